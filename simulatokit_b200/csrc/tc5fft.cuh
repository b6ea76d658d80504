// tc5fft.cuh -- the bf16x3 form's radix-16 DFT stages on the fifth-generation tensor cores (tcgen05, TMEM).
//
// A tile of LINES lines of length N = R * 16 * 16 (R = 1 or 2) in shared memory is transformed by a radix-R Stockham
// stage on the CUDA cores (R = 2 only, folded into the next stage's gather) and two radix-16 stages (Ns = R, 16 R) as
// tensor-core products. A radix-16 stage is one matrix product per block of 128 vectors:
//     D[v][2s + a] = sum_{r, b} A[v][2r + b] B[2s + a][2r + b]       (v: vector, r: input, s: output; a, b: re / im)
// with A the twiddled inputs as (re, im) pairs and B the real form of the DFT matrix F[s][r] = e^{-+2 pi i s r / 16}:
// B[2s][2r] = B[2s+1][2r+1] = Re F, B[2s][2r+1] = -Im F, B[2s+1][2r] = Im F. One elected thread issues
// tcgen05.mma (kind::f16, BF16 operands from shared memory, M = 128, N = 32, K = 16, float32 accumulators in tensor
// memory) and commits to an mbarrier; every thread then reads its row of D with tcgen05.ld.
//
// Precision. The data are split in three BF16 terms, x = x_hi + x_lo + x_lo2 (x_lo = bf16(x - x_hi), x_lo2 =
// bf16(x - x_hi - x_lo), about 24 bits), and so is B (B_hi + B_lo + B_lo2, from float64). Six products are summed:
// hi x lo2, hi x lo, lo x lo, lo2 x hi, lo x hi, hi x hi (A term x B term, small ones first); the dropped products are
// below 2^-24 of the result. With a two-term data split the rounding of x_lo (2^-18 of x) is correlated across the
// many equal values of a plane wave or a vacuum region and moved the total intensity by about 1e-5 per slice; with
// three terms it is about 1e-8. The tensor core's accumulator does not round to nearest when it adds a small product
// to a large sum, so no product is added to hi x hi inside it: the twelve-instruction order adds hi x hi last, and
// the stacked order keeps it in a column block of its own that the threads add in float32.
//
// Shared memory of a block: per block of 128 vectors three A planes (hi, lo, lo2), each K-major without swizzle: the
// 16-byte chunk c (K = 8c .. 8c + 7, i.e. inputs r = 4c .. 4c + 3) of row v at c * kTc5Lbo + v * 16 (core matrices
// of 8 rows x 16 bytes, 128 bytes apart along M: SBO = 128; chunks kTc5Lbo apart along K: LBO). kTc5Lbo = 2080 rather
// than 2048 spreads the 4-byte scatter of the second stage over all 32 banks. Then the B operand of each direction:
// the three terms' 32 rows stacked (rows 0-31 B_lo2, 32-63 B_lo, 64-95 B_hi), 4 chunks with LBO 1536, SBO 128, so
// that one descriptor covers B_hi (N = 32, from row 64), B_lo and B_hi (N = 64, from row 32) or all three (N = 96).
//
// Products. Either twelve instructions of N = 32, each A term times each B term it pairs with accumulating into one
// 32-column D (the default), or six of N = 96, 64, 32 (`stack`): A_hi times [B_lo2 B_lo B_hi], A_lo times
// [B_lo B_hi] and A_lo2 times B_hi into three 32-column blocks of D, (hi lo2 + lo lo + lo2 hi, hi lo + lo hi, hi hi),
// which the threads add, the two small blocks first, as they read them.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "tcfft.cuh"
#include "tma.cuh"

namespace simk {

constexpr uint32_t kTc5Lbo = 2080;                        // bytes between K chunks of an A plane
constexpr uint32_t kTc5Plane = 3 * kTc5Lbo + 2048;        // one A plane (4 chunks of 128 rows x 16 bytes)
constexpr uint32_t kTc5BLbo = 96 * 16;                    // bytes between K chunks of a direction's B (96 rows)
constexpr uint32_t kTc5BBytes = 4 * kTc5BLbo;             // one direction's B (3 terms x 32 rows x 64 bytes)
// Shared-memory bytes of the engine for MB blocks of 128 vectors: the A planes, then both directions' B.
constexpr uint32_t tc5_smem_bytes(int mb) { return (uint32_t)mb * 3u * kTc5Plane + 2u * kTc5BBytes; }
// Tensor-memory columns per block of 128 vectors: 32 float32 accumulator columns, or 128 (96 used) with the stacked
// products; a power of two, at least 32.
__host__ __device__ constexpr uint32_t tc5_tmem_cols(int mb, bool stack = false) {
    return stack ? (uint32_t)mb * 128u : (mb <= 1 ? 32u : (mb <= 2 ? 64u : 128u));
}
__host__ __device__ constexpr uint32_t tc5_block_cols(bool stack) { return stack ? 128u : 32u; }
// Instruction descriptor of kind::f16: D float32 (bits 4-5 = 1), A and B BF16 (bits 7-9 = 1, 10-12 = 1), both K-major,
// N >> 3 in bits 17-22, M >> 4 in bits 24-28 (M = 128; N = 32, 64 or 96, multiples of 16 as M = 128 requires).
__host__ __device__ constexpr uint32_t tc5_idesc(uint32_t n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

// ---- tcgen05 instructions ---------------------------------------------------------------------------------------------
// One warp allocates `ncols` tensor-memory columns and writes their address to *slot (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major without swizzle: start, LBO (K direction), SBO (M / N direction), all in
// bytes (multiples of 16); version 1 (bits 46-47), base offset 0, layout type 0.
__device__ __forceinline__ uint64_t tc5_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// D (tensor memory) = A B^T (+ D when accumulate): M = 128, K = 16, N from the instruction descriptor, issued by the
// calling thread alone.
__device__ __forceinline__ void tc5_mma(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                        uint32_t accumulate) {
    const uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2),
        "r"(mask3)
        : "memory");
}
// Arrives on `bar` once every tcgen05.mma this thread issued before has completed.
__device__ __forceinline__ void tc5_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
// 16 consecutive float32 columns of this thread's tensor-memory lane (the warp's quarter of the lanes), waited for
// inside the same statement so that no use of the registers can be scheduled before the load completes.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t tc5_bits(__nv_bfloat162 v) { return *reinterpret_cast<uint32_t*>(&v); }

// (re, im) -> three bf16x2 words, re in the low half: hi = bf16(x), lo = bf16(x - hi), lo2 = bf16(x - hi - lo); the
// differences are exact in float32 and are taken as packed pairs (one sub.f32x2 each, the same bits as two subs).
__device__ __forceinline__ void tc5_split3(float2 x, uint32_t& h, uint32_t& l, uint32_t& l2) {
    const __nv_bfloat162 hh = __floats2bfloat162_rn(x.x, x.y);
    const float2 r = psub(x, __bfloat1622float2(hh));
    const __nv_bfloat162 ll = __floats2bfloat162_rn(r.x, r.y);
    const float2 r2 = psub(r, __bfloat1622float2(ll));
    h = tc5_bits(hh);
    l = tc5_bits(ll);
    l2 = tc5_bits(__floats2bfloat162_rn(r2.x, r2.y));
}

// Polls of a wait for the tensor core: a stage's products finish within microseconds, so a wait this long means the
// products never completed (the caller records the error and abandons the tile).
constexpr uint32_t kTc5WaitPolls = 1u << 20;

// ---- per-block state ----------------------------------------------------------------------------------------------
struct Tc5 {
    uint32_t a_base;   // shared address of the A planes
    uint32_t b_base;   // shared address of the B matrices
    uint8_t* a_ptr;    // generic pointer to the A planes
    uint32_t tmem;     // tensor-memory address of the accumulators (lane 0)
    uint64_t* bar;     // the MMA completion barrier
    uint32_t phase;    // its next parity
    int stack;         // six stacked products (N = 96, 64, 32) instead of twelve of N = 32
};

// The six B matrices (forward, inverse) x (hi, lo, lo2) into shared memory at `b` by all `nthreads` threads, from
// the exact ratio s r / 16 in float64.
__device__ __forceinline__ void tc5_build_b(uint8_t* b, int tid, int nthreads) {
    for (int e = tid; e < 2 * 32 * 32; e += nthreads) {
        const int inv = e >> 10, n = (e >> 5) & 31, k = e & 31;
        const int s = n >> 1, a = n & 1, r = k >> 1, bb = k & 1;
        double sn, cs;
        sincospi(-(double)((s * r) & 15) / 8.0, &sn, &cs);  // F = e^{-2 pi i s r / 16} = cs + i sn
        const double im = inv ? -sn : sn;                    // the inverse takes conj(F)
        const double val = a == 0 ? (bb == 0 ? cs : -im) : (bb == 0 ? im : cs);
        const __nv_bfloat16 h = __double2bfloat16(val);
        const double r1 = val - (double)__bfloat162float(h);
        const __nv_bfloat16 l = __double2bfloat16(r1);
        const __nv_bfloat16 l2 = __double2bfloat16(r1 - (double)__bfloat162float(l));
        // row n of B_lo2, B_lo, B_hi sits at row n, 32 + n, 64 + n of the direction's stacked matrix
        const uint32_t off = (uint32_t)(k >> 3) * kTc5BLbo + (uint32_t)n * 16u + (uint32_t)(k & 7) * 2u;
        uint8_t* bd = b + inv * kTc5BBytes + off;
        *reinterpret_cast<__nv_bfloat16*>(bd) = l2;
        *reinterpret_cast<__nv_bfloat16*>(bd + 32 * 16) = l;
        *reinterpret_cast<__nv_bfloat16*>(bd + 64 * 16) = h;
    }
}

// Thread 0: the products of every block of 128 vectors, then a commit to the barrier.
template <int MB, int DIR>
__device__ __forceinline__ void tc5_issue(const Tc5& c) {
    tc_fence_after();
    constexpr int inv = DIR > 0 ? 1 : 0;
    const uint32_t bbase = c.b_base + (uint32_t)inv * kTc5BBytes;
    const uint32_t bcols = tc5_block_cols(c.stack != 0);
#pragma unroll
    for (int mb = 0; mb < MB; ++mb) {
        const uint32_t d = c.tmem + (uint32_t)mb * bcols;
        if (c.stack) {
            // A_hi x [B_lo2 B_lo B_hi] (N = 96 from row 0, initialises all three blocks), A_lo x [B_lo B_hi] (N = 64
            // from row 32), A_lo2 x B_hi (N = 32 from row 64), every one into the blocks from column 0
#pragma unroll
            for (int pa = 0; pa < 3; ++pa) {
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    const uint64_t ad = tc5_desc(c.a_base + (uint32_t)(mb * 3 + pa) * kTc5Plane + 2u * kk * kTc5Lbo,
                                                 kTc5Lbo, 128);
                    const uint64_t bd =
                        tc5_desc(bbase + (uint32_t)pa * 32u * 16u + 2u * kk * kTc5BLbo, kTc5BLbo, 128);
                    tc5_mma(d, ad, bd, tc5_idesc(96u - 32u * (uint32_t)pa), (pa | kk) != 0 ? 1u : 0u);
                }
            }
        } else {
            // (A plane, B row block): hi x lo2, hi x lo, lo x lo, lo2 x hi, lo x hi, hi x hi into one 32-column D
            constexpr int pa[6] = {0, 0, 1, 2, 1, 0};
            constexpr int tb[6] = {0, 1, 1, 2, 2, 2};
#pragma unroll
            for (int t = 0; t < 6; ++t) {
#pragma unroll
                for (int kk = 0; kk < 2; ++kk) {
                    const uint64_t ad = tc5_desc(c.a_base + (uint32_t)(mb * 3 + pa[t]) * kTc5Plane + 2u * kk * kTc5Lbo,
                                                 kTc5Lbo, 128);
                    const uint64_t bd = tc5_desc(bbase + (uint32_t)tb[t] * 32u * 16u + 2u * kk * kTc5BLbo, kTc5BLbo, 128);
                    tc5_mma(d, ad, bd, tc5_idesc(32), (t | kk) != 0 ? 1u : 0u);
                }
            }
        }
    }
    tc5_commit(c.bar);
}

// This thread's 16 accumulator columns (outputs 8 h .. 8 h + 7) of its vector: one block, or the sum of the three
// stacked blocks, the two small ones first.
__device__ __forceinline__ void tc5_read(const Tc5& c, uint32_t taddr, float (&d)[16]) {
    tmem_ld16(taddr, d);
    if (c.stack) {
        float e[16], f[16];
        tmem_ld16(taddr + 32u, e);
        tmem_ld16(taddr + 64u, f);
#pragma unroll
        for (int i = 0; i < 16; i += 2) {  // (d + e) + f on (re, im) pairs: add.f32x2, the same bits as scalar adds
            const float2 s = padd(padd(make_float2(d[i], d[i + 1]), make_float2(e[i], e[i + 1])),
                                  make_float2(f[i], f[i + 1]));
            d[i] = s.x;
            d[i + 1] = s.y;
        }
    }
}

// The tile's line FFT. Thread (warp w, lane l) owns vector v = 128 mb + 32 (w % 4) + l, mb = w / 8, and half h =
// (w / 4) % 2 of it (inputs r and outputs s in 8 h .. 8 h + 7); v is line v % LINES, vector j = v / LINES of a column
// tile (neighbouring lanes read neighbouring columns) and line v / NV, j = v % NV of a row tile. The input is read
// from the float32 tile `src` in its natural layout (column tiles: idx LINES + line; row tiles: line N + idx), each
// value times pre[same offset] * scale (PRE_MUL), times scale (PRE_SCALE) or as it is; the output is left in z[i],
// i < 8, the transform's element j + NV (8 h + i) of line `line`. Returns false when a wait for the tensor core ran
// out (the caller abandons the tile). Every thread calls it; it ends after a barrier at which every thread has read
// its last output, and it does not write `src`. line_out, idx0_out: z[i] is element idx0_out + NV i of line line_out.
template <int N, int LINES, bool COLS, int DIR, int PRE>
__device__ __forceinline__ bool tc5_fft(const float2* __restrict__ src, const float2* __restrict__ pre, float scale,
                                        const float2* __restrict__ tw, Tc5& c, int tid, float2 (&z)[8], int& line_out,
                                        int& idx0_out) {
    constexpr int R = N / 256;
    static_assert(R == 1 || R == 2, "tcgen05 line lengths: 256 and 512");
    constexpr int NV = N / 16;           // vectors per line in a radix-16 stage
    constexpr int V = LINES * NV;        // vectors in the tile
    constexpr int MB = V / 128;
    static_assert(V % 128 == 0, "blocks of 128 vectors");
    constexpr int NSA = R, NSB = 16 * R;  // the two radix-16 stages' spans
    const int warp = tid >> 5, lane = tid & 31;
    const int mb = warp >> 3, h = (warp >> 2) & 1, q = warp & 3;
    const int v = mb * 128 + q * 32 + lane;
    const int line = COLS ? v % LINES : v / NV;
    const int j = COLS ? v / LINES : v % NV;
    line_out = line;
    idx0_out = j + NV * 8 * h;
    auto nat = [&](int idx) { return COLS ? idx * LINES + line : line * N + idx; };
    auto load = [&](int idx) {
        const int o = nat(idx);
        float2 x = src[o];
        if constexpr (PRE == PRE_MUL) x = cmul(x, pre[o]) * scale;
        else if constexpr (PRE == PRE_SCALE) x = x * scale;
        return x;
    };
    auto row_of = [&](int jj) { return COLS ? jj * LINES + line : line * NV + jj; };  // vector (line, jj) -> A row
    uint8_t* a_blk = c.a_ptr;  // plane p of block b at (b * 3 + p) * kTc5Plane
    const uint32_t lane_base = (uint32_t)(q * 32) << 16;
    const uint32_t d_col = c.tmem + lane_base + (uint32_t)mb * tc5_block_cols(c.stack != 0) + (uint32_t)h * 16u;

    // ---- stage A: gather (radix-2 first stage folded in for R = 2), twiddle, split, write A rows ----
    {
        const int k = j % NSA;
        uint32_t hw[8], lw[8], l2w[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int r = 8 * h + i;
            const int p = j + r * NV;
            float2 x;
            if constexpr (R == 2) {
                const int m = p >> 1;
                const float2 a = load(m), b = load(m + N / 2);
                x = (p & 1) ? a - b : a + b;
            } else {
                x = load(p);
            }
            if constexpr (NSA > 1) {
                const float2 w = __ldg(tw + k * r * (N / (16 * NSA)));
                x = (DIR < 0) ? cmul(x, w) : cmulc(x, w);
            }
            tc5_split3(x, hw[i], lw[i], l2w[i]);
        }
        uint8_t* rowp = a_blk + (size_t)(v >> 7) * 3 * kTc5Plane + (size_t)(v & 127) * 16;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const uint32_t off = (uint32_t)(2 * h + e) * kTc5Lbo;
            *reinterpret_cast<uint4*>(rowp + 0 * kTc5Plane + off) = make_uint4(hw[4 * e], hw[4 * e + 1], hw[4 * e + 2], hw[4 * e + 3]);
            *reinterpret_cast<uint4*>(rowp + 1 * kTc5Plane + off) = make_uint4(lw[4 * e], lw[4 * e + 1], lw[4 * e + 2], lw[4 * e + 3]);
            *reinterpret_cast<uint4*>(rowp + 2 * kTc5Plane + off) = make_uint4(l2w[4 * e], l2w[4 * e + 1], l2w[4 * e + 2], l2w[4 * e + 3]);
        }
    }
    fence_proxy_async_shared();
    __syncthreads();
    if (tid == 0) tc5_issue<MB, DIR>(c);
    bool ok = mbar_wait_bounded(c.bar, c.phase, kTc5WaitPolls);
    c.phase ^= 1u;
    tc_fence_after();
    float d[16];
    if (ok) tc5_read(c, d_col, d);
    // ---- stage B: the outputs of stage A, twiddled for stage B and split, scattered into the A rows they feed ----
    // Output s = 8 h + i of stage A sits at (j - k) 16 + k + s NSA (k = j mod NSA) and is input rb of stage-B vector jb:
    // for R = 2, jb = k + 2 s and rb = j / 2; for R = 1, jb = s and rb = j. So along i the stage-B vector steps by
    // NSA (its A row by NSA LINES for column tiles, NSA for row tiles), the input rb is fixed, and the twiddle
    // W_N^{jb rb} steps by NSA rb: one base address and constant strides per thread, all in one 128-vector block.
    {
        const int k = j % NSA;
        const int rb = (R == 2) ? (j >> 1) : j;
        const int vb0 = row_of(R == 2 ? k + 16 * h : 8 * h);
        constexpr int kRowStep = NSA * (COLS ? LINES : 1);
        uint8_t* p0 = a_blk + (size_t)(vb0 >> 7) * 3 * kTc5Plane + (size_t)(vb0 & 127) * 16 +
                      (size_t)(rb >> 2) * kTc5Lbo + (size_t)(rb & 3) * 4;
        const float2* w0 = tw + (R == 2 ? (k + 16 * h) : 8 * h) * rb;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            float2 x = make_float2(d[2 * i], d[2 * i + 1]);
            const float2 w = __ldg(w0 + i * NSA * rb);
            x = (DIR < 0) ? cmul(x, w) : cmulc(x, w);
            uint32_t hh, ll, l2;
            tc5_split3(x, hh, ll, l2);
            uint8_t* p = p0 + i * kRowStep * 16;
            *reinterpret_cast<uint32_t*>(p) = hh;
            *reinterpret_cast<uint32_t*>(p + kTc5Plane) = ll;
            *reinterpret_cast<uint32_t*>(p + 2 * kTc5Plane) = l2;
        }
    }
    tc_fence_before();
    fence_proxy_async_shared();
    __syncthreads();
    if (tid == 0) tc5_issue<MB, DIR>(c);
    ok = mbar_wait_bounded(c.bar, c.phase, kTc5WaitPolls) && ok;
    c.phase ^= 1u;
    tc_fence_after();
    if (ok) tc5_read(c, d_col, d);
#pragma unroll
    for (int i = 0; i < 8; ++i) z[i] = make_float2(d[2 * i], d[2 * i + 1]);
    tc_fence_before();
    __syncthreads();  // every thread has read D and its inputs: the next transform may write the A planes and D
    return ok;
}

}  // namespace simk
