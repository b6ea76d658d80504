// tcfft.cuh -- the bf16x3 form's line FFT: radix-16 DFT stages as tensor-core products of split-BF16 operands.
//
// A tile of LINES lines of length N (N = R * 16 * 16, R in {1, 2, 3, 4, 8}) sits in shared memory and is transformed
// by Stockham stages: one radix-R stage on the CUDA cores (Ns = 1; skipped when R = 1), then two radix-16
// stages (Ns = R, then 16 R). A radix-16 stage multiplies each group of 8 twiddled 16-point vectors by the DFT matrix
// F[a][b] = e^{-2 pi i ab / 16} with mma.sync.m16n8k16 (bf16 operands, float32 accumulators), real-ified as
//     Re y = Re F Re x - Im F Im x,   Im y = Im F Re x + Re F Im x
// (conjugated F for the inverse). The data are split in two bf16 terms, x = x_hi + x_lo with x_hi = bf16(x) and
// x_lo = bf16(x - x_hi) (about 16 significant bits); the constant matrix in three, F = F_hi + F_lo + F_lo2, and each
// product is taken as F_hi x_hi + F_hi x_lo + F_lo x_hi + F_lo2 x_hi. The F_lo2 term matters although it is tiny: with
// F to 16 bits only, F_hi + F_lo is a fixed non-unitary matrix (singular values of F/4 up to 1 + 2e-6) whose norm gain,
// +9e-7 per stage, adds up coherently over the 8 stages of every slice; with it the gain is below 1e-8 and what remains
// is the random rounding of x_lo and the dropped lo x lo terms (about 3e-6 relative per stage). Twiddles (W_N^m, float32,
// from the context's plan) and the radix-R butterflies are float32 on the CUDA cores.
//
// Stockham stage with radix Q and span Ns over a line x of length N: for j in [0, N/Q), k = j mod Ns,
//     u_r = x[j + r N/Q] W_{Q Ns}^{k r},   x'[(j - k) Q + k + r Ns] = sum_s u_s W_Q^{r s}.
// Stages run out of place between the tile's stage buffer and one scratch tile, with one block barrier each.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "fft.cuh"

namespace simk {

// XOR swizzle of float2 offsets inside a tile: x ^ sum_i ((x >> a_i) & (2^w_i - 1)) << b_i. Every term moves higher
// bits into bits 0-3 (a_i >= b_i + w_i), so the map is a bijection that keeps each aligned block of 16 float2 in place
// (the tiles are multiples of 16 float2). Chosen per tile shape by an exhaustive search over the warp-wide access
// patterns of the stages below (8-byte accesses, counted per half-warp): 1.0-1.44 x the conflict-free wavefront count,
// against 2.4-3.7 x for the natural layout.
struct Xor3 {
    int a0, w0, b0, a1, w1, b1, a2, w2, b2;
};

template <int N, int LINES, bool COLS> constexpr Xor3 tile_swizzle() {
    if constexpr (!COLS) {
        if constexpr (N == 256) return {4, 3, 1, 1, 1, 0, 4, 2, 2};
        else if constexpr (N == 512) return {4, 3, 1, 5, 3, 0, 1, 1, 0};
        else if constexpr (N == 768) return {5, 2, 2, 2, 2, 0, 0, 0, 0};
        else if constexpr (N == 1024) return {4, 4, 0, 6, 3, 0, 0, 0, 0};
        else return {5, 4, 0, 7, 3, 0, 4, 3, 0};
    } else if constexpr (LINES == 2) {
        if constexpr (N == 256) return {4, 3, 1, 5, 3, 0, 0, 0, 0};
        else if constexpr (N == 512) return {6, 3, 0, 4, 4, 0, 3, 2, 0};
        else if constexpr (N == 768) return {5, 4, 0, 6, 1, 1, 2, 1, 1};
        else if constexpr (N == 1024) return {5, 4, 0, 3, 3, 0, 7, 3, 0};
        else return {4, 2, 2, 6, 4, 0, 8, 3, 0};
    } else if constexpr (LINES == 4) {
        if constexpr (N == 256) return {6, 3, 0, 4, 4, 0, 0, 0, 0};
        else if constexpr (N == 512) return {5, 4, 0, 7, 3, 0, 3, 2, 1};
        else if constexpr (N == 768) return {5, 4, 0, 1, 1, 0, 5, 1, 0};
        else if constexpr (N == 1024) return {6, 4, 0, 4, 2, 2, 8, 3, 0};
        else return {7, 4, 0, 4, 3, 1, 9, 3, 0};
    } else {
        if constexpr (N == 256) return {5, 4, 0, 7, 3, 0, 4, 1, 0};
        else if constexpr (N == 512) return {6, 4, 0, 4, 1, 3, 8, 3, 0};
        else if constexpr (N == 768) return {6, 4, 0, 2, 1, 0, 4, 3, 0};
        else return {7, 4, 0, 4, 2, 2, 9, 3, 0};
    }
}

// Lines of the tile in shared memory: column tiles interleave LINES columns (element idx of line c at natural offset
// idx LINES + c), row tiles hold whole rows (at c N + idx). `nat` is that natural offset (the layout the TMA copies
// produce, and of the staged P / t tiles); `at` the swizzled working layout every stage writes.
template <int N, int LINES, bool COLS> struct TileLayout {
    static constexpr Xor3 S = tile_swizzle<N, LINES, COLS>();
    __device__ __forceinline__ static int nat(int line, int idx) { return COLS ? idx * LINES + line : line * N + idx; }
    __device__ __forceinline__ static int swz(int x) {
        return x ^ (((x >> S.a0) & ((1 << S.w0) - 1)) << S.b0) ^ (((x >> S.a1) & ((1 << S.w1) - 1)) << S.b1) ^
               (((x >> S.a2) & ((1 << S.w2) - 1)) << S.b2);
    }
    __device__ __forceinline__ static int at(int line, int idx) { return swz(nat(line, idx)); }
    template <bool NAT> __device__ __forceinline__ static int in(int line, int idx) {
        return NAT ? nat(line, idx) : at(line, idx);
    }
};

// m16k16 A fragments (row-major; lane g = lane / 4, q = lane % 4 holds rows g, g + 8 and columns 2q, 2q + 1, 2q + 8,
// 2q + 9) of Re F and Im F of the forward 16-point DFT, each split into three bf16 terms.
struct Dft16Frags {
    uint32_t rh[4], rl[4], rl2[4], ih[4], il[4], il2[4];
};

__device__ __forceinline__ uint32_t bf162_bits(__nv_bfloat162 v) { return *reinterpret_cast<uint32_t*>(&v); }

// (a, b) -> hi = bf16x2(a, b), lo = bf16x2(a - hi.a, b - hi.b); a in the low half, as the fragments want.
__device__ __forceinline__ void split_bf16x2(float a, float b, uint32_t& hi, uint32_t& lo) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    const float2 hf = __bfloat1622float2(h);
    hi = bf162_bits(h);
    lo = bf162_bits(__floats2bfloat162_rn(a - hf.x, b - hf.y));
}

// The same in three terms, from float64: a = hi + lo + lo2 to about 24 bits.
__device__ __forceinline__ void split3_bf16x2(double a, double b, uint32_t& hi, uint32_t& lo, uint32_t& lo2) {
    const __nv_bfloat162 h = __floats2bfloat162_rn((float)a, (float)b);
    const float2 hf = __bfloat1622float2(h);
    const double ra = a - hf.x, rb = b - hf.y;
    const __nv_bfloat162 l = __floats2bfloat162_rn((float)ra, (float)rb);
    const float2 lf = __bfloat1622float2(l);
    hi = bf162_bits(h);
    lo = bf162_bits(l);
    lo2 = bf162_bits(__floats2bfloat162_rn((float)(ra - lf.x), (float)(rb - lf.y)));
}

__device__ __forceinline__ Dft16Frags dft16_frags(int lane) {
    const int g = lane >> 2, q = lane & 3;
    Dft16Frags f;
#pragma unroll
    for (int reg = 0; reg < 4; ++reg) {
        const int row = g + ((reg & 1) ? 8 : 0);
        const int col = 2 * q + ((reg & 2) ? 8 : 0);
        double re[2], im[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int m = (row * (col + h)) & 15;  // e^{-2 pi i m / 16} from the exact ratio
            sincospi(-(double)m / 8.0, &im[h], &re[h]);
        }
        split3_bf16x2(re[0], re[1], f.rh[reg], f.rl[reg], f.rl2[reg]);
        split3_bf16x2(im[0], im[1], f.ih[reg], f.il[reg], f.il2[reg]);
    }
    return f;
}

// Not volatile: the instruction has outputs, and without the qualifier the compiler may interleave independent
// accumulator chains instead of issuing every product in program order.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <bool NEG> __device__ __forceinline__ void negate_if(uint32_t (&o)[4], const uint32_t (&a)[4]) {
    constexpr uint32_t S = NEG ? 0x80008000u : 0u;
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = a[i] ^ S;  // bf16 sign bits
}

// The complex 16-point DFT of one group in split BF16, both accumulators at once:
//     dr += R xr + S1 I xi,   di += S2 I xr + R xi   (S1 = -1, S2 = +1 forward; S1 = +1, S2 = -1 inverse),
// each real product as (A_hi + A_lo + A_lo2)(B_hi + B_lo) without the lo x lo terms, the small terms first so that
// they are not lost against the large ones in the float32 accumulators. The two accumulators' chains alternate so
// that consecutive products are independent.
template <int DIR>
__device__ __forceinline__ void dft16_split(float (&dr)[4], float (&di)[4], const Dft16Frags& F,
                                            const uint32_t (&xrh)[2], const uint32_t (&xrl)[2],
                                            const uint32_t (&xih)[2], const uint32_t (&xil)[2]) {
    uint32_t i1h[4], i1l[4], i1l2[4], i2h[4], i2l[4], i2l2[4];
    negate_if<(DIR < 0)>(i1h, F.ih);
    negate_if<(DIR < 0)>(i1l, F.il);
    negate_if<(DIR < 0)>(i1l2, F.il2);
    negate_if<(DIR > 0)>(i2h, F.ih);
    negate_if<(DIR > 0)>(i2l, F.il);
    negate_if<(DIR > 0)>(i2l2, F.il2);
    mma_bf16(dr, F.rl2, xrh[0], xrh[1]);
    mma_bf16(di, i2l2, xrh[0], xrh[1]);
    mma_bf16(dr, i1l2, xih[0], xih[1]);
    mma_bf16(di, F.rl2, xih[0], xih[1]);
    mma_bf16(dr, F.rl, xrh[0], xrh[1]);
    mma_bf16(di, i2l, xrh[0], xrh[1]);
    mma_bf16(dr, i1l, xih[0], xih[1]);
    mma_bf16(di, F.rl, xih[0], xih[1]);
    mma_bf16(dr, F.rh, xrl[0], xrl[1]);
    mma_bf16(di, i2h, xrl[0], xrl[1]);
    mma_bf16(dr, i1h, xil[0], xil[1]);
    mma_bf16(di, F.rh, xil[0], xil[1]);
    mma_bf16(dr, F.rh, xrh[0], xrh[1]);
    mma_bf16(di, i2h, xrh[0], xrh[1]);
    mma_bf16(dr, i1h, xih[0], xih[1]);
    mma_bf16(di, F.rh, xih[0], xih[1]);
}

// A copy of v the compiler cannot see through. The stages' shared-memory addresses depend only on the thread, so
// without it they are hoisted out of the persistent tile loop and held in registers for every stage at once (spills);
// with it they are recomputed per tile on the otherwise idle integer pipe.
__device__ __forceinline__ int opaque(int v) {
    int r;
    asm volatile("mov.b32 %0, %1;" : "=r"(r) : "r"(v));
    return r;
}

// What the first stage of a transform does to each element as it loads it: nothing, x scale, or x pre[idx] scale
// (pre: a tile of the same layout, e.g. the propagator or transmission rows staged with the wave).
enum { PRE_NONE = 0, PRE_SCALE = 1, PRE_MUL = 2 };

template <int PRE>
__device__ __forceinline__ float2 pre_apply(float2 v, const float2* __restrict__ pre, int a, float scale) {  // a: natural
    if constexpr (PRE == PRE_SCALE) return v * scale;
    else if constexpr (PRE == PRE_MUL) return cmul(v, pre[a]) * scale;
    else return v;
}

// One radix-16 stage on the tensor cores, out of place (src -> dst, then one barrier). LINES N / 256 warps, two groups
// of 8 vectors each: a group takes LG lines (adjacent columns of a column tile, so that one access touches
// neighbouring words) times 8 / LG consecutive j. Each group's outputs are stored as soon as its products are done.
template <int N, int LINES, bool COLS, int NS, int DIR, int PRE, bool IN_NAT>
__device__ __forceinline__ void tc_stage16(const float2* __restrict__ src, float2* __restrict__ dst,
                                           const float2* __restrict__ pre, float scale,
                                           const float2* __restrict__ tw, const Dft16Frags& F, int warp, int lane) {
    constexpr int NV = N / 16;                             // 16-point vectors per line
    constexpr int LG = COLS ? (LINES < 8 ? LINES : 8) : 1;  // lines per group
    constexpr int JG = 8 / LG;                             // vectors per line per group
    constexpr int GPL = NV / JG;                           // groups per block of LG lines
    constexpr int NWARPS = LINES * N / 256;
    static_assert(NV % JG == 0 && LINES % LG == 0 && (LINES * N) % 256 == 0, "tile shape");
    using L = TileLayout<N, LINES, COLS>;
    lane = opaque(lane);
    warp = opaque(warp);
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int gi = warp + s * NWARPS;
        const int lb = gi / GPL, jb = gi - lb * GPL;
        float2 x[4];
        {
            const int line = lb * LG + g % LG;  // this lane's vector: B column n = g
            const int j = jb * JG + g / LG;
            const int k = j % NS;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int r = 2 * q + (e & 1) + ((e & 2) ? 8 : 0);
                float2 v = pre_apply<PRE>(src[L::template in<IN_NAT>(line, j + r * NV)], pre,
                                          L::nat(line, j + r * NV), scale);
                if constexpr (NS > 1) {
                    const float2 w = __ldg(tw + k * r * (N / (16 * NS)));
                    v = (DIR < 0) ? cmul(v, w) : cmulc(v, w);
                }
                x[e] = v;
            }
        }
        uint32_t xrh[2], xrl[2], xih[2], xil[2];
        split_bf16x2(x[0].x, x[1].x, xrh[0], xrl[0]);
        split_bf16x2(x[2].x, x[3].x, xrh[1], xrl[1]);
        split_bf16x2(x[0].y, x[1].y, xih[0], xil[0]);
        split_bf16x2(x[2].y, x[3].y, xih[1], xil[1]);
        float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
        // forward: Re y = R xr - I xi, Im y = I xr + R xi; inverse (conjugate F): Re y = R xr + I xi, Im y = -I xr + R xi
        dft16_split<DIR>(acc[0], acc[1], F, xrh, xrl, xih, xil);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            // accumulator e: row (output index) g + 8 (e >> 1), column (vector) n = 2q + (e & 1)
            const int n = 2 * q + (e & 1);
            const int rr = g + ((e & 2) ? 8 : 0);
            const int line = lb * LG + n % LG;
            const int j = jb * JG + n / LG;
            const int k = j % NS;
            dst[L::at(line, (j - k) * 16 + k + rr * NS)] = make_float2(acc[0][e], acc[1][e]);
        }
    }
    __syncthreads();
}

// The first stage, radix R on the CUDA cores (Ns = 1: no twiddles), out of place: 8 / R butterflies per thread (for
// R = 3 the last round is partial).
template <int N, int LINES, bool COLS, int R, int DIR, int PRE, bool IN_NAT>
__device__ __forceinline__ void cc_stage_first(const float2* __restrict__ src, float2* __restrict__ dst,
                                               const float2* __restrict__ pre, float scale, int tid) {
    constexpr int NT = LINES * N / 8;
    constexpr int M = N / R;
    constexpr int NBF = LINES * M;           // butterflies in the tile
    constexpr int NB = (NBF + NT - 1) / NT;  // rounds
    using L = TileLayout<N, LINES, COLS>;
    tid = opaque(tid);
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int bi = tid + NT * b;
        if (NBF % NT != 0 && bi >= NBF) break;
        const int line = COLS ? bi % LINES : bi / M;
        const int j = COLS ? bi / LINES : bi % M;
        float2 u[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
            u[r] = pre_apply<PRE>(src[L::template in<IN_NAT>(line, j + r * M)], pre, L::nat(line, j + r * M), scale);
        if constexpr (R == 2) bfly2<DIR>(u);
        else if constexpr (R == 3) bfly3<DIR>(u);
        else if constexpr (R == 4) bfly4<DIR>(u);
        else bfly8<DIR>(u);
#pragma unroll
        for (int r = 0; r < R; ++r) dst[L::at(line, j * R + r)] = u[r];
    }
    __syncthreads();
}

template <int N> struct TcPlan {
    static constexpr int R = N / 256;
    static constexpr bool ok = (N % 256 == 0) && (R == 1 || R == 2 || R == 3 || R == 4 || R == 8);
    static constexpr int stages = (R == 1) ? 2 : 3;
};

// The whole line FFT of the tile, ping-ponging between a (which holds the input: natural layout when IN_NAT, e.g.
// straight from a TMA copy, else the working layout) and b; returns the buffer that holds the output (working layout
// TileLayout::at, natural order of the transform): b after an odd number of stages, a after an even one. DIR < 0
// forward (e^{-}), > 0 inverse (unnormalised). The caller's block has LINES N / 8 threads; tid is the linear thread
// index; every thread has finished reading b before the call.
template <int N, int LINES, bool COLS, int DIR, int PRE, bool IN_NAT>
__device__ __forceinline__ float2* tc_fft(float2* __restrict__ a, float2* __restrict__ b,
                                          const float2* __restrict__ pre, float scale,
                                          const float2* __restrict__ tw, const Dft16Frags& F, int tid) {
    static_assert(TcPlan<N>::ok, "bf16x3 line length");
    constexpr int R = TcPlan<N>::R;
    const int warp = tid >> 5, lane = tid & 31;
    if constexpr (R == 1) {
        tc_stage16<N, LINES, COLS, 1, DIR, PRE, IN_NAT>(a, b, pre, scale, tw, F, warp, lane);
        tc_stage16<N, LINES, COLS, 16, DIR, PRE_NONE, false>(b, a, nullptr, 1.0f, tw, F, warp, lane);
        return a;
    } else {
        cc_stage_first<N, LINES, COLS, R, DIR, PRE, IN_NAT>(a, b, pre, scale, tid);
        tc_stage16<N, LINES, COLS, R, DIR, PRE_NONE, false>(b, a, nullptr, 1.0f, tw, F, warp, lane);
        tc_stage16<N, LINES, COLS, 16 * R, DIR, PRE_NONE, false>(a, b, nullptr, 1.0f, tw, F, warp, lane);
        return b;
    }
}

}  // namespace simk
