// tcfft.cuh -- the bf16x3 form's line FFT: radix-16 DFT stages as tensor-core products of split-BF16 operands.
//
// A tile of LINES lines of length N (N = R * 16 * 16, R in {1, 2, 3, 4, 8}) sits in shared memory and is transformed in
// place by Stockham stages: one radix-R stage on the CUDA cores (Ns = 1; skipped when R = 1), then two radix-16
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
// Each stage reads its whole tile into registers (or tensor-core accumulators), synchronises the block, and writes
// the outputs in place.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "fft.cuh"

namespace simk {

// Lines of the tile in shared memory: column tiles interleave LINES columns (element idx of line c at idx LINES + c),
// row tiles hold whole rows (at c N + idx).
template <int N, int LINES, bool COLS> struct TileLayout {
    __device__ __forceinline__ static int at(int line, int idx) { return COLS ? idx * LINES + line : line * N + idx; }
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

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// d += (A_hi + A_lo + A_lo2)(B_hi + B_lo) without the lo x lo terms; NEG negates A (bf16 sign bits). The small
// terms go first so that they are not lost against the large one in the float32 accumulator.
template <bool NEG>
__device__ __forceinline__ void mma_split(float (&d)[4], const uint32_t (&ah)[4], const uint32_t (&al)[4],
                                          const uint32_t (&al2)[4], const uint32_t (&bh)[2], const uint32_t (&bl)[2]) {
    constexpr uint32_t S = NEG ? 0x80008000u : 0u;
    const uint32_t h[4] = {ah[0] ^ S, ah[1] ^ S, ah[2] ^ S, ah[3] ^ S};
    const uint32_t l[4] = {al[0] ^ S, al[1] ^ S, al[2] ^ S, al[3] ^ S};
    const uint32_t l2[4] = {al2[0] ^ S, al2[1] ^ S, al2[2] ^ S, al2[3] ^ S};
    mma_bf16(d, l2, bh[0], bh[1]);
    mma_bf16(d, l, bh[0], bh[1]);
    mma_bf16(d, h, bl[0], bl[1]);
    mma_bf16(d, h, bh[0], bh[1]);
}

// What the first stage of a transform does to each element as it loads it: nothing, x scale, or x pre[idx] scale
// (pre: a tile of the same layout, e.g. the propagator or transmission rows staged with the wave).
enum { PRE_NONE = 0, PRE_SCALE = 1, PRE_MUL = 2 };

template <int PRE>
__device__ __forceinline__ float2 pre_apply(float2 v, const float2* __restrict__ pre, int a, float scale) {
    if constexpr (PRE == PRE_SCALE) return v * scale;
    else if constexpr (PRE == PRE_MUL) return cmul(v, pre[a]) * scale;
    else return v;
}

// One radix-16 stage on the tensor cores. LINES N / 256 warps, two groups of 8 vectors each: a group takes LG lines
// (adjacent columns of a column tile, so that one access touches neighbouring words) times 8 / LG consecutive j.
template <int N, int LINES, bool COLS, int NS, int DIR, int PRE>
__device__ __forceinline__ void tc_stage16(float2* __restrict__ buf, const float2* __restrict__ pre, float scale,
                                           const float2* __restrict__ tw, const Dft16Frags& F, int warp, int lane) {
    constexpr int NV = N / 16;                             // 16-point vectors per line
    constexpr int LG = COLS ? (LINES < 8 ? LINES : 8) : 1;  // lines per group
    constexpr int JG = 8 / LG;                             // vectors per line per group
    constexpr int GPL = NV / JG;                           // groups per block of LG lines
    constexpr int NWARPS = LINES * N / 256;
    static_assert(NV % JG == 0 && LINES % LG == 0 && (LINES * N) % 256 == 0, "tile shape");
    using L = TileLayout<N, LINES, COLS>;
    const int g = lane >> 2, q = lane & 3;
    float acc[2][2][4];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int gi = warp + s * NWARPS;
        const int lb = gi / GPL, jb = gi - lb * GPL;
        const int line = lb * LG + g % LG;  // this lane's vector: B column n = g
        const int j = jb * JG + g / LG;
        const int k = j % NS;
        float2 x[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int r = 2 * q + (e & 1) + ((e & 2) ? 8 : 0);
            const int a = L::at(line, j + r * NV);
            float2 v = pre_apply<PRE>(buf[a], pre, a, scale);
            if constexpr (NS > 1) {
                const float2 w = __ldg(tw + k * r * (N / (16 * NS)));
                v = (DIR < 0) ? cmul(v, w) : cmulc(v, w);
            }
            x[e] = v;
        }
        uint32_t xrh[2], xrl[2], xih[2], xil[2];
        split_bf16x2(x[0].x, x[1].x, xrh[0], xrl[0]);
        split_bf16x2(x[2].x, x[3].x, xrh[1], xrl[1]);
        split_bf16x2(x[0].y, x[1].y, xih[0], xil[0]);
        split_bf16x2(x[2].y, x[3].y, xih[1], xil[1]);
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[s][0][e] = acc[s][1][e] = 0.0f;
        // forward: Re y = R xr - I xi, Im y = I xr + R xi; inverse (conjugate F): Re y = R xr + I xi, Im y = -I xr + R xi
        mma_split<false>(acc[s][0], F.rh, F.rl, F.rl2, xrh, xrl);
        mma_split<(DIR < 0)>(acc[s][0], F.ih, F.il, F.il2, xih, xil);
        mma_split<(DIR > 0)>(acc[s][1], F.ih, F.il, F.il2, xrh, xrl);
        mma_split<false>(acc[s][1], F.rh, F.rl, F.rl2, xih, xil);
    }
    __syncthreads();  // every input of the stage has been read
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const int gi = warp + s * NWARPS;
        const int lb = gi / GPL, jb = gi - lb * GPL;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            // accumulator e: row (output index) g + 8 (e >> 1), column (vector) n = 2q + (e & 1)
            const int n = 2 * q + (e & 1);
            const int rr = g + ((e & 2) ? 8 : 0);
            const int line = lb * LG + n % LG;
            const int j = jb * JG + n / LG;
            const int k = j % NS;
            buf[L::at(line, (j - k) * 16 + k + rr * NS)] = make_float2(acc[s][0][e], acc[s][1][e]);
        }
    }
    __syncthreads();
}

// The first stage, radix R on the CUDA cores (Ns = 1: no twiddles): 8 / R butterflies per thread (for R = 3 the
// last round is partial).
template <int N, int LINES, bool COLS, int R, int DIR, int PRE>
__device__ __forceinline__ void cc_stage_first(float2* __restrict__ buf, const float2* __restrict__ pre, float scale,
                                               int tid) {
    constexpr int NT = LINES * N / 8;
    constexpr int M = N / R;
    constexpr int NBF = LINES * M;           // butterflies in the tile
    constexpr int NB = (NBF + NT - 1) / NT;  // rounds
    using L = TileLayout<N, LINES, COLS>;
    float2 u[NB][R];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int bi = tid + NT * b;
        if (NBF % NT != 0 && bi >= NBF) break;
        const int line = COLS ? bi % LINES : bi / M;
        const int j = COLS ? bi / LINES : bi % M;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int a = L::at(line, j + r * M);
            u[b][r] = pre_apply<PRE>(buf[a], pre, a, scale);
        }
        if constexpr (R == 2) bfly2<DIR>(u[b]);
        else if constexpr (R == 3) bfly3<DIR>(u[b]);
        else if constexpr (R == 4) bfly4<DIR>(u[b]);
        else bfly8<DIR>(u[b]);
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int bi = tid + NT * b;
        if (NBF % NT != 0 && bi >= NBF) break;
        const int line = COLS ? bi % LINES : bi / M;
        const int j = COLS ? bi / LINES : bi % M;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[L::at(line, j * R + r)] = u[b][r];
    }
    __syncthreads();
}

template <int N> struct TcPlan {
    static constexpr int R = N / 256;
    static constexpr bool ok = (N % 256 == 0) && (R == 1 || R == 2 || R == 3 || R == 4 || R == 8);
};

// The whole line FFT of the tile, in place (natural order in and out). DIR < 0 forward (e^{-}), > 0 inverse
// (unnormalised). The caller's block has LINES N / 8 threads; tid is the linear thread index.
template <int N, int LINES, bool COLS, int DIR, int PRE>
__device__ __forceinline__ void tc_fft(float2* __restrict__ buf, const float2* __restrict__ pre, float scale,
                                       const float2* __restrict__ tw, const Dft16Frags& F, int tid) {
    static_assert(TcPlan<N>::ok, "bf16x3 line length");
    constexpr int R = TcPlan<N>::R;
    const int warp = tid >> 5, lane = tid & 31;
    if constexpr (R == 1) {
        tc_stage16<N, LINES, COLS, 1, DIR, PRE>(buf, pre, scale, tw, F, warp, lane);
        tc_stage16<N, LINES, COLS, 16, DIR, PRE_NONE>(buf, nullptr, 1.0f, tw, F, warp, lane);
    } else {
        cc_stage_first<N, LINES, COLS, R, DIR, PRE>(buf, pre, scale, tid);
        tc_stage16<N, LINES, COLS, R, DIR, PRE_NONE>(buf, nullptr, 1.0f, tw, F, warp, lane);
        tc_stage16<N, LINES, COLS, 16 * R, DIR, PRE_NONE>(buf, nullptr, 1.0f, tw, F, warp, lane);
    }
}

}  // namespace simk
