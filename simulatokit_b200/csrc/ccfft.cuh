// ccfft.cuh -- float32 line FFT of a shared-memory tile on the CUDA cores, for the fused passes at lengths that are not
// powers of two (N = 2^a 3^b 5^c with N % 8 == 0): 384, 640, 768, 1536, ...
//
// Compile-time Stockham plan: radix 8 while it divides, then 4, 2, 3, 5. A stage with radix R and span Ns reads
// u_r = x[j + r N/R] W_{R Ns}^{(j mod Ns) r}, takes the R-point DFT (the butterflies of fft.cuh) and writes
// x'[(j - j mod Ns) R + j mod Ns + r Ns]; the tile ping-pongs between the TMA stage buffer and a scratch tile with one
// block barrier per stage, like the tensor-core engine (tcfft.cuh), in an XOR-swizzled working layout found by
// exhaustive search over these stages' warp access patterns (conflict-free for every shape searched). Twiddles W_N^m
// come from the context's float32 plan table.
#pragma once

#include "tcfft.cuh"

namespace simk {

constexpr int cc_radix(int n, int s) {
    // the s-th radix of the plan for n (0 when past the end)
    for (int i = 0; i <= s; ++i) {
        int r = 0;
        if (n % 8 == 0) r = 8;
        else if (n % 4 == 0) r = 4;
        else if (n % 2 == 0) r = 2;
        else if (n % 3 == 0) r = 3;
        else if (n % 5 == 0) r = 5;
        if (r == 0 || n == 1) return 0;
        if (i == s) return r;
        n /= r;
    }
    return 0;
}

constexpr int cc_stages(int n) {
    int s = 0;
    while (cc_radix(n, s)) ++s;
    return s;
}

constexpr bool cc_plannable(int n) {
    int m = n;
    for (int r : {2, 3, 5})
        while (m % r == 0) m /= r;
    return m == 1 && n % 8 == 0 && n >= 64;
}

// Swizzled working layout of the float32 engine (the natural layout is TileLayout's).
template <int N, int LINES, bool COLS> struct CcLayout {
    __device__ __forceinline__ static int nat(int line, int idx) { return COLS ? idx * LINES + line : line * N + idx; }
    __device__ __forceinline__ static int at(int line, int idx) {
        const int x = nat(line, idx);
        const int s = (x >> 4) & 7;
        return COLS ? x ^ (s << 1) : x ^ s ^ (s << 1);
    }
    template <bool NAT> __device__ __forceinline__ static int in(int line, int idx) {
        return NAT ? nat(line, idx) : at(line, idx);
    }
};

template <int R, int DIR> __device__ __forceinline__ void bfly_r(float2* u) {
    if constexpr (R == 2) bfly2<DIR>(u);
    else if constexpr (R == 3) bfly3<DIR>(u);
    else if constexpr (R == 4) bfly4<DIR>(u);
    else if constexpr (R == 5) bfly5<DIR>(u);
    else bfly8<DIR>(u);
}

template <int N, int LINES, bool COLS, int R, int NS, int DIR, int PRE, bool IN_NAT>
__device__ __forceinline__ void cc_stage(const float2* __restrict__ src, float2* __restrict__ dst,
                                         const float2* __restrict__ pre, float scale, const float2* __restrict__ tw,
                                         int tid) {
    constexpr int NT = LINES * N / 8;
    constexpr int M = N / R;
    constexpr int NBF = LINES * M;           // butterflies in the tile
    constexpr int NB = (NBF + NT - 1) / NT;  // rounds
    using L = CcLayout<N, LINES, COLS>;
    tid = opaque(tid);
#pragma unroll
    for (int b = 0; b < NB; ++b) {
        const int bi = tid + NT * b;
        if (NBF % NT != 0 && bi >= NBF) break;
        const int line = COLS ? bi % LINES : bi / M;
        const int j = COLS ? bi / LINES : bi % M;
        const int k = j % NS;
        float2 u[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            float2 v = pre_apply<PRE>(src[L::template in<IN_NAT>(line, j + r * M)], pre, L::nat(line, j + r * M),
                                      scale);
            if constexpr (NS > 1) {
                if (r > 0) {
                    const float2 w = __ldg(tw + k * r * (N / (R * NS)));
                    v = (DIR < 0) ? cmul(v, w) : cmulc(v, w);
                }
            }
            u[r] = v;
        }
        bfly_r<R, DIR>(u);
#pragma unroll
        for (int r = 0; r < R; ++r) dst[L::at(line, (j - k) * R + k + r * NS)] = u[r];
    }
    __syncthreads();
}

// Stages S.. of the plan, alternating a -> b -> a ...; returns the buffer holding the result.
template <int N, int LINES, bool COLS, int DIR, int PRE, bool IN_NAT, int S, int NS>
__device__ __forceinline__ float2* cc_stages_from(float2* __restrict__ a, float2* __restrict__ b,
                                                  const float2* __restrict__ pre, float scale,
                                                  const float2* __restrict__ tw, int tid) {
    constexpr int R = cc_radix(N, S);
    if constexpr (R == 0) {
        return a;
    } else {
        cc_stage<N, LINES, COLS, R, NS, DIR, (S == 0 ? PRE : PRE_NONE), (S == 0 ? IN_NAT : false)>(a, b, pre, scale,
                                                                                                  tw, tid);
        return cc_stages_from<N, LINES, COLS, DIR, PRE, IN_NAT, S + 1, NS * R>(b, a, pre, scale, tw, tid);
    }
}

// The whole line FFT of the tile: input in a (natural layout when IN_NAT, else the working layout), output in the
// returned buffer (a or b) in the working layout CcLayout::at, natural order. DIR < 0 forward, > 0 inverse
// (unnormalised). The caller's block has LINES N / 8 threads; every thread has finished reading b before the call.
template <int N, int LINES, bool COLS, int DIR, int PRE, bool IN_NAT>
__device__ __forceinline__ float2* cc_fft(float2* __restrict__ a, float2* __restrict__ b,
                                          const float2* __restrict__ pre, float scale,
                                          const float2* __restrict__ tw, int tid) {
    static_assert(cc_plannable(N), "float32 shared-memory engine: N = 2^a 3^b 5^c, N % 8 == 0");
    return cc_stages_from<N, LINES, COLS, DIR, PRE, IN_NAT, 0, 1>(a, b, pre, scale, tw, tid);
}

}  // namespace simk
