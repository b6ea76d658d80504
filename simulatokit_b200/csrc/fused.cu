// fused.cu -- the fused, batched form of the multislice step.
//
// One slice of every wave of a batch is two passes over HBM (32 N bytes per probe.slice step):
//   row pass    (along y, contiguous):  [row IFFT] -> x t_j (x scale) -> [row FFT]
//   column pass (along x, stride ny):   column FFT -> x P(dz_j) / N -> column IFFT      (slices 0 .. S-2)
//                                       column FFT -> x P(dz_j)     -> store k-space     (the last slice)
// The probe is generated inside the first column pass (Psi0 . r_x . r_y -> column IFFT) and the detectors read the
// last column pass's k-space wave: FFT2(IFFT2(P Phi)) = P Phi, so |FFT2(exit)|^2 = |P Phi|^2 without two transforms.
//
// Each line transform is register-resident: with E elements per thread and T = n / E threads per line, thread t holds
// elements t + T i (i < E). A Stockham pass of radix R (R | E) then reads its butterfly inputs from the thread's own
// registers, and the last pass writes them back to the same slots, so a transform of P passes exchanges data through
// shared memory P - 1 times. Loads and stores of t + T i are coalesced along rows; columns are read as tiles of TC
// neighbouring columns so that consecutive threads read consecutive addresses.
#include <algorithm>

#include "engine.cuh"
#include "ccfft.cuh"
#include "tc5fft.cuh"
#include "tcfft.cuh"
#include "tma.cuh"

namespace simk {

constexpr int kMaxRegPasses = 12;
// Threads per CTA by elements per thread, so that the register file holds E complex values per thread unspilled.
constexpr int cols_threads(int E) { return E <= 8 ? 1024 : (E <= 12 ? 512 : 256); }
constexpr int rows_threads(int E) { return E <= 12 ? 512 : 256; }

struct RegPlan {
    int n, E, T, npass;
    int fac[kMaxRegPasses];
    const float2* tw;  // n entries e^{-2 pi i k / n}
};

// Shared-memory slot of element idx of a line: rows pad one float2 per 16 (no bank conflicts on the strided
// scatter); column tiles interleave the TC columns of the tile.
struct SmemLine {
    float2* base;
    int stride;  // 1 for rows (padded), TC for column tiles
    __device__ __forceinline__ float2& at(int idx) const {
        return stride == 1 ? base[idx + (idx >> 4)] : base[idx * stride];
    }
};

// ---- one register pass ----------------------------------------------------------------------------------------------
// Butterflies jj = t + T q (q < E/R) on v[q + r E/R]; with `scatter`, the outputs go to their Stockham positions
// (jj - k) R + k + r Ns in shared memory, k = jj mod Ns.
template <int E, int R, int DIR>
__device__ __forceinline__ void reg_pass(float2 (&v)[E], int t, int T, int Ns, int n, const float2* __restrict__ tw,
                                         const SmemLine& sm, bool scatter) {
    constexpr int Q = E / R;
    const int tstride = n / (Ns * R);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        float2 u[R];
#pragma unroll
        for (int r = 0; r < R; ++r) u[r] = v[q + r * Q];
        const int jj = t + T * q;
        const int k = jj % Ns;
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                const float2 w = __ldg(tw + k * r * tstride);
                u[r] = (DIR < 0) ? cmul(u[r], w) : cmulc(u[r], w);
            }
        }
        if (R == 2) bfly2<DIR>(u);
        else if (R == 3) bfly3<DIR>(u);
        else if (R == 4) bfly4<DIR>(u);
        else if (R == 5) bfly5<DIR>(u);
        else if (R == 8) bfly8<DIR>(u);
        else if (R == 16) bfly16<DIR>(u);
        if (scatter) {
            const int o = (jj - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) sm.at(o + r * Ns) = u[r];
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) v[q + r * Q] = u[r];
        }
    }
}

template <int E, int DIR>
__device__ __forceinline__ void reg_pass_any(float2 (&v)[E], int R, int t, int T, int Ns, int n,
                                             const float2* __restrict__ tw, const SmemLine& sm, bool scatter) {
    switch (R) {
        case 2: if constexpr (E % 2 == 0) reg_pass<E, 2, DIR>(v, t, T, Ns, n, tw, sm, scatter); break;
        case 3: if constexpr (E % 3 == 0) reg_pass<E, 3, DIR>(v, t, T, Ns, n, tw, sm, scatter); break;
        case 4: if constexpr (E % 4 == 0) reg_pass<E, 4, DIR>(v, t, T, Ns, n, tw, sm, scatter); break;
        case 5: if constexpr (E % 5 == 0) reg_pass<E, 5, DIR>(v, t, T, Ns, n, tw, sm, scatter); break;
        case 8: if constexpr (E % 8 == 0) reg_pass<E, 8, DIR>(v, t, T, Ns, n, tw, sm, scatter); break;
        case 16: if constexpr (E % 16 == 0) reg_pass<E, 16, DIR>(v, t, T, Ns, n, tw, sm, scatter); break;
        default: break;
    }
}

// The whole transform of one line held as v[i] = x[t + T i]; result in the same layout.
template <int E, int DIR>
__device__ __forceinline__ void reg_fft(float2 (&v)[E], int t, const RegPlan& p, const SmemLine& sm) {
    const int T = p.T;
    int Ns = 1;
    for (int f = 0; f < p.npass; ++f) {
        const int R = p.fac[f];
        const bool scatter = (f + 1 < p.npass);
        reg_pass_any<E, DIR>(v, R, t, T, Ns, p.n, p.tw, sm, scatter);
        if (scatter) {
            __syncthreads();
#pragma unroll
            for (int i = 0; i < E; ++i) v[i] = sm.at(t + T * i);
            __syncthreads();
        }
        Ns *= R;
    }
}

// ---- row pass -------------------------------------------------------------------------------------------------------
// rows r = (wave, ix) of `count` waves; RB rows per CTA (blockDim = (T, RB)).
template <int E>
__global__ void __launch_bounds__(rows_threads(E)) fused_rows_kernel(float2* __restrict__ psi, const float2* __restrict__ tmul,
                                                         RegPlan p, int nx, long long nrows, int inv, int fwd,
                                                         float scale, const float2* const* __restrict__ t_of_wave) {
    extern __shared__ __align__(16) float2 smem_rows[];
    const int t = threadIdx.x;
    const int rr = threadIdx.y;
    const int ny = p.n;
    const int lds = ny + ny / 16 + 1;
    SmemLine sm{smem_rows + rr * lds, 1};
    const long long r = (long long)blockIdx.x * blockDim.y + rr;
    const bool active = r < nrows;
    const long long rc = active ? r : nrows - 1;  // inactive rows recompute the last row and do not store
    float2* row = psi + rc * ny;
    float2 v[E];
#pragma unroll
    for (int i = 0; i < E; ++i) v[i] = row[t + p.T * i];
    if (inv) reg_fft<E, +1>(v, t, p, sm);
    if (tmul || t_of_wave) {
        const int ix = (int)(rc % nx);
        const float2* tr = (t_of_wave ? t_of_wave[rc / nx] : tmul) + (long long)ix * ny;
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = cmul(v[i], __ldg(tr + t + p.T * i)) * scale;
    } else if (scale != 1.0f) {
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = v[i] * scale;
    }
    if (fwd) reg_fft<E, -1>(v, t, p, sm);
    if (active) {
#pragma unroll
        for (int i = 0; i < E; ++i) row[t + p.T * i] = v[i];
    }
}

// ---- column pass ----------------------------------------------------------------------------------------------------
// mode 0: FFT -> x P * pscale -> IFFT;  mode 1: FFT -> x P * pscale (k-space out);  mode 2: probe spectrum -> IFFT.
// blockDim = (TC, T); grid = (ny / TC, count).
struct ColArgs {
    float2* psi;
    const float2* P;
    float pscale;
    int mode;
    int ny;
    const float2* spectrum;
    const float2* rx;
    const float2* ry;
    const int* p_row;  // job tables: wave b uses the propagator P + p_row[b] N (null: every wave uses P)
    int p_blocks;      // job tables: propagators stacked at P (for the tensor map)
    FusedDetect det;   // mode 3: detection in the epilogue
    int* det_groups;   // mode 3: receives the column groups of the partial sums (the launch's ny / TC)
};

// The propagator of wave b.
__device__ __forceinline__ const float2* col_P(const ColArgs& a, long long b, long long N) {
    return a.p_row ? a.P + (long long)a.p_row[b] * N : a.P;
}

template <int E>
__global__ void __launch_bounds__(cols_threads(E)) fused_cols_kernel(ColArgs a, RegPlan p) {
    extern __shared__ __align__(16) float2 smem_cols[];
    const int c = threadIdx.x, TC = blockDim.x;
    const int t = threadIdx.y;
    const int nx = p.n, ny = a.ny;
    const int iy = blockIdx.x * TC + c;
    const long long b = blockIdx.y;
    const long long N = (long long)nx * ny;
    SmemLine sm{smem_cols + c, TC};
    float2* col = a.psi + b * N + iy;
    float2 v[E];
    if (a.mode == 2) {
        const float2 ryv = a.ry[b * ny + iy];
#pragma unroll
        for (int i = 0; i < E; ++i) {
            const int ix = t + p.T * i;
            v[i] = cmul(cmul(__ldg(a.spectrum + (long long)ix * ny + iy), __ldg(a.rx + b * nx + ix)), ryv);
        }
        reg_fft<E, +1>(v, t, p, sm);
    } else {
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = col[(long long)(t + p.T * i) * ny];
        reg_fft<E, -1>(v, t, p, sm);
        const float2* P = col_P(a, b, N);
#pragma unroll
        for (int i = 0; i < E; ++i) v[i] = cmul(v[i], __ldg(P + (long long)(t + p.T * i) * ny + iy)) * a.pscale;
        if (a.mode == 0) reg_fft<E, +1>(v, t, p, sm);
    }
#pragma unroll
    for (int i = 0; i < E; ++i) col[(long long)(t + p.T * i) * ny] = v[i];
}

// ---- compile-time plans for n = 2^L -----------------------------------------------------------------------------------
// E = 8 elements per thread, T = n / 8 threads per line, radix-8 passes then one radix-2 or radix-4 pass when L is not a
// multiple of 3. Every Ns, twiddle stride and shared-memory offset is a compile-time constant, each thread's twiddles
// (the same for every transform it runs) are loaded once into registers, and shared memory is addressed through the
// swizzle idx ^ ((idx >> 3) & 15), which makes every scatter and gather of these plans free of bank conflicts.
constexpr int ct_log2(int n) { return n <= 1 ? 0 : 1 + ct_log2(n / 2); }
template <int N> struct Pow2 {
    static constexpr int L = ct_log2(N);
    static constexpr int T = N / 8;
    static constexpr int NP = (L + 2) / 3;
    static constexpr int radix(int f) { return (f < L / 3) ? 8 : (1 << (L % 3)); }
    static constexpr int ns(int f) { return f == 0 ? 1 : ns(f - 1) * radix(f - 1); }
};

__device__ __forceinline__ int swz(int idx) { return idx ^ ((idx >> 3) & 15); }

// Element idx of a line in shared memory: rows (STRIDE 0) contiguous, column tiles interleave STRIDE columns.
template <int STRIDE> struct SmemCT {
    float2* base;
    __device__ __forceinline__ float2& at(int idx) const {
        if constexpr (STRIDE == 0) return base[swz(idx)];
        else return base[swz(idx) * STRIDE];
    }
    // the slot of an index already swizzled
    __device__ __forceinline__ float2& slot(int s) const {
        if constexpr (STRIDE == 0) return base[s];
        else return base[s * STRIDE];
    }
};

// Per-thread twiddles: pass f >= 1 uses w[f - 1][q (R - 1) + r - 1] = W_n^{k r n / (Ns R)}, k = (t + T q) mod Ns.
template <int N> struct TwRegs {
    float2 w[Pow2<N>::NP > 1 ? Pow2<N>::NP - 1 : 1][7];
};

// `tw` holds W_{N S}^m (S > 1: the table of a length that N divides; W_N^m = W_{N S}^{m S}).
template <int N, int F, int S = 1>
__device__ __forceinline__ void tw_load(TwRegs<N>& tr, unsigned t, const float2* __restrict__ tw) {
    using P = Pow2<N>;
    if constexpr (F < P::NP) {
        constexpr int R = P::radix(F), NS = P::ns(F), Q = 8 / R, TSTRIDE = N / (NS * R);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const unsigned k = (t + P::T * q) & (NS - 1);
#pragma unroll
            for (int r = 1; r < R; ++r) tr.w[F - 1][q * (R - 1) + r - 1] = __ldg(tw + k * (r * TSTRIDE) * S);
        }
        tw_load<N, F + 1, S>(tr, t, tw);
    }
}

// The barrier of one line's exchange: the whole block (LT = 0), or only the LT threads of the line (whole warps, from
// warp 32 (id - 1) / ... on): one warp needs no barrier beyond __syncwarp; more use the named barrier `id` (1-15).
template <int LT>
__device__ __forceinline__ void line_sync(int id) {
    if constexpr (LT == 0) __syncthreads();
    else if constexpr (LT == 32) __syncwarp();
    else asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(LT) : "memory");
}

template <int N, int F, int DIR, int STRIDE, int LT = 0>
__device__ __forceinline__ void ct_fft_from(float2 (&v)[8], unsigned t, const TwRegs<N>& tr,
                                            const SmemCT<STRIDE>& sm, int bar_id = 0) {
    using P = Pow2<N>;
    if constexpr (F < P::NP) {
        constexpr int R = P::radix(F), NS = P::ns(F), Q = 8 / R;
        constexpr bool SC = (F + 1 < P::NP);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            float2 u[R];
#pragma unroll
            for (int r = 0; r < R; ++r) u[r] = v[q + r * Q];
            if constexpr (F > 0) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    const float2 w = tr.w[F - 1][q * (R - 1) + r - 1];
                    u[r] = (DIR < 0) ? cmul(u[r], w) : cmulc(u[r], w);
                }
            }
            if constexpr (R == 2) bfly2<DIR>(u);
            else if constexpr (R == 4) bfly4<DIR>(u);
            else bfly8<DIR>(u);
            if constexpr (SC) {
                const int jj = (int)t + P::T * q;
                const int k = jj & (NS - 1);
                const int o = (jj - k) * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) sm.at(o + r * NS) = u[r];
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) v[q + r * Q] = u[r];
            }
        }
        if constexpr (SC) {
            line_sync<LT>(bar_id);
            // swz(t + T i) = (a ^ c_i) + T i with a = t ^ ((t >> 3) mod 16) per thread and c_i = (T / 8) i mod 16 a
            // constant of the unrolled loop (the carries of t + T i never reach the bits the swizzle flips): each
            // gather address is one of at most 16 / (T / 8) per-thread bases plus an immediate offset
            const int a = (int)t ^ (((int)t >> 3) & 15);
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = sm.slot((a ^ (((P::T >> 3) * i) & 15)) + P::T * i);
            line_sync<LT>(bar_id);
        }
        ct_fft_from<N, F + 1, DIR, STRIDE, LT>(v, t, tr, sm, bar_id);
    }
}

// ---- column pairs (engine 5): one thread transforms the same rows of two adjacent columns -----------------------------
// Thread (c, t) of a column tile eight columns wide holds columns 2c and 2c + 1 of rows t + T i: every load and store of
// the tile moves both as one 16-byte access, and the exchanges keep the pair together in one float4 slot. Pair c's
// exchange region is N float4 slots, slot s at swz(s) ^ 2c: a quarter warp (two t, four c) then reaches eight
// different 16-byte bank groups in every scatter and gather of these plans (bit 0 of the swizzled slot tells the two t
// apart, 2c the four pairs). The twiddles depend on t only, so both columns share them. `after_first_sync` runs right
// after the first barrier of the transform (by then every thread has finished what preceded the transform).
template <int N, int F, int DIR, typename Hook>
__device__ __forceinline__ void ct2_fft_from(float2 (&v0)[8], float2 (&v1)[8], unsigned t, const TwRegs<N>& tr,
                                             float4* __restrict__ region, int xc, Hook&& after_first_sync) {
    using P = Pow2<N>;
    if constexpr (F < P::NP) {
        constexpr int R = P::radix(F), NS = P::ns(F), Q = 8 / R;
        constexpr bool SC = (F + 1 < P::NP);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            float2 a[R], b[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                a[r] = v0[q + r * Q];
                b[r] = v1[q + r * Q];
            }
            if constexpr (F > 0) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    const float2 w = tr.w[F - 1][q * (R - 1) + r - 1];
                    a[r] = (DIR < 0) ? cmul(a[r], w) : cmulc(a[r], w);
                    b[r] = (DIR < 0) ? cmul(b[r], w) : cmulc(b[r], w);
                }
            }
            if constexpr (R == 2) {
                bfly2<DIR>(a);
                bfly2<DIR>(b);
            } else if constexpr (R == 4) {
                bfly4<DIR>(a);
                bfly4<DIR>(b);
            } else {
                bfly8<DIR>(a);
                bfly8<DIR>(b);
            }
            if constexpr (SC) {
                const int jj = (int)t + P::T * q;
                const int k = jj & (NS - 1);
                const int o = (jj - k) * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) region[swz(o + r * NS) ^ xc] = make_float4(a[r].x, a[r].y, b[r].x, b[r].y);
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    v0[q + r * Q] = a[r];
                    v1[q + r * Q] = b[r];
                }
            }
        }
        if constexpr (SC) {
            __syncthreads();
            if constexpr (F == 0) after_first_sync();
            // as in ct_fft_from: swz(t + T i) ^ xc = (a ^ c_i) + T i with the per-thread a = swz(t) ^ xc (xc < 8 and
            // swz(t) < T leave T i's bits alone)
            const int a0 = ((int)t ^ (((int)t >> 3) & 15)) ^ xc;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const float4 x = region[(a0 ^ (((P::T >> 3) * i) & 15)) + P::T * i];
                v0[i] = make_float2(x.x, x.y);
                v1[i] = make_float2(x.z, x.w);
            }
            __syncthreads();
        }
        ct2_fft_from<N, F + 1, DIR>(v0, v1, t, tr, region, xc, after_first_sync);
    }
}

// ---- composite lengths N = R M (R = 3 or 5, M a power of two >= 64): the register engine on R sub-lines ---------------
// A line's N / 8 threads form R sub-lines of TS = M / 8 threads; thread (g, u) is sub-line g, thread u. Decimation in
// frequency from natural order (comp_dif_in, then the M-point register transform of each sub-line):
//     X[R k1 + g] = sum_{n1} W_M^{n1 k1} y_g[n1],   y_g[n1] = W_N^{n1 g} sum_{n2} x[n1 + M n2] W_R^{n2 g},
// so thread (g, u) ends with X[R (u + TS i) + g] in v[i]. Decimation in time back to natural order: the M-point
// transform of X[R . + g] (v in that order), w_g[n1] = W_N^{n1 g} z_g[n1] into an exchange tile (comp_dit_twiddle),
// and after the line's barrier x[n1 + M g] = sum_{k2} W_R^{g k2} w_{k2}[n1] (comp_dit_out). Every W is taken in the
// transform's direction; the R-point sums are the butterflies of fft.cuh with output g selected.
template <int N> struct CompPlan {
    static constexpr int R = (N % 3 == 0) ? 3 : 5;
    static constexpr int M = N / R;
    static constexpr int TS = M / 8;
};
constexpr bool comp_length(int n) {
    for (int r : {3, 5}) {
        if (n % r) continue;
        const int m = n / r;
        if (m >= 64 && (m & (m - 1)) == 0) return true;
    }
    return false;
}
template <int R, int DIR> __device__ __forceinline__ float2 comp_dft_out(float2 (&x)[R], int g) {
    if constexpr (R == 3) bfly3<DIR>(x);
    else bfly5<DIR>(x);
    float2 y = x[0];
#pragma unroll
    for (int r = 1; r < R; ++r)
        if (g == r) y = x[r];
    return y;
}
// ld(idx): element idx of the line in natural order; tw: the N-entry table W_N^m.
template <int N, int DIR, typename Ld>
__device__ __forceinline__ void comp_dif_in(float2 (&v)[8], int g, int u, const float2* __restrict__ tw, Ld&& ld) {
    using C = CompPlan<N>;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int n1 = u + C::TS * i;
        float2 x[C::R];
#pragma unroll
        for (int r = 0; r < C::R; ++r) x[r] = ld(n1 + C::M * r);
        const float2 y = comp_dft_out<C::R, DIR>(x, g);
        const float2 w = __ldg(tw + n1 * g);  // n1 g < M R = N
        v[i] = (DIR < 0) ? cmul(y, w) : cmulc(y, w);
        // keeps the next point's loads after this one: hoisting all R * 8 loads spills under the register cap
        asm volatile("" ::: "memory");
    }
}
// st(slot, value): slot g M + n1 of the exchange tile.
template <int N, int DIR, typename St>
__device__ __forceinline__ void comp_dit_twiddle(const float2 (&v)[8], int g, int u, const float2* __restrict__ tw,
                                                 St&& st) {
    using C = CompPlan<N>;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int n1 = u + C::TS * i;
        const float2 w = __ldg(tw + n1 * g);
        st(g * C::M + n1, (DIR < 0) ? cmul(v[i], w) : cmulc(v[i], w));
    }
}
// ld(slot): slot k2 M + n1 of the exchange tile; v[i] = x[u + TS i + M g].
template <int N, int DIR, typename Ld>
__device__ __forceinline__ void comp_dit_out(float2 (&v)[8], int g, int u, Ld&& ld) {
    using C = CompPlan<N>;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int n1 = u + C::TS * i;
        float2 x[C::R];
#pragma unroll
        for (int r = 0; r < C::R; ++r) x[r] = ld(r * C::M + n1);
        v[i] = comp_dft_out<C::R, DIR>(x, g);
        asm volatile("" ::: "memory");  // as in comp_dif_in
    }
}

// rows: blockDim = (N / 8, RB); row r = (wave, ix) of nrows = count * nx
template <int N>
__global__ void __launch_bounds__(256) fused_rows_ct(float2* __restrict__ psi, const float2* __restrict__ tmul,
                                                     const float2* __restrict__ tw, unsigned nx, unsigned nrows,
                                                     int inv, int fwd, float scale,
                                                     const float2* const* __restrict__ t_of_wave) {
    extern __shared__ __align__(16) float2 smem_rows_ct[];
    constexpr int T = N / 8;
    const unsigned t = threadIdx.x;
    const unsigned r = blockIdx.x * blockDim.y + threadIdx.y;
    const bool active = r < nrows;
    const unsigned rc = active ? r : nrows - 1;  // inactive rows recompute the last row and do not store
    SmemCT<0> sm{smem_rows_ct + threadIdx.y * N};
    TwRegs<N> tr;
    tw_load<N, 1>(tr, t, tw);
    float2* row = psi + (size_t)rc * N;
    float2 v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = row[t + T * i];
    if (inv) ct_fft_from<N, 0, +1>(v, t, tr, sm);
    if (tmul || t_of_wave) {
        const float2* trow = (t_of_wave ? t_of_wave[rc / nx] : tmul) + (size_t)(rc % nx) * N;
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = cmul(v[i], __ldg(trow + t + T * i)) * scale;
    } else if (scale != 1.0f) {
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = v[i] * scale;
    }
    if (fwd) ct_fft_from<N, 0, -1>(v, t, tr, sm);
    if (active) {
#pragma unroll
        for (int i = 0; i < 8; ++i) row[t + T * i] = v[i];
    }
}

// columns: blockDim = (TC, N / 8), grid = (ny / TC, count). MODE 0: FFT -> x P pscale -> IFFT; 1: FFT -> x P pscale;
// 2: probe spectrum Psi0 r_x r_y -> IFFT.
template <int N, int TC, int MODE>
__global__ void __launch_bounds__(TC * (N / 8)) fused_cols_ct(ColArgs a, const float2* __restrict__ tw) {
    extern __shared__ __align__(16) float2 smem_cols_ct[];
    constexpr int T = N / 8;
    const int c = threadIdx.x;
    const unsigned t = threadIdx.y;
    const int ny = a.ny;
    const int iy = blockIdx.x * TC + c;
    const size_t b = blockIdx.y;
    SmemCT<TC> sm{smem_cols_ct + c};
    TwRegs<N> tr;
    tw_load<N, 1>(tr, t, tw);
    float2* col = a.psi + b * (size_t)N * ny + iy;
    float2 v[8];
    if constexpr (MODE == 2) {
        const float2 ryv = a.ry[b * ny + iy];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int ix = (int)t + T * i;
            v[i] = cmul(cmul(__ldg(a.spectrum + (size_t)ix * ny + iy), __ldg(a.rx + b * N + ix)), ryv);
        }
        ct_fft_from<N, 0, +1>(v, t, tr, sm);
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = col[(size_t)(t + T * i) * ny];
        ct_fft_from<N, 0, -1>(v, t, tr, sm);
        const float2* P = col_P(a, (long long)b, (long long)N * ny);
#pragma unroll
        for (int i = 0; i < 8; ++i) v[i] = cmul(v[i], __ldg(P + (size_t)(t + T * i) * ny + iy)) * a.pscale;
        if constexpr (MODE == 0) ct_fft_from<N, 0, +1>(v, t, tr, sm);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) col[(size_t)(t + T * i) * ny] = v[i];
}

// ---- detection in the last column pass's epilogue ----------------------------------------------------------------------
// MODE 3 of the column pass: FFT -> x P as MODE 1, then every channel detector (annular, centre of mass, segmented) is
// summed from the finished tile while it is still in shared memory, so the k-space wave need not be written and read
// back (it is stored only when pixelated or binned detectors want it). Per (wave, column group, channel) one float64
// partial: each thread sums its strided share of the group's entries in order, the warp reduces with shuffles, the
// warps' sums are added in warp order; k_detect_fold then adds the groups in order. Fixed order throughout, so scans
// stay bit-deterministic.
struct DetectArgs {
    const int* ptr;    // [groups C + 1]
    const int2* ent;   // (local index ix TC + c, weight bits)
    double* partial;   // [wave][groups][C]
    int n_ch;          // C
    int groups;        // ny / TC
    int store;         // also store the k-space tile
};

// `tile`: the finished tile of wave b, column group g, natural [row][TC] layout; `red`: NT / 32 * C doubles of free
// shared memory. Ends with the partials written; the caller's barrier must follow before `red` or `tile` is reused.
template <int NT>
__device__ __forceinline__ void detect_tile(const float2* __restrict__ tile, const DetectArgs& d, int b, int g, int tid,
                                            double* __restrict__ red) {
    constexpr int NW = NT / 32;
    const int lane = tid & 31, warp = tid >> 5;
    const int* ptr = d.ptr + (size_t)g * d.n_ch;
    for (int ch = 0; ch < d.n_ch; ++ch) {
        const int e1 = __ldg(ptr + ch + 1);
        double sum = 0.0;
        for (int e = __ldg(ptr + ch) + tid; e < e1; e += NT) {
            const int2 q = __ldg(d.ent + e);
            const float2 v = tile[q.x];
            sum += (double)((v.x * v.x + v.y * v.y) * __int_as_float(q.y));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) red[ch * NW + warp] = sum;
    }
    __syncthreads();
    for (int ch = tid; ch < d.n_ch; ch += NT) {
        double t = 0.0;
        for (int w = 0; w < NW; ++w) t += red[ch * NW + w];
        d.partial[((size_t)b * d.groups + g) * d.n_ch + ch] = t;
    }
}

// ---- the persistent TMA-pipelined passes (power-of-two lengths) --------------------------------------------------------
// Each CTA walks its tiles blockIdx.x, blockIdx.x + gridDim.x, ...: thread 0 starts the asynchronous copies of the
// next tile (the waves and the matching rows of t or P) into the other shared-memory stage before the CTA transforms
// the current one, so copies overlap arithmetic and no global load sits inside a transform. The wave part of a stage
// doubles as the transform's exchange buffer once it has been read. A wait that runs out sets *err, waits (bounded)
// for the copy it started and makes the whole CTA return.

// Thread 0: wait for stage s, phase (it >> 1) & 1; on timeout record it and drain the other stage's copy.
__device__ __forceinline__ void stage_wait(uint64_t* full, int s, int it, bool next_issued, int* err, int* abort_flag) {
    if (!mbar_wait_bounded(&full[s], (uint32_t)((it >> 1) & 1))) {
        atomicExch(err, 1);
        *abort_flag = 1;
        if (next_issued) mbar_wait_bounded(&full[s ^ 1], (uint32_t)(((it + 1) >> 1) & 1));
    }
}

// columns: tile = (wave b, TC columns from iy0); a stage holds the wave tile and the P tile, N x TC each (engine 5:
// the wave tile only, beside one P buffer).
// Engines: 0 register-resident float32 Cooley-Tukey passes (powers of two); 1 radix-16 stages as mma.sync products of
// split-BF16 operands on a shared-memory tile (tcfft.cuh, the bf16x3 form); 2 float32 shared-memory Stockham
// (ccfft.cuh); 3 radix-16 stages as tcgen05.mma products (tc5fft.cuh, the bf16x3 form at 256 and 512); 4 the composite
// register engine (lengths 3 or 5 times a power of two: R sub-lines of engine 0); 5 engine 0 on column pairs (8- or
// 16-column tiles, two adjacent columns a thread; MODE 2 there generates the probes from their spectrum).
// Height of the column pass's TMA boxes: the largest divisor of N that is at most 256 (the box limit).
constexpr int tma_box_rows(int n) {
    for (int h = 256; h > 1; --h)
        if (n % h == 0) return h;
    return 1;
}
// Rows per tile of the row pass: the largest power of two with RB N / 8 <= max_threads (256; 384 for the composite
// engine, whose row blocks then match its two 384-thread column blocks an SM).
constexpr int rows_per_tile(int n, int max_threads = 256) {
    int r = 1;
    while (2 * r * (n / 8) <= max_threads) r *= 2;
    return r;
}
constexpr int rows_tile(int n, int eng) { return rows_per_tile(n, eng == 4 ? 384 : 256); }

// State an engine keeps per thread: register twiddles (0, 5), the DFT-16 fragments (1), nothing (2), the tcgen05 block
// state (3), the sub-lines' register twiddles (4).
template <int N, int ENG>
using EngineState = std::conditional_t<
    ENG == 0 || ENG == 5, TwRegs<N>,
    std::conditional_t<ENG == 1, Dft16Frags,
                       std::conditional_t<ENG == 3, Tc5, std::conditional_t<ENG == 4, TwRegs<CompPlan<N>::M>, int>>>>;

// The tcgen05 engine (3) takes lines of 256 and 512 points in tiles of whole 128-vector blocks.
constexpr bool tc5_tile(int n, int lines) { return (n == 256 || n == 512) && (n * lines) % 2048 == 0; }
constexpr int tc5_blocks(int n, int lines) { return n * lines / 2048; }

// Engine 3's set-up, by every thread of the block: tensor memory (warp 0), the B matrices, the MMA barrier.
template <int MB>
__device__ __forceinline__ Tc5 tc5_setup(uint8_t* area, uint32_t* tmem_slot, uint64_t* mma_bar, int tid, int nthreads,
                                         int stack) {
    if (tid < 32) tmem_alloc(tmem_slot, tc5_tmem_cols(MB, stack != 0));
    tc5_build_b(area + (size_t)MB * 3 * kTc5Plane, tid, nthreads);
    if (tid == 0) {
        mbar_init(mma_bar, 1);
        fence_barrier_init();
    }
    fence_proxy_async_shared();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    Tc5 c;
    c.a_ptr = area;
    c.a_base = smem_u32(area);
    c.b_base = c.a_base + (uint32_t)MB * 3u * kTc5Plane;
    c.tmem = *tmem_slot;
    c.bar = mma_bar;
    c.phase = 0;
    c.stack = stack;
    return c;
}

// Engine 3's release: after every thread's last tensor-memory access (and, when a wait ran out, one more bounded
// wait for the products in flight), warp 0 frees the columns.
template <int MB>
__device__ __forceinline__ void tc5_release(const Tc5& c, int tid, bool aborted) {
    tc_fence_before();
    __syncthreads();
    if (aborted && tid == 0) mbar_wait_bounded(c.bar, c.phase ^ 1u, kTc5WaitPolls);
    __syncthreads();
    if (tid < 32) {
        tc_fence_after();
        tmem_dealloc(c.tmem, tc5_tmem_cols(MB, c.stack != 0));
    }
}

// Blocks per SM the engines ask the compiler for. The tensor-core engine: two when a block has at most 256 threads
// (at most 128 registers a thread). The float32 register engine: three for its 256-thread blocks (at most 85
// registers; 512^2 fits without spills and gains a third block per SM). The float32 shared-memory engine keeps the
// compiler's choice (capped at 84 registers it spilled and lost 12 % at 768^2). The composite-length register engine:
// two blocks of up to 384 threads (80 registers; the 768^2 column pass spills 84 bytes and is still the fastest
// choice measured, 0.86 ms a launch against 0.90 ms for one block at 168 registers), three of up to 256 threads (112
// registers: the row pass spilled 240 bytes at four blocks and 80 registers and ran 6 % slower).
constexpr int tc_min_blocks(int threads, int eng) {
    if (eng == 1 || eng == 3) return threads <= 256 ? 2 : 1;
    if (eng == 0) return threads == 256 ? 3 : 1;
    if (eng == 4) return threads <= 256 ? 3 : (threads <= 384 ? 2 : 1);
    if (eng == 5) return threads <= 256 ? 2 : 1;
    return 1;
}
// Threads across a column tile: one per column, or one per column pair (engine 5).
constexpr int cols_tx(int tc, int eng) { return eng == 5 ? tc / 2 : tc; }

template <int N, int TC, int MODE, int ENG>
__global__ void __launch_bounds__(cols_tx(TC, ENG) * (N / 8), tc_min_blocks(cols_tx(TC, ENG) * (N / 8), ENG))
    fused_cols_tma(const __grid_constant__ CUtensorMap map,
                                                               const __grid_constant__ CUtensorMap pmap,
                                                               float2* __restrict__ psi, float pscale, int ny,
                                                               int count, const float2* __restrict__ tw, int* err,
                                                               const int* __restrict__ p_row, const DetectArgs det,
                                                               int tc5_stack, const float2* __restrict__ rx,
                                                               const float2* __restrict__ ry) {
    extern __shared__ __align__(128) unsigned char smem_tma[];
    constexpr int T = N / 8;
    constexpr int BOXH = tma_box_rows(N);
    constexpr int NBOX = N / BOXH;
    constexpr int TILE = N * TC;  // float2 per tile
    // engine 5: a stage holds only the wave tile and the P tile has one buffer of its own (refilled for the next tile
    // once the multiply is done), so that two CTAs of eight-column tiles fit an SM
    constexpr bool PSEP = (ENG == 5);
    constexpr int TX = cols_tx(TC, ENG);
    constexpr int SST = (PSEP ? 1 : 2) * TILE;  // float2 per stage
    constexpr uint32_t STAGE_BYTES = (uint32_t)SST * sizeof(float2);
    __shared__ __align__(8) uint64_t full[2];
    __shared__ __align__(8) uint64_t pfull;
    __shared__ int abort_flag;
    __shared__ uint32_t tmem_slot;
    __shared__ __align__(8) uint64_t mma_bar;
    __shared__ double red5[PSEP && MODE == 3 ? TX * T / 32 * 64 : 1];  // engine 5's detector sums (C <= 64)
    float2* stages = reinterpret_cast<float2*>(smem_tma);
    [[maybe_unused]] float2* const ptile = stages + 2 * SST;  // engine 5's P tile (the spectrum's in MODE 2)
    const int c = threadIdx.x;
    const unsigned t = threadIdx.y;
    const int tid = (int)t * TX + c;
    const unsigned tiles_per_wave = (unsigned)(ny / TC);
    const unsigned ntiles = (unsigned)count * tiles_per_wave;  // < 2^31: checked by the launcher
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        mbar_init(&pfull, 1);
        fence_barrier_init();
        abort_flag = 0;
    }
    __syncthreads();
    [[maybe_unused]] EngineState<N, ENG> eng;
    if constexpr (ENG == 0 || ENG == 5) tw_load<N, 1>(eng, t, tw);
    else if constexpr (ENG == 4) tw_load<CompPlan<N>::M, 1, CompPlan<N>::R>(eng, t % CompPlan<N>::TS, tw);
    else if constexpr (ENG == 1) eng = dft16_frags(tid & 31);
    else if constexpr (ENG == 3)
        eng = tc5_setup<tc5_blocks(N, TC)>(smem_tma + 4 * (size_t)TILE * sizeof(float2), &tmem_slot, &mma_bar, tid,
                                           TC * T, tc5_stack);
    auto issue = [&](unsigned tile, int s) {
        const int b = (int)(tile / tiles_per_wave);
        const int iy0 = (int)(tile - (unsigned)b * tiles_per_wave) * TC;
        float2* dst = stages + s * SST;
        const int prow = p_row ? p_row[b] * N : 0;  // job tables: this wave's propagator among the stacked ones
        if constexpr (MODE == 2) {
            mbar_arrive_expect_tx(&full[s], 0);  // probes: no wave to load, the phase completes at once
            return;
        }
        mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
#pragma unroll
        for (int k = 0; k < NBOX; ++k) {
            tma_load_2d(dst + k * BOXH * TC, &map, &full[s], 2 * iy0, b * N + k * BOXH);
            if constexpr (!PSEP) tma_load_2d(dst + TILE + k * BOXH * TC, &pmap, &full[s], 2 * iy0, prow + k * BOXH);
        }
    };
    // engine 5: the P tile of `tile` into its own buffer, completing on pfull (one phase per tile)
    [[maybe_unused]] auto issue_p = [&](unsigned tile) {
        const int b = (int)(tile / tiles_per_wave);
        const int iy0 = (int)(tile - (unsigned)b * tiles_per_wave) * TC;
        const int prow = (MODE != 2 && p_row) ? p_row[b] * N : 0;
        mbar_arrive_expect_tx(&pfull, (uint32_t)TILE * sizeof(float2));
#pragma unroll
        for (int k = 0; k < NBOX; ++k) tma_load_2d(ptile + k * BOXH * TC, &pmap, &pfull, 2 * iy0, prow + k * BOXH);
    };
    unsigned tile = blockIdx.x;
    if (tid == 0 && tile < ntiles) {
        issue(tile, 0);
        if constexpr (PSEP) issue_p(tile);
    }
    for (int it = 0; tile < ntiles; tile += gridDim.x, ++it) {
        const int s = it & 1;
        float2* buf = stages + s * SST;
        const float2* pbuf = PSEP ? ptile : buf + TILE;
        const unsigned next = tile + gridDim.x;
        if (tid == 0) {
            // the previous tile's TMA store must have read its shared-memory source (a stage or the scratch tile)
            // before the next copy into a stage and before this tile's transforms write the scratch tile; after an
            // abandoned tile no further copy starts, and the one in flight is waited for
            bulk_wait_read();
            const bool more = !abort_flag && next < ntiles;
            if (more) issue(next, s ^ 1);
            stage_wait(full, s, it, more, err, &abort_flag);
            if constexpr (PSEP) {
                // this tile's P, issued at the start or once the previous tile's multiply was done; waited for after
                // an abandoned wave copy too, so that no copy is in flight when the block leaves
                if (!mbar_wait_bounded(&pfull, (uint32_t)(it & 1))) {
                    atomicExch(err, 1);
                    if (!abort_flag && more) mbar_wait_bounded(&full[s ^ 1], (uint32_t)(((it + 1) >> 1) & 1));
                    abort_flag = 1;
                }
            }
        }
        __syncthreads();
        if (abort_flag) break;
        const int b = (int)(tile / tiles_per_wave);
        const int iy = (int)(tile - (unsigned)b * tiles_per_wave) * TC + c;
        const float2* store_src = buf;  // where the finished tile lies in its natural layout
        if constexpr (ENG == 0) {
            float2 v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = buf[(t + T * i) * TC + c];
            __syncthreads();  // the wave tile has been read: it becomes the exchange buffer
            SmemCT<TC> sm{buf + c};
            ct_fft_from<N, 0, -1>(v, t, eng, sm);
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = cmul(v[i], pbuf[(t + T * i) * TC + c]) * pscale;
            if constexpr (MODE == 0) ct_fft_from<N, 0, +1>(v, t, eng, sm);
            // back into the stage tile in its natural [row][TC] layout (every exchange read is behind a barrier);
            // thread 0 stores the tile with TMA after the barrier below
#pragma unroll
            for (int i = 0; i < 8; ++i) buf[(t + T * i) * TC + c] = v[i];
            store_src = buf;
        } else if constexpr (ENG == 5) {
            // column pairs: thread (c, t) holds columns 2c, 2c + 1 of rows t + T i (one 16-byte access per row)
            static_assert(TX == 4 || TX == 8, "column pairs: four or eight pairs a tile");
            float4* const tile4 = reinterpret_cast<float4*>(buf);
            const float4* const p4 = reinterpret_cast<const float4*>(pbuf);
            float4* const region = tile4 + c * N;
            // the slot XOR that spreads a quarter warp (two t and four pairs, or one t and eight) over the bank groups
            const int xc = (TX == 4) ? 2 * c : c;
            // behind the first barrier of the transform that follows the last read of the P buffer, every thread has
            // read it: the next tile's P (or spectrum) may come
            auto next_p = [&] {
                if (tid == 0 && !abort_flag && next < ntiles) issue_p(next);
            };
            float2 v0[8], v1[8];
            if constexpr (MODE == 2) {
                // probes: the spectrum tile (in the P buffer) times the shift ramps r_x[ix] r_y[iy] of wave b, then the
                // inverse transform; nothing is read from the stage
                const int col = iy + c;  // iy - c + 2 c: the pair's first column
                const float2 ry0 = __ldg(ry + (size_t)b * ny + col), ry1 = __ldg(ry + (size_t)b * ny + col + 1);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int ix = (int)t + T * i;
                    const float4 sp = p4[ix * TX + c];
                    const float2 r = __ldg(rx + (size_t)b * N + ix);
                    v0[i] = cmul(cmul(make_float2(sp.x, sp.y), r), ry0);
                    v1[i] = cmul(cmul(make_float2(sp.z, sp.w), r), ry1);
                }
                ct2_fft_from<N, 0, +1>(v0, v1, t, eng, region, xc, next_p);
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float4 x = tile4[(t + T * i) * TX + c];
                    v0[i] = make_float2(x.x, x.y);
                    v1[i] = make_float2(x.z, x.w);
                }
                __syncthreads();  // the wave tile has been read: it becomes the pairs' exchange regions
                ct2_fft_from<N, 0, -1>(v0, v1, t, eng, region, xc, [] {});
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float4 pp = p4[(t + T * i) * TX + c];
                    v0[i] = cmul(v0[i], make_float2(pp.x, pp.y)) * pscale;
                    v1[i] = cmul(v1[i], make_float2(pp.z, pp.w)) * pscale;
                }
                if constexpr (MODE == 0) ct2_fft_from<N, 0, +1>(v0, v1, t, eng, region, xc, next_p);
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
                tile4[(t + T * i) * TX + c] = make_float4(v0[i].x, v0[i].y, v1[i].x, v1[i].y);
            store_src = buf;
        } else if constexpr (ENG == 4) {
            // composite length: R sub-lines of TS threads per column; a sub-line's exchanges use its own part of the
            // wave tile and synchronise the TC TS threads of sub-line g (whole warps: threads t = TS g .. of every
            // column), with the named barrier 1 + g
            using C = CompPlan<N>;
            const int g = (int)t / C::TS, u = (int)t % C::TS;
            float2 v[8];
            comp_dif_in<N, -1>(v, g, u, tw, [&](int idx) { return buf[idx * TC + c]; });
            __syncthreads();  // every sub-line has read the wave tile: its parts become the exchange buffers
            const SmemCT<TC> sm{buf + g * C::M * TC + c};
            ct_fft_from<C::M, 0, -1, TC, C::TS * TC>(v, (unsigned)u, eng, sm, 1 + g);
            float2* out = buf + TILE;  // the P tile takes the result once every thread has multiplied by it
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int idx = C::R * (u + C::TS * i) + g;  // v[i] = X[idx]
                v[i] = cmul(v[i], pbuf[idx * TC + c]) * pscale;
                if constexpr (MODE != 0) out[idx * TC + c] = v[i];  // each slot is read and written by its thread
            }
            if constexpr (MODE == 0) {
                ct_fft_from<C::M, 0, +1, TC, C::TS * TC>(v, (unsigned)u, eng, sm, 1 + g);
                comp_dit_twiddle<N, +1>(v, g, u, tw, [&](int slot, float2 x) { buf[slot * TC + c] = x; });
                __syncthreads();  // the sub-lines' twiddled transforms are in the wave tile; P has been read
                comp_dit_out<N, +1>(v, g, u, [&](int slot) { return buf[slot * TC + c]; });
#pragma unroll
                for (int i = 0; i < 8; ++i) out[(u + C::TS * i + C::M * g) * TC + c] = v[i];
            }
            store_src = out;
        } else if constexpr (ENG == 2) {
            using L = CcLayout<N, TC, true>;
            float2* scratch = stages + 4 * TILE;
            float2* out = cc_fft<N, TC, true, -1, PRE_NONE, true>(buf, scratch, nullptr, 1.0f, tw, tid);
            if constexpr (MODE == 0) {
                float2* other = (out == buf) ? scratch : buf;
                out = cc_fft<N, TC, true, +1, PRE_MUL, false>(out, other, pbuf, pscale, tw, tid);
            }
            float2 v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                v[i] = out[L::at(c, (int)t + T * i)];
                if constexpr (MODE == 1 || MODE == 3) v[i] = cmul(v[i], pbuf[L::nat(c, (int)t + T * i)]) * pscale;
            }
            __syncthreads();  // every thread has read `out`: it takes the tile in its natural [row][TC] layout
#pragma unroll
            for (int i = 0; i < 8; ++i) out[(t + T * i) * TC + c] = v[i];
            store_src = out;
        } else if constexpr (ENG == 3) {
            constexpr int NV = N / 16;
            float2 z[8];
            int ln, i0;
            bool ok = tc5_fft<N, TC, true, -1, PRE_NONE>(buf, nullptr, 1.0f, tw, eng, tid, z, ln, i0);
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int o = (i0 + NV * i) * TC + ln;
                buf[o] = cmul(z[i], pbuf[o]) * pscale;
            }
            if constexpr (MODE == 0) {
                __syncthreads();  // the spectrum times P is in the stage: the inverse transform gathers from it
                ok = tc5_fft<N, TC, true, +1, PRE_NONE>(buf, nullptr, 1.0f, tw, eng, tid, z, ln, i0) && ok;
#pragma unroll
                for (int i = 0; i < 8; ++i) buf[(i0 + NV * i) * TC + ln] = z[i];
            }
            if (!ok) {
                atomicExch(err, 1);
                abort_flag = 1;
            }
            store_src = buf;
        } else {
            using L = TileLayout<N, TC, true>;
            float2* scratch = stages + 4 * TILE;
            float2* out = tc_fft<N, TC, true, -1, PRE_NONE, true>(buf, scratch, nullptr, 1.0f, tw, eng, tid);
            if constexpr (MODE == 0) {
                float2* other = (out == buf) ? scratch : buf;
                out = tc_fft<N, TC, true, +1, PRE_MUL, false>(out, other, pbuf, pscale, tw, eng, tid);
            }
            float2 v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                v[i] = out[L::at(c, (int)t + T * i)];
                if constexpr (MODE == 1 || MODE == 3) v[i] = cmul(v[i], pbuf[L::nat(c, (int)t + T * i)]) * pscale;
            }
            __syncthreads();  // every thread has read `out`: it takes the tile in its natural [row][TC] layout
#pragma unroll
            for (int i = 0; i < 8; ++i) out[(t + T * i) * TC + c] = v[i];
            store_src = out;
        }
        fence_proxy_async_shared();
        __syncthreads();  // every thread is done with the stage before its next copy
        if (tid == 0 && (MODE != 3 || det.store)) {
            const int iy0 = iy - c;
#pragma unroll
            for (int k = 0; k < NBOX; ++k) tma_store_2d(&map, store_src + k * BOXH * TC, 2 * iy0, b * N + k * BOXH);
            bulk_commit();
        }
        if constexpr (PSEP && MODE != 0 && MODE != 2) {
            // without an inverse transform the P tile is free from the barrier above on
            if (tid == 0 && !abort_flag && next < ntiles) issue_p(next);
        }
        if constexpr (MODE == 3) {
            // the tile the result is not in holds the warps' sums (TILE float2 >= NT / 32 * C doubles, C <= 64): the P
            // tile (read by now), or for the composite engine, whose result is in the P tile, the wave tile; engine 5,
            // whose P buffer is being refilled, has an array of its own
            double* sums = PSEP ? red5 : reinterpret_cast<double*>((ENG == 4) ? buf : buf + TILE);
            detect_tile<TX * T>(store_src, det, b, (iy - c) / TC, tid, sums);
            fence_proxy_async_shared();  // the sums were written by this proxy; the next copy into the stage by TMA
            __syncthreads();  // the partials' reads of the tile and of the sums precede the next copy into the stage
        }
    }
    if (tid == 0) bulk_wait_all();  // the stores read this block's shared memory: finish them before it is freed
    if constexpr (ENG == 3) tc5_release<tc5_blocks(N, TC)>(eng, tid, abort_flag != 0);
}

// rows: tile = RB consecutive rows of one wave (nx % RB == 0); a stage holds those RB rows and the RB rows of t.
// IFW >= 0 fixes the transforms at compile time (bit 0: inverse, bit 1: forward; the composite engine's instantiations,
// so that each holds only its own path's registers); -1 takes inv and fwd as given.
template <int N, int RB, int ENG, int IFW = -1>
__global__ void __launch_bounds__(RB * (N / 8), tc_min_blocks(RB * (N / 8), ENG)) fused_rows_tma(float2* __restrict__ psi,
                                                               const float2* __restrict__ tmul,
                                                               const float2* __restrict__ tw, int nx, int nrows,
                                                               int inv, int fwd, float scale, int* err,
                                                               const float2* const* __restrict__ t_of_wave,
                                                               int tc5_stack) {
    extern __shared__ __align__(128) unsigned char smem_rtma[];
    if constexpr (IFW >= 0) {
        inv = IFW & 1;
        fwd = (IFW >> 1) & 1;
    }
    constexpr int T = N / 8;
    constexpr int TILE = N * RB;
    __shared__ __align__(8) uint64_t full[2];
    __shared__ int abort_flag;
    __shared__ uint32_t tmem_slot;
    __shared__ __align__(8) uint64_t mma_bar;
    float2* stages = reinterpret_cast<float2*>(smem_rtma);
    const unsigned t = threadIdx.x;
    const int rr = threadIdx.y;
    const int tid = rr * T + (int)t;
    const int ntiles = nrows / RB;
    const bool with_t = (tmul != nullptr) || (t_of_wave != nullptr);
    const uint32_t bytes = (uint32_t)(TILE * sizeof(float2));
    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_barrier_init();
        abort_flag = 0;
    }
    __syncthreads();
    [[maybe_unused]] EngineState<N, ENG> eng;
    if constexpr (ENG == 0) tw_load<N, 1>(eng, t, tw);
    else if constexpr (ENG == 4) tw_load<CompPlan<N>::M, 1, CompPlan<N>::R>(eng, t % CompPlan<N>::TS, tw);
    else if constexpr (ENG == 1) eng = dft16_frags(tid & 31);
    else if constexpr (ENG == 3)
        eng = tc5_setup<tc5_blocks(N, RB)>(smem_rtma + 4 * (size_t)TILE * sizeof(float2), &tmem_slot, &mma_bar, tid,
                                           RB * T, tc5_stack);
    // the finished rows go back by a bulk store from the stage: its wave rows (ENG 0, 3) or its rows of t (ENG 4)
    constexpr bool kStoreFromStage = (ENG == 0 || ENG == 3 || ENG == 4);
    auto issue = [&](int tile, int s) {
        float2* dst = stages + s * 2 * TILE;
        const int row0 = tile * RB;
        // ENG 0, 3 and 4 store each tile from its stage: the previous tile's store must have read the stage first
        if constexpr (kStoreFromStage) bulk_wait_read();
        mbar_arrive_expect_tx(&full[s], with_t ? 2 * bytes : bytes);
        bulk_load(dst, psi + (size_t)row0 * N, bytes, &full[s]);
        if (with_t) {
            const float2* tb = t_of_wave ? t_of_wave[row0 / nx] : tmul;  // job tables: this wave's transmission
            bulk_load(dst + TILE, tb + (size_t)(row0 % nx) * N, bytes, &full[s]);
        }
    };
    int tile = blockIdx.x;
    if (tid == 0 && tile < ntiles) issue(tile, 0);
    for (int it = 0; tile < ntiles; tile += gridDim.x, ++it) {
        const int s = it & 1;
        float2* buf = stages + s * 2 * TILE;
        const float2* tbuf = buf + TILE;
        const int next = tile + gridDim.x;
        if (tid == 0) {
            const bool more = !abort_flag && next < ntiles;  // after an abandoned tile no further copy starts
            if (more) issue(next, s ^ 1);
            stage_wait(full, s, it, more, err, &abort_flag);
        }
        __syncthreads();
        if (abort_flag) break;
        float2* row = psi + (size_t)(tile * RB + rr) * N;
        if constexpr (ENG == 0) {
            // a row's exchanges stay in its own part of the stage: only the row's threads synchronise
            constexpr int LT = (RB > 1 && T % 32 == 0 && RB < 16) ? T : 0;
            const int bar = 1 + rr;
            float2 v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = buf[rr * N + t + T * i];
            line_sync<LT>(bar);
            SmemCT<0> sm{buf + rr * N};
            if (inv) ct_fft_from<N, 0, +1, 0, LT>(v, t, eng, sm, bar);
            if (with_t) {
#pragma unroll
                for (int i = 0; i < 8; ++i) v[i] = cmul(v[i], tbuf[rr * N + t + T * i]) * scale;
            } else if (scale != 1.0f) {
#pragma unroll
                for (int i = 0; i < 8; ++i) v[i] = v[i] * scale;
            }
            if (fwd) ct_fft_from<N, 0, -1, 0, LT>(v, t, eng, sm, bar);
            // back into the stage rows (every exchange read is behind a barrier); thread 0 stores them after the
            // barrier below
#pragma unroll
            for (int i = 0; i < 8; ++i) buf[rr * N + t + T * i] = v[i];
        } else if constexpr (ENG == 4) {
            // composite length: R sub-lines of TS threads per row. The row's barrier: its T threads (named 1 + rr)
            // when they are whole warps and the tile has several rows, else the block; a sub-line's: __syncwarp when
            // it lies in one warp, else the named barrier 1 + RB + R rr + g
            using C = CompPlan<N>;
            constexpr int LT = (RB > 1 && T % 32 == 0 && RB < 16) ? T : 0;
            constexpr int LS = C::TS <= 32 ? 32 : C::TS;
            static_assert(LS == 32 || RB + RB * C::R <= 15, "named barriers 1..15");
            const int g = (int)t / C::TS, u = (int)t % C::TS;
            const int line_bar = 1 + rr, sub_bar = 1 + RB + rr * C::R + g;
            float2* line = buf + rr * N;
            float2* tout = buf + TILE + rr * N;  // the row's part of the t tile takes the result
            const float2* trow = tbuf + rr * N;
            float2 v[8];
            if (inv || fwd) {
                if (inv) {
                    comp_dif_in<N, +1>(v, g, u, tw, [&](int idx) { return line[idx]; });
                } else if (with_t) {  // the forward transform alone: t multiplies the row before it
                    comp_dif_in<N, -1>(v, g, u, tw, [&](int idx) { return cmul(line[idx], trow[idx]) * scale; });
                } else {
                    comp_dif_in<N, -1>(v, g, u, tw, [&](int idx) { return line[idx] * scale; });
                }
                line_sync<LT>(line_bar);  // the row has been read: its sub-line parts become exchange buffers
                const SmemCT<0> sm{line + g * C::M};
                if (inv) {
                    ct_fft_from<C::M, 0, +1, 0, LS>(v, (unsigned)u, eng, sm, sub_bar);
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        const int idx = C::R * (u + C::TS * i) + g;  // v[i] = element idx
                        v[i] = with_t ? cmul(v[i], trow[idx]) * scale : v[i] * scale;
                    }
                } else {
                    ct_fft_from<C::M, 0, -1, 0, LS>(v, (unsigned)u, eng, sm, sub_bar);
                }
                if (inv && fwd) {
                    ct_fft_from<C::M, 0, -1, 0, LS>(v, (unsigned)u, eng, sm, sub_bar);
                    comp_dit_twiddle<N, -1>(v, g, u, tw, [&](int slot, float2 x) { line[slot] = x; });
                    line_sync<LT>(line_bar);  // the sub-lines' twiddled transforms are in the row; t has been read
                    comp_dit_out<N, -1>(v, g, u, [&](int slot) { return line[slot]; });
#pragma unroll
                    for (int i = 0; i < 8; ++i) tout[u + C::TS * i + C::M * g] = v[i];
                } else {
                    // one transform: element R k1 + g in v, read (inverse) or no longer read (forward) at that slot
#pragma unroll
                    for (int i = 0; i < 8; ++i) tout[C::R * (u + C::TS * i) + g] = v[i];
                }
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int idx = (int)t + T * i;
                    v[i] = with_t ? cmul(line[idx], trow[idx]) * scale : line[idx] * scale;
                    tout[idx] = v[i];
                }
            }
        } else if constexpr (ENG == 3) {
            constexpr int NV = N / 16;
            float2 z[8];
            int ln, i0;
            bool ok = true;
            if (inv) {
                ok = tc5_fft<N, RB, false, +1, PRE_NONE>(buf, nullptr, 1.0f, tw, eng, tid, z, ln, i0);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int o = ln * N + i0 + NV * i;
                    buf[o] = with_t ? cmul(z[i], tbuf[o]) * scale : z[i] * scale;
                }
                if (fwd) {
                    __syncthreads();  // the rows times t are in the stage: the forward transform gathers from them
                    ok = tc5_fft<N, RB, false, -1, PRE_NONE>(buf, nullptr, 1.0f, tw, eng, tid, z, ln, i0) && ok;
                }
            } else if (fwd) {
                if (with_t) ok = tc5_fft<N, RB, false, -1, PRE_MUL>(buf, tbuf, scale, tw, eng, tid, z, ln, i0);
                else ok = tc5_fft<N, RB, false, -1, PRE_SCALE>(buf, nullptr, scale, tw, eng, tid, z, ln, i0);
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int o = rr * N + (int)t + T * i;
                    buf[o] = with_t ? cmul(buf[o], tbuf[o]) * scale : buf[o] * scale;
                }
            }
            if (fwd) {
#pragma unroll
                for (int i = 0; i < 8; ++i) buf[ln * N + i0 + NV * i] = z[i];
            }
            if (!ok) {
                atomicExch(err, 1);
                abort_flag = 1;
            }
        } else if constexpr (ENG == 2) {
            using L = CcLayout<N, RB, false>;
            float2* scratch = stages + 4 * TILE;
            float2* out = buf;
            if (inv) out = cc_fft<N, RB, false, +1, PRE_NONE, true>(buf, scratch, nullptr, 1.0f, tw, tid);
            if (fwd) {
                float2* other = (out == buf) ? scratch : buf;
                if (inv) {
                    if (with_t) out = cc_fft<N, RB, false, -1, PRE_MUL, false>(out, other, tbuf, scale, tw, tid);
                    else out = cc_fft<N, RB, false, -1, PRE_SCALE, false>(out, other, nullptr, scale, tw, tid);
                } else {
                    if (with_t) out = cc_fft<N, RB, false, -1, PRE_MUL, true>(out, other, tbuf, scale, tw, tid);
                    else out = cc_fft<N, RB, false, -1, PRE_SCALE, true>(out, other, nullptr, scale, tw, tid);
                }
            }
            const bool moved = inv || fwd;  // a transform ran: the tile is in the working layout
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int idx = (int)t + T * i;
                float2 v = out[moved ? L::at(rr, idx) : L::nat(rr, idx)];
                if (!fwd) v = with_t ? cmul(v, tbuf[L::nat(rr, idx)]) * scale : v * scale;
                row[idx] = v;
            }
        } else {
            using L = TileLayout<N, RB, false>;
            float2* scratch = stages + 4 * TILE;
            float2* out = buf;
            if (inv) out = tc_fft<N, RB, false, +1, PRE_NONE, true>(buf, scratch, nullptr, 1.0f, tw, eng, tid);
            if (fwd) {
                float2* other = (out == buf) ? scratch : buf;
                if (inv) {
                    if (with_t) out = tc_fft<N, RB, false, -1, PRE_MUL, false>(out, other, tbuf, scale, tw, eng, tid);
                    else out = tc_fft<N, RB, false, -1, PRE_SCALE, false>(out, other, nullptr, scale, tw, eng, tid);
                } else {
                    if (with_t) out = tc_fft<N, RB, false, -1, PRE_MUL, true>(out, other, tbuf, scale, tw, eng, tid);
                    else out = tc_fft<N, RB, false, -1, PRE_SCALE, true>(out, other, nullptr, scale, tw, eng, tid);
                }
            }
            const bool moved = inv || fwd;  // a transform ran: the tile is in the working layout
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int idx = (int)t + T * i;
                float2 v = out[moved ? L::at(rr, idx) : L::nat(rr, idx)];
                if (!fwd) v = with_t ? cmul(v, tbuf[L::nat(rr, idx)]) * scale : v * scale;
                row[idx] = v;
            }
        }
        fence_proxy_async_shared();
        __syncthreads();  // every thread is done with the stage before its next copy
        if constexpr (kStoreFromStage) {
            if (tid == 0) {
                bulk_store(psi + (size_t)tile * RB * N, ENG == 4 ? buf + TILE : buf, bytes);
                bulk_commit();
            }
        }
    }
    if constexpr (kStoreFromStage) {
        if (tid == 0) bulk_wait_all();  // the stores read this block's shared memory: finish them before it is freed
    }
    if constexpr (ENG == 3) tc5_release<tc5_blocks(N, RB)>(eng, tid, abort_flag != 0);
}

// ---- plans and launches ---------------------------------------------------------------------------------------------
namespace {

bool factor_with(int n, int E, std::vector<int>& out) {
    out.clear();
    int rest = n;
    for (int r : {16, 8, 4, 2, 5, 3}) {
        if (E % r) continue;
        while (rest % r == 0 && rest > 1) {
            out.push_back(r);
            rest /= r;
        }
    }
    return rest == 1;
}

struct RegChoice {
    int E = 0;
    std::vector<int> fac;
};

RegChoice choose(int n) {
    RegChoice best;
    for (int E : {8, 16, 12, 20, 24}) {
        std::vector<int> f;
        if (n % E) continue;
        const int T = n / E;
        if (T < 4 || T > 256) continue;
        if (!factor_with(n, E, f)) continue;
        if ((int)f.size() > kMaxRegPasses) continue;
        if (best.E == 0 || f.size() < best.fac.size()) {
            best.E = E;
            best.fac = f;
        }
    }
    return best;
}

RegPlan reg_plan(Context& ctx, int n) {
    RegChoice ch = choose(n);
    SIMK_REQUIRE(ch.E != 0, "no register FFT plan for length " + std::to_string(n));
    RegPlan p{};
    p.n = n;
    p.E = ch.E;
    p.T = n / ch.E;
    p.npass = (int)ch.fac.size();
    for (int i = 0; i < p.npass; ++i) p.fac[i] = ch.fac[i];
    p.tw = static_cast<const float2*>(ctx.plan(n, 32).tw.ptr);
    return p;
}

template <int E>
void launch_rows_e(Context& ctx, const RegPlan& p, float2* psi, const float2* tmul, int nx, long long nrows, int inv,
                   int fwd, float scale) {
    const int RB = std::max(1, std::min(8, std::min(256, rows_threads(E)) / p.T));
    SIMK_REQUIRE(RB * p.T <= rows_threads(E), "row tile too large");
    const int lds = p.n + p.n / 16 + 1;
    const size_t smem = (size_t)RB * lds * sizeof(float2);
    static bool set = false;
    if (!set) {
        SIMK_CUDA(cudaFuncSetAttribute(fused_rows_kernel<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
        set = true;
    }
    dim3 block(p.T, RB);
    const long long blocks = (nrows + RB - 1) / RB;
    fused_rows_kernel<E><<<(unsigned)blocks, block, smem, ctx.stream>>>(psi, tmul, p, nx, nrows, inv, fwd, scale,
                                                                        ctx.wave_t);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
}

template <int E>
void launch_cols_e(Context& ctx, const RegPlan& p, const ColArgs& a, int count) {
    int TC = 16;
    while (TC > 1 && (TC * p.T > cols_threads(E) || a.ny % TC)) TC /= 2;
    SIMK_REQUIRE(TC * p.T <= cols_threads(E), "column tile too large");
    const size_t smem = (size_t)TC * p.n * sizeof(float2);
    static bool set = false;
    if (!set) {
        SIMK_CUDA(cudaFuncSetAttribute(fused_cols_kernel<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
        set = true;
    }
    SIMK_REQUIRE(smem <= 160 * 1024, "column tile too large");
    dim3 block(TC, p.T);
    dim3 grid(a.ny / TC, count);
    fused_cols_kernel<E><<<grid, block, smem, ctx.stream>>>(a, p);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
}

template <int N>
void launch_rows_ct(Context& ctx, const RegPlan& p, float2* psi, const float2* tmul, int nx, long long nrows, int inv,
                    int fwd, float scale) {
    constexpr int T = N / 8;
    constexpr int RB = (256 / T) > 0 ? (256 / T) : 1;
    const size_t smem = (size_t)RB * N * sizeof(float2);
    static bool set = false;
    if (!set) {
        SIMK_CUDA(cudaFuncSetAttribute(fused_rows_ct<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
        set = true;
    }
    SIMK_REQUIRE(nrows < (1LL << 31), "too many rows in one batch");
    dim3 block(T, RB);
    const long long blocks = (nrows + RB - 1) / RB;
    fused_rows_ct<N><<<(unsigned)blocks, block, smem, ctx.stream>>>(psi, tmul, p.tw, (unsigned)nx, (unsigned)nrows,
                                                                    inv, fwd, scale, ctx.wave_t);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
}

template <int N, int TC, int MODE>
void launch_cols_ct_m(Context& ctx, const RegPlan& p, const ColArgs& a, int count) {
    constexpr int T = N / 8;
    const size_t smem = (size_t)TC * N * sizeof(float2);
    static bool set = false;
    if (!set) {
        SIMK_CUDA(cudaFuncSetAttribute(fused_cols_ct<N, TC, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       160 * 1024));
        set = true;
    }
    dim3 block(TC, T);
    dim3 grid(a.ny / TC, count);
    fused_cols_ct<N, TC, MODE><<<grid, block, smem, ctx.stream>>>(a, p.tw);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
}



void ensure_err_flag(Context& ctx) {
    if (!ctx.err_flag.ptr) {
        ctx.err_flag.alloc(sizeof(int));
        SIMK_CUDA(cudaMemsetAsync(ctx.err_flag.ptr, 0, sizeof(int), ctx.stream));
    }
    if (ctx.sm_count == 0) SIMK_CUDA(cudaDeviceGetAttribute(&ctx.sm_count, cudaDevAttrMultiProcessorCount, ctx.device));
}

// Dynamic shared memory of a TMA pass: two stages of (wave tile, t or P tile), plus the shared-memory engines' scratch
// tile (1, 2) or the tcgen05 engine's operands (3).
constexpr size_t tma_pass_smem(int n, int lines, int eng) {
    return eng == 3   ? 4 * (size_t)n * lines * sizeof(float2) + tc5_smem_bytes(tc5_blocks(n, lines))
           : eng == 5 ? 3 * (size_t)n * lines * sizeof(float2)  // two wave stages and one P tile
                      : (eng != 0 && eng != 4 ? 5 : 4) * (size_t)n * lines * sizeof(float2);
}

// Blocks of `kern` (threads, dynamic shared memory) that fit on one SM by its registers, shared memory, threads and
// block slots, from the kernel's and the device's attributes. cudaOccupancyMaxActiveBlocksPerMultiprocessor reported
// one block for the tcgen05 passes where two fit (101 KB of shared memory and 128 registers a thread; the profiler's
// limits place two), so the persistent passes ask for the largest shared-memory carveout and take the larger of the
// two figures. The passes' blocks never wait on one another, so a block that does not find room only starts later.
int fitting_blocks(const void* kern, int threads, size_t dyn_smem, int device) {
    cudaFuncAttributes fa;
    SIMK_CUDA(cudaFuncGetAttributes(&fa, kern));
    int regs = 0, smem = 0, reserved = 0, max_threads = 0, max_blocks = 0;
    SIMK_CUDA(cudaDeviceGetAttribute(&regs, cudaDevAttrMaxRegistersPerMultiprocessor, device));
    SIMK_CUDA(cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device));
    SIMK_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device));
    SIMK_CUDA(cudaDeviceGetAttribute(&max_threads, cudaDevAttrMaxThreadsPerMultiProcessor, device));
    SIMK_CUDA(cudaDeviceGetAttribute(&max_blocks, cudaDevAttrMaxBlocksPerMultiprocessor, device));
    const int warps = (threads + 31) / 32;
    const int regs_per_warp = ((fa.numRegs * 32 + 255) / 256) * 256;  // allocated per warp in units of 256
    const long long block_smem = (long long)fa.sharedSizeBytes + (long long)dyn_smem + reserved;
    int n = max_blocks;
    if (regs_per_warp > 0) n = std::min(n, regs / (regs_per_warp * warps));
    if (block_smem > 0) n = (int)std::min<long long>(n, smem / block_smem);
    n = std::min(n, max_threads / std::max(1, threads));
    return std::max(0, n);
}

// Blocks per SM of a persistent pass: the occupancy, and for the tcgen05 engine at most what tensor memory holds.
inline int pass_blocks_per_sm(int occupancy, int eng, int mb, bool stack) {
    if (eng == 3) occupancy = std::min(occupancy, 512 / (int)tc5_tmem_cols(mb, stack));
    return occupancy;
}

template <int N, int ENG, int IFW = -1>
bool launch_rows_tma_k(Context& ctx, const RegPlan& p, float2* psi, const float2* tmul, int nx, long long nrows,
                       int inv, int fwd, float scale) {
    constexpr int T = N / 8;
    constexpr int RB = rows_tile(N, ENG);
    if constexpr (ENG == 3 && !tc5_tile(N, RB)) {
        return false;
    } else {
    if (nx % RB || nrows % RB || nrows >= (1LL << 31)) return false;
    const size_t smem = tma_pass_smem(N, RB, ENG);
    auto kern = fused_rows_tma<N, RB, ENG, IFW>;
    static int occupancy = -1;
    if (occupancy < 0) {
        SIMK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        SIMK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        SIMK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occupancy, kern, RB * T, smem));
        occupancy = std::max(occupancy, fitting_blocks((const void*)kern, RB * T, smem, ctx.device));
    }
    const int stack = ctx.tcgen05 == 2 ? 1 : 0;
    const int blocks_per_sm = pass_blocks_per_sm(occupancy, ENG, ENG == 3 ? tc5_blocks(N, RB) : 0, stack != 0);
    if (blocks_per_sm <= 0) return false;
    ensure_err_flag(ctx);
    const long long ntiles = nrows / RB;
    const int grid = (int)std::min<long long>(ntiles, (long long)blocks_per_sm * ctx.sm_count);
    kern<<<grid, dim3(T, RB), smem, ctx.stream>>>(psi, tmul, p.tw, nx, (int)nrows, inv, fwd, scale,
                                                  ctx.err_flag.as<int>(), ctx.wave_t, stack);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
    return true;
    }
}

// The composite engine's row pass is instantiated per (inverse, forward) pair; the other engines take them at run time.
template <int N, int ENG>
bool launch_rows_tma(Context& ctx, const RegPlan& p, float2* psi, const float2* tmul, int nx, long long nrows, int inv,
                     int fwd, float scale) {
    if constexpr (ENG == 4) {
        switch ((inv ? 1 : 0) | (fwd ? 2 : 0)) {
            case 0: return launch_rows_tma_k<N, ENG, 0>(ctx, p, psi, tmul, nx, nrows, 0, 0, scale);
            case 1: return launch_rows_tma_k<N, ENG, 1>(ctx, p, psi, tmul, nx, nrows, 1, 0, scale);
            case 2: return launch_rows_tma_k<N, ENG, 2>(ctx, p, psi, tmul, nx, nrows, 0, 1, scale);
            default: return launch_rows_tma_k<N, ENG, 3>(ctx, p, psi, tmul, nx, nrows, 1, 1, scale);
        }
    } else {
        return launch_rows_tma_k<N, ENG>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale);
    }
}

template <int N, int TC, int MODE, int ENG>
bool launch_cols_tma_m(Context& ctx, const RegPlan& p, const ColArgs& a, int count) {
    constexpr int T = N / 8;
    constexpr int BOXH = tma_box_rows(N);
    if constexpr (ENG == 3 && !tc5_tile(N, TC)) {
        return false;
    } else {
    const size_t smem = tma_pass_smem(N, TC, ENG);
    auto kern = fused_cols_tma<N, TC, MODE, ENG>;
    static int occupancy = -1;
    if (occupancy < 0) {
        SIMK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        SIMK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        SIMK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occupancy, kern, cols_tx(TC, ENG) * T, smem));
        occupancy = std::max(occupancy, fitting_blocks((const void*)kern, cols_tx(TC, ENG) * T, smem, ctx.device));
    }
    const int stack = ctx.tcgen05 == 2 ? 1 : 0;
    const int blocks_per_sm = pass_blocks_per_sm(occupancy, ENG, ENG == 3 ? tc5_blocks(N, TC) : 0, stack != 0);
    if (blocks_per_sm <= 0) return false;
    ensure_err_flag(ctx);
    const CUtensorMap map = encode_tensor_map_2d(a.psi, 2ULL * a.ny, (unsigned long long)count * N, 2 * TC, BOXH);
    // the P tiles, or for the probes (MODE 2) the spectrum's
    const CUtensorMap pmap =
        MODE == 2 ? encode_tensor_map_2d(const_cast<float2*>(a.spectrum), 2ULL * a.ny, (unsigned long long)N, 2 * TC, BOXH)
                  : encode_tensor_map_2d(const_cast<float2*>(a.P), 2ULL * a.ny,
                                         (unsigned long long)std::max(1, a.p_blocks) * N, 2 * TC, BOXH);
    const long long ntiles = (long long)count * (a.ny / TC);
    if (ntiles >= (1LL << 31)) return false;
    DetectArgs det{};
    if constexpr (MODE == 3) {
        const DetectorPlan::TileChannels& tch = a.det.plan->tiles(TC);
        det.ptr = tch.ptr.as<int>();
        det.ent = tch.ent.as<int2>();
        det.partial = a.det.partial;
        det.n_ch = a.det.plan->n_channels;
        det.groups = tch.groups;
        det.store = a.det.store;
        if (a.det_groups) *a.det_groups = tch.groups;
    }
    const int grid = (int)std::min<long long>(ntiles, (long long)blocks_per_sm * ctx.sm_count);
    kern<<<grid, dim3(cols_tx(TC, ENG), T), smem, ctx.stream>>>(map, pmap, a.psi, a.pscale, a.ny, count, p.tw,
                                                  ctx.err_flag.as<int>(), a.p_row, det, stack, a.rx, a.ry);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
    return true;
    }
}

template <int N, int TC, int ENG = 0>
bool launch_cols_tma(Context& ctx, const RegPlan& p, const ColArgs& a, int count) {
    if (TC < 2 || a.ny % TC) return false;  // the TMA box's inner extent must be a multiple of 16 bytes
    if (a.mode == 0) return launch_cols_tma_m<N, TC, 0, ENG>(ctx, p, a, count);
    if (a.mode == 1) return launch_cols_tma_m<N, TC, 1, ENG>(ctx, p, a, count);
    if (a.mode == 3) return launch_cols_tma_m<N, TC, 3, ENG>(ctx, p, a, count);
    if constexpr (ENG == 5) {
        if (a.mode == 2) return launch_cols_tma_m<N, TC, 2, ENG>(ctx, p, a, count);  // probes from their spectrum
    }
    return false;
}

template <int N, int TC>
void launch_cols_ct(Context& ctx, const RegPlan& p, const ColArgs& a, int count) {
    switch (a.mode) {
        case 0: launch_cols_ct_m<N, TC, 0>(ctx, p, a, count); break;
        case 1: launch_cols_ct_m<N, TC, 1>(ctx, p, a, count); break;
        default: launch_cols_ct_m<N, TC, 2>(ctx, p, a, count); break;
    }
}

bool rows_ct(Context& ctx, const RegPlan& p, float2* psi, const float2* tmul, int nx, long long nrows, int inv, int fwd,
             float scale) {
    if (ctx.tma) {
        bool done = false;
        switch (p.n) {
            case 256: done = launch_rows_tma<256, 0>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); break;
            case 512: done = launch_rows_tma<512, 0>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); break;
            case 1024: done = launch_rows_tma<1024, 0>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); break;
            case 2048: done = launch_rows_tma<2048, 0>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); break;
            default: break;
        }
        if (done) return true;
    }
    switch (p.n) {
        case 128: launch_rows_ct<128>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); return true;
        case 256: launch_rows_ct<256>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); return true;
        case 512: launch_rows_ct<512>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); return true;
        case 1024: launch_rows_ct<1024>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); return true;
        case 2048: launch_rows_ct<2048>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); return true;
        default: return false;
    }
}

template <int N>
bool cols_ct_tc(Context& ctx, const RegPlan& p, const ColArgs& a, int count, int tc) {
    // TC x N/8 threads per CTA, at most 1024
    if (tc * (N / 8) > 1024 || a.ny % tc) return false;
    // column pairs (engine 5, every mode including the probes' generation): tiles of 8 columns at 512 and 1024 (one
    // 512-thread CTA an SM there) and 16 at 256, where the column tile is automatic or that
    if constexpr (N == 512 || N == 256 || N == 1024) {
        constexpr int TP = (N == 256) ? 16 : 8;
        if (ctx.tma && ctx.paired && (ctx.col_tile == 0 || ctx.col_tile == TP) && a.ny % TP == 0 &&
            launch_cols_tma<N, TP, 5>(ctx, p, a, count))
            return true;
    }
    if (ctx.tma && a.mode != 2) {
        switch (tc) {
            case 2: if (launch_cols_tma<N, 2>(ctx, p, a, count)) return true; break;
            case 4: if (launch_cols_tma<N, 4>(ctx, p, a, count)) return true; break;
            case 8: if constexpr (8 * (N / 8) <= 1024) { if (launch_cols_tma<N, 8>(ctx, p, a, count)) return true; } break;
            default: break;
        }
    }
    if (a.mode == 3) return false;  // detection in the epilogue runs on the TMA passes only
    switch (tc) {
        case 1: launch_cols_ct<N, 1>(ctx, p, a, count); return true;
        case 2: launch_cols_ct<N, 2>(ctx, p, a, count); return true;
        case 4: launch_cols_ct<N, 4>(ctx, p, a, count); return true;
        case 8: if constexpr (8 * (N / 8) <= 1024) { launch_cols_ct<N, 8>(ctx, p, a, count); return true; } return false;
        case 16: if constexpr (16 * (N / 8) <= 1024) { launch_cols_ct<N, 16>(ctx, p, a, count); return true; } return false;
        default: return false;
    }
}

// Column tile width: the context's SIMK_OPT_COL_TILE, else 4 columns (three CTAs per SM at 512).
bool cols_ct(Context& ctx, const RegPlan& p, const ColArgs& a, int count) {
    int tc = ctx.col_tile > 0 ? ctx.col_tile : 4;
    while (tc > 1 && (a.ny % tc || tc * (p.n / 8) > 1024)) tc /= 2;
    switch (p.n) {
        case 128: return cols_ct_tc<128>(ctx, p, a, count, tc);
        case 256: return cols_ct_tc<256>(ctx, p, a, count, tc);
        case 512: return cols_ct_tc<512>(ctx, p, a, count, tc);
        case 1024: return cols_ct_tc<1024>(ctx, p, a, count, tc);
        case 2048: return cols_ct_tc<2048>(ctx, p, a, count, tc);
        default: return false;
    }
}

// ---- the bf16x3 form: the same TMA passes with tensor-core line FFTs ---------------------------------------------------
bool rows_tc(Context& ctx, const RegPlan& p, float2* psi, const float2* tmul, int nx, long long nrows, int inv, int fwd,
             float scale) {
    if (ctx.tcgen05) {  // the tcgen05 engine where its tiles fit, else the mma.sync engine
        if (p.n == 256 && launch_rows_tma<256, 3>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale)) return true;
        if (p.n == 512 && launch_rows_tma<512, 3>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale)) return true;
    }
    switch (p.n) {
        case 256: return launch_rows_tma<256, 1>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale);
        case 512: return launch_rows_tma<512, 1>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale);
        case 768: return launch_rows_tma<768, 1>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale);
        case 1024: return launch_rows_tma<1024, 1>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale);
        case 2048: return launch_rows_tma<2048, 1>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale);
        default: return false;
    }
}

// The widest column tile (at most the context's SIMK_OPT_COL_TILE, default 4) whose two stages fit in shared memory.
template <int N>
bool cols_tc_n(Context& ctx, const RegPlan& p, const ColArgs& a, int count, int tc) {
    for (; tc >= 2; tc /= 2) {
        switch (tc) {
            case 8:
                if constexpr (8 * (N / 8) <= 1024) {
                    if (launch_cols_tma<N, 8, 1>(ctx, p, a, count)) return true;
                }
                break;
            case 4:
                if constexpr (4 * (N / 8) <= 1024) {
                    if (launch_cols_tma<N, 4, 1>(ctx, p, a, count)) return true;
                }
                break;
            case 2:
                if (launch_cols_tma<N, 2, 1>(ctx, p, a, count)) return true;
                break;
            default: break;
        }
    }
    return false;
}

// The tcgen05 engine's column tiles are whole 128-vector blocks: 8 columns at 256, 4 or 8 at 512.
template <int N>
bool cols_tc5(Context& ctx, const RegPlan& p, const ColArgs& a, int count) {
    if constexpr (N == 512) {
        if (ctx.col_tile == 8 && launch_cols_tma<512, 8, 3>(ctx, p, a, count)) return true;
        return launch_cols_tma<512, 4, 3>(ctx, p, a, count);
    } else {
        return launch_cols_tma<N, 8, 3>(ctx, p, a, count);
    }
}

bool cols_tc(Context& ctx, const RegPlan& p, const ColArgs& a, int count) {
    if (ctx.tcgen05) {
        if (p.n == 256 && cols_tc5<256>(ctx, p, a, count)) return true;
        if (p.n == 512 && cols_tc5<512>(ctx, p, a, count)) return true;
    }
    int tc = ctx.col_tile > 0 ? ctx.col_tile : 4;
    switch (p.n) {
        case 256: return cols_tc_n<256>(ctx, p, a, count, tc);
        case 512: return cols_tc_n<512>(ctx, p, a, count, tc);
        case 768: return cols_tc_n<768>(ctx, p, a, count, tc);
        case 1024: return cols_tc_n<1024>(ctx, p, a, count, tc);
        case 2048: return cols_tc_n<2048>(ctx, p, a, count, tc);
        default: return false;
    }
}

// ---- the float32 fused form at lengths that are not powers of two: the TMA passes with the composite-length register
// engine (4) where N = 3 or 5 times a power of two, else the shared-memory engine (2); SIMK_OPT_COMPOSITE = 0 keeps 2 ---
template <int N>
bool rows_cc_n(Context& ctx, const RegPlan& p, float2* psi, const float2* tmul, int nx, long long nrows, int inv,
               int fwd, float scale) {
    if constexpr (comp_length(N)) {
        if (ctx.composite && launch_rows_tma<N, 4>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale)) return true;
    }
    return launch_rows_tma<N, 2>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale);
}

bool rows_cc(Context& ctx, const RegPlan& p, float2* psi, const float2* tmul, int nx, long long nrows, int inv, int fwd,
             float scale) {
    switch (p.n) {
        case 384: return rows_cc_n<384>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale);
        case 640: return rows_cc_n<640>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale);
        case 768: return rows_cc_n<768>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale);
        case 1536: return rows_cc_n<1536>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale);
        default: return false;
    }
}

template <int N, int TC>
bool cols_cc_tc(Context& ctx, const RegPlan& p, const ColArgs& a, int count) {
    if constexpr (TC * (N / 8) > 1024) {
        return false;
    } else {
        if constexpr (comp_length(N)) {
            if (ctx.composite && launch_cols_tma<N, TC, 4>(ctx, p, a, count)) return true;
        }
        return launch_cols_tma<N, TC, 2>(ctx, p, a, count);
    }
}

template <int N>
bool cols_cc_n(Context& ctx, const RegPlan& p, const ColArgs& a, int count, int tc) {
    for (; tc >= 2; tc /= 2) {
        switch (tc) {
            case 8: if (cols_cc_tc<N, 8>(ctx, p, a, count)) return true; break;
            case 4: if (cols_cc_tc<N, 4>(ctx, p, a, count)) return true; break;
            case 2: if (cols_cc_tc<N, 2>(ctx, p, a, count)) return true; break;
            default: break;
        }
    }
    return false;
}

bool cols_cc(Context& ctx, const RegPlan& p, const ColArgs& a, int count) {
    const int tc = ctx.col_tile > 0 ? ctx.col_tile : 4;
    switch (p.n) {
        case 384: return cols_cc_n<384>(ctx, p, a, count, tc);
        case 640: return cols_cc_n<640>(ctx, p, a, count, tc);
        case 768: return cols_cc_n<768>(ctx, p, a, count, tc);
        case 1536: return cols_cc_n<1536>(ctx, p, a, count, tc);
        default: return false;
    }
}

bool tc_length(int n) { return n == 256 || n == 512 || n == 768 || n == 1024 || n == 2048; }

void launch_rows(Context& ctx, const RegPlan& p, float2* psi, const float2* tmul, int nx, long long nrows, int inv,
                 int fwd, float scale) {
    KernelTimer timer(ctx, "fused_rows", 16.0 * (double)nrows * p.n);
    if (ctx.form == SIMK_FORM_BF16X3) {
        if (!rows_tc(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale))
            throw Error(SIMK_ERR_INVALID, "the bf16x3 form has no row pass for length " + std::to_string(p.n));
        return;
    }
    if (rows_ct(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale)) return;
    if (ctx.tma && rows_cc(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale)) return;
    switch (p.E) {
        case 8: launch_rows_e<8>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); break;
        case 12: launch_rows_e<12>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); break;
        case 16: launch_rows_e<16>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); break;
        case 20: launch_rows_e<20>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); break;
        case 24: launch_rows_e<24>(ctx, p, psi, tmul, nx, nrows, inv, fwd, scale); break;
        default: throw Error(SIMK_ERR_INVALID, "unsupported register plan");
    }
}

// Mode 3 (detection in the epilogue) where a TMA pass takes it, else mode 1; returns the column groups of the
// detection's partial sums (0: the caller detects from the stored k-space waves).
int launch_cols(Context& ctx, const RegPlan& p, const ColArgs& a_in, int count) {
    ColArgs a = a_in;
    if (a.mode != 2 && ctx.wave_p) {  // job tables: per-wave propagators stacked at a.P
        a.p_row = ctx.wave_p;
        a.p_blocks = ctx.wave_p_blocks;
    }
    const double bytes = (a.mode == 2 ? 8.0 : 16.0) * (double)p.n * a.ny * count;
    KernelTimer timer(ctx, "fused_cols", bytes);
    int groups = 0;
    if (a.mode == 3) {
        a.det_groups = &groups;
        const bool done = ctx.form == SIMK_FORM_BF16X3 ? cols_tc(ctx, p, a, count)
                                                       : (cols_ct(ctx, p, a, count) ||
                                                          (ctx.tma && cols_cc(ctx, p, a, count)));
        if (done) return groups;
        a.mode = 1;
        groups = 0;
    }
    if (ctx.form == SIMK_FORM_BF16X3 && a.mode != 2) {  // the probe's inverse transform (mode 2) stays float32
        if (!cols_tc(ctx, p, a, count))
            throw Error(SIMK_ERR_INVALID, "the bf16x3 form has no column pass for length " + std::to_string(p.n));
        return 0;
    }
    if (cols_ct(ctx, p, a, count)) return 0;
    if (ctx.tma && a.mode != 2 && cols_cc(ctx, p, a, count)) return 0;
    switch (p.E) {
        case 8: launch_cols_e<8>(ctx, p, a, count); break;
        case 12: launch_cols_e<12>(ctx, p, a, count); break;
        case 16: launch_cols_e<16>(ctx, p, a, count); break;
        case 20: launch_cols_e<20>(ctx, p, a, count); break;
        case 24: launch_cols_e<24>(ctx, p, a, count); break;
        default: throw Error(SIMK_ERR_INVALID, "unsupported register plan");
    }
    return 0;
}

}  // namespace


CUtensorMap encode_tensor_map_2d(void* base, unsigned long long inner, unsigned long long rows, unsigned box_inner,
                                 unsigned box_rows) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        SIMK_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        SIMK_REQUIRE(fn != nullptr && q == cudaDriverEntryPointSuccess, "cuTensorMapEncodeTiled is not available");
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    SIMK_REQUIRE(((uintptr_t)base % 16) == 0, "TMA base address must be 16-byte aligned");
    SIMK_REQUIRE((inner * sizeof(float)) % 16 == 0, "TMA row pitch must be a multiple of 16 bytes");
    SIMK_REQUIRE((box_inner * sizeof(float)) % 16 == 0 && box_inner <= 256 && box_rows <= 256, "bad TMA box");
    CUtensorMap map;
    const cuuint64_t dims[2] = {inner, rows};
    const cuuint64_t strides[1] = {inner * sizeof(float)};
    const cuuint32_t box[2] = {box_inner, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = encode(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw Error(SIMK_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return map;
}

bool fused_supported(Context& ctx, const GridGeom& g) {
    if (ctx.form == SIMK_FORM_BF16X3) {
        SIMK_REQUIRE(tc_length(g.nx) && tc_length(g.ny),
                     "the bf16x3 form covers grid sides of 256, 512, 768, 1024 and 2048 points");
        SIMK_REQUIRE(ctx.tma, "the bf16x3 form runs on the TMA-pipelined passes (SIMK_OPT_TMA must be on)");
        return true;
    }
    return choose(g.nx).E != 0 && choose(g.ny).E != 0;
}

namespace {
int propagate_fused_eager(Context& ctx, PotentialImpl& pot, double energy, double tx, double ty, float2* psi,
                          int count, bool probe_rows_pending, const std::function<void(int, bool)>& on_slice,
                          bool kspace_last, const FusedDetect* det);

template <typename T> void key_append(std::string& k, const T& v) {
    k.append(reinterpret_cast<const char*>(&v), sizeof(T));
}
}  // namespace

// The slice loop of one batch: 2 launches per slice. With SIMK_OPT_GRAPHS (and no per-kernel timing, no per-slice
// callback) the loop is replayed from a CUDA graph: the first time a key is seen it runs eagerly (creating the
// propagators, the error flag and the launch configurations), the second time it is captured and instantiated, and
// from then on one graph launch replaces the 2 S kernel launches. The key holds every pointer and setting the
// recorded launches read, so a replay never sees a freed or different buffer.
int propagate_fused(Context& ctx, PotentialImpl& pot, double energy, double tx, double ty, float2* psi, int count,
                    bool probe_rows_pending, const std::function<void(int, bool)>& on_slice, bool kspace_last,
                    const FusedDetect* det) {
    if (!kspace_last) det = nullptr;
    if (!ctx.graphs || ctx.timing || on_slice)
        return propagate_fused_eager(ctx, pot, energy, tx, ty, psi, count, probe_rows_pending, on_slice, kspace_last,
                                     det);
    std::string key;
    key_append(key, psi);
    key_append(key, count);
    key_append(key, pot.t.ptr);
    key_append(key, pot.g.nx);
    key_append(key, pot.g.ny);
    key_append(key, probe_rows_pending);
    key_append(key, kspace_last);
    key_append(key, ctx.form);
    key_append(key, ctx.col_tile);
    key_append(key, ctx.paired);
    key_append(key, ctx.tma);
    key_append(key, ctx.tcgen05);
    key_append(key, ctx.composite);
    key_append(key, ctx.stream);
    const FusedDetect nodet{};
    const FusedDetect& d = det ? *det : nodet;
    key_append(key, d.plan);
    key_append(key, d.partial);
    key_append(key, d.store);
    for (int j = 0; j < pot.n_slices(); ++j) key_append(key, ctx.propagator(pot.g, energy, pot.dz[j], tx, ty).p.ptr);
    auto it = ctx.slice_graphs.find(key);
    if (it != ctx.slice_graphs.end()) {
        SIMK_CUDA(cudaGraphLaunch(it->second.exec, ctx.stream));
        ctx.launches += it->second.launches;
        return it->second.det_groups;
    }
    if (ctx.slice_seen.insert(key).second)
        return propagate_fused_eager(ctx, pot, energy, tx, ty, psi, count, probe_rows_pending, nullptr, kspace_last,
                                     det);
    if (ctx.slice_graphs.size() >= 64) ctx.drop_graphs();
    const int64_t before = ctx.launches;
    cudaGraph_t graph = nullptr;
    int groups = 0;
    SIMK_CUDA(cudaStreamBeginCapture(ctx.stream, cudaStreamCaptureModeThreadLocal));
    try {
        groups = propagate_fused_eager(ctx, pot, energy, tx, ty, psi, count, probe_rows_pending, nullptr, kspace_last,
                                       det);
    } catch (...) {
        cudaStreamEndCapture(ctx.stream, &graph);
        if (graph) cudaGraphDestroy(graph);
        ctx.launches = before;
        throw;
    }
    SIMK_CUDA(cudaStreamEndCapture(ctx.stream, &graph));
    const int64_t n = ctx.launches - before;
    ctx.launches = before;
    cudaGraphExec_t exec = nullptr;
    const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    SIMK_CUDA(e);
    ctx.slice_graphs[key] = Context::SliceGraph{exec, n, groups};
    SIMK_CUDA(cudaGraphLaunch(exec, ctx.stream));
    ctx.launches += n;
    return groups;
}

namespace {
int propagate_fused_eager(Context& ctx, PotentialImpl& pot, double energy, double tx, double ty, float2* psi,
                          int count, bool probe_rows_pending, const std::function<void(int, bool)>& on_slice,
                          bool kspace_last, const FusedDetect* det) {
    int groups = 0;
    const GridGeom& g = pot.g;
    const long long N = g.count();
    const RegPlan prow = reg_plan(ctx, g.ny);
    const RegPlan pcol = reg_plan(ctx, g.nx);
    const int S = pot.n_slices();
    const float invN = 1.0f / (float)N;
    for (int j = 0; j < S; ++j) {
        // rows: complete the previous inverse transform (or the probe's), x t_j, forward
        const bool inv = (j > 0) || probe_rows_pending;
        const float rscale = (j == 0 && probe_rows_pending) ? invN : 1.0f;
        launch_rows(ctx, prow, psi, pot.t.as<float2>() + (long long)j * N, g.nx, (long long)count * g.nx, inv ? 1 : 0,
                    1, rscale);
        const Propagator& P = ctx.propagator(g, energy, pot.dz[j], tx, ty);
        const bool last = (j == S - 1);
        ColArgs a{};
        a.psi = psi;
        a.P = P.p.as<float2>();
        a.ny = g.ny;
        if (last && kspace_last) {
            a.mode = det ? 3 : 1;
            if (det) a.det = *det;
            a.pscale = 1.0f;
        } else {
            a.mode = 0;
            a.pscale = invN;
        }
        const int gr = launch_cols(ctx, pcol, a, count);
        if (last) groups = gr;
        if (on_slice) on_slice(j, last && kspace_last);
    }
    return groups;
}

}  // namespace

// The waves after slice j are in "row spectrum" form (columns inverse-transformed, rows not): the row IFFT that
// completes them, in place.
void finish_rows(Context& ctx, const GridGeom& g, float2* psi, int count) {
    const RegPlan prow = reg_plan(ctx, g.ny);
    launch_rows(ctx, prow, psi, nullptr, g.nx, (long long)count * g.nx, 1, 0, 1.0f);
}

int exit_spectra_fused(Context& ctx, PotentialImpl& pot, const simk_probe& probe, const float2* spectrum,
                       const double* positions_dev, long long first, int b, const FusedDetect* det) {
    const GridGeom& g = pot.g;
    float2* psi = ctx.work_a.as<float2>();
    launch_ramps(ctx, g, positions_dev, first, b, ctx.rx.as<float2>(), ctx.ry.as<float2>());
    const RegPlan pcol = reg_plan(ctx, g.nx);
    ColArgs a{};
    a.psi = psi;
    a.mode = 2;
    a.ny = g.ny;
    a.spectrum = spectrum;
    a.rx = ctx.rx.as<float2>();
    a.ry = ctx.ry.as<float2>();
    a.pscale = 1.0f;
    launch_cols(ctx, pcol, a, b);
    return propagate_fused(ctx, pot, probe.energy, probe.tilt_x, probe.tilt_y, psi, b, true, nullptr, true, det);
}

void scan_fused_batch(Context& ctx, PotentialImpl& pot, const simk_probe& probe, const float2* spectrum,
                      const double* positions_dev, long long first, int b, DetectorPlan& dplan,
                      double* const* outputs_dev, double weight) {
    const GridGeom& g = pot.g;
    const long long N = g.count();
    // channel detectors are summed in the last column pass when it runs on the TMA passes (at most 64 channels)
    FusedDetect fd{};
    const bool fuse = dplan.n_channels > 0 && dplan.n_channels <= 64 && ctx.tma && ctx.epilogue_detect;
    if (fuse) {
        ctx.det_partial.ensure((size_t)b * (g.ny / 2) * dplan.n_channels * sizeof(double));
        fd.plan = &dplan;
        fd.partial = ctx.det_partial.as<double>();
        fd.store = dplan.has_pixel_outputs ? 1 : 0;
    }
    const int groups = exit_spectra_fused(ctx, pot, probe, spectrum, positions_dev, first, b, fuse ? &fd : nullptr);
    {
        KernelTimer t(ctx, "detect", groups ? 0.0 : 8.0 * (double)N * b);
        if (groups) launch_detect_fold(ctx, dplan, fd.partial, groups, b, first, outputs_dev, weight);
        if (!groups || dplan.has_pixel_outputs)
            launch_detect(ctx, dplan, g, ctx.work_a.as<float2>(), b, first, outputs_dev, weight, 1.0f, groups == 0);
    }
}

// ---- autotuning ------------------------------------------------------------------------------------------------------
// Candidates are timed on one slice step (row pass + column pass) of the potential's first transmission and
// propagator over a scratch batch of waves (values do not change the time), with CUDA events after a warm-up: first
// every (column tile, TMA) pair at a batch of up to 256 waves, then batch sizes from 32 waves up to what half of the
// free device memory holds (the scan's wave buffer and its copy) for the winner. The figure of merit is time per
// wave-step; of the batches, the largest within 2 % of the fastest is kept.
Context::Tuned autotune(Context& ctx, PotentialImpl& pot, double energy, double tx, double ty, long long max_waves) {
    const GridGeom& g = pot.g;
    std::string key;
    key_append(key, g.nx);
    key_append(key, g.ny);
    key_append(key, ctx.form);
    auto it = ctx.tuned.find(key);
    if (it != ctx.tuned.end()) {
        ctx.last_tuned = it->second;
        return it->second;
    }
    const long long N = g.count();
    size_t free_b = 0, total_b = 0;
    SIMK_CUDA(cudaMemGetInfo(&free_b, &total_b));
    long long cap = (long long)(free_b / 2 / (2 * (size_t)N * sizeof(float2)));
    cap = std::max(1LL, std::min(cap, 1024LL));  // per grid, not per call: the caller's batches cap themselves
    (void)max_waves;
    const RegPlan prw = reg_plan(ctx, g.ny);
    const RegPlan pcl = reg_plan(ctx, g.nx);
    const Propagator& P = ctx.propagator(g, energy, pot.dz[0], tx, ty);
    DeviceBuffer buf((size_t)cap * N * sizeof(float2));
    SIMK_CUDA(cudaMemsetAsync(buf.ptr, 0, (size_t)cap * N * sizeof(float2), ctx.stream));
    const int save_tc = ctx.col_tile, save_tma = ctx.tma, save_timing = ctx.timing;
    const int save_comp = ctx.composite, save_tc5 = ctx.tcgen05;
    ctx.timing = 0;
    // the engines to choose from: the composite register engine or the shared-memory one (fused form, lengths 3 or 5
    // times a power of two), the tcgen05 engine's two product orders or the mma.sync engine (bf16x3 form, 256, 512)
    std::vector<int> engines{-1};
    const bool comp_side = comp_length(g.nx) || comp_length(g.ny);
    const bool tc5_side = (g.nx == 256 || g.nx == 512) && (g.ny == 256 || g.ny == 512);
    if (ctx.form == SIMK_FORM_FUSED && comp_side) engines = {1, 0};
    if (ctx.form == SIMK_FORM_BF16X3 && tc5_side) engines = {2, 1, 0};
    auto set_engine = [&](int e) {
        if (e < 0) return;
        if (ctx.form == SIMK_FORM_FUSED) ctx.composite = e;
        else ctx.tcgen05 = e;
    };
    cudaEvent_t e0, e1;
    SIMK_CUDA(cudaEventCreate(&e0));
    SIMK_CUDA(cudaEventCreate(&e1));
    auto step = [&](long long b) {
        launch_rows(ctx, prw, buf.as<float2>(), pot.t.as<float2>(), g.nx, b * g.nx, 1, 1, 1.0f);
        ColArgs a{};
        a.psi = buf.as<float2>();
        a.P = P.p.as<float2>();
        a.ny = g.ny;
        a.mode = 0;
        a.pscale = 1.0f / (float)N;
        launch_cols(ctx, pcl, a, (int)b);
    };
    auto time_per_wave = [&](long long b) {
        step(b);  // warm-up (first launches set attributes and occupancy)
        SIMK_CUDA(cudaEventRecord(e0, ctx.stream));
        for (int r = 0; r < 2; ++r) step(b);
        SIMK_CUDA(cudaEventRecord(e1, ctx.stream));
        SIMK_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        SIMK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return (double)ms / (2.0 * (double)b);
    };
    Context::Tuned best;
    double best_t = 1e300;
    try {
        const long long b0 = std::min(cap, 256LL);
        for (int eng : engines) {
            set_engine(eng);
            for (int tma : {1, 0}) {
                if (tma && !save_tma) continue;
                if (!tma && ctx.form == SIMK_FORM_BF16X3) continue;  // the tensor-core form runs on the TMA passes only
                if (!tma && eng == 0 && ctx.form == SIMK_FORM_FUSED) continue;  // the engines differ on TMA passes only
                for (int tc : {2, 4, 8, 16}) {
                    if (g.ny % tc || tc * (g.nx / 8) > 1024) continue;
                    // 16 columns only where the column pairs take them (256^2)
                    if (tc == 16 && !(ctx.paired && g.nx == 256 && ctx.form == SIMK_FORM_FUSED && tma)) continue;
                    ctx.tma = tma;
                    ctx.col_tile = tc;
                    const double t = time_per_wave(b0);
                    if (t < best_t) {
                        best_t = t;
                        best.col_tile = tc;
                        best.tma = tma;
                        best.batch = b0;
                        best.engine = eng;
                    }
                }
            }
        }
        ctx.tma = best.tma;
        ctx.col_tile = best.col_tile;
        set_engine(best.engine);
        // batch: the largest whose time per wave is within 2 % of the fastest, since the per-batch work that is not
        // timed here (probe generation, detection, launches) favours large batches
        std::vector<std::pair<long long, double>> bt{{best.batch, best_t}};
        for (long long b = 32; b <= cap; b *= 2)
            if (b != best.batch) bt.push_back({b, time_per_wave(b)});
        double fastest = 1e300;
        for (auto& x : bt) fastest = std::min(fastest, x.second);
        for (auto& x : bt)
            if (x.second <= 1.02 * fastest && x.first > best.batch) best.batch = x.first;
        for (auto& x : bt)
            if (x.first == best.batch) best_t = x.second;
    } catch (...) {
        ctx.col_tile = save_tc;
        ctx.tma = save_tma;
        ctx.timing = save_timing;
        ctx.composite = save_comp;
        ctx.tcgen05 = save_tc5;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    ctx.col_tile = save_tc;
    ctx.tma = save_tma;
    ctx.timing = save_timing;
    ctx.composite = save_comp;
    ctx.tcgen05 = save_tc5;
    SIMK_CUDA(cudaEventDestroy(e0));
    SIMK_CUDA(cudaEventDestroy(e1));
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));  // the scratch batch is freed on return
    ctx.tuned[key] = best;
    ctx.last_tuned = best;
    return best;
}

// ---- job tables -------------------------------------------------------------------------------------------------------
// Independent jobs (own grid, potential, energy, slice count; plane wave or probe) in the fewest launches: jobs of one
// grid shape form a group whose waves sit side by side, sorted by slice count, so that at slice step s the jobs still
// running are a prefix of the group. One row pass and one column pass per step advance that prefix, each wave reading
// its own transmission slice and propagator through the context's wave table (wave_t, wave_p): the transmissions stay
// in each potential's stack, the propagators are stacked once per group for the column pass's tensor map. The jobs
// that end at step s complete their row inverse transform and write |exit wave|^2. With the plain form the jobs run
// one after another through the plain path instead (the sequential baseline).
namespace {
__global__ void k_fill_c(float2* __restrict__ psi, long long n, float2 v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        psi[i] = v;
}
__global__ void k_intensity(const float2* __restrict__ psi, long long n, double* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float2 v = psi[i];
        out[i] = (double)v.x * v.x + (double)v.y * v.y;
    }
}
int grid_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 16)); }

// Buffers the incident probes of a job table share, grown to the largest grid once: the jobs' probes are formed one
// after another on one stream, so no job allocates, frees or waits.
struct ProbeScratch {
    DeviceBuffer spectrum, tmp, norm, rx, ry;
    DeviceBuffer positions;  // (x, y) of every job, uploaded once
};

// The incident wave of job j (index `job` of the table) into psi (N float2): ones, or the probe IFFT(Psi0 r_x r_y) at
// (x, y).
void incident_wave(Context& ctx, const JobSpec& j, int job, ProbeScratch& sc, float2* psi) {
    const GridGeom& g = j.pot->g;
    const long long N = g.count();
    if (!j.probe) {
        k_fill_c<<<grid_for(N), 256, 0, ctx.stream>>>(psi, N, make_float2(1.0f, 0.0f));
        ++ctx.launches;
        SIMK_CUDA(cudaGetLastError());
        return;
    }
    simk_probe pr = j.probe_spec;
    pr.energy = j.energy;
    probe_spectrum_into(ctx, g, pr, sc.spectrum, sc.tmp, sc.norm);
    sc.rx.ensure(g.nx * sizeof(float2));
    sc.ry.ensure(g.ny * sizeof(float2));
    launch_ramps(ctx, g, sc.positions.as<double>(), job, 1, sc.rx.as<float2>(), sc.ry.as<float2>());
    launch_probes(ctx, g, sc.spectrum.as<float2>(), sc.rx.as<float2>(), sc.ry.as<float2>(), 1, psi, 1.0f);
    fft2(ctx.plan(g.ny, 32), ctx.plan(g.nx, 32), psi, g.nx, g.ny, 1, +1, 1.0 / (double)N, ctx.stream, &ctx.launches);
}

// The scratch for the table's probes: sized for the largest probe grid, and every job's position on the device.
void probe_scratch(Context& ctx, const std::vector<JobSpec>& jobs, ProbeScratch& sc) {
    long long n_max = 0;
    int nx_max = 0, ny_max = 0;
    std::vector<double> xy(2 * jobs.size());
    for (size_t i = 0; i < jobs.size(); ++i) {
        xy[2 * i] = jobs[i].x;
        xy[2 * i + 1] = jobs[i].y;
        if (!jobs[i].probe) continue;
        n_max = std::max(n_max, jobs[i].pot->g.count());
        nx_max = std::max(nx_max, jobs[i].pot->g.nx);
        ny_max = std::max(ny_max, jobs[i].pot->g.ny);
    }
    if (n_max == 0) return;
    sc.spectrum.ensure(n_max * sizeof(float2));
    sc.tmp.ensure(n_max * sizeof(double2));
    sc.norm.ensure(sizeof(double));
    sc.rx.ensure(nx_max * sizeof(float2));
    sc.ry.ensure(ny_max * sizeof(float2));
    sc.positions.ensure(xy.size() * sizeof(double));
    SIMK_CUDA(cudaMemcpyAsync(sc.positions.ptr, xy.data(), xy.size() * sizeof(double), cudaMemcpyHostToDevice,
                              ctx.stream));
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));  // the host copy of the positions is freed on return
}

// One grid shape's jobs in a fused job-table run: their waves, intensities, per-step tables and stream.
struct GroupRun {
    std::vector<int> ids;     // job indices, longest first
    std::vector<int> slices;  // their slice counts
    int G = 0, S = 0, nx = 0, ny = 0, first_in_order = 0, pblocks = 0;
    long long N = 0;
    DeviceBuffer waves, inten, pstack, dt, dp;
    cudaStream_t stream = nullptr;
};

// The groups' streams and their start event: on exit (also by an exception) the context's stream is restored, every
// stream drained and destroyed.
struct StreamsScope {
    Context& c;
    cudaStream_t home;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> events;
    ~StreamsScope() {
        c.stream = home;
        for (auto st : streams) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        for (auto e : events) cudaEventDestroy(e);
    }
};

// A job table's capture: on exit by an exception during the capture the capture is ended and its graph dropped, so the
// streams can be drained; the instantiated graph is destroyed with it.
struct TableGraph {
    cudaStream_t origin = nullptr;
    bool capturing = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ~TableGraph() {
        if (capturing) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(origin, &g);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();  // an invalidated capture leaves its error behind
        }
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

// The last fused job table captured as a graph, kept in the context for a call with the same jobs: its groups'
// buffers and tables, the instantiated graph and the events its nodes record. A repeat then computes the incident
// waves into the same buffers and launches the graph again, without capturing or instantiating it.
struct TableCache {
    std::vector<GroupRun> runs;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaEvent_t> events;
    std::vector<std::pair<int, int>> event_jobs;
    std::vector<int> order;
    long long kernels = 0;
    ~TableCache() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto e : events) cudaEventDestroy(e);
    }
};

// Everything the captured schedule depends on: the settings that choose its kernels, and per job the potential (its
// address, transmissions, grid, slice thicknesses), energy, incident wave and position.
std::string table_key(const Context& ctx, const std::vector<JobSpec>& jobs) {
    std::string k;
    auto add = [&](const void* p, size_t n) { k.append(static_cast<const char*>(p), n); };
    const int opts[] = {ctx.form, ctx.tma, ctx.col_tile, ctx.composite, ctx.tcgen05, ctx.paired};
    add(opts, sizeof(opts));
    for (const JobSpec& j : jobs) {
        const void* ids[] = {j.pot, j.pot->t.ptr};
        add(ids, sizeof(ids));
        const double geo[] = {(double)j.pot->g.nx, (double)j.pot->g.ny, j.pot->g.ex, j.pot->g.ey, j.energy,
                              j.probe ? 1.0 : 0.0, j.x, j.y};
        add(geo, sizeof(geo));
        add(j.pot->dz.data(), j.pot->dz.size() * sizeof(double));
        if (j.probe) add(&j.probe_spec, sizeof(j.probe_spec));
    }
    return k;
}

// Resets the context's wave table when a job run ends, also by an exception.
struct WaveTableScope {
    Context& c;
    ~WaveTableScope() {
        c.wave_t = nullptr;
        c.wave_p = nullptr;
        c.wave_p_blocks = 0;
    }
};
}  // namespace

void run_job_table(Context& ctx, const std::vector<JobSpec>& jobs, double* done_ms) {
    const int n = (int)jobs.size();
    if (n == 0) return;
    std::map<const PotentialImpl*, double> energy_of;
    for (int i = 0; i < n; ++i) {
        const JobSpec& j = jobs[i];
        SIMK_REQUIRE(j.pot && j.intensity, "job " + std::to_string(i) + ": null potential or output");
        SIMK_REQUIRE(std::isfinite(j.energy) && j.energy > 0, "job " + std::to_string(i) + ": energy must be > 0");
        SIMK_REQUIRE(!j.probe || (std::isfinite(j.x) && std::isfinite(j.y)), "job " + std::to_string(i) +
                                                                               ": invalid probe position");
        auto it = energy_of.find(j.pot);
        SIMK_REQUIRE(it == energy_of.end() || it->second == j.energy,
                     "job " + std::to_string(i) + ": a potential shared by jobs of different energies");
        energy_of[j.pot] = j.energy;
    }
    for (auto& kv : energy_of) prepare_transmissions(ctx, *const_cast<PotentialImpl*>(kv.first), kv.second);
    const bool capture = ctx.form != SIMK_FORM_PLAIN && ctx.graphs && !ctx.timing;
    const std::string key = capture ? table_key(ctx, jobs) : std::string();
    if (capture && ctx.table_cache && ctx.table_cache_key == key) {
        // the same jobs again: their incident waves into the kept buffers, and one launch of the kept graph
        TableCache& tc = *static_cast<TableCache*>(ctx.table_cache.get());
        ProbeScratch sc;
        probe_scratch(ctx, jobs, sc);
        cudaEvent_t start;
        SIMK_CUDA(cudaEventCreate(&start));
        try {
            SIMK_CUDA(cudaEventRecord(start, ctx.stream));
            for (auto& gr : tc.runs)
                for (int w = 0; w < gr.G; ++w)
                    incident_wave(ctx, jobs[gr.ids[w]], gr.ids[w], sc, gr.waves.as<float2>() + (long long)w * gr.N);
            SIMK_CUDA(cudaGraphLaunch(tc.exec, ctx.stream));
            for (auto& gr : tc.runs)
                for (int w = 0; w < gr.G; ++w)
                    SIMK_CUDA(cudaMemcpyAsync(jobs[gr.ids[w]].intensity, gr.inten.as<double>() + (long long)w * gr.N,
                                              gr.N * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
            SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
            check_device_error(ctx);
            for (size_t k = 0; k < tc.events.size(); ++k) {
                float ms = 0;
                SIMK_CUDA(cudaEventElapsedTime(&ms, start, tc.events[k]));
                if (done_ms)
                    for (int q = tc.event_jobs[k].first; q < tc.event_jobs[k].second; ++q) done_ms[tc.order[q]] = ms;
            }
        } catch (...) {
            cudaStreamSynchronize(ctx.stream);
            cudaEventDestroy(start);
            throw;
        }
        cudaEventDestroy(start);
        ctx.table_launches = 1;
        ctx.table_kernels = tc.kernels;
        ctx.table_shapes = (int)tc.runs.size();
        return;
    }
    ctx.table_cache.reset();  // another table: the kept one's buffers go before this one's are allocated
    ctx.table_cache_key.clear();
    // the groups: jobs of one grid shape, longest first
    std::map<std::pair<int, int>, std::vector<int>> groups;
    for (int i = 0; i < n; ++i) groups[{jobs[i].pot->g.nx, jobs[i].pot->g.ny}].push_back(i);
    for (auto& kv : groups)
        std::stable_sort(kv.second.begin(), kv.second.end(), [&](int a, int b) {
            return jobs[a].pot->n_slices() > jobs[b].pot->n_slices();
        });
    auto tilt = [&](const JobSpec& j, int k) {
        return j.probe ? (k == 0 ? j.probe_spec.tilt_x : j.probe_spec.tilt_y) : 0.0;
    };
    ProbeScratch probes;  // the incident probes' buffers, kept to the end of the call
    probe_scratch(ctx, jobs, probes);
    cudaEvent_t start;
    SIMK_CUDA(cudaEventCreate(&start));
    std::vector<cudaEvent_t> events;
    std::vector<std::pair<int, int>> event_jobs;  // (first, last) indices into `order` completed at each event
    std::vector<int> order;
    SIMK_CUDA(cudaEventRecord(start, ctx.stream));
    WaveTableScope scope{ctx};
    std::vector<GroupRun> runs;  // the fused form's groups, set up first, then advanced side by side
    runs.reserve(groups.size());
    cudaGraph_t table_graph = nullptr;  // the captured schedule, until the context keeps it
    cudaGraphExec_t table_exec = nullptr;
    auto drop_graph = [&] {
        if (table_exec) cudaGraphExecDestroy(table_exec);
        if (table_graph) cudaGraphDestroy(table_graph);
        table_exec = nullptr;
        table_graph = nullptr;
    };
    try {
        for (auto& kv : groups) {
            const std::vector<int>& ids = kv.second;
            const int G = (int)ids.size();
            const GridGeom& g0 = jobs[ids[0]].pot->g;
            const long long N = g0.count();
            const int nx = g0.nx, ny = g0.ny;
            const int S = jobs[ids[0]].pot->n_slices();
            DeviceBuffer waves((size_t)G * N * sizeof(float2)), inten((size_t)G * N * sizeof(double));
            float2* psi = waves.as<float2>();
            for (int w = 0; w < G; ++w) incident_wave(ctx, jobs[ids[w]], ids[w], probes, psi + (long long)w * N);
            const int first_in_order = (int)order.size();
            order.insert(order.end(), ids.begin(), ids.end());
            if (ctx.form == SIMK_FORM_PLAIN) {
                // the sequential baseline: each job alone through the plain path
                for (int w = 0; w < G; ++w) {
                    const JobSpec& j = jobs[ids[w]];
                    propagate_plain(ctx, *j.pot, j.energy, tilt(j, 0), tilt(j, 1), psi + (long long)w * N, 1, true,
                                    nullptr);
                    k_intensity<<<grid_for(N), 256, 0, ctx.stream>>>(psi + (long long)w * N, N,
                                                                      inten.as<double>() + (long long)w * N);
                    ++ctx.launches;
                    cudaEvent_t e;
                    SIMK_CUDA(cudaEventCreate(&e));
                    SIMK_CUDA(cudaEventRecord(e, ctx.stream));
                    events.push_back(e);
                    event_jobs.push_back({first_in_order + w, first_in_order + w + 1});
                }
                for (int w = 0; w < G; ++w)
                    SIMK_CUDA(cudaMemcpyAsync(jobs[ids[w]].intensity, inten.as<double>() + (long long)w * N,
                                              N * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
                SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
                continue;
            }
            // per step: each wave's transmission slice and propagator block
            GroupRun& gr = runs.emplace_back();
            gr.ids = ids;
            gr.G = G;
            gr.S = S;
            gr.N = N;
            gr.nx = nx;
            gr.ny = ny;
            gr.first_in_order = first_in_order;
            gr.waves = std::move(waves);
            gr.inten = std::move(inten);
            std::vector<const float2*> tptr((size_t)S * G, nullptr);
            std::vector<int> prow((size_t)S * G, 0);
            std::vector<const float2*> pblocks;
            std::map<const float2*, int> block_of;
            for (int w = 0; w < G; ++w) {
                const JobSpec& j = jobs[ids[w]];
                for (int s = 0; s < j.pot->n_slices(); ++s) {
                    tptr[(size_t)s * G + w] = j.pot->t.as<float2>() + (long long)s * N;
                    const float2* P = ctx.propagator(j.pot->g, j.energy, j.pot->dz[s], tilt(j, 0), tilt(j, 1))
                                          .p.as<float2>();
                    auto it = block_of.find(P);
                    if (it == block_of.end()) {
                        it = block_of.emplace(P, (int)pblocks.size()).first;
                        pblocks.push_back(P);
                    }
                    prow[(size_t)s * G + w] = it->second;
                }
            }
            gr.pblocks = (int)pblocks.size();
            gr.pstack.alloc(pblocks.size() * N * sizeof(float2));
            gr.dt.alloc(tptr.size() * sizeof(float2*));
            gr.dp.alloc(prow.size() * sizeof(int));
            for (size_t b = 0; b < pblocks.size(); ++b)
                SIMK_CUDA(cudaMemcpyAsync(gr.pstack.as<float2>() + (long long)b * N, pblocks[b], N * sizeof(float2),
                                          cudaMemcpyDeviceToDevice, ctx.stream));
            SIMK_CUDA(cudaMemcpyAsync(gr.dt.ptr, tptr.data(), tptr.size() * sizeof(float2*), cudaMemcpyHostToDevice,
                                      ctx.stream));
            SIMK_CUDA(cudaMemcpyAsync(gr.dp.ptr, prow.data(), prow.size() * sizeof(int), cudaMemcpyHostToDevice,
                                      ctx.stream));
            gr.slices.resize(G);
            for (int w = 0; w < G; ++w) gr.slices[w] = jobs[ids[w]].pot->n_slices();
            SIMK_CUDA(cudaStreamSynchronize(ctx.stream));  // the host tables above are freed on return
        }
        // The groups' slice steps, each group on its own stream so that the shapes run side by side (the launches of a
        // step depend only on the same group's previous step): step s of every group still running, in turn. With
        // SIMK_OPT_GRAPHS (and no per-kernel timing) the whole schedule, every shape and step, the finishing row
        // passes and the intensities, is captured as one CUDA graph and run by one launch.
        if (!runs.empty()) {
            cudaStream_t home = ctx.stream;
            StreamsScope streams{ctx, home};
            for (auto& gr : runs) {
                cudaStream_t st;
                SIMK_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
                streams.streams.push_back(st);
                gr.stream = st;
            }
            // what the launches create on first use exists before a capture: the plans and the error flag
            for (auto& gr : runs) {
                reg_plan(ctx, gr.nx);
                reg_plan(ctx, gr.ny);
            }
            ensure_err_flag(ctx);
            TableGraph tg;
            tg.origin = home;
            if (capture) {
                SIMK_CUDA(cudaStreamBeginCapture(home, cudaStreamCaptureModeRelaxed));
                tg.capturing = true;
            }
            const long long launches0 = ctx.launches;
            cudaEvent_t go;
            SIMK_CUDA(cudaEventCreateWithFlags(&go, cudaEventDisableTiming));
            streams.events.push_back(go);
            SIMK_CUDA(cudaEventRecord(go, home));
            for (auto& gr : runs) SIMK_CUDA(cudaStreamWaitEvent(gr.stream, go, 0));
            int max_s = 0;
            for (auto& gr : runs) max_s = std::max(max_s, gr.S);
            for (int s = 0; s < max_s; ++s) {
                for (auto& gr : runs) {
                    if (s >= gr.S) continue;
                    ctx.stream = gr.stream;
                    const int G = gr.G;
                    auto active = [&](int ss) {  // jobs with more than ss slices: a prefix
                        int a = 0;
                        while (a < G && gr.slices[a] > ss) ++a;
                        return a;
                    };
                    const int A = active(s);
                    const RegPlan prw = reg_plan(ctx, gr.ny);
                    const RegPlan pcl = reg_plan(ctx, gr.nx);
                    float2* psi = gr.waves.as<float2>();
                    ctx.wave_t = gr.dt.as<const float2*>() + (size_t)s * G;
                    ctx.wave_p = gr.dp.as<int>() + (size_t)s * G;
                    ctx.wave_p_blocks = gr.pblocks;
                    launch_rows(ctx, prw, psi, nullptr, gr.nx, (long long)A * gr.nx, s > 0 ? 1 : 0, 1, 1.0f);
                    ColArgs a{};
                    a.psi = psi;
                    a.P = gr.pstack.as<float2>();
                    a.ny = gr.ny;
                    a.mode = 0;
                    a.pscale = 1.0f / (float)gr.N;
                    launch_cols(ctx, pcl, a, A);
                    ctx.wave_t = nullptr;
                    ctx.wave_p = nullptr;
                    ctx.wave_p_blocks = 0;
                    const int A1 = active(s + 1);
                    if (A1 == A) continue;
                    // jobs A1 .. A-1 have ended: complete their row inverse transform, intensities out
                    const GridGeom g1{gr.nx, gr.ny, 0.0, 0.0};
                    finish_rows(ctx, g1, psi + (long long)A1 * gr.N, A - A1);
                    k_intensity<<<grid_for((long long)(A - A1) * gr.N), 256, 0, ctx.stream>>>(
                        psi + (long long)A1 * gr.N, (long long)(A - A1) * gr.N, gr.inten.as<double>() + (long long)A1 * gr.N);
                    ++ctx.launches;
                    cudaEvent_t e;
                    SIMK_CUDA(cudaEventCreate(&e));
                    // inside a capture an external record becomes a node of the graph that records the event
                    SIMK_CUDA(cudaEventRecordWithFlags(e, ctx.stream, capture ? cudaEventRecordExternal : 0));
                    events.push_back(e);
                    event_jobs.push_back({gr.first_in_order + A1, gr.first_in_order + A});
                }
            }
            ctx.stream = home;
            for (auto& gr : runs) {  // every group's stream joins the origin stream
                cudaEvent_t j;
                SIMK_CUDA(cudaEventCreateWithFlags(&j, cudaEventDisableTiming));
                streams.events.push_back(j);
                SIMK_CUDA(cudaEventRecord(j, gr.stream));
                SIMK_CUDA(cudaStreamWaitEvent(home, j, 0));
            }
            ctx.table_kernels = ctx.launches - launches0;
            ctx.table_shapes = (int)runs.size();
            if (capture) {
                tg.capturing = false;
                SIMK_CUDA(cudaStreamEndCapture(home, &tg.graph));
                SIMK_CUDA(cudaGraphInstantiate(&tg.exec, tg.graph, 0));
                SIMK_CUDA(cudaGraphLaunch(tg.exec, home));
                ctx.table_launches = 1;
                table_graph = tg.graph;  // from here on owned by this call (then by the context's cache)
                table_exec = tg.exec;
                tg.graph = nullptr;
                tg.exec = nullptr;
            } else {
                ctx.table_launches = ctx.table_kernels;
            }
            for (auto& gr : runs) {
                for (int w = 0; w < gr.G; ++w)
                    SIMK_CUDA(cudaMemcpyAsync(jobs[gr.ids[w]].intensity, gr.inten.as<double>() + (long long)w * gr.N,
                                              gr.N * sizeof(double), cudaMemcpyDeviceToHost, home));
            }
            SIMK_CUDA(cudaStreamSynchronize(home));
        }
        SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
        check_device_error(ctx);
        for (size_t k = 0; k < events.size(); ++k) {
            float ms = 0;
            SIMK_CUDA(cudaEventElapsedTime(&ms, start, events[k]));
            if (done_ms)
                for (int q = event_jobs[k].first; q < event_jobs[k].second; ++q) done_ms[order[q]] = ms;
        }
        if (table_exec) {
            // kept for a call with the same jobs: the groups' buffers, the graph and the events its nodes record
            auto tc = std::make_shared<TableCache>();
            tc->runs = std::move(runs);
            tc->graph = table_graph;
            tc->exec = table_exec;
            tc->events = std::move(events);
            tc->event_jobs = std::move(event_jobs);
            tc->order = std::move(order);
            tc->kernels = ctx.table_kernels;
            events.clear();
            table_graph = nullptr;
            table_exec = nullptr;
            ctx.table_cache = std::static_pointer_cast<void>(tc);
            ctx.table_cache_key = key;
        }
    } catch (...) {
        drop_graph();
        cudaStreamSynchronize(ctx.stream);
        for (auto e : events) cudaEventDestroy(e);
        cudaEventDestroy(start);
        throw;
    }
    for (auto e : events) cudaEventDestroy(e);
    cudaEventDestroy(start);
}

}  // namespace simk
