// fft.cuh -- batched complex line FFTs for sm_100a: radix butterflies, the shared-memory Stockham pass (any length,
// Bluestein's chirp-z for large prime factors), and the host-side plans.
//
// Conventions are NumPy's (Sources/SimulatoCore/FFT2D.swift:1-8): forward unnormalised with e^{-2 pi i jk/n},
// inverse with e^{+2 pi i jk/n}; the caller applies 1/(nx ny). The Stockham autosort pass with radix R after Ns
// points have been combined reads v[r] = a[j + r n/R], twiddles v[r] by W_n^{(j mod Ns) r n/(Ns R)}, takes the
// R-point DFT and writes b[(j - j mod Ns) R + j mod Ns + r Ns]. Twiddles come from tables computed in float64 from
// exact integer phases (as MixedRadixPlan.swift:72-99 does) and rounded once.
#pragma once

#include "common.cuh"

namespace simk {

constexpr int kMaxFactors = 24;
constexpr int kMaxGenericRadix = 64;

// ---- butterflies, DIR = -1 forward, +1 inverse ----------------------------------------------------------------------
template <int DIR, typename V> __device__ __forceinline__ void bfly2(V* v) {
    V a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
}
template <int DIR, typename V> __device__ __forceinline__ void bfly4(V* v) {
    V a = v[0] + v[2], b = v[0] - v[2], c = v[1] + v[3], d = mul_si(v[1] - v[3], DIR);
    v[0] = a + c;
    v[2] = a - c;
    v[1] = b + d;
    v[3] = b - d;
}
template <int DIR, typename V> __device__ __forceinline__ void bfly3(V* v) {
    using R = decltype(V::x);
    const R h = (R)0.86602540378443864676;  // sin(2 pi / 3)
    V t1 = v[1] + v[2];
    V t2 = v[0] - t1 * (R)0.5;
    V t3 = mul_si(v[1] - v[2], (R)DIR * h);
    v[0] = v[0] + t1;
    v[1] = t2 + t3;
    v[2] = t2 - t3;
}
template <int DIR, typename V> __device__ __forceinline__ void bfly5(V* v) {
    using R = decltype(V::x);
    const R c1 = (R)0.30901699437494742410, c2 = (R)-0.80901699437494742410;  // cos(2pi/5), cos(4pi/5)
    const R s1 = (R)0.95105651629515357212, s2 = (R)0.58778525229247312917;   // sin(2pi/5), sin(4pi/5)
    V a1 = v[1] + v[4], b1 = v[1] - v[4], a2 = v[2] + v[3], b2 = v[2] - v[3];
    V x0 = v[0];
    V p1 = x0 + a1 * c1 + a2 * c2;
    V p2 = x0 + a1 * c2 + a2 * c1;
    V q1 = mul_si(b1 * s1 + b2 * s2, (R)DIR);
    V q2 = mul_si(b1 * s2 - b2 * s1, (R)DIR);
    v[0] = x0 + a1 + a2;
    v[1] = p1 + q1;
    v[4] = p1 - q1;
    v[2] = p2 + q2;
    v[3] = p2 - q2;
}
template <int DIR, typename V> __device__ __forceinline__ void bfly8(V* v) {
    using R = decltype(V::x);
    const R c = (R)0.70710678118654752440;
    V e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    bfly4<DIR>(e);
    bfly4<DIR>(o);
    V o1 = mk<V>((o[1].x - DIR * o[1].y) * c, (o[1].y + DIR * o[1].x) * c);
    V o2 = mul_si(o[2], (R)DIR);
    V o3 = mk<V>((-o[3].x - DIR * o[3].y) * c, (-o[3].y + DIR * o[3].x) * c);
    v[0] = e[0] + o[0];
    v[4] = e[0] - o[0];
    v[1] = e[1] + o1;
    v[5] = e[1] - o1;
    v[2] = e[2] + o2;
    v[6] = e[2] - o2;
    v[3] = e[3] + o3;
    v[7] = e[3] - o3;
}
template <int DIR, typename V> __device__ __forceinline__ void bfly16(V* v) {
    using R = decltype(V::x);
    const R c1 = (R)0.92387953251128675613, s1 = (R)0.38268343236508977173, c2 = (R)0.70710678118654752440;
    V e[8], o[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        e[i] = v[2 * i];
        o[i] = v[2 * i + 1];
    }
    bfly8<DIR>(e);
    bfly8<DIR>(o);
    const R wr[8] = {(R)1, c1, c2, s1, (R)0, -s1, -c2, -c1};
    const R wi[8] = {(R)0, s1, c2, c1, (R)1, c1, c2, s1};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        V w = mk<V>(wr[k], (R)DIR * wi[k]);
        V t = (k == 0) ? o[0] : cmul(o[k], w);
        v[k] = e[k] + t;
        v[k + 8] = e[k] - t;
    }
}
// ---- float32 butterflies on packed pairs ------------------------------------------------------------------------------
// sm_100's add/sub/mul/fma.rn.f32x2 take a complex value as one 64-bit register pair, so a complex add is one
// instruction instead of two. Multiplication by +-i becomes the swapped pair times (-+1, +-1) inside one packed FMA:
// the products are exact, so every lane rounds as the scalar forms above do and the results are the same bits. These
// overloads are more specialised than the templates above and serve every float2 butterfly of radix 2, 4 and 8.
__device__ __forceinline__ unsigned long long pk(float2 a) {
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
    return r;
}
__device__ __forceinline__ float2 upk(unsigned long long r) {
    float2 a;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
    return a;
}
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
    return upk(r);
}
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
    return upk(r);
}
__device__ __forceinline__ float2 pmul(float2 a, float2 b) {
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)));
    return upk(r);
}
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) {
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(pk(a)), "l"(pk(b)), "l"(pk(c)));
    return upk(r);
}
__device__ __forceinline__ float2 swp(float2 a) { return make_float2(a.y, a.x); }

template <int DIR> __device__ __forceinline__ void bfly2(float2* v) {
    const float2 a = v[0], b = v[1];
    v[0] = padd(a, b);
    v[1] = psub(a, b);
}
template <int DIR> __device__ __forceinline__ void bfly4(float2* v) {
    const float2 a = padd(v[0], v[2]), b = psub(v[0], v[2]), c = padd(v[1], v[3]), e = psub(v[1], v[3]);
    // d = (v1 - v3) i DIR = (-DIR e.y, DIR e.x): b +- d = (e.y, e.x) (-+DIR, +-DIR) + b
    const float2 es = swp(e);
    v[0] = padd(a, c);
    v[2] = psub(a, c);
    v[1] = pfma(es, make_float2((float)-DIR, (float)DIR), b);
    v[3] = pfma(es, make_float2((float)DIR, (float)-DIR), b);
}
template <int DIR> __device__ __forceinline__ void bfly8(float2* v) {
    const float c = 0.70710678118654752440f;
    float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    bfly4<DIR>(e);
    bfly4<DIR>(o);
    // o1 = ((o.x - DIR o.y) c, (o.y + DIR o.x) c); o3 = ((-o.x - DIR o.y) c, (-o.y + DIR o.x) c)
    //    = ((o.x + DIR o.y) (-c), (o.y - DIR o.x) (-c))
    const float2 o1 = pmul(pfma(swp(o[1]), make_float2((float)-DIR, (float)DIR), o[1]), make_float2(c, c));
    const float2 o3 = pmul(pfma(swp(o[3]), make_float2((float)DIR, (float)-DIR), o[3]), make_float2(-c, -c));
    v[0] = padd(e[0], o[0]);
    v[4] = psub(e[0], o[0]);
    v[1] = padd(e[1], o1);
    v[5] = psub(e[1], o1);
    // e2 +- o2, o2 = o[2] i DIR
    const float2 s2 = swp(o[2]);
    v[2] = pfma(s2, make_float2((float)-DIR, (float)DIR), e[2]);
    v[6] = pfma(s2, make_float2((float)DIR, (float)-DIR), e[2]);
    v[3] = padd(e[3], o3);
    v[7] = psub(e[3], o3);
}

// The p-point DFT by its definition, for odd prime radices (7, 11, ...): W_p^{rq} from a table of cos/sin(2 pi k/p).
template <int DIR, typename V>
__device__ __forceinline__ void dft_direct(V* v, int R, const double* ctab, const double* stab) {
    using Rt = decltype(V::x);
    V out[kMaxGenericRadix];
    for (int q = 0; q < R; ++q) {
        V acc = v[0];
        int e = 0;
        for (int r = 1; r < R; ++r) {
            e += q;
            if (e >= R) e -= R;
            V w = mk<V>((Rt)ctab[e], (Rt)DIR * (Rt)stab[e]);
            acc = acc + cmul(v[r], w);
        }
        out[q] = acc;
    }
    for (int q = 0; q < R; ++q) v[q] = out[q];
}

// ---- plans ----------------------------------------------------------------------------------------------------------
// Device view of a line plan, passed by value.
struct LinePlanDev {
    int n;          // line length
    int m;          // work length: n, or Bluestein's padded power of two
    int nfac;       // passes over the work length
    int bluestein;  // 1: chirp-z
    int fac[kMaxFactors];
    const void* tw;      // m entries W_m^k = e^{-2 pi i k/m}, complex of the plan's precision
    const void* chirp;   // n entries e^{-i pi (k^2 mod 2n)/n} (Bluestein)
    const void* khat;    // m entries: the DFT of the conjugate chirp kernel, divided by m (Bluestein)
    const double* rad_cos;  // per generic radix p: cos(2 pi k / p), k < p, packed at rad_off[pass]
    const double* rad_sin;
    int rad_off[kMaxFactors];
};

struct LinePlan {
    int n = 0, m = 0, precision = 32;
    bool bluestein = false;
    std::vector<int> factors;
    DeviceBuffer tw, chirp, khat, rad_cos, rad_sin;
    std::vector<int> rad_off;
    LinePlanDev dev() const;
};

// Radices of a length for the GPU (16, 8, 4, 2, then 3, 5, 7, then other primes <= kMaxGenericRadix); empty when a
// prime factor is larger (Bluestein).
std::vector<int> gpu_factorization(int n);
std::unique_ptr<LinePlan> make_line_plan(int n, int precision);

// Launch a batched line transform in place: line l (0 <= l < nlines) starts at
// (l / lines_per_batch) * batch_stride + (l % lines_per_batch) * line_stride, element e at + e * elem_stride.
// dir = -1 forward, +1 inverse (unnormalised); every output is multiplied by `scale`.
void launch_line_fft(const LinePlan& plan, void* data, long long nlines, int lines_per_batch, long long line_stride,
                     long long elem_stride, long long batch_stride, int dir, double scale, cudaStream_t stream,
                     int64_t* launches);

// 2-D transform of `count` nx x ny fields in place: rows (along y) then columns (along x).
void fft2(const LinePlan& row_plan, const LinePlan& col_plan, void* data, int nx, int ny, long long count, int dir,
          double scale, cudaStream_t stream, int64_t* launches);

// ---- the generic shared-memory Stockham pass, used by the kernels in fft.cu and engine.cu --------------------------
template <int DIR, int R, typename V>
__device__ __forceinline__ void stockham_pass_fixed(const V* __restrict__ src, V* __restrict__ dst, int n, int Ns,
                                                    const V* __restrict__ tw, int lines, int lds, int tid,
                                                    int nthreads) {
    const int nb = n / R;
    const int tstride = n / (Ns * R);
    for (int t = tid; t < lines * nb; t += nthreads) {
        const int l = t / nb;
        const int j = t - l * nb;
        const int k = j % Ns;
        const V* s = src + l * lds;
        V* d = dst + l * lds;
        V v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = s[j + r * nb];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                V w = tw[k * r * tstride];
                v[r] = (DIR < 0) ? cmul(v[r], w) : cmulc(v[r], w);
            }
        }
        if (R == 2) bfly2<DIR>(v);
        else if (R == 3) bfly3<DIR>(v);
        else if (R == 4) bfly4<DIR>(v);
        else if (R == 5) bfly5<DIR>(v);
        else if (R == 8) bfly8<DIR>(v);
        else if (R == 16) bfly16<DIR>(v);
        const int o = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) d[o + r * Ns] = v[r];
    }
}

template <int DIR, typename V>
__device__ __forceinline__ void stockham_pass_generic(const V* __restrict__ src, V* __restrict__ dst, int n, int Ns,
                                                      int R, const V* __restrict__ tw, const double* ctab,
                                                      const double* stab, int lines, int lds, int tid, int nthreads) {
    const int nb = n / R;
    const int tstride = n / (Ns * R);
    for (int t = tid; t < lines * nb; t += nthreads) {
        const int l = t / nb;
        const int j = t - l * nb;
        const int k = j % Ns;
        const V* s = src + l * lds;
        V* d = dst + l * lds;
        V v[kMaxGenericRadix];
        for (int r = 0; r < R; ++r) v[r] = s[j + r * nb];
        if (Ns > 1)
            for (int r = 1; r < R; ++r) {
                V w = tw[k * r * tstride];
                v[r] = (DIR < 0) ? cmul(v[r], w) : cmulc(v[r], w);
            }
        dft_direct<DIR>(v, R, ctab, stab);
        const int o = (j - k) * R + k;
        for (int r = 0; r < R; ++r) d[o + r * Ns] = v[r];
    }
}

// All passes of one transform of length plan.m over `lines` lines in shared memory. Input in a, scratch b; returns
// the buffer that holds the result. Ends with a __syncthreads().
template <int DIR, typename V>
__device__ V* stockham_lines(V* a, V* b, const LinePlanDev& p, int lines, int lds) {
    const V* tw = static_cast<const V*>(p.tw);
    const int tid = threadIdx.x, nth = blockDim.x;
    int Ns = 1;
    for (int f = 0; f < p.nfac; ++f) {
        const int R = p.fac[f];
        switch (R) {
            case 2: stockham_pass_fixed<DIR, 2>(a, b, p.m, Ns, tw, lines, lds, tid, nth); break;
            case 3: stockham_pass_fixed<DIR, 3>(a, b, p.m, Ns, tw, lines, lds, tid, nth); break;
            case 4: stockham_pass_fixed<DIR, 4>(a, b, p.m, Ns, tw, lines, lds, tid, nth); break;
            case 5: stockham_pass_fixed<DIR, 5>(a, b, p.m, Ns, tw, lines, lds, tid, nth); break;
            case 8: stockham_pass_fixed<DIR, 8>(a, b, p.m, Ns, tw, lines, lds, tid, nth); break;
            case 16: stockham_pass_fixed<DIR, 16>(a, b, p.m, Ns, tw, lines, lds, tid, nth); break;
            default:
                stockham_pass_generic<DIR>(a, b, p.m, Ns, R, tw, p.rad_cos + p.rad_off[f], p.rad_sin + p.rad_off[f],
                                           lines, lds, tid, nth);
        }
        __syncthreads();
        V* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

}  // namespace simk
