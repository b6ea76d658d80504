// surrogate.cu -- a small MLP that stands in for the per-(atom, slice) quadrature of the finite-projection potential.
//
// The network C(Z, rho, z) is a cumulative profile: with the element's 16-float embedding and the features
// ((log rho + 1.5) / 2, asinh(z / rho) / 4) -- the radius and one slice edge in the u variable of finite.cu's
// quadrature -- it returns the share of the infinite projection below z, so that
//     P(rho; zl, zu) = P_inf(rho) (C(Z, rho, zu) - C(Z, rho, zl)),
// P_inf the analytic infinite projection. Slices therefore add exactly, and the loss is the absolute error of the
// fraction F = P / P_inf, i.e. of P in units of the full projection at that radius -- the error that matters for the
// summed potential. Network: 18 -> 64 -> 64 -> 64 -> 1 with SiLU.
// Training (on the device, by the kernels below): samples drawn uniformly in log rho, zl and the slab thickness inside
// the trained domain, labelled by the float64 quadrature itself; each sample runs the network at both edges (rows b and
// B + b of a doubled batch) and back-propagates +dF and -dF; mean-squared error; Adam. A training step is two launches:
// k_sg_train runs the forward and backward pass of 32 samples per block with every contraction on the tensor cores
// (mma.sync TF32, operands split in two terms: float32 accuracy) and writes the block's gradient; k_sg_reduce_adam adds
// the blocks' gradients in block order and takes the Adam step. Every reduction runs in a fixed order, so training is
// deterministic for a seed. Inference: tensor-core tiles of 16 queries per warp (k_sg_infer), f16 weights and
// activations (SiLU in f16x2), float32 accumulation.
//
// Parameter layout (float32, kSurrogateParams values): emb[103][16] | W1[64][18] b1[64] | W2[64][64] b2[64] |
// W3[64][64] b3[64] | W4[64] b4[1].
#include <algorithm>
#include <cmath>
#include <cuda_fp16.h>
#include <random>

#include "finite.cuh"
#include "surrogate.cuh"

namespace simk {

namespace {
constexpr int OFF_EMB = 0;
constexpr int OFF_W1 = OFF_EMB + 103 * kEmbed;
constexpr int OFF_B1 = OFF_W1 + kHidden * kIn;
constexpr int OFF_W2 = OFF_B1 + kHidden;
constexpr int OFF_B2 = OFF_W2 + kHidden * kHidden;
constexpr int OFF_W3 = OFF_B2 + kHidden;
constexpr int OFF_B3 = OFF_W3 + kHidden * kHidden;
constexpr int OFF_W4 = OFF_B3 + kHidden;
constexpr int OFF_B4 = OFF_W4 + kHidden;
static_assert(OFF_B4 + 1 == kSurrogateParams, "parameter layout");

inline int blocks_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 32)); }

__device__ __forceinline__ float silu(float x) { return x / (1.0f + __expf(-x)); }
__device__ __forceinline__ float silu_grad(float x) {
    const float s = 1.0f / (1.0f + __expf(-x));
    return s * (1.0f + x * (1.0f - s));
}
}  // namespace

__host__ __device__ inline void surrogate_features(double rho, double z, float* f) {
    f[0] = (float)((log(rho) + 1.5) / 2.0);
    f[1] = (float)(asinh(z / rho) / 4.0);
}

// ---- training: one fused forward + backward per block of samples, on the tensor cores ----------------------------
// A block takes kTrSamples samples: rows 0 .. kTrSamples - 1 are their upper-edge rows, the next kTrSamples their
// lower-edge rows. Every contraction of the forward and backward pass is a warp-level tensor-core product
// (mma.sync m16n8k8, TF32 operands split in two terms, x = x_hi + x_lo, with the three products hi hi + hi lo + lo hi:
// float32 accuracy), from float32 operands in shared memory. The block writes the gradient of its samples for every
// parameter to its own row of `partial`; k_sg_reduce_adam adds the rows in block order (fixed, so training is
// deterministic for a seed) and takes the Adam step.
constexpr int kTrSamples = 32;
constexpr int kTrRows = 2 * kTrSamples;
constexpr int kTrThreads = 256;
constexpr int kTrWarps = kTrThreads / 32;
constexpr int kIn8 = 24;          // layer-1 inputs padded to whole k-steps of 8
constexpr int kLdH = kHidden + 4; // row pitch of [row][64] buffers (4 mod 32: conflict-free fragment loads)
constexpr int kLd1 = kIn8 + 4;    // row pitch of [row][24] buffers
// shared memory, in floats
constexpr int kTrW1 = 0;                            // W1 [64][kLd1] (inputs 18 .. 23 zero)
constexpr int kTrW2 = kTrW1 + kHidden * kLd1;       // W2 [64][kLdH]
constexpr int kTrW3 = kTrW2 + kHidden * kLdH;       // W3 [64][kLdH]
constexpr int kTrVec = kTrW3 + kHidden * kLdH;      // b1 b2 b3 W4 [64 each], b4
constexpr int kTrX0 = kTrVec + 4 * kHidden + 4;     // X0 [rows][kLd1]
constexpr int kTrA1 = kTrX0 + kTrRows * kLd1;       // pre-activations A1, A2, A3 [rows][kLdH]
constexpr int kTrA2 = kTrA1 + kTrRows * kLdH;
constexpr int kTrA3 = kTrA2 + kTrRows * kLdH;
constexpr int kTrH = kTrA3 + kTrRows * kLdH;        // an activation SiLU(A) [rows][kLdH]
constexpr int kTrD0 = kTrH + kTrRows * kLdH;        // gradients of the pre-activations [rows][kLdH], two buffers
constexpr int kTrD1 = kTrD0 + kTrRows * kLdH;
constexpr int kTrY = kTrD1 + kTrRows * kLdH;        // y [rows], dy [rows]
constexpr int kTrDy = kTrY + kTrRows;
constexpr int kTrZ = kTrDy + kTrRows;               // Z of every row (int)
constexpr int kTrFloats = kTrZ + kTrRows;
constexpr size_t kTrSmem = (size_t)kTrFloats * sizeof(float);

__device__ __forceinline__ void tf32_split(float x, uint32_t& hi, uint32_t& lo) {
    uint32_t h, l;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
    const float r = x - __uint_as_float(h);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(r));
    hi = h;
    lo = l;
}

__device__ __forceinline__ void mma_tf32_1688(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// C[M][N] = sum_k A(m, k) B(k, n) over K, tiles of 16 x 8 spread over the block's warps; `store(m, n, value)` takes the
// result. Fragments (g = lane / 4, q = lane % 4): A (g, q), (g + 8, q), (g, q + 4), (g + 8, q + 4); B (q, g),
// (q + 4, g); C (g, 2q), (g, 2q + 1), (g + 8, 2q), (g + 8, 2q + 1).
template <int M, int N, int K, typename FA, typename FB, typename FS>
__device__ __forceinline__ void tr_gemm(FA a, FB b, FS store, int warp, int lane) {
    constexpr int TN = N / 8, NT = (M / 16) * TN;
    static_assert(M % 16 == 0 && N % 8 == 0 && K % 8 == 0, "tile shape");
    const int g = lane >> 2, q = lane & 3;
    for (int t = warp; t < NT; t += kTrWarps) {
        const int m0 = (t / TN) * 16, n0 = (t % TN) * 8;
        float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 4
        for (int k0 = 0; k0 < K; k0 += 8) {
            uint32_t ah[4], al[4], bh0, bl0, bh1, bl1;
            tf32_split(a(m0 + g, k0 + q), ah[0], al[0]);
            tf32_split(a(m0 + g + 8, k0 + q), ah[1], al[1]);
            tf32_split(a(m0 + g, k0 + q + 4), ah[2], al[2]);
            tf32_split(a(m0 + g + 8, k0 + q + 4), ah[3], al[3]);
            tf32_split(b(k0 + q, n0 + g), bh0, bl0);
            tf32_split(b(k0 + q + 4, n0 + g), bh1, bl1);
            mma_tf32_1688(acc, al, bh0, bh1);
            mma_tf32_1688(acc, ah, bl0, bl1);
            mma_tf32_1688(acc, ah, bh0, bh1);
        }
        store(m0 + g, n0 + 2 * q, acc[0]);
        store(m0 + g, n0 + 2 * q + 1, acc[1]);
        store(m0 + g + 8, n0 + 2 * q, acc[2]);
        store(m0 + g + 8, n0 + 2 * q + 1, acc[3]);
    }
}

// One forward and backward pass of samples [blockIdx.x kTrSamples, +kTrSamples) of a doubled batch of B samples (row b
// and row B + b of z and feats: the upper and the lower edge of sample b): the per-block gradients into
// partial[blockIdx.x][kSurrogateParams] and, with loss_terms, each sample's squared error.
__global__ void __launch_bounds__(kTrThreads) k_sg_train(const float* __restrict__ params, const int* __restrict__ z,
                                                         const float* __restrict__ feats,
                                                         const float* __restrict__ target, int B,
                                                         float* __restrict__ partial, double* __restrict__ loss_terms) {
    extern __shared__ __align__(16) float sm_tr[];
    float* W1 = sm_tr + kTrW1;
    float* W2 = sm_tr + kTrW2;
    float* W3 = sm_tr + kTrW3;
    float* vec = sm_tr + kTrVec;  // b1 b2 b3 W4 b4
    float* X0 = sm_tr + kTrX0;
    float* A1 = sm_tr + kTrA1;
    float* A2 = sm_tr + kTrA2;
    float* A3 = sm_tr + kTrA3;
    float* H = sm_tr + kTrH;
    float* D0 = sm_tr + kTrD0;
    float* D1 = sm_tr + kTrD1;
    float* y = sm_tr + kTrY;
    float* dy = sm_tr + kTrDy;
    int* zr = reinterpret_cast<int*>(sm_tr + kTrZ);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int s0 = blockIdx.x * kTrSamples;
    float* out = partial + (size_t)blockIdx.x * kSurrogateParams;
    // ---- parameters and inputs ----
    for (int i = tid; i < kHidden * kLd1; i += kTrThreads) {
        const int n = i / kLd1, k = i % kLd1;
        W1[i] = k < kIn ? params[OFF_W1 + n * kIn + k] : 0.0f;
    }
    for (int i = tid; i < kHidden * kHidden; i += kTrThreads) {
        const int n = i / kHidden, k = i % kHidden;
        W2[n * kLdH + k] = params[OFF_W2 + i];
        W3[n * kLdH + k] = params[OFF_W3 + i];
    }
    for (int i = tid; i < kHidden; i += kTrThreads) {
        vec[i] = params[OFF_B1 + i];
        vec[kHidden + i] = params[OFF_B2 + i];
        vec[2 * kHidden + i] = params[OFF_B3 + i];
        vec[3 * kHidden + i] = params[OFF_W4 + i];
    }
    if (tid == 0) vec[4 * kHidden] = params[OFF_B4];
    for (int i = tid; i < kTrRows * kLd1; i += kTrThreads) {
        const int r = i / kLd1, k = i % kLd1;
        const int smp = s0 + (r % kTrSamples);
        const bool ok = smp < B;
        const long long row = ok ? (r < kTrSamples ? smp : (long long)B + smp) : 0;
        const int zz = ok ? z[row] : 1;
        if (k == 0) zr[r] = ok ? zz : 0;
        float v = 0.0f;
        if (ok) {
            if (k < kEmbed) v = params[OFF_EMB + (zz - 1) * kEmbed + k];
            else if (k < kIn) v = feats[row * 2 + (k - kEmbed)];
        }
        X0[r * kLd1 + k] = v;
    }
    __syncthreads();
    // ---- forward ----
    const float* b1 = vec;
    const float* b2 = vec + kHidden;
    const float* b3 = vec + 2 * kHidden;
    const float* w4 = vec + 3 * kHidden;
    tr_gemm<kTrRows, kHidden, kIn8>([&](int m, int k) { return X0[m * kLd1 + k]; },
                                    [&](int k, int n) { return W1[n * kLd1 + k]; },
                                    [&](int m, int n, float v) {
                                        const float a = v + b1[n];
                                        A1[m * kLdH + n] = a;
                                        H[m * kLdH + n] = silu(a);
                                    },
                                    warp, lane);
    __syncthreads();
    tr_gemm<kTrRows, kHidden, kHidden>([&](int m, int k) { return H[m * kLdH + k]; },
                                       [&](int k, int n) { return W2[n * kLdH + k]; },
                                       [&](int m, int n, float v) { A2[m * kLdH + n] = v + b2[n]; }, warp, lane);
    __syncthreads();
    for (int i = tid; i < kTrRows * kHidden; i += kTrThreads) {
        const int m = i / kHidden, n = i % kHidden;
        H[m * kLdH + n] = silu(A2[m * kLdH + n]);
    }
    __syncthreads();
    tr_gemm<kTrRows, kHidden, kHidden>([&](int m, int k) { return H[m * kLdH + k]; },
                                       [&](int k, int n) { return W3[n * kLdH + k]; },
                                       [&](int m, int n, float v) { A3[m * kLdH + n] = v + b3[n]; }, warp, lane);
    __syncthreads();
    // output layer: y = b4 + sum_k silu(A3) W4, one warp per row, lanes over k, shuffle tree (fixed order)
    for (int m = warp; m < kTrRows; m += kTrWarps) {
        float sum = silu(A3[m * kLdH + lane]) * w4[lane] + silu(A3[m * kLdH + lane + 32]) * w4[lane + 32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) y[m] = sum + vec[4 * kHidden];
    }
    __syncthreads();
    // ---- loss: F_hat = y(upper) - y(lower); dL/dy = +-2 e / B ----
    if (tid < kTrSamples) {
        const int smp = s0 + tid;
        float d = 0.0f;
        if (smp < B) {
            const float e = (y[tid] - y[kTrSamples + tid]) - target[smp];
            d = 2.0f * e / (float)B;
            if (loss_terms) loss_terms[smp] = (double)e * (double)e;
        }
        dy[tid] = d;
        dy[kTrSamples + tid] = -d;
    }
    __syncthreads();
    // ---- backward ----
    // output layer: gW4[k] = sum_m dy silu(A3), gb4 = sum_m dy; D0 = dy W4 silu'(A3)
    for (int k = tid; k < kHidden; k += kTrThreads) {
        float g = 0.0f;
        for (int m = 0; m < kTrRows; ++m) g += dy[m] * silu(A3[m * kLdH + k]);
        out[OFF_W4 + k] = g;
    }
    if (tid == kHidden) {
        float g = 0.0f;
        for (int m = 0; m < kTrRows; ++m) g += dy[m];
        out[OFF_B4] = g;
    }
    for (int i = tid; i < kTrRows * kHidden; i += kTrThreads) {
        const int m = i / kHidden, n = i % kHidden;
        D0[m * kLdH + n] = dy[m] * w4[n] * silu_grad(A3[m * kLdH + n]);
    }
    __syncthreads();
    // layer 3 (H = silu(A2) still holds its input): gW3 = D0^T H, gb3 = colsum D0; D1 = (D0 W3) silu'(A2)
    tr_gemm<kHidden, kHidden, kTrRows>([&](int n, int m) { return D0[m * kLdH + n]; },
                                       [&](int m, int k) { return H[m * kLdH + k]; },
                                       [&](int n, int k, float v) { out[OFF_W3 + n * kHidden + k] = v; }, warp, lane);
    tr_gemm<kTrRows, kHidden, kHidden>([&](int m, int n) { return D0[m * kLdH + n]; },
                                       [&](int n, int k) { return W3[n * kLdH + k]; },
                                       [&](int m, int k, float v) { D1[m * kLdH + k] = v * silu_grad(A2[m * kLdH + k]); },
                                       warp, lane);
    for (int n = tid; n < kHidden; n += kTrThreads) {
        float g = 0.0f;
        for (int m = 0; m < kTrRows; ++m) g += D0[m * kLdH + n];
        out[OFF_B3 + n] = g;
    }
    __syncthreads();
    for (int i = tid; i < kTrRows * kHidden; i += kTrThreads) {
        const int m = i / kHidden, n = i % kHidden;
        H[m * kLdH + n] = silu(A1[m * kLdH + n]);
    }
    __syncthreads();
    // layer 2: gW2 = D1^T silu(A1), gb2; D0 = (D1 W2) silu'(A1)
    tr_gemm<kHidden, kHidden, kTrRows>([&](int n, int m) { return D1[m * kLdH + n]; },
                                       [&](int m, int k) { return H[m * kLdH + k]; },
                                       [&](int n, int k, float v) { out[OFF_W2 + n * kHidden + k] = v; }, warp, lane);
    tr_gemm<kTrRows, kHidden, kHidden>([&](int m, int n) { return D1[m * kLdH + n]; },
                                       [&](int n, int k) { return W2[n * kLdH + k]; },
                                       [&](int m, int k, float v) { D0[m * kLdH + k] = v * silu_grad(A1[m * kLdH + k]); },
                                       warp, lane);
    for (int n = tid; n < kHidden; n += kTrThreads) {
        float g = 0.0f;
        for (int m = 0; m < kTrRows; ++m) g += D1[m * kLdH + n];
        out[OFF_B2 + n] = g;
    }
    __syncthreads();
    // layer 1: gW1 = D0^T X0 (inputs 0 .. 17), gb1; dX0 = D0 W1 (the embedding's 16 inputs) into H
    tr_gemm<kHidden, kIn8, kTrRows>([&](int n, int m) { return D0[m * kLdH + n]; },
                                    [&](int m, int k) { return X0[m * kLd1 + k]; },
                                    [&](int n, int k, float v) {
                                        if (k < kIn) out[OFF_W1 + n * kIn + k] = v;
                                    },
                                    warp, lane);
    tr_gemm<kTrRows, kEmbed, kHidden>([&](int m, int n) { return D0[m * kLdH + n]; },
                                      [&](int n, int k) { return W1[n * kLd1 + k]; },
                                      [&](int m, int k, float v) { H[m * kLdH + k] = v; }, warp, lane);
    for (int n = tid; n < kHidden; n += kTrThreads) {
        float g = 0.0f;
        for (int m = 0; m < kTrRows; ++m) g += D0[m * kLdH + n];
        out[OFF_B1 + n] = g;
    }
    __syncthreads();
    // embedding: gEmb[Z][k] = sum over the block's rows of element Z, in row order (zero for the others)
    for (int i = tid; i < 103 * kEmbed; i += kTrThreads) {
        const int zz = i / kEmbed + 1, k = i % kEmbed;
        float g = 0.0f;
        for (int m = 0; m < kTrRows; ++m)
            if (zr[m] == zz) g += H[m * kLdH + k];
        out[OFF_EMB + i] = g;
    }
}

// g = sum over the blocks' rows of `partial` in block order; with lr > 0 also the Adam step on p.
__global__ void k_sg_reduce_adam(const float* __restrict__ partial, int blocks, float* __restrict__ grads,
                                 float* __restrict__ p, float* __restrict__ m, float* __restrict__ v, int n, float lr,
                                 float b1, float b2, float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float gi = 0.0f;
        for (int b = 0; b < blocks; ++b) gi += partial[(size_t)b * n + i];
        grads[i] = gi;
        if (lr > 0.0f) {
            const float mi = b1 * m[i] + (1.0f - b1) * gi;
            const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
            m[i] = mi;
            v[i] = vi;
            p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        }
    }
}

// ---- fused inference ---------------------------------------------------------------------------------------------
// Each warp evaluates 16 queries (Z, rho, zl, zu) at a time as 32 rows of the network -- rows 0-15 the upper edges,
// rows 16-31 the lower edges -- with mma.sync m16n8k16 (f16 operands, float32 accumulators):
//     F = C(zu) - C(zl),   P = P_inf(rho) F.
// Each block stages the float32 matrices once as f16 [out][in] rows in shared memory (which is the col-major B operand
// itself; row pitches padded by 16 bytes so that the 8 rows one fragment load touches fall into distinct banks);
// biases and the 64 -> 1 layer stay float32. The accumulators of one layer, after bias and SiLU, are re-packed in
// registers as the next layer's A fragments (the m16n8 accumulator layout of two neighbouring n-tiles is the m16k16 A
// layout), so activations never leave the registers. The 64 -> 1 layer is a quad shuffle-reduction, and the upper and
// lower rows of a query end in the same lane. f16 rather than bf16: the activations and weights are of order one, and
// the 11-bit significand keeps the rounding of the hidden activations well below the network's fit.
struct SgQueryPairs {  // queries from a profile table: pair p, radius k
    const FinitePair* pairs;
    const int* pair_ids;      // the table rows this launch fills
    int npairs;
    const int* elem_z;        // Z of each element index of the potential
    const float2* rho_f0;     // [element][nr]: the table's radius rho and the feature (log rho + 1.5) / 2
    const double* pinf;       // [element][nr]: P_inf at the table's radii
    int nr;
};

constexpr int kTcIn = 32;                            // layer-1 inputs padded to two k-steps
constexpr int kTcLd1 = kTcIn + 8;                    // padded row pitches (f16 elements)
constexpr int kTcLd = kHidden + 8;
constexpr int kTcW1 = kHidden * kTcLd1;
constexpr int kTcW = kHidden * kTcLd;
constexpr int kTcWarps = 4;
constexpr int kTcSmem = (kTcW1 + 2 * kTcW) * 2 + (4 * kHidden + 2) * 4 + kTcWarps * 32 * kTcLd1 * 2;

__device__ __forceinline__ void mma_f16_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_f16(float lo, float hi) {
    const __half2 v = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// SiLU of two accumulators as a packed f16 pair: silu(x) = x sigmoid(x) = h + h tanh(h) with h = x / 2, in f16x2 with
// the hardware tanh approximation (one special-function operation per pair; the result is rounded to f16 for the
// next layer in any case). The float32 SiLU of training needs an exponential and a reciprocal per value, which
// made the activations, not the products, the inference's bottleneck.
__device__ __forceinline__ uint32_t silu_f16x2(float a, float b) {
    const __half2 h = __hmul2(__floats2half2_rn(a, b), __float2half2_rn(0.5f));
    uint32_t t;
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(t) : "r"(*reinterpret_cast<const uint32_t*>(&h)));
    const __half2 y = __hfma2(h, *reinterpret_cast<const __half2*>(&t), h);
    return *reinterpret_cast<const uint32_t*>(&y);
}

// One hidden layer on 32 rows: acc = A (KS k-steps of 16) x W^T + bias, then SiLU into `out` as the next layer's A
// fragments (4 k-steps of 16). Fragment layouts of m16n8k16 (g = lane / 4, q = lane % 4): A registers hold
// (row g, k 2q..2q+1), (row g+8, k 2q..), (row g, k 2q+8..), (row g+8, k 2q+8..); B registers (k 2q.., n g) and
// (k 2q+8.., n g); accumulators (row g, n 2q, 2q+1) and (row g+8, n 2q, 2q+1).
template <int KS>
__device__ __forceinline__ void tc_layer(const uint32_t (&a)[2][KS][4], const __half* __restrict__ W, int ldw,
                                         const float* __restrict__ bias, int lane, uint32_t (&out)[2][4][4]) {
    const int g = lane >> 2, q = lane & 3;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const int n = nt * 8 + g;
        const float b0 = bias[nt * 8 + 2 * q], b1 = bias[nt * 8 + 2 * q + 1];
        float acc[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            acc[mt][0] = b0;
            acc[mt][1] = b1;
            acc[mt][2] = b0;
            acc[mt][3] = b1;
        }
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
            const uint32_t w0 = *reinterpret_cast<const uint32_t*>(W + n * ldw + ks * 16 + 2 * q);
            const uint32_t w1 = *reinterpret_cast<const uint32_t*>(W + n * ldw + ks * 16 + 8 + 2 * q);
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) mma_f16_16816(acc[mt], a[mt][ks], w0, w1);
        }
        // n-tile nt holds columns nt*8 .. nt*8+7: the first (nt even) or second half of the next layer's k-step nt/2
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const uint32_t lo = silu_f16x2(acc[mt][0], acc[mt][1]);
            const uint32_t hi = silu_f16x2(acc[mt][2], acc[mt][3]);
            out[mt][nt >> 1][(nt & 1) * 2] = lo;
            out[mt][nt >> 1][(nt & 1) * 2 + 1] = hi;
        }
    }
}

template <bool FROM_PAIRS>
__global__ void __launch_bounds__(kTcWarps * 32) k_sg_infer(const float* __restrict__ params, SgQueryPairs q,
                                                          const int* __restrict__ qz, const double* __restrict__ qrho,
                                                          const double* __restrict__ qzl,
                                                          const double* __restrict__ qzu,
                                                          const double* __restrict__ qpinf, int nq,
                                                          double* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_sg[];
    __half* W1 = reinterpret_cast<__half*>(smem_sg);                 // [64][kTcLd1]
    __half* W2 = W1 + kTcW1;                                         // [64][kTcLd]
    __half* W3 = W2 + kTcW;                                          // [64][kTcLd]
    float* bias = reinterpret_cast<float*>(W3 + kTcW);               // b1 b2 b3 [64 each], W4 [64], b4
    __half* xs = reinterpret_cast<__half*>(bias + 4 * kHidden + 2);  // per warp [32][kTcLd1]
    for (int i = threadIdx.x; i < kTcW1; i += blockDim.x) {
        const int n = i / kTcLd1, k = i % kTcLd1;
        W1[i] = __float2half_rn(k < kIn ? params[OFF_W1 + n * kIn + k] : 0.0f);
    }
    for (int i = threadIdx.x; i < kTcW; i += blockDim.x) {
        const int n = i / kTcLd, k = i % kTcLd;
        W2[i] = __float2half_rn(k < kHidden ? params[OFF_W2 + n * kHidden + k] : 0.0f);
        W3[i] = __float2half_rn(k < kHidden ? params[OFF_W3 + n * kHidden + k] : 0.0f);
    }
    for (int i = threadIdx.x; i < kHidden; i += blockDim.x) {
        bias[i] = params[OFF_B1 + i];
        bias[kHidden + i] = params[OFF_B2 + i];
        bias[2 * kHidden + i] = params[OFF_B3 + i];
        bias[3 * kHidden + i] = params[OFF_W4 + i];
    }
    if (threadIdx.x == 0) bias[4 * kHidden] = params[OFF_B4];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, qd = lane & 3;
    __half* x = xs + warp * 32 * kTcLd1;
    const float* w4 = bias + 3 * kHidden;
    const long long total = FROM_PAIRS ? (long long)q.npairs * q.nr : nq;
    const long long groups = (total + 15) / 16;
    for (long long grp = (long long)blockIdx.x * kTcWarps + warp; grp < groups;
         grp += (long long)gridDim.x * kTcWarps) {
        // lane l < 16 stages the upper-edge row of query grp*16 + l, lane 16 + l the lower-edge row of the same query
        const long long qi = grp * 16 + (lane & 15);
        const bool valid = qi < total;
        int z = 1;
        double pinf = 0.0;
        float f[2] = {0.0f, 0.0f};
        long long dst = 0;
        if (valid) {
            if (FROM_PAIRS) {
                // the table's radius k of this element: its radius and first feature come from a per-build table,
                // the edge feature asinh(z / rho) / 4 in float32 (it is rounded to f16 for the network anyway)
                const int p = q.pair_ids[qi / q.nr], k = (int)(qi % q.nr);
                const FinitePair pr = q.pairs[p];
                z = q.elem_z[pr.elem];
                const float2 rf = q.rho_f0[(size_t)pr.elem * q.nr + k];
                f[0] = rf.y;
                f[1] = 0.25f * asinhf((float)(lane < 16 ? pr.zu : pr.zl) / rf.x);
                pinf = q.pinf[(size_t)pr.elem * q.nr + k];
                dst = (long long)p * q.nr + k;
            } else {
                z = qz[qi];
                surrogate_features(qrho[qi], lane < 16 ? qzu[qi] : qzl[qi], f);
                pinf = qpinf[qi];
                dst = qi;
            }
        }
        {
            __half* row = x + lane * kTcLd1;
            const float* emb = params + OFF_EMB + (z - 1) * kEmbed;
#pragma unroll
            for (int k = 0; k < kEmbed; k += 2)
                *reinterpret_cast<uint32_t*>(row + k) = pack_f16(__ldg(emb + k), __ldg(emb + k + 1));
            *reinterpret_cast<uint32_t*>(row + kEmbed) = pack_f16(f[0], f[1]);
#pragma unroll
            for (int k = kIn; k < kTcIn; k += 2) *reinterpret_cast<uint32_t*>(row + k) = 0u;
        }
        __syncwarp();
        uint32_t a1[2][2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int ks = 0; ks < 2; ++ks) {
                const __half* r0 = x + (mt * 16 + g) * kTcLd1 + ks * 16 + 2 * qd;
                const __half* r1 = r0 + 8 * kTcLd1;
                a1[mt][ks][0] = *reinterpret_cast<const uint32_t*>(r0);
                a1[mt][ks][1] = *reinterpret_cast<const uint32_t*>(r1);
                a1[mt][ks][2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
                a1[mt][ks][3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
            }
        __syncwarp();  // the rows are rewritten by the next group
        uint32_t h1[2][4][4], h2[2][4][4], h3[2][4][4];
        tc_layer<2>(a1, W1, kTcLd1, bias, lane, h1);
        tc_layer<4>(h1, W2, kTcLd, bias + kHidden, lane, h2);
        tc_layer<4>(h2, W3, kTcLd, bias + 2 * kHidden, lane, h3);
        // 64 -> 1: this lane holds columns ks*16 + 2qd + {0, 1} (+8) of rows g and g + 8 of each m-tile
        float y[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int ks = 0; ks < 4; ++ks)
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const float2 f2 = __half22float2(*reinterpret_cast<const __half2*>(&h3[mt][ks][r]));
                    const int c = ks * 16 + 2 * qd + ((r & 2) ? 8 : 0);
                    y[mt][r & 1] += f2.x * w4[c] + f2.y * w4[c + 1];
                }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                y[mt][h] += __shfl_xor_sync(0xffffffffu, y[mt][h], 1);
                y[mt][h] += __shfl_xor_sync(0xffffffffu, y[mt][h], 2);
            }
        // m-tile 0 holds the upper edges, m-tile 1 the lower: rows g and g + 8 are queries g and g + 8 (b4 cancels)
        const float F0 = y[0][0] - y[1][0], F1 = y[0][1] - y[1][1];
        // lane l < 16 takes query l from the first lane of quad l % 8
        const float Fa = __shfl_sync(0xffffffffu, F0, (lane & 7) << 2);
        const float Fb = __shfl_sync(0xffffffffu, F1, (lane & 7) << 2);
        const float F = (lane & 8) ? Fb : Fa;
        if (lane < 16 && valid) out[dst] = pinf * (double)F;
    }
}

// ---- host --------------------------------------------------------------------------------------------------------
double infinite_profile(int z, double rho) {
    const ElementAB e = element_ab(z);
    double s = 0.0;
    for (int t = 0; t < 5; ++t)
        s += 2.0 * e.A[t] / e.B[t] * std::cyl_bessel_k(0.0, e.B[t] * rho) + e.A[t] * rho * std::cyl_bessel_k(1.0, e.B[t] * rho);
    return 2.0 * s;
}

namespace {

struct Batch {  // a doubled batch: rows b (upper edge) and B + b (lower edge); per-block gradient rows
    DeviceBuffer z, feats, target, loss, partial;
    void ensure(int B) {
        const int R = 2 * B;
        z.ensure(R * sizeof(int));
        feats.ensure((size_t)R * 2 * sizeof(float));
        target.ensure(B * sizeof(float));
        loss.ensure(B * sizeof(double));
        partial.ensure((size_t)train_blocks(B) * kSurrogateParams * sizeof(float));
    }
    static int train_blocks(int B) { return (B + kTrSamples - 1) / kTrSamples; }
};

// Host rows of one doubled batch from samples [first, first + B).
void fill_rows(const std::vector<int>& z, const std::vector<double>& rho, const std::vector<double>& zl,
               const std::vector<double>& zu, size_t first, int B, std::vector<int>& rz, std::vector<float>& rf) {
    rz.resize(2 * B);
    rf.resize(4 * (size_t)B);
    for (int b = 0; b < B; ++b) {
        const size_t i = first + b;
        rz[b] = rz[B + b] = z[i];
        surrogate_features(rho[i], zu[i], rf.data() + 2 * b);
        surrogate_features(rho[i], zl[i], rf.data() + 2 * (B + b));
    }
}

void set_train_smem() {
    static bool set = false;
    if (!set) {
        SIMK_CUDA(cudaFuncSetAttribute(k_sg_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrSmem));
        set = true;
    }
}

// Forward and backward of the doubled batch at (z, feats, target): the gradient into G (and, with lr > 0, the Adam step
// on P with moments m, v); returns the loss when asked (then it synchronises).
double forward_backward(Context& ctx, float* P, float* G, const int* z, const float* feats, const float* target, int B,
                        Batch& b, bool want_loss, float lr = 0.0f, float* m = nullptr, float* v = nullptr,
                        float c1 = 1.0f, float c2 = 1.0f) {
    cudaStream_t st = ctx.stream;
    set_train_smem();
    const int blocks = Batch::train_blocks(B);
    k_sg_train<<<blocks, kTrThreads, kTrSmem, st>>>(P, z, feats, target, B, b.partial.as<float>(),
                                                    want_loss ? b.loss.as<double>() : nullptr);
    k_sg_reduce_adam<<<(kSurrogateParams + 255) / 256, 256, 0, st>>>(b.partial.as<float>(), blocks, G, P, m, v,
                                                                    kSurrogateParams, lr, 0.9f, 0.999f, 1e-8f, c1, c2);
    ctx.launches += 2;
    SIMK_CUDA(cudaGetLastError());
    if (!want_loss) return 0.0;
    std::vector<double> terms(B);
    SIMK_CUDA(cudaMemcpyAsync(terms.data(), b.loss.ptr, B * sizeof(double), cudaMemcpyDeviceToHost, st));
    SIMK_CUDA(cudaStreamSynchronize(st));
    double sum = 0.0;
    for (double t : terms) sum += t;
    return sum / B;
}

void set_infer_smem() {
    static bool set = false;
    if (!set) {
        SIMK_CUDA(cudaFuncSetAttribute(k_sg_infer<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
        SIMK_CUDA(cudaFuncSetAttribute(k_sg_infer<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
        set = true;
    }
}

// Persistent grid: at most 4 blocks of 128 threads x 128 registers per SM, and no more warps than 16-query groups.
inline int infer_blocks(const Context& ctx, long long queries) {
    const long long groups = (queries + 15) / 16;
    return (int)std::max<long long>(1, std::min<long long>((groups + kTcWarps - 1) / kTcWarps,
                                                           4LL * ctx.sm_count));
}

}  // namespace

// Samples of the trained domain: Z from the list, log rho uniform in [rho_min, R_c(Z)], zl uniform in [-R_c, R_c),
// thickness uniform in (0, min(max_thickness, R_c - zl)].
void draw_samples(const SurrogateImpl& s, std::mt19937_64& rng, int n, std::vector<int>& z, std::vector<double>& rho,
                  std::vector<double>& zl, std::vector<double>& zu) {
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::uniform_int_distribution<int> E(0, (int)s.elements.size() - 1);
    z.resize(n);
    rho.resize(n);
    zl.resize(n);
    zu.resize(n);
    for (int i = 0; i < n; ++i) {
        const int e = E(rng);
        const double rc = s.rcut[e];
        z[i] = s.elements[e];
        rho[i] = s.rho_min * std::pow(rc / s.rho_min, U(rng));
        zl[i] = -rc + 2.0 * rc * U(rng);
        const double tmax = std::min(s.max_thickness, rc - zl[i]);
        zu[i] = zl[i] + std::max(1e-4, tmax * U(rng));
    }
}

void surrogate_quadrature_points(Context& ctx, const std::vector<int>& z, const std::vector<double>& rho,
                                 const std::vector<double>& zl, const std::vector<double>& zu, double* out_dev) {
    const int n = (int)z.size();
    std::vector<int> els(z);
    std::sort(els.begin(), els.end());
    els.erase(std::unique(els.begin(), els.end()), els.end());
    std::vector<ElementAB> ab;
    for (int zz : els) ab.push_back(element_ab(zz));
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = (int)(std::lower_bound(els.begin(), els.end(), z[i]) - els.begin());
    DeviceBuffer dab(ab.size() * sizeof(ElementAB)), didx(n * sizeof(int)), dr(n * sizeof(double)),
        dl(n * sizeof(double)), du(n * sizeof(double));
    SIMK_CUDA(cudaMemcpy(dab.ptr, ab.data(), ab.size() * sizeof(ElementAB), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemcpy(didx.ptr, idx.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemcpy(dr.ptr, rho.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemcpy(dl.ptr, zl.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemcpy(du.ptr, zu.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    finite_points(ctx, dab.as<ElementAB>(), n, didx.as<int>(), dr.as<double>(), dl.as<double>(), du.as<double>(),
                  out_dev);
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
}

std::unique_ptr<SurrogateImpl> surrogate_train(Context& ctx, const std::vector<int>& elements, long long n_samples,
                                               int steps, int batch, double lr, unsigned long long seed,
                                               double max_thickness, double rho_min) {
    SIMK_REQUIRE(!elements.empty(), "no element to train on");
    SIMK_REQUIRE(n_samples >= batch && batch >= 1 && steps >= 1, "need n_samples >= batch >= 1 and steps >= 1");
    auto s = std::make_unique<SurrogateImpl>();
    s->elements = elements;
    std::sort(s->elements.begin(), s->elements.end());
    s->elements.erase(std::unique(s->elements.begin(), s->elements.end()), s->elements.end());
    for (int z : s->elements) {
        SIMK_REQUIRE(z >= 1 && z <= 103, "unsupported element");
        s->rcut.push_back(finite_cutoff(z));
    }
    s->max_thickness = max_thickness;
    s->rho_min = rho_min;
    s->params.alloc(kSurrogateParams * sizeof(float));
    s->grads.alloc(kSurrogateParams * sizeof(float));
    s->m.alloc(kSurrogateParams * sizeof(float));
    s->v.alloc(kSurrogateParams * sizeof(float));
    // initial weights: U(-1/sqrt(fan_in), 1/sqrt(fan_in)), biases zero, embedding N(0, 0.1)
    std::mt19937_64 rng(seed);
    std::vector<float> p(kSurrogateParams, 0.0f);
    std::normal_distribution<float> N01(0.0f, 0.1f);
    for (int i = OFF_EMB; i < OFF_W1; ++i) p[i] = N01(rng);
    auto fill = [&](int off, int count, int fan_in) {
        std::uniform_real_distribution<float> U(-1.0f / std::sqrt((float)fan_in), 1.0f / std::sqrt((float)fan_in));
        for (int i = 0; i < count; ++i) p[off + i] = U(rng);
    };
    fill(OFF_W1, kHidden * kIn, kIn);
    fill(OFF_W2, kHidden * kHidden, kHidden);
    fill(OFF_W3, kHidden * kHidden, kHidden);
    fill(OFF_W4, kHidden, kHidden);
    SIMK_CUDA(cudaMemcpy(s->params.ptr, p.data(), kSurrogateParams * sizeof(float), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemset(s->m.ptr, 0, kSurrogateParams * sizeof(float)));
    SIMK_CUDA(cudaMemset(s->v.ptr, 0, kSurrogateParams * sizeof(float)));
    // the training set, labelled F = P / P_inf with P by the float64 device quadrature
    const long long n = n_samples;
    std::vector<int> all_z(n);
    std::vector<double> all_rho(n), all_zl(n), all_zu(n);
    std::vector<float> all_F(n);
    {
        DeviceBuffer P(std::min<long long>(n, 1 << 20) * sizeof(double));
        std::vector<int> z;
        std::vector<double> rho, zl, zu;
        for (long long first = 0; first < n; first += (1 << 20)) {
            const int m = (int)std::min<long long>(1 << 20, n - first);
            draw_samples(*s, rng, m, z, rho, zl, zu);
            surrogate_quadrature_points(ctx, z, rho, zl, zu, P.as<double>());
            std::vector<double> hp(m);
            SIMK_CUDA(cudaMemcpy(hp.data(), P.ptr, m * sizeof(double), cudaMemcpyDeviceToHost));
            for (int i = 0; i < m; ++i) {
                all_z[first + i] = z[i];
                all_rho[first + i] = rho[i];
                all_zl[first + i] = zl[i];
                all_zu[first + i] = zu[i];
                all_F[first + i] = (float)(hp[i] / infinite_profile(z[i], rho[i]));
            }
        }
    }
    // device copies of the doubled rows of every batch
    const long long nb = n / batch;
    DeviceBuffer rows_z((size_t)nb * 2 * batch * sizeof(int)), rows_f((size_t)nb * 4 * batch * sizeof(float));
    {
        std::vector<int> rz;
        std::vector<float> rf;
        for (long long k = 0; k < nb; ++k) {
            fill_rows(all_z, all_rho, all_zl, all_zu, (size_t)k * batch, batch, rz, rf);
            SIMK_CUDA(cudaMemcpy(rows_z.as<int>() + k * 2 * batch, rz.data(), rz.size() * sizeof(int),
                                 cudaMemcpyHostToDevice));
            SIMK_CUDA(cudaMemcpy(rows_f.as<float>() + k * 4 * batch, rf.data(), rf.size() * sizeof(float),
                                 cudaMemcpyHostToDevice));
        }
    }
    DeviceBuffer targets((size_t)n * sizeof(float));
    SIMK_CUDA(cudaMemcpy(targets.ptr, all_F.data(), n * sizeof(float), cudaMemcpyHostToDevice));
    Batch b;
    b.ensure(batch);
    const float b1 = 0.9f, b2 = 0.999f;
    double loss = 0.0;
    for (int step = 0; step < steps; ++step) {
        const long long k = step % nb;
        const bool want = (step == steps - 1);
        // cosine decay from lr to lr / 20
        const double lr_t = lr * (0.05 + 0.95 * 0.5 * (1.0 + std::cos(M_PI * step / (double)steps)));
        const float c1 = 1.0f - std::pow(b1, (float)(step + 1)), c2 = 1.0f - std::pow(b2, (float)(step + 1));
        const double l = forward_backward(ctx, s->params.as<float>(), s->grads.as<float>(),
                                          rows_z.as<int>() + k * 2 * batch, rows_f.as<float>() + k * 4 * batch,
                                          targets.as<float>() + k * batch, batch, b, want, (float)lr_t,
                                          s->m.as<float>(), s->v.as<float>(), c1, c2);
        if (want) loss = l;
    }
    SIMK_CUDA(cudaGetLastError());
    s->train_loss = loss;
    s->steps = steps;
    s->samples = n;
    // held-out judgement by the quadrature: 4096 fresh samples, error |dP| / P_inf(rho) = |dF|
    std::vector<int> z;
    std::vector<double> rho, zl, zu;
    draw_samples(*s, rng, 4096, z, rho, zl, zu);
    std::vector<double> q(4096), e(4096);
    DeviceBuffer dq(4096 * sizeof(double));
    surrogate_quadrature_points(ctx, z, rho, zl, zu, dq.as<double>());
    SIMK_CUDA(cudaMemcpy(q.data(), dq.ptr, 4096 * sizeof(double), cudaMemcpyDeviceToHost));
    surrogate_evaluate(ctx, *s, z, rho, zl, zu, e.data());
    double mx = 0.0, rms = 0.0;
    for (int i = 0; i < 4096; ++i) {
        const double r = std::fabs(e[i] - q[i]) / infinite_profile(z[i], rho[i]);
        mx = std::max(mx, r);
        rms += r * r;
    }
    s->val_max_rel = mx;
    s->val_rms_rel = std::sqrt(rms / 4096.0);
    return s;
}

void surrogate_evaluate(Context& ctx, const SurrogateImpl& s, const std::vector<int>& z, const std::vector<double>& rho,
                        const std::vector<double>& zl, const std::vector<double>& zu, double* out_host) {
    const int n = (int)z.size();
    if (n == 0) return;
    set_infer_smem();
    std::vector<double> pinf(n);
    for (int i = 0; i < n; ++i) pinf[i] = infinite_profile(z[i], rho[i]);
    DeviceBuffer dz(n * sizeof(int)), dr(n * sizeof(double)), dl(n * sizeof(double)), du(n * sizeof(double)),
        dp(n * sizeof(double)), dout(n * sizeof(double));
    SIMK_CUDA(cudaMemcpy(dz.ptr, z.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemcpy(dr.ptr, rho.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemcpy(dl.ptr, zl.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemcpy(du.ptr, zu.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemcpy(dp.ptr, pinf.data(), n * sizeof(double), cudaMemcpyHostToDevice));
    SgQueryPairs q{};
    k_sg_infer<false><<<infer_blocks(ctx, n), kTcWarps * 32, kTcSmem, ctx.stream>>>(
        s.params.as<float>(), q, dz.as<int>(), dr.as<double>(), dl.as<double>(), du.as<double>(),
        dp.as<double>(), n, dout.as<double>());
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
    SIMK_CUDA(cudaMemcpyAsync(out_host, dout.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
}

void surrogate_profiles(Context& ctx, const SurrogateImpl& s, const FiniteDevice& d, const int* pair_ids_dev,
                        int npairs, const int* elem_z_dev, const float2* rho_f0_dev, const double* pinf_dev, int nr,
                        double* table) {
    if (npairs == 0) return;
    set_infer_smem();
    SgQueryPairs q{d.pairs, pair_ids_dev, npairs, elem_z_dev, rho_f0_dev, pinf_dev, nr};
    KernelTimer t(ctx, "surrogate_infer", 0.0);
    k_sg_infer<true><<<infer_blocks(ctx, (long long)npairs * nr), kTcWarps * 32, kTcSmem, ctx.stream>>>(
        s.params.as<float>(), q, nullptr, nullptr, nullptr, nullptr, nullptr, 0, table);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
}

double surrogate_gradients(Context& ctx, SurrogateImpl& s, const std::vector<int>& z, const std::vector<double>& rho,
                           const std::vector<double>& zl, const std::vector<double>& zu,
                           const std::vector<double>& target, float* grads_host) {
    const int B = (int)z.size();
    SIMK_REQUIRE(B >= 1, "empty batch");
    Batch b;
    b.ensure(B);
    std::vector<int> rz;
    std::vector<float> rf, y(B);
    fill_rows(z, rho, zl, zu, 0, B, rz, rf);
    for (int i = 0; i < B; ++i) y[i] = (float)target[i];
    SIMK_CUDA(cudaMemcpy(b.z.ptr, rz.data(), rz.size() * sizeof(int), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemcpy(b.feats.ptr, rf.data(), rf.size() * sizeof(float), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemcpy(b.target.ptr, y.data(), B * sizeof(float), cudaMemcpyHostToDevice));
    const double loss = forward_backward(ctx, s.params.as<float>(), s.grads.as<float>(), b.z.as<int>(),
                                         b.feats.as<float>(), b.target.as<float>(), B, b, true);
    SIMK_CUDA(cudaMemcpy(grads_host, s.grads.ptr, kSurrogateParams * sizeof(float), cudaMemcpyDeviceToHost));
    return loss;
}

}  // namespace simk
