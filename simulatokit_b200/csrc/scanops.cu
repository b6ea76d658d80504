// scanops.cu -- scan post-processing on the device (ScanOperations.swift:12-167, IntegratedCenterOfMass.swift:11-41,
// ImageOperations.swift:140-176): the Gaussian source size, Poisson noise and the integral of a gradient field.
//
// All three run once per finished scan on scan-sized float64 arrays that stay on the device. The Gaussian filter is
// a separable periodic convolution, one pass per scan axis, every output summed in the reference's order with
// explicitly rounded multiplies and adds (no contraction into FMA), so the result is bit-equal to the reference's
// float64 loop given the same weights, which the host computes as the reference does. The Poisson sampler is the
// reference's (Knuth's product below a mean of 10, Hoermann's PTRS above) on the kit's xoshiro256** generator; each
// value and sample has a generator of its own (the reference runs one stream through all values in order, a chain a
// GPU cannot split), so a seed gives the same noise on every run and any split of the work, not the reference's bits.
#include <algorithm>
#include <cmath>

#include "fft.cuh"
#include "scanops.cuh"

namespace simk {

namespace {

inline int blocks_for(long long n, int threads = 256) {
    return (int)std::max<long long>(1, std::min<long long>((n + threads - 1) / threads, 148LL * 16));
}

// ---- Gaussian source size -------------------------------------------------------------------------------------------

// One periodic pass along an axis of length L with element stride `stride` (the array is [outer][L][stride]):
// out[e] = sum_j w[j] in[base + ((k + j - r) mod L) stride], j = 0 .. taps - 1 in order, k the axis index of e.
// Used where the staged form below does not apply (strides below 32, radii beyond its shared memory).
__global__ void k_gauss_axis(const double* __restrict__ in, double* __restrict__ out, long long total, int L,
                             long long stride, const double* __restrict__ w, int taps, int radius) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long k = (e / stride) % L;
        const long long base = e - k * stride;
        long long idx = ((k - radius) % L + L) % L;
        double acc = 0.0;
        for (int j = 0; j < taps; ++j) {
            acc = __dadd_rn(acc, __dmul_rn(__ldg(w + j), __ldg(in + base + idx * stride)));
            if (++idx == L) idx = 0;
        }
        out[e] = acc;
    }
}

// The same pass for axes whose element stride is at least 32 (a scan's values): a block takes 32 neighbouring columns
// i0 .. i0 + 31 of one outer index and nk consecutive outputs k0 .. k0 + nk - 1 along the axis (the whole axis when it
// fits, else windows of kTileOutputs), and stages rows k0 - r .. k0 + nk + r - 1 (indices mod L) in shared memory, one
// coalesced 256-byte asynchronous copy (cp.async) per row, into one of two buffers: the next tile's rows are in flight
// while the current tile is computed. Output k reads staged rows k - k0 + j, j < taps, with no index wrapping. Each
// warp computes kQ consecutive outputs per lane, the taps in chunks of kQ: a chunk's 2 kQ - 1 staged values and kQ
// weights are loaded once into registers for kQ x kQ multiply-adds. Every output is still summed over j in order with
// the same rounding as k_gauss_axis, so the two give identical bits.
constexpr int kWholeAxis = 256;
constexpr int kTileOutputs = 64;
constexpr int kQ = 8;
constexpr int kMaxStagedRows = 384;                    // rows of real data
constexpr int kStagedAlloc = kMaxStagedRows + 2 * kQ;  // plus the zero rows a ragged chunk may read

__host__ __device__ inline int staged_outputs(int L, int radius) {
    return (L <= kWholeAxis && L + 2 * radius <= kMaxStagedRows) ? L : kTileOutputs;
}

struct AxisTile {
    long long base;  // element (outer index, axis 0, this lane's column)
    bool valid;      // this lane's column exists
    int k0, nk, rows;
};

__device__ __forceinline__ AxisTile axis_tile(int t, int k_tiles, int col_tiles, int KT, int L, long long stride,
                                              int radius, int lane) {
    AxisTile a;
    const int kt = t % k_tiles;
    const int rest = t / k_tiles;
    const int ct = rest % col_tiles;
    const int o = rest / col_tiles;
    const long long i = (long long)ct * 32 + lane;
    a.valid = i < stride;
    a.base = (long long)o * L * stride + i;
    a.k0 = kt * KT;
    a.nk = min(KT, L - a.k0);
    a.rows = a.nk + 2 * radius;
    return a;
}

// Staged row r of `buf` <- axis index (k0 - radius + r) mod L of this lane's column (asynchronously), zeros past the
// tile's rows and for a missing column; each warp takes rows grp, grp + ngrp, ...
__device__ __forceinline__ void stage_rows(double* buf, const double* __restrict__ in, const AxisTile& a, int L,
                                           long long stride, int radius, int grp, int ngrp, int lane) {
    int ax = ((a.k0 - radius + grp) % L + L) % L;
    for (int r = grp; r < a.rows + 2 * kQ; r += ngrp) {
        double* dst = buf + r * 32 + lane;
        if (r < a.rows && a.valid) {
            const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(in + a.base + (long long)ax * stride)
                         : "memory");
        } else {
            *dst = 0.0;
        }
        ax += ngrp;
        while (ax >= L) ax -= L;
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

__global__ void k_gauss_axis_tiled(const double* __restrict__ in, double* __restrict__ out, int L, long long stride,
                                   int col_tiles, int tiles, const double* __restrict__ w, int taps, int radius) {
    extern __shared__ double staged[];  // two buffers of (KT + 2 radius + 2 kQ) x 32
    const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5, ngrp = blockDim.x >> 5;
    const int KT = staged_outputs(L, radius);
    const int k_tiles = (L + KT - 1) / KT;
    const int chunks = (taps + kQ - 1) / kQ;
    const int buf_rows = KT + 2 * radius + 2 * kQ;
    int t = blockIdx.x;
    if (t >= tiles) return;
    AxisTile cur = axis_tile(t, k_tiles, col_tiles, KT, L, stride, radius, lane);
    int which = 0;
    stage_rows(staged, in, cur, L, stride, radius, grp, ngrp, lane);
    for (; t < tiles; t += gridDim.x) {
        const int tn = t + gridDim.x;
        AxisTile next = cur;
        if (tn < tiles) {
            next = axis_tile(tn, k_tiles, col_tiles, KT, L, stride, radius, lane);
            stage_rows(staged + (which ^ 1) * buf_rows * 32, in, next, L, stride, radius, grp, ngrp, lane);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();  // this tile's rows are in shared memory
        const double* tile = staged + which * buf_rows * 32;
        for (int kk0 = grp * kQ; kk0 < cur.nk; kk0 += ngrp * kQ) {
            double acc[kQ];
#pragma unroll
            for (int q = 0; q < kQ; ++q) acc[q] = 0.0;
            for (int c = 0; c < chunks; ++c) {
                const int jb = c * kQ;
                double x[2 * kQ - 1];
#pragma unroll
                for (int m = 0; m < 2 * kQ - 1; ++m) x[m] = tile[(kk0 + jb + m) * 32 + lane];
#pragma unroll
                for (int jj = 0; jj < kQ; ++jj) {
                    if (jb + jj < taps) {
                        const double wj = __ldg(w + jb + jj);
#pragma unroll
                        for (int q = 0; q < kQ; ++q) acc[q] = __dadd_rn(acc[q], __dmul_rn(wj, x[q + jj]));
                    }
                }
            }
            if (cur.valid) {
                double* o_ptr = out + cur.base + (long long)(cur.k0 + kk0) * stride;
#pragma unroll
                for (int q = 0; q < kQ; ++q)
                    if (kk0 + q < cur.nk) o_ptr[(long long)q * stride] = acc[q];
            }
        }
        __syncthreads();  // this buffer's reads are done before the next-but-one tile is staged into it
        cur = next;
        which ^= 1;
    }
}

// ---- Poisson noise --------------------------------------------------------------------------------------------------

struct Xoshiro {
    uint64_t s[4];
};

__device__ __forceinline__ uint64_t splitmix_finalise(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ uint64_t rotl64(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }

// GaussianGenerator's seeding (FrozenPhonons.swift:14-40): four SplitMix64 outputs.
__device__ __forceinline__ void seed_xoshiro(Xoshiro& g, uint64_t seed) {
    uint64_t x = seed;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        x += 0x9E3779B97F4A7C15ULL;
        g.s[i] = splitmix_finalise(x);
    }
}

__device__ __forceinline__ uint64_t next_u64(Xoshiro& g) {
    const uint64_t result = rotl64(g.s[1] * 5, 7) * 9;
    const uint64_t t = g.s[1] << 17;
    g.s[2] ^= g.s[0];
    g.s[3] ^= g.s[1];
    g.s[1] ^= g.s[2];
    g.s[0] ^= g.s[3];
    g.s[2] ^= t;
    g.s[3] = rotl64(g.s[3], 45);
    return result;
}

// PoissonSampler.uniform: the top 53 bits over 2^53.
__device__ __forceinline__ double uniform53(Xoshiro& g) {
    return (double)(next_u64(g) >> 11) * (1.0 / 9007199254740992.0);
}

constexpr int kKnuthLimit = 1 << 20;  // a mean below 10 needs about mean + 1 products
constexpr int kPtrsLimit = 1 << 16;   // PTRS accepts over 90 % of its attempts

// PoissonSampler.draw (ScanOperations.swift:137-166) with its arithmetic in the reference's order. `err` bit 1: an
// attempt limit was reached (never for a finite mean in practice); the value is then 0.
__device__ double poisson_draw(double lambda, Xoshiro& g, int* err) {
    if (lambda <= 0.0) return 0.0;
    if (lambda < 10.0) {
        const double limit = exp(-lambda);
        double product = uniform53(g);
        int k = 0;
        while (product > limit) {
            product = __dmul_rn(product, uniform53(g));
            if (++k >= kKnuthLimit) {
                atomicOr(err, 1);
                return 0.0;
            }
        }
        return (double)k;
    }
    const double slam = sqrt(lambda), loglam = log(lambda);
    const double b = __dadd_rn(0.931, __dmul_rn(2.53, slam));
    const double a = __dadd_rn(-0.059, __dmul_rn(0.02483, b));
    const double invalpha = __dadd_rn(1.1239, __ddiv_rn(1.1328, __dsub_rn(b, 3.4)));
    const double vr = __dsub_rn(0.9277, __ddiv_rn(3.6224, __dsub_rn(b, 2.0)));
    for (int attempt = 0; attempt < kPtrsLimit; ++attempt) {
        const double u = __dsub_rn(uniform53(g), 0.5);
        const double v = uniform53(g);
        const double us = __dsub_rn(0.5, fabs(u));
        if (us <= 0.0) continue;
        const double t = __dadd_rn(__ddiv_rn(__dmul_rn(2.0, a), us), b);
        const double kd = floor(__dadd_rn(__dadd_rn(__dmul_rn(t, u), lambda), 0.43));
        if (!(isfinite(kd) && fabs(kd) < 9e18)) continue;
        const long long k = (long long)kd;
        if (us >= 0.07 && v <= vr) return (double)k;
        if (k < 0 || (us < 0.013 && v > us)) continue;
        const double lhs = __dsub_rn(__dadd_rn(log(v), log(invalpha)),
                                     log(__dadd_rn(__ddiv_rn(a, __dmul_rn(us, us)), b)));
        const double rhs = __dsub_rn(__dadd_rn(-lambda, __dmul_rn((double)k, loglam)), lgamma((double)k + 1.0));
        if (lhs <= rhs) return (double)k;
    }
    atomicOr(err, 1);
    return 0.0;
}

// out[s count + i] for every value i and sample s, each drawn from the generator seeded by mix(mix(seed) + s count + i),
// the mix of a frozen-phonon configuration's seed (FrozenPhonons.swift:122-130). err bit 2: a value times the dose is
// not finite (the reference's sampler would never return); its draws are then 0.
__global__ void k_poisson(const double* __restrict__ in, double* __restrict__ out, long long count, int samples,
                          double dose, uint64_t seed, int* err) {
    const uint64_t mixed = splitmix_finalise(seed + 0x9E3779B97F4A7C15ULL);  // mix(seed), shared by every value
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x) {
        const double m = __dmul_rn(in[i], dose);
        if (!isfinite(m)) atomicOr(err, 2);
        const double lambda = (isfinite(m) && m > 0.0) ? m : 0.0;
        for (int s = 0; s < samples; ++s) {
            const long long e = (long long)s * count + i;
            double k = 0.0;
            if (lambda > 0.0) {
                Xoshiro g;
                seed_xoshiro(g, splitmix_finalise(mixed + (uint64_t)e + 0x9E3779B97F4A7C15ULL));
                k = poisson_draw(lambda, g, err);
            }
            out[e] = k;
        }
    }
}

// The reference's own stream (ScanOperations.swift:80-117): one generator seeded by `seed`, every sample's values drawn
// in order, so that a seed gives the reference's draws. The number of uniforms a draw takes depends on the draws, so
// the chain cannot be split: one thread walks it. err bits as k_poisson.
__global__ void k_poisson_sequential(const double* __restrict__ in, double* __restrict__ out, long long count,
                                     int samples, double dose, uint64_t seed, int* err) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    Xoshiro g;
    seed_xoshiro(g, seed);
    for (int s = 0; s < samples; ++s)
        for (long long i = 0; i < count; ++i) {
            const double m = __dmul_rn(in[i], dose);
            if (!isfinite(m)) {
                atomicOr(err, 2);
                out[(long long)s * count + i] = 0.0;
                continue;
            }
            out[(long long)s * count + i] = poisson_draw(m > 0.0 ? m : 0.0, g, err);
        }
}

// ---- integrated gradient --------------------------------------------------------------------------------------------

__global__ void k_gradient_load(const double* __restrict__ gx, const double* __restrict__ gy, long long stride,
                                long long n, double2* __restrict__ z) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        z[i] = make_double2(gx[i * stride], 0.0);
        z[n + i] = make_double2(gy[i * stride], 0.0);
    }
}

// NumPy's fftfreq(n, d) at index i: (i or i - n) times 1 / (n d), the scale rounded once as the reference does.
__device__ __forceinline__ double freq(int i, int n, double scale) {
    const int positive = (n - 1) / 2 + 1;
    return __dmul_rn((double)(i < positive ? i : i - n), scale);
}

// T^ = (kx g^x + ky g^y) / (2 pi i |k|^2) into z[0, n) (ImageOperations.swift:151-162).
__global__ void k_gradient_divide(double2* __restrict__ z, int nx, int ny, double sx_scale, double sy_scale) {
    const long long n = (long long)nx * ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i / ny), iy = (int)(i - (long long)ix * ny);
        const double kx = freq(ix, nx, sx_scale), ky = freq(iy, ny, sy_scale);
        double k = __dadd_rn(__dmul_rn(kx, kx), __dmul_rn(ky, ky));
        if (k == 0.0) k = 1e-12;
        const double2 fx = z[i], fy = z[n + i];
        const double a = __dadd_rn(__dmul_rn(fx.x, kx), __dmul_rn(fy.x, ky));
        const double b = __dadd_rn(__dmul_rn(fx.y, kx), __dmul_rn(fy.y, ky));
        const double c = __dmul_rn(2.0 * 3.14159265358979323846, k);
        z[i] = make_double2(__ddiv_rn(b, c), -__ddiv_rn(a, c));
    }
}

// One block: the minimum of the real parts (order-independent, so deterministic).
__global__ void k_real_min(const double2* __restrict__ z, long long n, double* __restrict__ out) {
    __shared__ double part[256];
    double m = INFINITY;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) m = fmin(m, z[i].x);
    part[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) part[threadIdx.x] = fmin(part[threadIdx.x], part[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0];
}

__global__ void k_sub_min(const double2* __restrict__ z, long long n, const double* __restrict__ low,
                          double* __restrict__ out) {
    const double m = *low;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = __dsub_rn(z[i].x, m);
}

}  // namespace

std::vector<double> gaussian_weights(double s) {
    const int radius = (int)(4.0 * s + 0.5);
    std::vector<double> w;
    w.reserve(2 * radius + 1);
    for (int x = -radius; x <= radius; ++x) w.push_back(std::exp(-0.5 * (double)(x * x) / (s * s)));
    double sum = 0.0;
    for (double v : w) sum += v;
    for (double& v : w) v /= sum;
    return w;
}

void gaussian_source_size_device(Context& ctx, int nx, int ny, long long v, double sigma_x, double sigma_y,
                                 double sampling_x, double sampling_y, const double* in, double* out) {
    SIMK_REQUIRE(std::isfinite(sigma_x) && std::isfinite(sigma_y) && sigma_x >= 0 && sigma_y >= 0,
                 "the source size must be finite and non-negative, got (" + std::to_string(sigma_x) + ", " +
                     std::to_string(sigma_y) + ") A");
    SIMK_REQUIRE(std::isfinite(sampling_x) && std::isfinite(sampling_y) && sampling_x > 0 && sampling_y > 0,
                 "the scan sampling must be finite and positive, got (" + std::to_string(sampling_x) + ", " +
                     std::to_string(sampling_y) + ") A");
    SIMK_REQUIRE(nx >= 1 && ny >= 1 && v >= 1, "the scan needs at least one position and one value");
    SIMK_REQUIRE(v <= (1LL << 40) / ((long long)nx * ny), "the scan holds more than 2^40 values");
    SIMK_REQUIRE((uintptr_t)in % sizeof(double) == 0 && (uintptr_t)out % sizeof(double) == 0,
                 "the values must be 8-byte aligned float64 arrays");
    const long long total = (long long)nx * ny * v;
    struct AxisPass {
        int L;
        long long stride;
        double sigma_px;
    };
    std::vector<AxisPass> passes;
    // along y (the second scan axis) then x, as scipy filters the axes in order
    if (sigma_y / sampling_y > 0) passes.push_back({ny, v, sigma_y / sampling_y});
    if (sigma_x / sampling_x > 0) passes.push_back({nx, (long long)ny * v, sigma_x / sampling_x});
    if (passes.empty()) {
        if (out != in) {
            SIMK_CUDA(cudaMemcpyAsync(out, in, total * sizeof(double), cudaMemcpyDeviceToDevice, ctx.stream));
            SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
        }
        return;
    }
    // one pass: in -> out (in -> work -> copy when they alias); two: in -> work -> out
    double* work = nullptr;
    if (passes.size() == 2 || out == in) {
        ctx.post_work.ensure(total * sizeof(double));
        work = ctx.post_work.as<double>();
    }
    std::vector<double> w_all;
    std::vector<size_t> w_off;
    for (const AxisPass& p : passes) {
        const std::vector<double> w = gaussian_weights(p.sigma_px);
        w_off.push_back(w_all.size());
        w_all.insert(w_all.end(), w.begin(), w.end());
    }
    w_off.push_back(w_all.size());
    ctx.post_weights.ensure(w_all.size() * sizeof(double));
    SIMK_CUDA(cudaMemcpyAsync(ctx.post_weights.ptr, w_all.data(), w_all.size() * sizeof(double),
                              cudaMemcpyHostToDevice, ctx.stream));
    const double* src = in;
    for (size_t p = 0; p < passes.size(); ++p) {
        const int taps = (int)(w_off[p + 1] - w_off[p]);
        const bool last = p + 1 == passes.size();
        double* dst = (last && src != out) ? out : work;
        const int L = passes[p].L, radius = taps / 2;
        const long long stride = passes[p].stride;
        const int rows = staged_outputs(L, radius) + 2 * radius;
        const double* w = ctx.post_weights.as<double>() + w_off[p];
        {
            KernelTimer t(ctx, "gauss_axis", 16.0 * (double)total);
            if (stride >= 32 && rows <= kMaxStagedRows) {
                // the launch limit for this device (set on every call: contexts on other threads may do the same)
                SIMK_CUDA(cudaFuncSetAttribute(k_gauss_axis_tiled, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               2 * kStagedAlloc * 32 * (int)sizeof(double)));
                const long long outer = total / ((long long)L * stride);
                const int KT = staged_outputs(L, radius);
                const long long col_tiles = (stride + 31) / 32;
                const long long tiles = outer * col_tiles * ((L + KT - 1) / KT);
                SIMK_REQUIRE(tiles < (1LL << 31), "the scan's values are too many for one filter launch");
                const size_t smem = 2 * (size_t)(rows + 2 * kQ) * 32 * sizeof(double);  // two staging buffers
                int per_sm = 0;
                SIMK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gauss_axis_tiled, 256, smem));
                const long long resident = (long long)ctx.sm_count * std::max(1, per_sm);
                const int grid = (int)std::max<long long>(1, std::min<long long>(tiles, resident));
                k_gauss_axis_tiled<<<grid, 256, smem, ctx.stream>>>(src, dst, L, stride, (int)col_tiles, (int)tiles,
                                                                     w, taps, radius);
            } else {
                k_gauss_axis<<<blocks_for(total), 256, 0, ctx.stream>>>(src, dst, total, L, stride, w, taps, radius);
            }
        }
        ++ctx.launches;
        SIMK_CUDA(cudaGetLastError());
        src = dst;
    }
    if (src != out)
        SIMK_CUDA(cudaMemcpyAsync(out, src, total * sizeof(double), cudaMemcpyDeviceToDevice, ctx.stream));
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
}

void poisson_noise_device(Context& ctx, long long count, const double* in, double dose, int samples, uint64_t seed,
                          double* out) {
    SIMK_REQUIRE(std::isfinite(dose) && dose >= 0, "the dose must be finite and non-negative, got " + std::to_string(dose));
    SIMK_REQUIRE(samples >= 1, "samples must be at least 1, got " + std::to_string(samples));
    SIMK_REQUIRE(count >= 0, "negative value count");
    SIMK_REQUIRE(samples == 1 || out != in, "several samples cannot overwrite their input");
    SIMK_REQUIRE(count <= (1LL << 40) / samples, "more than 2^40 values and samples");
    if (count == 0) return;
    ctx.post_flag.ensure(sizeof(int));
    SIMK_CUDA(cudaMemsetAsync(ctx.post_flag.ptr, 0, sizeof(int), ctx.stream));
    {
        KernelTimer t(ctx, "poisson", 8.0 * (double)count + 8.0 * (double)count * samples);
        if (ctx.poisson_stream == 1)
            k_poisson_sequential<<<1, 1, 0, ctx.stream>>>(in, out, count, samples, dose, seed, ctx.post_flag.as<int>());
        else
            k_poisson<<<blocks_for(count), 256, 0, ctx.stream>>>(in, out, count, samples, dose, seed,
                                                                 ctx.post_flag.as<int>());
    }
    ++ctx.launches;
    SIMK_CUDA(cudaGetLastError());
    int h = 0;
    SIMK_CUDA(cudaMemcpyAsync(&h, ctx.post_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
    SIMK_REQUIRE(!(h & 2), "a value times the dose is not finite: Poisson noise needs finite means");
    if (h & 1) throw Error(SIMK_ERR_CUDA, "the Poisson sampler reached its attempt limit");
}

void integrate_gradient_device(Context& ctx, int nx, int ny, double sampling_x, double sampling_y, const double* gx,
                               const double* gy, long long stride, double* out) {
    SIMK_REQUIRE(std::isfinite(sampling_x) && std::isfinite(sampling_y) && sampling_x > 0 && sampling_y > 0,
                 "invalid sampling (" + std::to_string(sampling_x) + ", " + std::to_string(sampling_y) + ") A");
    SIMK_REQUIRE(nx >= 2 && ny >= 2, "the gradient's images need at least 2 points per axis, got " +
                                         std::to_string(nx) + " x " + std::to_string(ny));
    SIMK_REQUIRE(stride >= 1, "the component stride must be at least 1");
    SIMK_REQUIRE((long long)nx * ny <= (1LL << 28), "the gradient's images hold more than 2^28 pixels");
    const long long n = (long long)nx * ny;
    ctx.post_spectra.ensure(2 * n * sizeof(double2));
    ctx.post_min.ensure(sizeof(double));
    double2* z = ctx.post_spectra.as<double2>();
    k_gradient_load<<<blocks_for(n), 256, 0, ctx.stream>>>(gx, gy, stride, n, z);
    ++ctx.launches;
    SIMK_CUDA(cudaGetLastError());
    const LinePlan& prow = ctx.plan(ny, 64);
    const LinePlan& pcol = ctx.plan(nx, 64);
    fft2(prow, pcol, z, nx, ny, 2, -1, 1.0, ctx.stream, &ctx.launches);
    k_gradient_divide<<<blocks_for(n), 256, 0, ctx.stream>>>(z, nx, ny, 1.0 / ((double)nx * sampling_x),
                                                             1.0 / ((double)ny * sampling_y));
    ++ctx.launches;
    SIMK_CUDA(cudaGetLastError());
    fft2(prow, pcol, z, nx, ny, 1, +1, 1.0 / (double)n, ctx.stream, &ctx.launches);
    k_real_min<<<1, 256, 0, ctx.stream>>>(z, n, ctx.post_min.as<double>());
    ++ctx.launches;
    SIMK_CUDA(cudaGetLastError());
    k_sub_min<<<blocks_for(n), 256, 0, ctx.stream>>>(z, n, ctx.post_min.as<double>(), out);
    ++ctx.launches;
    SIMK_CUDA(cudaGetLastError());
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
}

}  // namespace simk
