// noalloc.cu -- simk_probe_spectrum_noalloc: the probe spectrum Psi0 written into a caller-owned device buffer without
// any device allocation by the library.
//
// Who needs it: callers that embed this library inside a host framework which owns all device memory -- a caching
// allocator such as PyTorch's, an XLA/JAX custom call, or an application that pre-reserves its HBM budget -- where a
// cudaMalloc inside the call would bypass the framework's accounting and may synchronise the device. The regular
// entry point (simk_probe_spectrum) allocates a float64 work buffer and a norm scalar per call; this variant keeps its
// scratch in a fixed file-scope device array instead.
//
// Scratch: kNoallocPartials float64 partial sums plus one float64 norm, 32 KiB + 8 B in all, held by every device that
// loads the library until the process exits. One partial covers kNoallocChunk pixels, so a grid may have at most
// kNoallocPartials * kNoallocChunk = 4,194,304 pixels (2048 x 2048); larger grids are refused. Every call reuses the
// same array and leaves its last contents there; each call overwrites every partial it reads before reading it, so
// nothing needs clearing between calls. Calls whose work overlaps on the GPU (on different streams, or from different
// host threads without ordering) race on the shared array and must be serialised by the caller.
//
// Set-up: the first call on a device, with that device current, looks up the array's device address with
// cudaGetSymbolAddress and caches it; make that first call before any stream capture. The address belongs to the
// context the call runs in (the device's primary context, as the runtime API uses), so every later call that is not
// being captured looks it up again, which allocates nothing: a cudaDeviceReset between calls then cannot leave a stale
// pointer behind. A call made while its stream is being captured uses the cached address.
//
// Errors: a CUDA error already pending on the calling thread (left by the host framework's own work) is reported as
// such and left pending for its owner; nothing is launched then. Otherwise a launch error of this call is reported and
// cleared.
#include <mutex>

#include "common.cuh"

namespace simk {

constexpr int kNoallocPartials = 4096;
constexpr int kNoallocChunk = 1024;
constexpr int kNoallocMaxDevices = 64;

// [0, kNoallocPartials): per-block sums of |Psi|^2; [kNoallocPartials]: the total.
static __device__ __align__(256) double g_noalloc_scratch[kNoallocPartials + 1];

namespace {

struct NoallocProbe {
    int nx, ny;
    double dx, dy;
    double lambda, cutoff, dax, day;
    int soft, infinite;
    double ab[25];
};

// Psi0 before normalisation at pixel i: aperture . exp(-i chi), as Probe.centredSpectrum computes it
// (Sources/SimulatoProbe/Probe.swift:25-48, 113-136; Aberrations.swift:39-59), in float64.
__device__ double2 noalloc_probe_value(long long i, const NoallocProbe& p) {
    const int ix = (int)(i / p.ny), iy = (int)(i % p.ny);
    const double kx = fftfreq_at(ix, p.nx, p.dx), ky = fftfreq_at(iy, p.ny, p.dy);
    const double alpha = sqrt(kx * kx + ky * ky) * p.lambda;
    const double phi = atan2(ky, kx);
    double ap;
    if (p.infinite) ap = 1.0;
    else if (p.soft) {
        if (ix == 0 && iy == 0) ap = 1.0;
        else {
            const double a = cos(phi) * p.dax, b = sin(phi) * p.day;
            ap = fmin(fmax((p.cutoff - alpha) / sqrt(a * a + b * b) + 0.5, 0.0), 1.0);
        }
    } else ap = (alpha <= p.cutoff) ? 1.0 : 0.0;
    const double* c = p.ab;
    const double a2 = alpha * alpha;
    double x = 0.0;
    if (c[0] != 0 || c[1] != 0 || c[2] != 0) x = x + 1.0 / 2 * a2 * (c[0] + c[1] * cos(2 * (phi - c[2])));
    if (c[3] != 0 || c[4] != 0 || c[5] != 0 || c[6] != 0)
        x = x + 1.0 / 3 * (a2 * alpha) * (c[3] * cos(phi - c[4]) + c[5] * cos(3 * (phi - c[6])));
    if (c[7] != 0 || c[8] != 0 || c[9] != 0 || c[10] != 0 || c[11] != 0)
        x = x + 1.0 / 4 * (a2 * a2) * (c[7] + c[8] * cos(2 * (phi - c[9])) + c[10] * cos(4 * (phi - c[11])));
    if (c[12] != 0 || c[13] != 0 || c[14] != 0 || c[15] != 0 || c[16] != 0 || c[17] != 0)
        x = x + 1.0 / 5 * (a2 * a2 * alpha) *
                    (c[12] * cos(phi - c[13]) + c[14] * cos(3 * (phi - c[15])) + c[16] * cos(5 * (phi - c[17])));
    if (c[18] != 0 || c[19] != 0 || c[20] != 0 || c[21] != 0 || c[22] != 0 || c[23] != 0 || c[24] != 0)
        x = x + 1.0 / 6 * (a2 * a2 * a2) *
                    (c[18] + c[19] * cos(2 * (phi - c[20])) + c[21] * cos(4 * (phi - c[22])) +
                     c[23] * cos(6 * (phi - c[24])));
    const double chi = x * (2 * M_PI / p.lambda);
    double s, co;
    sincos(-chi, &s, &co);
    return make_double2(ap * co, ap * s);
}

// Block b sums |Psi0|^2 over pixels [b * chunk, (b + 1) * chunk) into partials[b] (fixed order: deterministic).
__global__ void k_noalloc_partials(NoallocProbe p, long long N, double* partials) {
    __shared__ double part[256];
    const long long first = (long long)blockIdx.x * kNoallocChunk;
    double s = 0.0;
    for (long long i = first + threadIdx.x; i < min(first + kNoallocChunk, N); i += blockDim.x) {
        const double2 v = noalloc_probe_value(i, p);
        s += v.x * v.x + v.y * v.y;
    }
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = part[0];
}

// One block: total = sum of the first `count` partials, in a fixed order.
__global__ void k_noalloc_total(double* scratch, int count) {
    __shared__ double part[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) s += scratch[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) scratch[kNoallocPartials] = part[0];
}

__global__ void k_noalloc_write(NoallocProbe p, long long N, const double* scratch, float2* out) {
    const double f = 1.0 / sqrt(scratch[kNoallocPartials]);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const double2 v = noalloc_probe_value(i, p);
        out[i] = make_float2((float)(v.x * f), (float)(v.y * f));
    }
}

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoallocMaxDevices] = {};

// The device address of the scratch array on the current device: looked up on the first call and on every call whose
// stream is not being captured; a call under capture takes the address cached by an earlier call.
double* noalloc_scratch_address(cudaStream_t stream) {
    int dev = 0;
    SIMK_CUDA(cudaGetDevice(&dev));
    SIMK_REQUIRE(dev >= 0 && dev < kNoallocMaxDevices, "device ordinal out of range");
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    SIMK_CUDA(cudaStreamIsCapturing(stream, &capture));
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev] || capture == cudaStreamCaptureStatusNone) {
        SIMK_REQUIRE(capture == cudaStreamCaptureStatusNone,
                     "simk_probe_spectrum_noalloc: the first call on a device must come before any stream capture");
        void* ptr = nullptr;
        SIMK_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        g_noalloc_ptr[dev] = static_cast<double*>(ptr);
    }
    return g_noalloc_ptr[dev];
}

}  // namespace

void probe_spectrum_noalloc(const simk_grid* grid, const simk_probe* probe, void* out_device, void* stream) {
    SIMK_REQUIRE(grid && probe && out_device, "null argument");
    SIMK_REQUIRE(grid->nx >= 2 && grid->ny >= 2, "grid lengths must be at least 2");
    SIMK_REQUIRE(std::isfinite(grid->extent_x) && std::isfinite(grid->extent_y) && grid->extent_x > 0 &&
                     grid->extent_y > 0,
                 "the extent must be finite and positive");
    const long long N = (long long)grid->nx * grid->ny;
    const long long max_pixels = (long long)kNoallocPartials * kNoallocChunk;
    if (N > max_pixels)
        throw Error(SIMK_ERR_INVALID, "simk_probe_spectrum_noalloc: grid of " + std::to_string(N) +
                                          " pixels exceeds the fixed scratch's maximum of " +
                                          std::to_string(max_pixels) + " pixels (2048 x 2048)");
    SIMK_REQUIRE(std::isfinite(probe->energy) && probe->energy > 0, "the energy must be finite and positive");
    SIMK_REQUIRE(probe->semiangle_mrad > 0 && !std::isnan(probe->semiangle_mrad), "invalid aperture");
    for (int i = 0; i < 25; ++i) SIMK_REQUIRE(std::isfinite(probe->aberrations[i]), "every aberration must be finite");
    NoallocProbe p{};
    p.nx = grid->nx;
    p.ny = grid->ny;
    p.dx = grid->extent_x / grid->nx;
    p.dy = grid->extent_y / grid->ny;
    p.lambda = wavelength(probe->energy);
    p.infinite = std::isinf(probe->semiangle_mrad) ? 1 : 0;
    p.soft = probe->soft ? 1 : 0;
    p.cutoff = probe->semiangle_mrad * 1e-3;
    p.dax = 1.0 / ((double)p.nx * p.dx) * 1e3 * p.lambda * 1e-3;
    p.day = 1.0 / ((double)p.ny * p.dy) * 1e3 * p.lambda * 1e-3;
    for (int i = 0; i < 25; ++i) p.ab[i] = probe->aberrations[i];
    // an error someone else left pending stays theirs: report it without clearing it, and launch nothing
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess)
        throw Error(SIMK_ERR_CUDA, std::string("simk_probe_spectrum_noalloc: a CUDA error was already pending on this "
                                               "thread (") + cudaGetErrorString(pending) + "); nothing was launched");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* scratch = noalloc_scratch_address(s);
    const int blocks = (int)((N + kNoallocChunk - 1) / kNoallocChunk);
    k_noalloc_partials<<<blocks, 256, 0, s>>>(p, N, scratch);
    k_noalloc_total<<<1, 256, 0, s>>>(scratch, blocks);
    const int wblocks = (int)std::min<long long>((N + 255) / 256, 148LL * 16);
    k_noalloc_write<<<wblocks, 256, 0, s>>>(p, N, scratch, static_cast<float2*>(out_device));
    SIMK_CUDA(cudaGetLastError());  // none was pending before the launches: an error here is this call's
}

}  // namespace simk
