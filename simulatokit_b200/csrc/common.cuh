// common.cuh -- shared types of libsimulato_cuda: complex helpers, the context, device buffers, error plumbing.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/simulato_cuda.h"

namespace simk {

// ---- errors ---------------------------------------------------------------------------------------------------------
struct Error : std::runtime_error {
    int status;
    Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        int st = (e == cudaErrorMemoryAllocation) ? SIMK_ERR_MEMORY : SIMK_ERR_CUDA;
        throw Error(st, std::string(what) + ": " + cudaGetErrorString(e));
    }
}
#define SIMK_CUDA(call) ::simk::check_cuda((call), #call)
#define SIMK_REQUIRE(cond, msg) \
    do { if (!(cond)) throw ::simk::Error(SIMK_ERR_INVALID, (msg)); } while (0)

// ---- complex arithmetic on float2 / double2 -------------------------------------------------------------------------
template <typename T> struct C2;
template <> struct C2<float> { using type = float2; };
template <> struct C2<double> { using type = double2; };
template <typename T> using c2_t = typename C2<T>::type;

template <typename V> __host__ __device__ __forceinline__ V mk(decltype(V::x) a, decltype(V::x) b) { V r; r.x = a; r.y = b; return r; }
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
    return mk<V>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename V> __host__ __device__ __forceinline__ V cmulc(V a, V b) {
    return mk<V>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename V> __host__ __device__ __forceinline__ V cconj(V a) { return mk<V>(a.x, -a.y); }
// multiply by s*i, s = +1 or -1: i(a + ib) = -b + ia
template <typename V, typename S> __host__ __device__ __forceinline__ V mul_si(V a, S s) { return mk<V>(-s * a.y, s * a.x); }
template <typename V> __host__ __device__ __forceinline__ decltype(V::x) cabs2(V a) { return a.x * a.x + a.y * a.y; }

// ---- device buffers -------------------------------------------------------------------------------------------------
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    explicit DeviceBuffer(size_t n) { alloc(n); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr; o.bytes = 0; }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) { release(); ptr = o.ptr; bytes = o.bytes; o.ptr = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DeviceBuffer() { release(); }
    void alloc(size_t n) {
        release();
        if (n == 0) return;
        SIMK_CUDA(cudaMalloc(&ptr, n));
        bytes = n;
    }
    void ensure(size_t n) { if (bytes < n) alloc(n); }
    void release() { if (ptr) { cudaFree(ptr); ptr = nullptr; bytes = 0; } }
    template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

// ---- geometry -------------------------------------------------------------------------------------------------------
struct GridGeom {
    int nx = 0, ny = 0;
    double ex = 0, ey = 0;
    double dx() const { return ex / nx; }
    double dy() const { return ey / ny; }
    long long count() const { return (long long)nx * ny; }
    bool operator<(const GridGeom& o) const { return std::tie(nx, ny, ex, ey) < std::tie(o.nx, o.ny, o.ex, o.ey); }
};

// NumPy's fftfreq(n, d)[i] (Sources/SimulatoCore/Grid.swift:82-86), usable on both sides.
__host__ __device__ inline double fftfreq_at(int i, int n, double d) {
    double val = 1.0 / ((double)n * d);
    int pos = (n - 1) / 2 + 1;
    return (double)(i < pos ? i : i - n) * val;
}

// sin(pi x), cos(pi x) on the host, x reduced to [-1, 1] first so the argument of sin/cos stays small.
inline void host_sincospi(double x, double* s, double* c) {
    double r = std::fmod(x, 2.0);
    if (r > 1.0) r -= 2.0;
    if (r < -1.0) r += 2.0;
    *s = std::sin(M_PI * r);
    *c = std::cos(M_PI * r);
}

// Relativistic wavelength [A] and interaction parameter (Sources/SimulatoCore/ElectronBeam.swift:21-43).
double wavelength(double energy);
double interaction_parameter(double energy);

}  // namespace simk
