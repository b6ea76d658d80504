// scanops.cuh -- scan post-processing on the device: the Gaussian source size, Poisson noise and the integration of a
// gradient field (integrated centre of mass). Inputs and outputs are float64 device arrays; the scan's values are
// row-major [scan x][scan y][values of one position].
#pragma once

#include "context.cuh"

namespace simk {

// ScanMeasurement.gaussianSourceSize (ScanOperations.swift:19-36): `in` [nx][ny][v] filtered periodically along the
// second scan axis with sigma_y / sampling_y pixels, then along the first with sigma_x / sampling_x, into `out`
// (which may equal `in`). Weights and summation order as the reference: bit-equal to its float64 loop.
void gaussian_source_size_device(Context& ctx, int nx, int ny, long long v, double sigma_x, double sigma_y,
                                 double sampling_x, double sampling_y, const double* in, double* out);

// Poisson noise for `dose` electrons per value (ScanOperations.swift:80-117): out[s count + i] ~ Poisson(max(in[i]
// dose, 0)) for s < samples, each value and sample drawn by the reference's sampler from a generator of its own seeded
// by mix(mix(seed) + s count + i). `out` may equal `in` when samples is 1.
void poisson_noise_device(Context& ctx, long long count, const double* in, double dose, int samples, uint64_t seed,
                          double* out);

// integrateGradient (ImageOperations.swift:140-167) on nx x ny images: gx[i stride], gy[i stride] for pixel i; the
// result (real part of the inverse transform less its minimum) into out[nx ny].
void integrate_gradient_device(Context& ctx, int nx, int ny, double sampling_x, double sampling_y, const double* gx,
                               const double* gy, long long stride, double* out);

// The periodic Gaussian weights of sigma_px pixels (ScanOperations.swift:43-50), as the host computes them.
std::vector<double> gaussian_weights(double sigma_px);

}  // namespace simk
