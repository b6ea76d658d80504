// physics.cu -- the float64 parts of the hot path on the device: the Lobato projected potential (infinite
// projection), the bandlimited transmission functions, the Fresnel propagators, the probe spectrum and shift ramps, and
// the detector maps with their reduction kernel.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "context.cuh"

namespace simk {

#include "lobato_table.inc"

// ---- beam (Sources/SimulatoCore/ElectronBeam.swift:21-43, PhysicalConstants.swift:8-31) ------------------------------
namespace {
constexpr double kPlanck = 6.62607004e-34, kElectronMass = 9.10938356e-31, kSpeedOfLight = 299792458.0,
                 kElementaryCharge = 1.6021766208e-19, kKappa = 0.0208865737082965;
constexpr double kAseKg = 6.0221408585491615e+26, kAseCoulomb = 6.241509125883258e+18,
                 kAseSecond = 98226947884640.62, kAseJoule = 6.241509125883258e+18;
}  // namespace

double wavelength(double energy) {
    const double c2 = kSpeedOfLight * kSpeedOfLight;
    return kPlanck * kSpeedOfLight / std::sqrt(energy * (2 * kElectronMass * c2 / kElementaryCharge + energy)) /
           kElementaryCharge * 1.0e10;
}

double interaction_parameter(double energy) {
    const double mass =
        (1 + kElementaryCharge * energy / (kElectronMass * (kSpeedOfLight * kSpeedOfLight))) * kElectronMass;
    const double hsj = kPlanck * kAseSecond * kAseJoule;
    return 2 * M_PI * mass * kAseKg * kElementaryCharge * kAseCoulomb * wavelength(energy) / (hsj * hsj);
}

// ---- device helpers -------------------------------------------------------------------------------------------------
__device__ __forceinline__ double antialias_at(int ix, int iy, const GridDev g) {
    // Sources/SimulatoCore/Antialias.swift:18-39: cutoff 0.6666666 / (2 max dx), taper 0.01 / max dx
    const double dmax = fmax(g.dx, g.dy);
    const double kc = 0.6666666 / dmax / 2.0;
    const double w = 0.01 / dmax;
    const double kx = fftfreq_at(ix, g.nx, g.dx), ky = fftfreq_at(iy, g.ny, g.dy);
    const double r = sqrt(kx * kx + ky * ky);
    if (r > kc) return 0.0;
    if (r > kc - w) return 0.5 * (1.0 + cos(M_PI * (r - kc + w) / w));
    return 1.0;
}

__global__ void k_zero_d2(double2* a, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        a[i] = make_double2(0.0, 0.0);
}

// f(k^2)/S(k) for one element (LobatoParameterization.swift:51-69; ProjectedPotential.swift:130-153).
__global__ void k_lobato_kernel(double* out, GridDev g, const double* AB, double pi, double pi2) {
    const long long N = (long long)g.nx * g.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i / g.ny), iy = (int)(i % g.ny);
        const double kx = fftfreq_at(ix, g.nx, g.dx), ky = fftfreq_at(iy, g.ny, g.dy);
        const double k2 = kx * kx + ky * ky;
        const double q = (4.0 * pi2) * k2;
        double sum = 0.0;
#pragma unroll
        for (int t = 0; t < 5; ++t) {
            const double A = AB[t], B = AB[5 + t];
            const double d = q + B * B;
            sum = sum + (A / B / d + A * B / (d * d));
        }
        const double f = (8.0 * pi) * sum;
        const double a = kx * g.dx, b = ky * g.dy;
        const double kk = sqrt(a * a + b * b);
        const double s = (ix == 0 && iy == 0) ? g.dx * g.dy : sin(kk) / kk * (g.dx * g.dy);
        out[i] = f / s;
    }
}

__global__ void k_scatter(double2* D, const int* pix, const double* w, int count) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
        D[pix[i]] = make_double2(w[i], 0.0);
}

// S += sum over the `count` spectra D_q (N apart) of D_q K_{elem[q]}, the elements in the given (increasing Z) order, so
// each pixel sees the same sequence of additions as one element at a time.
__global__ void k_accum_spectra(double2* S, const double2* D, const double* K, const int* elem, int count, long long N) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double2 s = S[i];
        for (int q = 0; q < count; ++q) {
            const double k = K[(long long)elem[q] * N + i];
            const double2 d = D[(long long)q * N + i];
            s = make_double2(s.x + d.x * k, s.y + d.y * k);
        }
        S[i] = s;
    }
}

__global__ void k_real_part(double* V, const double2* S, long long N) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        V[i] = S[i].x;
}

__global__ void k_exp_i_sigma_v(double2* T, const double* V, double sigma, long long N) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double s, c;
        sincos(sigma * V[i], &s, &c);  // sigma V in float64 before rounding
        T[i] = make_double2(c, s);
    }
}

// `count` fields of nx x ny, one after another.
__global__ void k_mul_antialias(double2* T, GridDev g, int count) {
    const long long N = (long long)g.nx * g.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N * count;
         i += (long long)gridDim.x * blockDim.x) {
        const long long k = i % N;
        const double a = antialias_at((int)(k / g.ny), (int)(k % g.ny), g);
        T[i] = make_double2(T[i].x * a, T[i].y * a);
    }
}

__global__ void k_to_float2(float2* out, const double2* in, long long N) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

// P = exp(-i pi lambda dz k^2) A, times e^{-2 pi i dz (kx tan tx + ky tan ty)} (Multislice.swift:108-130).
__global__ void k_propagator(float2* P, GridDev g, double lambda, double dz, double ttx, double tty, int tilted) {
    const long long N = (long long)g.nx * g.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i / g.ny), iy = (int)(i % g.ny);
        const double kx = fftfreq_at(ix, g.nx, g.dx), ky = fftfreq_at(iy, g.ny, g.dy);
        const double k2 = kx * kx + ky * ky;
        const double x = -k2 * M_PI * dz * lambda;  // float64 phase argument
        const double a = antialias_at(ix, iy, g);
        double s, c;
        sincos(x, &s, &c);
        double re = c * a, im = s * a;
        if (tilted) {
            const double t = -2.0 * M_PI * dz * (kx * ttx + ky * tty);
            double st, ct;
            sincos(t, &st, &ct);
            const double r2 = re * ct - im * st, i2 = re * st + im * ct;
            re = r2;
            im = i2;
        }
        P[i] = make_float2((float)re, (float)im);
    }
}

inline int blocks_for(long long n, int threads = 256) {
    long long b = (n + threads - 1) / threads;
    return (int)std::max<long long>(1, std::min<long long>(b, 148LL * 16));
}

const Propagator& Context::propagator(const GridGeom& g, double energy, double dzv, double tx, double ty) {
    auto key = std::make_tuple(g.nx, g.ny, g.ex, g.ey, energy, dzv, tx, ty);
    auto it = props.find(key);
    if (it != props.end()) return *it->second;
    auto p = std::make_unique<Propagator>();
    p->p.alloc(sizeof(float2) * g.count());
    const bool tilted = (tx != 0.0 || ty != 0.0);
    k_propagator<<<blocks_for(g.count()), 256, 0, stream>>>(p->p.as<float2>(), grid_dev(g), wavelength(energy), dzv,
                                                            std::tan(tx / 1e3), std::tan(ty / 1e3), tilted ? 1 : 0);
    SIMK_CUDA(cudaGetLastError());
    ++launches;
    auto& ref = *p;
    props[key] = std::move(p);
    return ref;
}

// ---- potential from atoms -------------------------------------------------------------------------------------------
void build_potential_from_atoms(Context& ctx, PotentialImpl& pot, int pi_choice, int n_atoms, const int* Z,
                                const double* xyz, const int* slice_of_atom) {
    const GridGeom& g = pot.g;
    const long long N = g.count();
    const int S = pot.n_slices();
    for (int a = 0; a < n_atoms; ++a) {
        SIMK_REQUIRE(Z[a] >= 1 && Z[a] <= 103, "unsupported element: Z = " + std::to_string(Z[a]));
        SIMK_REQUIRE(slice_of_atom[a] >= 0 && slice_of_atom[a] < S, "slice index out of range");
        SIMK_REQUIRE(std::isfinite(xyz[3 * a]) && std::isfinite(xyz[3 * a + 1]), "non-finite atom position");
    }
    // elements in increasing Z (ProjectedPotential.swift:158)
    std::vector<int> elements(Z, Z + n_atoms);
    std::sort(elements.begin(), elements.end());
    elements.erase(std::unique(elements.begin(), elements.end()), elements.end());
    const int E = (int)elements.size();
    // merged bilinear weights per (slice, element): atoms in structure order, weight by weight (add.at order,
    // ProjectedPotential.swift:178-201; merged per pixel as MetalEngine.swift:254-275)
    std::vector<int> pix;
    std::vector<double> wts;
    std::vector<long long> group_ptr(1, 0);
    std::vector<double> dense(N, 0.0);
    std::vector<char> touched(N, 0);
    std::vector<int> touched_list;
    std::vector<std::vector<int>> atoms_of(S * E);
    for (int a = 0; a < n_atoms; ++a) {
        int e = (int)(std::lower_bound(elements.begin(), elements.end(), Z[a]) - elements.begin());
        atoms_of[slice_of_atom[a] * E + e].push_back(a);
    }
    auto mod = [](long long v, long long m) { long long r = v % m; return r < 0 ? r + m : r; };
    for (int j = 0; j < S; ++j) {
        for (int e = 0; e < E; ++e) {
            const auto& list = atoms_of[j * E + e];
            touched_list.clear();
            for (int k = 0; k < 4; ++k) {
                for (int a : list) {
                    const double px = xyz[3 * a] / g.dx(), py = xyz[3 * a + 1] / g.dy();
                    const double r = std::floor(px), c = std::floor(py);
                    const double x = px - r, y = py - c, xy = x * y;
                    const double w = (k == 0) ? 1 + xy - y - x : (k == 1) ? x - xy : (k == 2) ? y - xy : xy;
                    const long long i = mod((long long)r + ((k == 1 || k == 3) ? 1 : 0), g.nx);
                    const long long jj = mod((long long)c + ((k >= 2) ? 1 : 0), g.ny);
                    const long long p = i * g.ny + jj;
                    if (!touched[p]) {
                        touched[p] = 1;
                        touched_list.push_back((int)p);
                    }
                    dense[p] += w;
                }
            }
            std::sort(touched_list.begin(), touched_list.end());
            for (int p : touched_list) {
                pix.push_back(p);
                wts.push_back(dense[p]);
                dense[p] = 0.0;
                touched[p] = 0;
            }
            group_ptr.push_back((long long)pix.size());
        }
    }
    // device: kernels f/S per element (float64), then per slice sum_e FFT(deltas_e) f_e/S -> IFFT -> Re
    DeviceBuffer& d_pix = ctx.pot_pix;
    DeviceBuffer& d_w = ctx.pot_w;
    d_pix.ensure(std::max<size_t>(1, pix.size() * sizeof(int)));
    d_w.ensure(std::max<size_t>(1, wts.size() * sizeof(double)));
    if (!pix.empty()) {
        SIMK_CUDA(cudaMemcpyAsync(d_pix.ptr, pix.data(), pix.size() * sizeof(int), cudaMemcpyHostToDevice, ctx.stream));
        SIMK_CUDA(cudaMemcpyAsync(d_w.ptr, wts.data(), wts.size() * sizeof(double), cudaMemcpyHostToDevice, ctx.stream));
    }
    DeviceBuffer& kern = ctx.pot_kern;
    DeviceBuffer& ab = ctx.pot_ab;
    kern.ensure(std::max<long long>(1, E) * N * sizeof(double));
    ab.ensure(std::max(1, E) * 10 * sizeof(double));
    std::vector<double> hab(std::max(1, E) * 10);
    const double pi = (pi_choice == SIMK_PI_ABTEM_FLOAT32) ? (double)(float)M_PI : M_PI;
    const double pi2 = (pi_choice == SIMK_PI_ABTEM_FLOAT32) ? (double)(float)(M_PI * M_PI) : M_PI * M_PI;
    for (int e = 0; e < E; ++e) {
        const double* p = kLobatoTable[elements[e] - 1];
        for (int t = 0; t < 5; ++t) {
            // A = pi^2 a / b^1.5 / kappa, B = 2 pi / sqrt(b) with the exact pi (LobatoParameterization.swift:38-44)
            hab[e * 10 + t] = M_PI * M_PI * p[t] / std::pow(p[5 + t], 1.5) / kKappa;
            hab[e * 10 + 5 + t] = 2 * M_PI / std::sqrt(p[5 + t]);
        }
    }
    SIMK_CUDA(cudaMemcpyAsync(ab.ptr, hab.data(), hab.size() * sizeof(double), cudaMemcpyHostToDevice, ctx.stream));
    for (int e = 0; e < E; ++e) {
        k_lobato_kernel<<<blocks_for(N), 256, 0, ctx.stream>>>(kern.as<double>() + e * N, grid_dev(g),
                                                                ab.as<double>() + e * 10, pi, pi2);
        ++ctx.launches;
    }
    SIMK_CUDA(cudaGetLastError());
    pot.V.alloc(std::max<long long>(1, S) * N * sizeof(double));
    // Slices go in groups: the delta images of a group's slices (the elements present in each, in increasing Z) are
    // transformed as one batch of at most `chunk` images (64 MiB, at least one slice's worth up to 256 MiB), each
    // slice's spectrum is accumulated from its own images in that order, and the group's spectra (at most `gmax`)
    // are transformed back together. A slice whose images exceed the batch is a group of its own, its images
    // transformed in turn. Every line transform and every pixel's sum is the same as one slice at a time.
    const long long img = N * (long long)sizeof(double2);
    const int gmax = (int)std::max<long long>(1, (64LL << 20) / img);
    const int chunk = (int)std::max<long long>(
        1, std::max<long long>(gmax, std::min<long long>(E, (256LL << 20) / img)));
    DeviceBuffer& spec = ctx.pot_spec;
    DeviceBuffer& delta = ctx.pot_delta;
    DeviceBuffer& d_elem = ctx.pot_elem;
    spec.ensure((size_t)std::min(gmax, std::max(1, S)) * img);
    delta.ensure((size_t)chunk * img);
    d_elem.ensure((size_t)std::max(1, S * E) * sizeof(int));
    std::vector<int> present;  // per slice, the elements with atoms in it, in increasing Z; concatenated over slices
    std::vector<int> present_ptr(1, 0);
    for (int j = 0; j < S; ++j) {
        for (int e = 0; e < E; ++e)
            if (group_ptr[j * E + e + 1] > group_ptr[j * E + e]) present.push_back(e);
        present_ptr.push_back((int)present.size());
    }
    if (!present.empty())
        SIMK_CUDA(cudaMemcpyAsync(d_elem.ptr, present.data(), present.size() * sizeof(int), cudaMemcpyHostToDevice,
                                  ctx.stream));
    const LinePlan& prow = ctx.plan(g.ny, 64);
    const LinePlan& pcol = ctx.plan(g.nx, 64);
    // delta image q (of the batch starting at q0) of slice j: its element's atoms scattered with their weights
    auto scatter = [&](int j, int q_global, int q_local) {
        const int e = present[q_global];
        const long long a0 = group_ptr[j * E + e], a1 = group_ptr[j * E + e + 1];
        k_scatter<<<blocks_for(a1 - a0), 256, 0, ctx.stream>>>(delta.as<double2>() + (long long)q_local * N,
                                                                d_pix.as<int>() + a0, d_w.as<double>() + a0,
                                                                (int)(a1 - a0));
        ++ctx.launches;
    };
    for (int j0 = 0; j0 < S;) {
        int j1 = j0 + 1;
        while (j1 < S && j1 - j0 < gmax && present_ptr[j1 + 1] - present_ptr[j0] <= chunk) ++j1;
        const int G = j1 - j0;
        const int imgs = present_ptr[j1] - present_ptr[j0];
        k_zero_d2<<<blocks_for((long long)G * N), 256, 0, ctx.stream>>>(spec.as<double2>(), (long long)G * N);
        ++ctx.launches;
        if (imgs <= chunk) {
            if (imgs > 0) {
                k_zero_d2<<<blocks_for((long long)imgs * N), 256, 0, ctx.stream>>>(delta.as<double2>(),
                                                                                   (long long)imgs * N);
                ++ctx.launches;
                for (int j = j0; j < j1; ++j)
                    for (int q = present_ptr[j]; q < present_ptr[j + 1]; ++q) scatter(j, q, q - present_ptr[j0]);
                fft2(prow, pcol, delta.ptr, g.nx, g.ny, imgs, -1, 1.0, ctx.stream, &ctx.launches);
                for (int j = j0; j < j1; ++j) {
                    const int nq = present_ptr[j + 1] - present_ptr[j];
                    if (nq == 0) continue;
                    k_accum_spectra<<<blocks_for(N), 256, 0, ctx.stream>>>(
                        spec.as<double2>() + (long long)(j - j0) * N,
                        delta.as<double2>() + (long long)(present_ptr[j] - present_ptr[j0]) * N, kern.as<double>(),
                        d_elem.as<int>() + present_ptr[j], nq, N);
                    ++ctx.launches;
                }
            }
        } else {  // G == 1: the slice's images in batches of `chunk`
            for (int q0 = present_ptr[j0]; q0 < present_ptr[j1]; q0 += chunk) {
                const int nq = std::min(chunk, present_ptr[j1] - q0);
                k_zero_d2<<<blocks_for((long long)nq * N), 256, 0, ctx.stream>>>(delta.as<double2>(),
                                                                                 (long long)nq * N);
                ++ctx.launches;
                for (int q = 0; q < nq; ++q) scatter(j0, q0 + q, q);
                fft2(prow, pcol, delta.ptr, g.nx, g.ny, nq, -1, 1.0, ctx.stream, &ctx.launches);
                k_accum_spectra<<<blocks_for(N), 256, 0, ctx.stream>>>(spec.as<double2>(), delta.as<double2>(),
                                                                        kern.as<double>(), d_elem.as<int>() + q0, nq,
                                                                        N);
                ++ctx.launches;
            }
        }
        fft2(prow, pcol, spec.ptr, g.nx, g.ny, G, +1, 1.0 / (double)N, ctx.stream, &ctx.launches);
        k_real_part<<<blocks_for((long long)G * N), 256, 0, ctx.stream>>>(pot.V.as<double>() + (long long)j0 * N,
                                                                          spec.as<double2>(), (long long)G * N);
        ++ctx.launches;
        j0 = j1;
    }
    SIMK_CUDA(cudaGetLastError());
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
}

// ---- transmissions (Multislice.swift:83-103) --------------------------------------------------------------------------
void prepare_transmissions(Context& ctx, PotentialImpl& pot, double energy) {
    if (pot.t_energy == energy && pot.t.ptr) return;
    const GridGeom& g = pot.g;
    const long long N = g.count();
    const int S = pot.n_slices();
    pot.t.alloc(std::max(1, S) * N * sizeof(float2));
    // slices in batches of up to 64 MiB of float64 fields, each line transformed as it would be alone
    const int C = (int)std::max<long long>(1, std::min<long long>(S, (64LL << 20) / (N * (long long)sizeof(double2))));
    DeviceBuffer& T = ctx.pot_delta;  // the builder's delta-image scratch, grown if needed
    T.ensure((size_t)C * N * sizeof(double2));
    const LinePlan& prow = ctx.plan(g.ny, 64);
    const LinePlan& pcol = ctx.plan(g.nx, 64);
    const double sigma = interaction_parameter(energy);
    for (int j0 = 0; j0 < S; j0 += C) {
        const int c = std::min(C, S - j0);
        const long long cn = (long long)c * N;
        k_exp_i_sigma_v<<<blocks_for(cn), 256, 0, ctx.stream>>>(T.as<double2>(), pot.V.as<double>() + (long long)j0 * N,
                                                                sigma, cn);
        ++ctx.launches;
        fft2(prow, pcol, T.ptr, g.nx, g.ny, c, -1, 1.0, ctx.stream, &ctx.launches);
        k_mul_antialias<<<blocks_for(cn), 256, 0, ctx.stream>>>(T.as<double2>(), grid_dev(g), c);
        ++ctx.launches;
        fft2(prow, pcol, T.ptr, g.nx, g.ny, c, +1, 1.0 / (double)N, ctx.stream, &ctx.launches);
        k_to_float2<<<blocks_for(cn), 256, 0, ctx.stream>>>(pot.t.as<float2>() + (long long)j0 * N, T.as<double2>(), cn);
        ++ctx.launches;
    }
    SIMK_CUDA(cudaGetLastError());
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
    pot.t_energy = energy;
}

// ---- probe (Probe.swift:25-156, Aberrations.swift:39-59) ---------------------------------------------------------------
struct ProbeDev {
    double lambda, cutoff, dax, day;
    int soft, infinite;
    double ab[25];
};

__device__ double chi_of(double alpha, double phi, const double* c, double lambda) {
    // coefficient order: C10 C12 phi12 C21 phi21 C23 phi23 C30 C32 phi32 C34 phi34 C41 phi41 C43 phi43 C45 phi45
    //                    C50 C52 phi52 C54 phi54 C56 phi56
    double x = 0.0;
    const double a2 = alpha * alpha;
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
    return x * (2 * M_PI / lambda);
}

__global__ void k_probe_spectrum(double2* out, GridDev g, ProbeDev p) {
    const long long N = (long long)g.nx * g.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i / g.ny), iy = (int)(i % g.ny);
        const double kx = fftfreq_at(ix, g.nx, g.dx), ky = fftfreq_at(iy, g.ny, g.dy);
        const double alpha = sqrt(kx * kx + ky * ky) * p.lambda;
        const double phi = atan2(ky, kx);
        double ap;
        if (p.infinite) ap = 1.0;
        else if (p.soft) {
            if (ix == 0 && iy == 0) ap = 1.0;
            else {
                const double a = cos(phi) * p.dax, b = sin(phi) * p.day;
                const double d = sqrt(a * a + b * b);
                ap = fmin(fmax((p.cutoff - alpha) / d + 0.5, 0.0), 1.0);
            }
        } else ap = (alpha <= p.cutoff) ? 1.0 : 0.0;
        const double chi = chi_of(alpha, phi, p.ab, p.lambda);
        double s, c;
        sincos(-chi, &s, &c);
        out[i] = make_double2(ap * c, ap * s);
    }
}

// ---- contrast transfer function (ContrastTransferFunction.swift:12-115) -------------------------------------------
// d chi / d alpha and abTEM's azimuthal term, in the coefficient order of chi_of.
__device__ double dchi_dalpha(double a, double p, const double* c, double lambda) {
    const double a2 = a * a, a3 = a2 * a, a4 = a3 * a, a5 = a4 * a;
    const double t1 = (c[1] * cos(2 * (p - c[2])) + c[0]) * a;
    const double t2 = (c[5] * cos(3 * (p - c[6])) + c[3] * cos(1 * (p - c[4]))) * a2;
    const double t3 = (c[10] * cos(4 * (p - c[11])) + c[8] * cos(2 * (p - c[9])) + c[7]) * a3;
    const double t4 = (c[16] * cos(5 * (p - c[17])) + c[14] * cos(3 * (p - c[15])) + c[12] * cos(1 * (p - c[13]))) * a4;
    const double t5 = (c[23] * cos(6 * (p - c[24])) + c[21] * cos(4 * (p - c[22])) + c[19] * cos(2 * (p - c[20])) +
                       c[18]) * a5;
    return 2 * M_PI / lambda * (t1 + t2 + t3 + t4 + t5);
}
__device__ double dchi_dphi(double a, double p, const double* c, double lambda) {
    const double a2 = a * a, a3 = a2 * a, a4 = a3 * a, a5 = a4 * a;
    const double t1 = 1 / 2.0 * (2.0 * c[1] * sin(2.0 * (p - c[2]))) * a;
    const double t2 = 1 / 3.0 * (3.0 * c[5] * sin(3.0 * (p - c[6])) + 1.0 * c[3] * sin(1.0 * (p - c[4]))) * a2;
    const double t3 = 1 / 4.0 * (4.0 * c[10] * sin(4.0 * (p - c[11])) + 2.0 * c[8] * sin(2.0 * (p - c[9]))) * a3;
    const double t4 = 1 / 5.0 * (5.0 * c[16] * sin(5.0 * (p - c[17])) + 3.0 * c[14] * sin(3.0 * (p - c[15])) +
                                 1.0 * c[12] * sin(1.0 * (p - c[13]))) * a4;
    const double t5 = (1 / 6.0) * (6.0 * c[23] * sin(6.0 * (p - c[24])) + 4.0 * c[21] * sin(4.0 * (p - c[22])) +
                                   2.0 * c[19] * sin(2.0 * (p - c[20]))) * a5;
    return -2 * M_PI / lambda * (t1 + t2 + t3 + t4 + t5);
}

struct CtfDev {
    double lambda, cutoff, dax, day, focal, beta;
    int soft, infinite;
    double ab[25];
};

// H = exp(-i chi) x E_s (beta != 0) x E_t (Delta != 0) x aperture (finite cutoff), float64, FFT order.
__global__ void k_ctf_kernel(double2* out, GridDev g, CtfDev c) {
    const long long N = (long long)g.nx * g.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i / g.ny), iy = (int)(i % g.ny);
        const double kx = fftfreq_at(ix, g.nx, g.dx), ky = fftfreq_at(iy, g.ny, g.dy);
        const double alpha = sqrt(kx * kx + ky * ky) * c.lambda;
        const double phi = atan2(ky, kx);
        double s, co;
        sincos(-chi_of(alpha, phi, c.ab, c.lambda), &s, &co);
        double f = 1.0;
        if (c.beta != 0.0) {
            const double b = c.beta / 1e3;
            const double dk = dchi_dalpha(alpha, phi, c.ab, c.lambda), dp = dchi_dphi(alpha, phi, c.ab, c.lambda);
            const double sign = b > 0 ? 1.0 : (b < 0 ? -1.0 : 0.0);
            f *= exp(-sign * (b / 2) * (b / 2) * (dk * dk + dp * dp));
        }
        if (c.focal != 0.0) {
            const double x = 0.5 * M_PI / c.lambda * c.focal * alpha * alpha;
            f *= exp(-(x * x));
        }
        if (!c.infinite) {
            double ap;
            if (c.soft) {
                if (ix == 0 && iy == 0) ap = 1.0;
                else {
                    const double a = cos(phi) * c.dax, b = sin(phi) * c.day;
                    ap = fmin(fmax((c.cutoff - alpha) / sqrt(a * a + b * b) + 0.5, 0.0), 1.0);
                }
            } else ap = (alpha <= c.cutoff) ? 1.0 : 0.0;
            f *= ap;
        }
        out[i] = make_double2(co * f, s * f);
    }
}

void ctf_kernel_device(Context& ctx, const GridGeom& g, double energy, const simk_ctf& ctf, DeviceBuffer& out_f64) {
    SIMK_REQUIRE(std::isfinite(energy) && energy > 0, "the energy must be finite and positive");
    SIMK_REQUIRE(ctf.semiangle_mrad > 0 && !std::isnan(ctf.semiangle_mrad), "invalid aperture");
    for (int i = 0; i < 25; ++i) SIMK_REQUIRE(std::isfinite(ctf.aberrations[i]), "every aberration must be finite");
    SIMK_REQUIRE(std::isfinite(ctf.focal_spread) && ctf.focal_spread >= 0, "focal spread must be finite and >= 0 A");
    SIMK_REQUIRE(std::isfinite(ctf.angular_spread) && ctf.angular_spread >= 0,
                 "angular spread must be finite and >= 0 mrad");
    const long long N = g.count();
    CtfDev c{};
    c.lambda = wavelength(energy);
    c.infinite = std::isinf(ctf.semiangle_mrad) ? 1 : 0;
    c.soft = ctf.soft ? 1 : 0;
    c.cutoff = ctf.semiangle_mrad * 1e-3;
    const double rsx = 1.0 / ((double)g.nx * g.dx()), rsy = 1.0 / ((double)g.ny * g.dy());
    c.dax = rsx * 1e3 * c.lambda * 1e-3;
    c.day = rsy * 1e3 * c.lambda * 1e-3;
    c.focal = ctf.focal_spread;
    c.beta = ctf.angular_spread;
    for (int i = 0; i < 25; ++i) c.ab[i] = ctf.aberrations[i];
    out_f64.alloc(N * sizeof(double2));
    k_ctf_kernel<<<blocks_for(N), 256, 0, ctx.stream>>>(out_f64.as<double2>(), grid_dev(g), c);
    ++ctx.launches;
    SIMK_CUDA(cudaGetLastError());
}

// Waves.applying: IFFT(FFT(psi) H) on batches of waves in float32 with the float64-computed kernel (1/N folded in).
void apply_ctf_device(Context& ctx, const GridGeom& g, double energy, const simk_ctf& ctf, int count,
                      const double* in_re, const double* in_im, double* out_re, double* out_im, double* out_intensity) {
    const long long N = g.count();
    DeviceBuffer h64, h32(N * sizeof(float2));
    ctf_kernel_device(ctx, g, energy, ctf, h64);
    k_to_float2<<<blocks_for(N), 256, 0, ctx.stream>>>(h32.as<float2>(), h64.as<double2>(), N);
    ++ctx.launches;
    SIMK_CUDA(cudaGetLastError());
    const long long B = std::max<long long>(1, std::min<long long>(count, (256LL << 20) / (N * (long long)sizeof(float2))));
    DeviceBuffer psi(B * N * sizeof(float2));
    std::vector<float2> h(B * N);
    const LinePlan& prow = ctx.plan(g.ny, 32);
    const LinePlan& pcol = ctx.plan(g.nx, 32);
    for (long long first = 0; first < count; first += B) {
        const int b = (int)std::min<long long>(B, count - first);
        for (long long i = 0; i < b * N; ++i)
            h[i] = make_float2((float)in_re[first * N + i], (float)in_im[first * N + i]);
        SIMK_CUDA(cudaMemcpyAsync(psi.ptr, h.data(), b * N * sizeof(float2), cudaMemcpyHostToDevice, ctx.stream));
        fft2(prow, pcol, psi.ptr, g.nx, g.ny, b, -1, 1.0, ctx.stream, &ctx.launches);
        launch_mul_broadcast(ctx, psi.as<float2>(), h32.as<float2>(), N, b, 1.0f / (float)N);
        fft2(prow, pcol, psi.ptr, g.nx, g.ny, b, +1, 1.0, ctx.stream, &ctx.launches);
        SIMK_CUDA(cudaMemcpyAsync(h.data(), psi.ptr, b * N * sizeof(float2), cudaMemcpyDeviceToHost, ctx.stream));
        SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
        for (long long i = 0; i < b * N; ++i) {
            const double re = h[i].x, im = h[i].y;
            if (out_re) {
                out_re[first * N + i] = re;
                out_im[first * N + i] = im;
            }
            if (out_intensity) out_intensity[first * N + i] = re * re + im * im;
        }
    }
}

// One block: the float64 sum of |a|^2 in a fixed order (deterministic).
__global__ void k_norm2(const double2* a, long long N, double* out) {
    __shared__ double part[1024];
    double s = 0.0;
    for (long long i = threadIdx.x; i < N; i += blockDim.x) s += a[i].x * a[i].x + a[i].y * a[i].y;
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0];
}

__global__ void k_scale_d2(double2* a, long long N, const double* norm2) {
    const double f = 1.0 / sqrt(*norm2);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        a[i] = make_double2(a[i].x * f, a[i].y * f);
}

namespace {
// The normalised probe spectrum in float64 into tmp (N double2, norm one double) and as complex64 into out.
void probe_spectrum_launch(Context& ctx, const GridGeom& g, const simk_probe& probe, double2* tmp, double* norm,
                           float2* out) {
    SIMK_REQUIRE(std::isfinite(probe.energy) && probe.energy > 0, "the energy must be finite and positive");
    SIMK_REQUIRE(probe.semiangle_mrad > 0 && !std::isnan(probe.semiangle_mrad), "invalid aperture");
    for (int i = 0; i < 25; ++i) SIMK_REQUIRE(std::isfinite(probe.aberrations[i]), "every aberration must be finite");
    const long long N = g.count();
    ProbeDev p{};
    p.lambda = wavelength(probe.energy);
    p.infinite = std::isinf(probe.semiangle_mrad) ? 1 : 0;
    p.soft = probe.soft ? 1 : 0;
    p.cutoff = probe.semiangle_mrad * 1e-3;
    const double rsx = 1.0 / ((double)g.nx * g.dx()), rsy = 1.0 / ((double)g.ny * g.dy());
    p.dax = rsx * 1e3 * p.lambda * 1e-3;
    p.day = rsy * 1e3 * p.lambda * 1e-3;
    for (int i = 0; i < 25; ++i) p.ab[i] = probe.aberrations[i];
    k_probe_spectrum<<<blocks_for(N), 256, 0, ctx.stream>>>(tmp, grid_dev(g), p);
    k_norm2<<<1, 1024, 0, ctx.stream>>>(tmp, N, norm);
    k_scale_d2<<<blocks_for(N), 256, 0, ctx.stream>>>(tmp, N, norm);
    k_to_float2<<<blocks_for(N), 256, 0, ctx.stream>>>(out, tmp, N);
    ctx.launches += 4;
    SIMK_CUDA(cudaGetLastError());
}
}  // namespace

void probe_spectrum_into(Context& ctx, const GridGeom& g, const simk_probe& probe, DeviceBuffer& out_f32,
                         DeviceBuffer& tmp, DeviceBuffer& norm) {
    const long long N = g.count();
    tmp.ensure(N * sizeof(double2));
    norm.ensure(sizeof(double));
    out_f32.ensure(N * sizeof(float2));
    probe_spectrum_launch(ctx, g, probe, tmp.as<double2>(), norm.as<double>(), out_f32.as<float2>());
}

void probe_spectrum_device(Context& ctx, const GridGeom& g, const simk_probe& probe, DeviceBuffer& out_f32,
                           DeviceBuffer* out_f64) {
    const long long N = g.count();
    DeviceBuffer tmp(N * sizeof(double2)), norm(sizeof(double));
    out_f32.alloc(N * sizeof(float2));
    probe_spectrum_launch(ctx, g, probe, tmp.as<double2>(), norm.as<double>(), out_f32.as<float2>());
    if (out_f64) {
        out_f64->alloc(N * sizeof(double2));
        SIMK_CUDA(cudaMemcpyAsync(out_f64->ptr, tmp.ptr, N * sizeof(double2), cudaMemcpyDeviceToDevice, ctx.stream));
    }
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
}

// r_x[ix] = exp(-2 pi i p_x[ix] u_x), u_x = x / dx, p_x = fftfreq(nx, 1) (Probe.swift:140-156), float64 phases.
__global__ void k_ramps(const double* positions, long long first, int count, GridDev g, float2* rx, float2* ry) {
    const int len = g.nx + g.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)count * len;
         i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / len), e = (int)(i % len);
        const double x = positions[2 * (first + b)], y = positions[2 * (first + b) + 1];
        double s, c;
        if (e < g.nx) {
            const double u = x / g.dx;
            sincospi(-2.0 * fftfreq_at(e, g.nx, 1.0) * u, &s, &c);
            rx[(long long)b * g.nx + e] = make_float2((float)c, (float)s);
        } else {
            const int iy = e - g.nx;
            const double u = y / g.dy;
            sincospi(-2.0 * fftfreq_at(iy, g.ny, 1.0) * u, &s, &c);
            ry[(long long)b * g.ny + iy] = make_float2((float)c, (float)s);
        }
    }
}

void launch_ramps(Context& ctx, const GridGeom& g, const double* positions_dev, long long first, int count, float2* rx,
                  float2* ry) {
    k_ramps<<<blocks_for((long long)count * (g.nx + g.ny)), 256, 0, ctx.stream>>>(positions_dev, first, count,
                                                                                  grid_dev(g), rx, ry);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
}

__global__ void k_probes(const float2* __restrict__ spectrum, const float2* __restrict__ rx,
                         const float2* __restrict__ ry, int nx, int ny, int count, float2* __restrict__ out,
                         float scale) {
    const long long N = (long long)nx * ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N * count;
         i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / N);
        const long long k = i - (long long)b * N;
        const int ix = (int)(k / ny), iy = (int)(k % ny);
        float2 v = cmul(cmul(spectrum[k], rx[(long long)b * nx + ix]), ry[(long long)b * ny + iy]);
        out[i] = v * scale;
    }
}

void launch_probes(Context& ctx, const GridGeom& g, const float2* spectrum, const float2* rx, const float2* ry,
                   int count, float2* out, float scale) {
    k_probes<<<blocks_for(g.count() * count), 256, 0, ctx.stream>>>(spectrum, rx, ry, g.nx, g.ny, count, out, scale);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
}

__global__ void k_mul_broadcast(float2* __restrict__ psi, const float2* __restrict__ f, long long n, int count,
                                float scale) {
    const long long total = n * count;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        psi[i] = cmul(psi[i], f[i % n]) * scale;
    }
}

void launch_mul_broadcast(Context& ctx, float2* psi, const float2* factor, long long n, int count, float scale) {
    k_mul_broadcast<<<blocks_for(n * count), 256, 0, ctx.stream>>>(psi, factor, n, count, scale);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
}

// ---- detectors (Sources/SimulatoDetector/Detectors.swift) -------------------------------------------------------------
namespace {
double round7(double x) { return std::nearbyint(x * 1e7) / 1e7; }  // np.round(x, 7), half to even

struct Angles {
    double ax, ay;  // angular sampling [mrad / px] (Detectors.swift:39-41)
};
Angles angular_sampling(const GridGeom& g, double energy) {
    const double lam = wavelength(energy);
    return {1.0 / ((double)g.nx * g.dx()) * lam * 1e3, 1.0 / ((double)g.ny * g.dy()) * lam * 1e3};
}
std::pair<int, int> cutoff_gpts(const GridGeom& g) {
    const double kcut = 2.0 / 3.0 / std::max(g.dx(), g.dy());
    auto size = [&](int n, double extent) {
        int m = (int)std::floor(round7(kcut * extent));
        if (m % 2 != n % 2) m += 1;
        return m;
    };
    return {size(g.nx, (double)g.nx * g.dx()), size(g.ny, (double)g.ny * g.dy())};
}
std::vector<int> crop_indices(int n, int m) {
    std::vector<int> out;
    if (m >= n) {
        for (int i = 0; i < n; ++i) out.push_back(i);
        return out;
    }
    const int low = (m % 2 == 1) ? m / 2 + 1 : m / 2, high = m / 2;
    for (int i = 0; i < low; ++i) out.push_back(i);
    for (int i = n - high; i < n; ++i) out.push_back(i);
    return out;
}
std::pair<int, int> pixelated_size(const GridGeom& g, int mode) {
    if (mode == SIMK_MAXANGLE_FULL) return {g.nx, g.ny};
    auto c = cutoff_gpts(g);
    if (mode == SIMK_MAXANGLE_CUTOFF) return c;
    auto v = [](int m, int n) {
        int k = (int)std::floor(round7((double)m / std::sqrt(2.0)));
        if (k % 2 != n % 2) k += 1;
        return k;
    };
    return {v(c.first, g.nx), v(c.second, g.ny)};
}
double annular_outer(const GridGeom& g, double energy, const simk_detector& d) {
    const Angles a = angular_sampling(g, energy);
    if (!d.has_outer) {
        auto c = cutoff_gpts(g);
        return std::floor(std::min((double)(c.first / 2) * a.ax, (double)(c.second / 2) * a.ay));
    }
    const double maximum = std::min((double)(g.nx / 2) * a.ax, (double)(g.ny / 2) * a.ay);
    const double o = d.outer;
    if (o > maximum && std::fabs(o - maximum) > 1e-5 + 1e-5 * std::fabs(o))
        throw Error(SIMK_ERR_INVALID, "outer " + std::to_string(o) + " mrad exceeds the maximum simulated angle " +
                                          std::to_string(maximum) + " mrad");
    return o;
}
std::vector<double> angles_of(int m, double d) {
    std::vector<double> a(m);
    for (int i = 0; i < m; ++i) a[i] = fftfreq_at(i, m, 1.0 / d / (double)m);
    return a;
}
}  // namespace

void detector_shape(const GridGeom& g, double energy, const simk_detector& d, int* ndim, int* shape) {
    switch (d.kind) {
        case SIMK_DET_ANNULAR: *ndim = 0; break;
        case SIMK_DET_PIXELATED: {
            auto s = pixelated_size(g, d.max_angle);
            *ndim = 2;
            shape[0] = std::min(s.first, g.nx);
            shape[1] = std::min(s.second, g.ny);
            break;
        }
        case SIMK_DET_COM: *ndim = 1; shape[0] = 2; break;
        case SIMK_DET_SEGMENTED: *ndim = 2; shape[0] = d.nr; shape[1] = d.nphi; break;
        case SIMK_DET_BINNED: *ndim = 2; shape[0] = d.nr; shape[1] = d.nphi; break;
        default: throw Error(SIMK_ERR_INVALID, "unknown detector kind");
    }
}

std::unique_ptr<DetectorPlan> build_detector_plan(Context& ctx, const GridGeom& g, double energy,
                                                  const simk_detector* dets, int n_dets) {
    auto plan = std::make_unique<DetectorPlan>();
    const Angles a = angular_sampling(g, energy);
    const double lam = wavelength(energy);
    std::vector<std::vector<std::pair<int, float>>> channels;
    std::vector<int> crop;
    for (int di = 0; di < n_dets; ++di) {
        const simk_detector& d = dets[di];
        int ndim, shape[2] = {1, 1};
        detector_shape(g, energy, d, &ndim, shape);
        plan->det_count.push_back(ndim == 0 ? 1 : ndim == 1 ? shape[0] : shape[0] * shape[1]);
        if (d.kind == SIMK_DET_ANNULAR) {
            SIMK_REQUIRE(std::isfinite(d.inner) && d.inner >= 0, "inner must be finite and >= 0");
            SIMK_REQUIRE(!d.has_outer || (std::isfinite(d.outer) && d.outer >= d.inner),
                         "outer must be finite and >= inner");
            const double o = annular_outer(g, energy, d);
            SIMK_REQUIRE(d.inner <= o, "inner exceeds the outer angle");
            auto ax = angles_of(g.nx, a.ax), ay = angles_of(g.ny, a.ay);
            const double i2 = d.inner * d.inner, o2 = o * o;
            std::vector<std::pair<int, float>> ch;
            for (int ix = 0; ix < g.nx; ++ix)
                for (int iy = 0; iy < g.ny; ++iy) {
                    const double a2 = ax[ix] * ax[ix] + ay[iy] * ay[iy];
                    if (a2 >= i2 && a2 < o2) ch.push_back({ix * g.ny + iy, 1.0f});
                }
            plan->det_first_channel.push_back((int)channels.size());
            plan->det_pixelated_offset.push_back(-1);
            channels.push_back(std::move(ch));
        } else if (d.kind == SIMK_DET_PIXELATED || d.kind == SIMK_DET_COM) {
            auto s = pixelated_size(g, d.max_angle);
            auto sx = crop_indices(g.nx, s.first), sy = crop_indices(g.ny, s.second);
            const int mx = (int)sx.size(), my = (int)sy.size();
            if (d.kind == SIMK_DET_PIXELATED) {
                plan->det_first_channel.push_back(-1);
                plan->det_pixelated_offset.push_back((int)crop.size());
                std::vector<int> map(mx * my);
                for (int cx = 0; cx < mx; ++cx)
                    for (int cy = 0; cy < my; ++cy)
                        map[((cx + mx / 2) % mx) * my + (cy + my / 2) % my] = sx[cx] * g.ny + sy[cy];
                crop.insert(crop.end(), map.begin(), map.end());
            } else {
                const double per = (d.units == SIMK_UNITS_MRAD) ? 1.0 : 1.0 / (lam * 1e3);
                std::vector<std::pair<int, float>> chx, chy;
                for (int cx = 0; cx < mx; ++cx)
                    for (int cy = 0; cy < my; ++cy) {
                        const int ox = (cx + mx / 2) % mx, oy = (cy + my / 2) % my;
                        const int p = sx[cx] * g.ny + sy[cy];
                        chx.push_back({p, (float)((double)(ox - mx / 2) * a.ax * per)});
                        chy.push_back({p, (float)((double)(oy - my / 2) * a.ay * per)});
                    }
                plan->det_first_channel.push_back((int)channels.size());
                plan->det_pixelated_offset.push_back(-1);
                channels.push_back(std::move(chx));
                channels.push_back(std::move(chy));
            }
        } else if (d.kind == SIMK_DET_SEGMENTED) {
            SIMK_REQUIRE(d.nr >= 1 && d.nphi >= 1, "bins must be at least 1");
            SIMK_REQUIRE(std::isfinite(d.inner) && std::isfinite(d.outer) && d.inner >= 0 && d.outer > d.inner &&
                             std::isfinite(d.rotation),
                         "need 0 <= inner < outer, finite, and a finite rotation");
            auto m = [&](int n, double dd) {
                int k = (int)(2 * std::ceil(d.outer / dd)) + 1;
                if (k % 2 != n % 2) k += 1;
                return std::min(k, n);
            };
            const int mx = m(g.nx, a.ax), my = m(g.ny, a.ay);
            auto sx = crop_indices(g.nx, mx), sy = crop_indices(g.ny, my);
            auto ax = angles_of(mx, a.ax), ay = angles_of(my, a.ay);
            const int nb = d.nr * d.nphi;
            std::vector<std::vector<std::pair<int, float>>> bins(nb);
            const double two_pi = 2 * M_PI;
            for (int cx = 0; cx < mx; ++cx)
                for (int cy = 0; cy < my; ++cy) {
                    const double alpha = std::sqrt(ax[cx] * ax[cx] + ay[cy] * ay[cy]);
                    if (!(alpha >= d.inner && alpha < d.outer)) continue;
                    double phi = std::fmod(std::atan2(ay[cy], ax[cx]) - d.rotation, two_pi);
                    if (phi < 0) phi += two_pi;
                    const int r = (int)std::floor((double)d.nr * (alpha - d.inner) / (d.outer - d.inner));
                    if (r >= d.nr) continue;
                    const double f = std::floor((double)d.nphi * (phi / two_pi));
                    const int az = (int)std::min(std::max(f, 0.0), (double)(d.nphi - 1));
                    bins[az + r * d.nphi].push_back({sx[cx] * g.ny + sy[cy], 1.0f});
                }
            plan->det_first_channel.push_back((int)channels.size());
            plan->det_pixelated_offset.push_back(-1);
            for (auto& b : bins) channels.push_back(std::move(b));
        } else if (d.kind == SIMK_DET_BINNED) {
            SIMK_REQUIRE(d.nr >= 1 && d.nphi >= 1 && d.nr <= 4096 && d.nphi <= 4096, "bins must be in 1..4096");
            const double wmax = std::min((g.nx / 2) * a.ax, (g.ny / 2) * a.ay);
            SIMK_REQUIRE(std::isfinite(d.outer) && d.outer > 0 && d.outer <= wmax,
                         "the binned window must lie within the largest simulated angle (" + std::to_string(wmax) +
                             " mrad)");
            auto b = std::make_unique<DetectorPlan::Binned>();
            b->det = di;
            b->nbx = d.nr;
            b->nby = d.nphi;
            // per axis: bin k covers [-outer + k w, -outer + (k + 1) w), pixel i covers [alpha_i - s/2, alpha_i + s/2)
            auto axis = [&](int n, double samp, int nb, DeviceBuffer& P, DeviceBuffer& I, DeviceBuffer& W) {
                const std::vector<double> al = angles_of(n, samp);
                const double bw = 2.0 * d.outer / nb;
                std::vector<int> ptr(1, 0), idx;
                std::vector<double> wt;
                for (int k = 0; k < nb; ++k) {
                    const double lo = -d.outer + k * bw, hi = lo + bw;
                    for (int i = 0; i < n; ++i) {
                        const double ov = std::min(hi, al[i] + 0.5 * samp) - std::max(lo, al[i] - 0.5 * samp);
                        if (ov > 0) {
                            idx.push_back(i);
                            wt.push_back(ov / samp);
                        }
                    }
                    ptr.push_back((int)idx.size());
                }
                P.alloc(ptr.size() * sizeof(int));
                SIMK_CUDA(cudaMemcpy(P.ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice));
                I.alloc(std::max<size_t>(1, idx.size()) * sizeof(int));
                W.alloc(std::max<size_t>(1, wt.size()) * sizeof(double));
                if (!idx.empty()) {
                    SIMK_CUDA(cudaMemcpy(I.ptr, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice));
                    SIMK_CUDA(cudaMemcpy(W.ptr, wt.data(), wt.size() * sizeof(double), cudaMemcpyHostToDevice));
                }
            };
            axis(g.nx, a.ax, d.nr, b->xp, b->xi, b->xw);
            axis(g.ny, a.ay, d.nphi, b->yp, b->yi, b->yw);
            plan->det_first_channel.push_back(-1);
            plan->det_pixelated_offset.push_back(-1);
            plan->binned.push_back(std::move(b));
        } else {
            throw Error(SIMK_ERR_INVALID, "unknown detector kind");
        }
    }
    plan->n_channels = (int)channels.size();
    std::vector<int> ptr(1, 0), pix;
    std::vector<float> w;
    for (auto& ch : channels) {
        for (auto& e : ch) {
            pix.push_back(e.first);
            w.push_back(e.second);
        }
        ptr.push_back((int)pix.size());
    }
    plan->host_chan_ptr = ptr;
    plan->host_chan_pix = pix;
    plan->host_chan_w = w;
    plan->grid_ny = g.ny;
    plan->has_pixel_outputs = !crop.empty() || !plan->binned.empty();
    plan->total_entries = (long long)pix.size();
    plan->total_crop = (long long)crop.size();
    plan->chan_ptr.alloc(ptr.size() * sizeof(int));
    SIMK_CUDA(cudaMemcpy(plan->chan_ptr.ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (!pix.empty()) {
        plan->chan_pix.alloc(pix.size() * sizeof(int));
        plan->chan_w.alloc(w.size() * sizeof(float));
        SIMK_CUDA(cudaMemcpy(plan->chan_pix.ptr, pix.data(), pix.size() * sizeof(int), cudaMemcpyHostToDevice));
        SIMK_CUDA(cudaMemcpy(plan->chan_w.ptr, w.data(), w.size() * sizeof(float), cudaMemcpyHostToDevice));
    }
    if (!crop.empty()) {
        plan->crop_src.alloc(crop.size() * sizeof(int));
        SIMK_CUDA(cudaMemcpy(plan->crop_src.ptr, crop.data(), crop.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    return plan;
}

const DetectorPlan::TileChannels& DetectorPlan::tiles(int tc) {
    for (auto& t : tile_channels)
        if (t->tc == tc) return *t;
    SIMK_REQUIRE(tc >= 1 && grid_ny % tc == 0, "column tile width must divide the grid");
    auto t = std::make_unique<TileChannels>();
    t->tc = tc;
    t->groups = grid_ny / tc;
    const int C = n_channels, G = t->groups;
    std::vector<std::vector<std::pair<int, float>>> lists((size_t)G * C);
    for (int ch = 0; ch < C; ++ch)
        for (int e = host_chan_ptr[ch]; e < host_chan_ptr[ch + 1]; ++e) {
            const int p = host_chan_pix[e], ix = p / grid_ny, iy = p % grid_ny;
            lists[(size_t)(iy / tc) * C + ch].push_back({ix * tc + iy % tc, host_chan_w[e]});
        }
    std::vector<int> ptr(1, 0);
    std::vector<int2> ent;
    ent.reserve(host_chan_pix.size());
    for (auto& l : lists) {
        std::sort(l.begin(), l.end(), [](const std::pair<int, float>& a, const std::pair<int, float>& b) {
            return a.first < b.first;
        });
        for (auto& e : l) {
            int bits;
            std::memcpy(&bits, &e.second, sizeof(int));
            ent.push_back(make_int2(e.first, bits));
        }
        ptr.push_back((int)ent.size());
    }
    t->ptr.alloc(ptr.size() * sizeof(int));
    SIMK_CUDA(cudaMemcpy(t->ptr.ptr, ptr.data(), ptr.size() * sizeof(int), cudaMemcpyHostToDevice));
    t->ent.alloc(std::max<size_t>(1, ent.size()) * sizeof(int2));
    if (!ent.empty())
        SIMK_CUDA(cudaMemcpy(t->ent.ptr, ent.data(), ent.size() * sizeof(int2), cudaMemcpyHostToDevice));
    tile_channels.push_back(std::move(t));
    return *tile_channels.back();
}

// One block per (position, channel): sum over the channel's pixels of |phi|^2 * scale * w in float64, in a fixed
// order (deterministic); adds weight * sum to the output of the channel's detector.
struct ChannelOut {
    double* out[16];
    int first_channel[16];
    int count[16];
    int n_det;
};

__device__ __forceinline__ int channel_owner(const ChannelOut& co, int c) {
    int d = 0;
    for (int k = 0; k < co.n_det; ++k)
        if (co.first_channel[k] >= 0 && c >= co.first_channel[k] && c < co.first_channel[k] + co.count[k]) d = k;
    return d;
}

// One thread per (position, channel): the column groups' partial sums in order (the fused pass's fixed-order block
// sums), weight times the total added to the channel's output.
__global__ void k_detect_fold(const double* __restrict__ partial, int groups, int n_channels, int count,
                              ChannelOut co, long long first_position, double weight) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count * n_channels) return;
    const int b = i / n_channels, c = i - b * n_channels;
    const double* p = partial + (size_t)b * groups * n_channels + c;
    double s = 0.0;
    for (int g = 0; g < groups; ++g) s += p[(size_t)g * n_channels];
    const int d = channel_owner(co, c);
    co.out[d][(first_position + b) * co.count[d] + (c - co.first_channel[d])] += weight * s;
}

__global__ void k_detect_channels(const float2* __restrict__ phi, long long N, const int* __restrict__ ptr,
                                  const int* __restrict__ pix, const float* __restrict__ w, int n_channels,
                                  ChannelOut co, long long first_position, double weight, float iscale) {
    __shared__ double part[256];
    const int b = blockIdx.y;
    const int c = blockIdx.x;
    const float2* p = phi + (long long)b * N;
    double s = 0.0;
    for (int i = ptr[c] + threadIdx.x; i < ptr[c + 1]; i += blockDim.x) {
        const float2 v = p[pix[i]];
        s += (double)((v.x * v.x + v.y * v.y) * iscale * w[i]);
    }
    part[threadIdx.x] = s;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) part[threadIdx.x] += part[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const int d = channel_owner(co, c);  // which detector owns channel c
        const int local = c - co.first_channel[d];
        double* o = co.out[d] + (first_position + b) * co.count[d] + local;
        *o += weight * part[0];
    }
}

__global__ void k_detect_pixelated(const float2* __restrict__ phi, long long N, const int* __restrict__ src, int m,
                                   double* out, long long first_position, int count, double weight, float iscale) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (long long)m * count;
         i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / m), o = (int)(i % m);
        const float2 v = phi[(long long)b * N + src[o]];
        out[(first_position + b) * m + o] += weight * (double)((v.x * v.x + v.y * v.y) * iscale);
    }
}

// Binned detector: one thread per (position, bin), the separable overlap weights over the bin's pixels summed in
// float64 in a fixed order.
__global__ void k_detect_binned(const float2* __restrict__ phi, long long N, int ny, const int* __restrict__ xp,
                                const int* __restrict__ xi, const double* __restrict__ xw, const int* __restrict__ yp,
                                const int* __restrict__ yi, const double* __restrict__ yw, int nbx, int nby,
                                double* out, long long first_position, int count, double weight, float iscale) {
    const long long m = (long long)nbx * nby;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m * count;
         i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / m);
        const long long o = i - (long long)b * m;
        const int bx = (int)(o / nby), by = (int)(o - (long long)bx * nby);
        const float2* w = phi + (long long)b * N;
        double s = 0.0;
        for (int p = xp[bx]; p < xp[bx + 1]; ++p) {
            const long long row = (long long)xi[p] * ny;
            double sy = 0.0;
            for (int q = yp[by]; q < yp[by + 1]; ++q) {
                const float2 v = w[row + yi[q]];
                sy += yw[q] * (double)((v.x * v.x + v.y * v.y) * iscale);
            }
            s += xw[p] * sy;
        }
        out[(first_position + b) * m + o] += weight * s;
    }
}

namespace {
ChannelOut channel_out(const DetectorPlan& plan, double* const* outputs_dev) {
    const int nd = (int)plan.det_count.size();
    SIMK_REQUIRE(nd <= 16, "at most 16 detectors per scan");
    ChannelOut co{};
    co.n_det = nd;
    for (int d = 0; d < nd; ++d) {
        co.out[d] = outputs_dev[d];
        co.first_channel[d] = plan.det_first_channel[d];
        co.count[d] = plan.det_count[d];
    }
    return co;
}
}  // namespace

void launch_detect_fold(Context& ctx, const DetectorPlan& plan, const double* partial, int groups, int count,
                        long long first_position, double* const* outputs_dev, double weight) {
    if (plan.n_channels == 0 || count == 0) return;
    const ChannelOut co = channel_out(plan, outputs_dev);
    const int n = count * plan.n_channels;
    k_detect_fold<<<(n + 127) / 128, 128, 0, ctx.stream>>>(partial, groups, plan.n_channels, count, co,
                                                           first_position, weight);
    ++ctx.launches;
    SIMK_CUDA(cudaGetLastError());
}

void launch_detect(Context& ctx, const DetectorPlan& plan, const GridGeom& g, const float2* phi, int count,
                   long long first_position, double* const* outputs_dev, double weight, float intensity_scale,
                   bool channels) {
    const long long N = g.count();
    const int nd = (int)plan.det_count.size();
    SIMK_REQUIRE(nd <= 16, "at most 16 detectors per scan");
    if (channels && plan.n_channels > 0) {
        const ChannelOut co = channel_out(plan, outputs_dev);
        dim3 grid(plan.n_channels, count);
        k_detect_channels<<<grid, 256, 0, ctx.stream>>>(phi, N, plan.chan_ptr.as<int>(), plan.chan_pix.as<int>(),
                                                        plan.chan_w.as<float>(), plan.n_channels, co, first_position,
                                                        weight, intensity_scale);
        ++ctx.launches;
    }
    for (int d = 0; d < nd; ++d) {
        if (plan.det_pixelated_offset[d] < 0) continue;
        const int m = plan.det_count[d];
        k_detect_pixelated<<<blocks_for((long long)m * count), 256, 0, ctx.stream>>>(
            phi, N, plan.crop_src.as<int>() + plan.det_pixelated_offset[d], m, outputs_dev[d], first_position, count,
            weight, intensity_scale);
        ++ctx.launches;
    }
    for (const auto& b : plan.binned) {
        const long long m = (long long)b->nbx * b->nby;
        k_detect_binned<<<blocks_for(m * count), 256, 0, ctx.stream>>>(
            phi, N, g.ny, b->xp.as<int>(), b->xi.as<int>(), b->xw.as<double>(), b->yp.as<int>(), b->yi.as<int>(),
            b->yw.as<double>(), b->nbx, b->nby, outputs_dev[b->det], first_position, count, weight, intensity_scale);
        ++ctx.launches;
    }
    SIMK_CUDA(cudaGetLastError());
}

}  // namespace simk
