// finite.cu -- the finite-projection Lobato potential: the real-space potential of each atom integrated over the part
// of each slice it reaches, splatted onto the grid.
//
// SimulatoKit has no finite projection (`Potential(projection="finite")` is listed as not ported, docs/parity.md:58,
// 251); the construction here is defined by the physics and anchored by identities the tests check: the integral over a
// thick slab is the infinite projection (the analytic 2 sum_i [2 A_i/B_i K0(B_i r) + A_i r K1(B_i r)] of
// tools/pins/potential-multislice/pins.py:432, whose 2-D transform is LobatoParameterization's f(k^2)), slices add,
// and the float64 device quadrature equals the float64 CPU restatement.
//
//   V(r) = sum_i A_i (2 / (B_i r) + 1) exp(-B_i r)               (A, B: LobatoParameterization.swift:38-44)
//   P(rho; zl, zu) = int_zl^zu V(sqrt(rho^2 + z^2)) dz
//                  = sum_i A_i int (2/B_i + rho cosh u) exp(-B_i rho cosh u) du,   z = rho sinh u
// The u-form is smooth; Gauss-Legendre (48 nodes each side of u = 0) reaches ~1e-15. An atom reaches rho <= R_c(Z)
// in the plane and |z - z_a| <= R_c(Z) along the beam, R_c the radius where V falls to 1e-3 V (bounded to
// [1, 6] A); rho is clamped below at min(dx, dy) / 2, the value abTEM uses inside its inner cutoff.
//
// Each (atom, slice) pair gets a radial profile on NR log-spaced radii between rho_min and R_c; each pixel then gathers,
// from the pairs of its slice binned in cells of side >= R_c (periodic in x and y), the profile interpolated cubically
// in log rho, in a fixed order (deterministic, no atomics).
#include <algorithm>
#include <cmath>

#include "finite.cuh"
#include "surrogate.cuh"

namespace simk {

#include "lobato_table.inc"

namespace {
constexpr double kKappaF = 0.0208865737082965;
__constant__ double c_gl_x[kGaussNodes];
__constant__ double c_gl_w[kGaussNodes];
bool g_gl_ready[64] = {};
}  // namespace

// Gauss-Legendre nodes and weights on [-1, 1] by Newton's iteration on P_n (the classical Golub-Welsch-free method).
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    for (int i = 0; i < (n + 1) / 2; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 0.0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            const double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        x[i] = -z;
        x[n - 1 - i] = z;
        w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

void ensure_gauss_nodes(Context& ctx) {
    if (g_gl_ready[ctx.device]) return;
    std::vector<double> x, w;
    gauss_legendre(kGaussNodes, x, w);
    SIMK_CUDA(cudaMemcpyToSymbol(c_gl_x, x.data(), sizeof(double) * kGaussNodes));
    SIMK_CUDA(cudaMemcpyToSymbol(c_gl_w, w.data(), sizeof(double) * kGaussNodes));
    g_gl_ready[ctx.device] = true;
}

ElementAB element_ab(int z) {
    const double* p = kLobatoTable[z - 1];
    ElementAB e{};
    for (int t = 0; t < 5; ++t) {
        e.A[t] = M_PI * M_PI * p[t] / std::pow(p[5 + t], 1.5) / kKappaF;
        e.B[t] = 2 * M_PI / std::sqrt(p[5 + t]);
    }
    return e;
}

double lobato_v3d(const ElementAB& e, double r) {
    double s = 0.0;
    for (int t = 0; t < 5; ++t) s += e.A[t] * (2.0 / (e.B[t] * r) + 1.0) * std::exp(-e.B[t] * r);
    return s;
}

double finite_cutoff(int z) {
    const ElementAB e = element_ab(z);
    double lo = 0.05, hi = 6.0;
    if (lobato_v3d(e, hi) > 1e-3) return hi;
    for (int i = 0; i < 100; ++i) {
        const double mid = 0.5 * (lo + hi);
        if (lobato_v3d(e, mid) > 1e-3) lo = mid;
        else hi = mid;
    }
    return std::max(1.0, hi);
}

__device__ double finite_profile_dev(const ElementAB& e, double rho, double zl, double zu) {
    if (!(zu > zl)) return 0.0;
    const double ul = asinh(zl / rho), uu = asinh(zu / rho);
    double total = 0.0;
    const int nparts = (ul < 0.0 && uu > 0.0) ? 2 : 1;
    for (int part = 0; part < nparts; ++part) {
        const double a = (nparts == 2) ? (part == 0 ? ul : 0.0) : ul;
        const double b = (nparts == 2) ? (part == 0 ? 0.0 : uu) : uu;
        const double h = 0.5 * (b - a), m = 0.5 * (b + a);
        double s = 0.0;
        for (int k = 0; k < kGaussNodes; ++k) {
            const double c = cosh(h * c_gl_x[k] + m);
            double f = 0.0;
#pragma unroll
            for (int t = 0; t < 5; ++t) f += e.A[t] * (2.0 / e.B[t] + rho * c) * exp(-e.B[t] * rho * c);
            s += c_gl_w[k] * f;
        }
        total += h * s;
    }
    return total;
}

// One profile value per (pair, radius): table[p * nr + k] = P(rho_k(e); zl_p, zu_p).
__global__ void k_finite_profiles(const FinitePair* __restrict__ pairs, int npairs, const ElementAB* __restrict__ elems,
                                  const double* __restrict__ rmin, const double* __restrict__ rcut, int nr,
                                  double* __restrict__ table) {
    const long long total = (long long)npairs * nr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int p = (int)(i / nr), k = (int)(i % nr);
        const FinitePair pr = pairs[p];
        const double r0 = rmin[pr.elem], r1 = rcut[pr.elem];
        const double rho = r0 * pow(r1 / r0, (double)k / (double)(nr - 1));
        table[i] = finite_profile_dev(elems[pr.elem], rho, pr.zl, pr.zu);
    }
}

// The same for a subset of the pairs.
__global__ void k_finite_profiles_ids(const FinitePair* __restrict__ pairs, const int* __restrict__ ids, int nids,
                                      const ElementAB* __restrict__ elems, const double* __restrict__ rmin,
                                      const double* __restrict__ rcut, int nr, double* __restrict__ table) {
    const long long total = (long long)nids * nr;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int p = ids[i / nr], k = (int)(i % nr);
        const FinitePair pr = pairs[p];
        const double r0 = rmin[pr.elem], r1 = rcut[pr.elem];
        const double rho = r0 * pow(r1 / r0, (double)k / (double)(nr - 1));
        table[(long long)p * nr + k] = finite_profile_dev(elems[pr.elem], rho, pr.zl, pr.zu);
    }
}

// Profile values at arbitrary (element, rho, zl, zu): the float64 quadrature itself, for tests and for training data.
__global__ void k_finite_points(const int* __restrict__ elem, const double* __restrict__ rho,
                                const double* __restrict__ zl, const double* __restrict__ zu, int n,
                                const ElementAB* __restrict__ elems, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = finite_profile_dev(elems[elem[i]], rho[i], zl[i], zu[i]);
}

// Catmull-Rom interpolation of the log-radial table row at fractional index s in [0, nr - 1].
__device__ __forceinline__ double interp_row(const double* row, int nr, double s) {
    int k = (int)floor(s);
    k = max(0, min(k, nr - 2));
    const double f = s - k;
    const double p1 = row[k], p2 = row[k + 1];
    const double p0 = (k > 0) ? row[k - 1] : 2.0 * p1 - p2;
    const double p3 = (k + 2 < nr) ? row[k + 2] : 2.0 * p2 - p1;
    return p1 + 0.5 * f * (p2 - p0 + f * (2.0 * p0 - 5.0 * p1 + 4.0 * p2 - p3 + f * (3.0 * (p1 - p2) + p3 - p0)));
}

// One thread per pixel of one slice: gather the pairs of the 3 x 3 (or all, if fewer) neighbouring cells.
__global__ void k_finite_splat(double* __restrict__ V, int nx, int ny, double dx, double dy, double lx, double ly,
                               const FinitePair* __restrict__ pairs, const int* __restrict__ cell_start,
                               const int* __restrict__ cell_pairs, int ncx, int ncy, const double* __restrict__ rmin,
                               const double* __restrict__ rcut, int nr, const double* __restrict__ table) {
    const long long N = (long long)nx * ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const int ix = (int)(i / ny), iy = (int)(i % ny);
        const double x = ix * dx, y = iy * dy;
        const int cx = min((int)(x / lx * ncx), ncx - 1), cy = min((int)(y / ly * ncy), ncy - 1);
        const int spanx = ncx >= 3 ? 3 : ncx, spany = ncy >= 3 ? 3 : ncy;
        double acc = 0.0;
        for (int a = 0; a < spanx; ++a) {
            const int gx = (ncx >= 3) ? (cx + a - 1 + ncx) % ncx : a;
            for (int b = 0; b < spany; ++b) {
                const int gy = (ncy >= 3) ? (cy + b - 1 + ncy) % ncy : b;
                const int c = gx * ncy + gy;
                for (int q = cell_start[c]; q < cell_start[c + 1]; ++q) {
                    const int p = cell_pairs[q];
                    const FinitePair pr = pairs[p];
                    double ddx = x - pr.x, ddy = y - pr.y;
                    ddx -= lx * rint(ddx / lx);
                    ddy -= ly * rint(ddy / ly);
                    const double r = sqrt(ddx * ddx + ddy * ddy);
                    const double rc = rcut[pr.elem];
                    if (r > rc) continue;
                    const double r0 = rmin[pr.elem];
                    const double rr = fmax(r, r0);
                    const double s = log(rr / r0) / log(rc / r0) * (double)(nr - 1);
                    acc += interp_row(table + (size_t)p * nr, nr, s);
                }
            }
        }
        V[i] = acc;
    }
}

namespace {
inline int blocks_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * 16)); }
}  // namespace

FiniteSetup finite_setup(const GridGeom& g, const std::vector<double>& dz, int n_atoms, const int* Z,
                         const double* xyz) {
    FiniteSetup s;
    std::vector<int> els(Z, Z + n_atoms);
    std::sort(els.begin(), els.end());
    els.erase(std::unique(els.begin(), els.end()), els.end());
    s.elements = els;
    const double rmin = 0.5 * std::min(g.dx(), g.dy());
    for (int z : els) {
        s.ab.push_back(element_ab(z));
        s.rcut.push_back(finite_cutoff(z));
        s.rmin.push_back(rmin);
    }
    const int S = (int)dz.size();
    std::vector<double> edges(S + 1, 0.0);
    for (int j = 0; j < S; ++j) edges[j + 1] = edges[j] + dz[j];
    s.slice_first.assign(S + 1, 0);
    for (int j = 0; j < S; ++j) {
        for (int a = 0; a < n_atoms; ++a) {
            const int e = (int)(std::lower_bound(els.begin(), els.end(), Z[a]) - els.begin());
            const double rc = s.rcut[e], za = xyz[3 * a + 2];
            const double zl = std::max(edges[j] - za, -rc), zu = std::min(edges[j + 1] - za, rc);
            if (!(zu > zl)) continue;
            FinitePair p{};
            p.elem = e;
            p.atom = a;
            p.zl = zl;
            p.zu = zu;
            p.x = xyz[3 * a];
            p.y = xyz[3 * a + 1];
            s.pairs.push_back(p);
        }
        s.slice_first[j + 1] = (int)s.pairs.size();
    }
    return s;
}

void finite_profiles_quadrature(Context& ctx, const FiniteDevice& d, long long npairs, int nr, double* table) {
    ensure_gauss_nodes(ctx);
    if (npairs == 0) return;
    k_finite_profiles<<<blocks_for(npairs * nr), 256, 0, ctx.stream>>>(d.pairs, (int)npairs, d.ab, d.rmin, d.rcut, nr,
                                                                      table);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
}

void finite_points(Context& ctx, const ElementAB* ab_dev, int n, const int* elem_dev, const double* rho_dev,
                   const double* zl_dev, const double* zu_dev, double* out_dev) {
    ensure_gauss_nodes(ctx);
    if (n == 0) return;
    k_finite_points<<<blocks_for(n), 256, 0, ctx.stream>>>(elem_dev, rho_dev, zl_dev, zu_dev, n, ab_dev, out_dev);
    SIMK_CUDA(cudaGetLastError());
    ++ctx.launches;
}

FiniteDevice upload_finite(Context& ctx, const FiniteSetup& s, DeviceBuffer& pairs, DeviceBuffer& ab,
                           DeviceBuffer& rmin, DeviceBuffer& rcut) {
    pairs.alloc(std::max<size_t>(1, s.pairs.size()) * sizeof(FinitePair));
    ab.alloc(std::max<size_t>(1, s.ab.size()) * sizeof(ElementAB));
    rmin.alloc(std::max<size_t>(1, s.rmin.size()) * sizeof(double));
    rcut.alloc(std::max<size_t>(1, s.rcut.size()) * sizeof(double));
    if (!s.pairs.empty())
        SIMK_CUDA(cudaMemcpy(pairs.ptr, s.pairs.data(), s.pairs.size() * sizeof(FinitePair), cudaMemcpyHostToDevice));
    if (!s.ab.empty()) {
        SIMK_CUDA(cudaMemcpy(ab.ptr, s.ab.data(), s.ab.size() * sizeof(ElementAB), cudaMemcpyHostToDevice));
        SIMK_CUDA(cudaMemcpy(rmin.ptr, s.rmin.data(), s.rmin.size() * sizeof(double), cudaMemcpyHostToDevice));
        SIMK_CUDA(cudaMemcpy(rcut.ptr, s.rcut.data(), s.rcut.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    FiniteDevice d{};
    d.pairs = pairs.as<FinitePair>();
    d.ab = ab.as<ElementAB>();
    d.rmin = rmin.as<double>();
    d.rcut = rcut.as<double>();
    return d;
}

void finite_splat(Context& ctx, PotentialImpl& pot, const FiniteSetup& s, const FiniteDevice& d, int nr,
                  const double* table) {
    const GridGeom& g = pot.g;
    const long long N = g.count();
    const int S = pot.n_slices();
    pot.V.alloc(std::max(1, S) * N * sizeof(double));
    double rcmax = 0.0;
    for (double r : s.rcut) rcmax = std::max(rcmax, r);
    const int ncx = std::max(1, (int)std::floor(g.ex / std::max(rcmax, 1e-9)));
    const int ncy = std::max(1, (int)std::floor(g.ey / std::max(rcmax, 1e-9)));
    DeviceBuffer cstart((size_t)(ncx * ncy + 1) * sizeof(int)), cpairs(std::max<size_t>(1, s.pairs.size()) * sizeof(int));
    std::vector<int> start(ncx * ncy + 1), order;
    for (int j = 0; j < S; ++j) {
        // bin the pairs of slice j by cell, in pair order (deterministic)
        std::vector<std::vector<int>> cells(ncx * ncy);
        for (int p = s.slice_first[j]; p < s.slice_first[j + 1]; ++p) {
            const FinitePair& pr = s.pairs[p];
            const double fx = pr.x / g.ex - std::floor(pr.x / g.ex), fy = pr.y / g.ey - std::floor(pr.y / g.ey);
            const int cx = std::min((int)(fx * ncx), ncx - 1), cy = std::min((int)(fy * ncy), ncy - 1);
            cells[cx * ncy + cy].push_back(p);
        }
        order.clear();
        for (int c = 0; c < ncx * ncy; ++c) {
            start[c] = (int)order.size();
            order.insert(order.end(), cells[c].begin(), cells[c].end());
        }
        start[ncx * ncy] = (int)order.size();
        SIMK_CUDA(cudaMemcpyAsync(cstart.ptr, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice,
                                  ctx.stream));
        if (!order.empty())
            SIMK_CUDA(cudaMemcpyAsync(cpairs.ptr, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice,
                                      ctx.stream));
        k_finite_splat<<<blocks_for(N), 256, 0, ctx.stream>>>(pot.V.as<double>() + (size_t)j * N, g.nx, g.ny, g.dx(),
                                                              g.dy(), g.ex, g.ey, d.pairs, cstart.as<int>(),
                                                              cpairs.as<int>(), ncx, ncy, d.rmin, d.rcut, nr, table);
        SIMK_CUDA(cudaGetLastError());
        ++ctx.launches;
        SIMK_CUDA(cudaStreamSynchronize(ctx.stream));  // the host vectors are reused for the next slice
    }
}


void build_potential_finite(Context& ctx, PotentialImpl& pot, int n_atoms, const int* Z, const double* xyz,
                            const SurrogateImpl* sg, double bound, int* used_surrogate, double* judged_max_rel) {
    for (int a = 0; a < n_atoms; ++a) {
        SIMK_REQUIRE(Z[a] >= 1 && Z[a] <= 103, "unsupported element: Z = " + std::to_string(Z[a]));
        SIMK_REQUIRE(std::isfinite(xyz[3 * a]) && std::isfinite(xyz[3 * a + 1]) && std::isfinite(xyz[3 * a + 2]),
                     "non-finite atom position");
    }
    const FiniteSetup s = finite_setup(pot.g, pot.dz, n_atoms, Z, xyz);
    DeviceBuffer dpairs, dab, drmin, drcut;
    const FiniteDevice d = upload_finite(ctx, s, dpairs, dab, drmin, drcut);
    const int nr = kProfileRadii;
    const long long np = (long long)s.pairs.size();
    DeviceBuffer table(std::max<long long>(1, np) * nr * sizeof(double));
    ensure_gauss_nodes(ctx);
    *used_surrogate = 0;
    *judged_max_rel = 0.0;
    std::vector<int> in_dom, out_dom;
    if (sg) {
        const double rmin = s.rmin.empty() ? 0.0 : s.rmin[0];
        for (long long p = 0; p < np; ++p) {
            const FinitePair& pr = s.pairs[p];
            const bool ok = sg->trained_on(s.elements[pr.elem]) && rmin >= sg->rho_min &&
                            (pr.zu - pr.zl) <= sg->max_thickness + 1e-12;
            (ok ? in_dom : out_dom).push_back((int)p);
        }
    } else {
        for (long long p = 0; p < np; ++p) out_dom.push_back((int)p);
    }
    auto run_quadrature = [&](const std::vector<int>& ids) {
        if (ids.empty()) return;
        DeviceBuffer did(ids.size() * sizeof(int));
        SIMK_CUDA(cudaMemcpy(did.ptr, ids.data(), ids.size() * sizeof(int), cudaMemcpyHostToDevice));
        KernelTimer t(ctx, "finite_quadrature", 0.0);
        k_finite_profiles_ids<<<blocks_for((long long)ids.size() * nr), 256, 0, ctx.stream>>>(
            d.pairs, did.as<int>(), (int)ids.size(), d.ab, d.rmin, d.rcut, nr, table.as<double>());
        SIMK_CUDA(cudaGetLastError());
        ++ctx.launches;
        SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
    };
    run_quadrature(out_dom);
    if (!in_dom.empty()) {
        DeviceBuffer did(in_dom.size() * sizeof(int)), dz(s.elements.size() * sizeof(int)),
            dpinf(s.elements.size() * nr * sizeof(double));
        std::vector<double> pinf(s.elements.size() * nr);
        std::vector<float2> rf(s.elements.size() * nr);
        for (size_t e = 0; e < s.elements.size(); ++e)
            for (int k = 0; k < nr; ++k) {
                const double rho = s.rmin[e] * std::pow(s.rcut[e] / s.rmin[e], (double)k / (double)(nr - 1));
                pinf[e * nr + k] = infinite_profile(s.elements[e], rho);
                rf[e * nr + k] = make_float2((float)rho, (float)((std::log(rho) + 1.5) / 2.0));
            }
        DeviceBuffer drf(rf.size() * sizeof(float2));
        SIMK_CUDA(cudaMemcpy(drf.ptr, rf.data(), rf.size() * sizeof(float2), cudaMemcpyHostToDevice));
        SIMK_CUDA(cudaMemcpy(did.ptr, in_dom.data(), in_dom.size() * sizeof(int), cudaMemcpyHostToDevice));
        SIMK_CUDA(cudaMemcpy(dz.ptr, s.elements.data(), s.elements.size() * sizeof(int), cudaMemcpyHostToDevice));
        SIMK_CUDA(cudaMemcpy(dpinf.ptr, pinf.data(), pinf.size() * sizeof(double), cudaMemcpyHostToDevice));
        surrogate_profiles(ctx, *sg, d, did.as<int>(), (int)in_dom.size(), dz.as<int>(), drf.as<float2>(),
                           dpinf.as<double>(), nr, table.as<double>());
        SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
        // the quadrature judges a fixed sample of the surrogate's entries: up to 512 pairs x 8 radii
        const int npick = (int)std::min<size_t>(512, in_dom.size());
        std::vector<int> zz, idx;
        std::vector<double> rho, zl, zu, got;
        for (int i = 0; i < npick; ++i) {
            const int p = in_dom[(size_t)i * in_dom.size() / npick];
            const FinitePair& pr = s.pairs[p];
            std::vector<double> row(nr);
            SIMK_CUDA(cudaMemcpy(row.data(), table.as<double>() + (size_t)p * nr, nr * sizeof(double),
                                 cudaMemcpyDeviceToHost));
            for (int j = 0; j < 8; ++j) {
                const int k = j * (nr - 1) / 7;
                const double r0 = s.rmin[pr.elem], r1 = s.rcut[pr.elem];
                zz.push_back(s.elements[pr.elem]);
                rho.push_back(r0 * std::pow(r1 / r0, (double)k / (double)(nr - 1)));
                zl.push_back(pr.zl);
                zu.push_back(pr.zu);
                got.push_back(row[k]);
            }
        }
        DeviceBuffer q(zz.size() * sizeof(double));
        surrogate_quadrature_points(ctx, zz, rho, zl, zu, q.as<double>());
        std::vector<double> hq(zz.size());
        SIMK_CUDA(cudaMemcpy(hq.data(), q.ptr, zz.size() * sizeof(double), cudaMemcpyDeviceToHost));
        double mx = 0.0;
        // error in units of the full projection at that radius, |dP| / P_inf(rho): the error of the summed potential
        for (size_t i = 0; i < hq.size(); ++i)
            mx = std::max(mx, std::fabs(got[i] - hq[i]) / infinite_profile(zz[i], rho[i]));
        *judged_max_rel = mx;
        if (mx <= bound) {
            *used_surrogate = 1;
        } else {
            run_quadrature(in_dom);  // the surrogate is outside its error bound here: the quadrature replaces it
        }
    }
    finite_splat(ctx, pot, s, d, nr, table.as<double>());
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
}

}  // namespace simk
