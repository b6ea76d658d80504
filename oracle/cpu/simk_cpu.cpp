// simk_cpu.cpp -- TEST INFRASTRUCTURE: a C++17 float64 restatement of SimulatoKit's `.cpu` STEM scan path, the timed
// CPU baseline and a second checker beside the NumPy oracle (oracle/simk_oracle.py). Never part of the CUDA library.
//
// Follows the reference's CPU path:
//   - FFT2D (Sources/SimulatoCore/FFT2D.swift:130-265): NumPy conventions (forward e^{-2 pi i jk/n} unnormalised,
//     inverse e^{+} with 1/(nx ny)), rows first then columns; per axis either a Stockham mixed-radix transform or
//     Bluestein's chirp-z on a power-of-two length >= max(16, 2n - 1) (FFT2D.swift:62-131), chosen by
//     MixedRadixPlan.prefersBluestein (MixedRadixPlan.swift:33-71: pocketfft's cost rule re-weighted). Where the
//     reference calls vDSP's DFT directly (f 2^m, f in {1, 3, 5, 15}, Grid.swift:61-67) this file runs its own Stockham
//     passes, the x86 stand-in for that tuned library transform. Twiddles come from exact integer phases
//     (MixedRadixPlan.swift:72-99). Several lines go through each pass at once, interleaved lane by lane, as the
//     reference runs two (SIMD2) per pass;
//   - Multislice.runCPU (Multislice.swift:132-157): psi <- IFFT2(FFT2(psi t_j) P(dz_j));
//   - Probe.build from the centred spectrum and the shift ramps (Probe.swift:113-156);
//   - DiffractionIntensity + annular detectors (Detectors.swift:28-36, 119-135): sum over a mask of |FFT2(exit)|^2;
//   - runCPUParallel (MetalMultislice.swift:28-47): positions spread over threads, each with its own buffers.
// The transmissions, propagators, spectrum and masks come from the NumPy oracle (float64), so this file restates the
// per-position hot loop, which is what the baseline times.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

namespace {

using cd = std::complex<double>;
constexpr int B = 8;  // lines per batch, interleaved: element i of lane b at [i * B + b]

// e^{sign 2 pi i k / n} from the exact ratio k / n (k reduced mod n).
cd unit_root(long long k, long long n, int sign) {
    k %= n;
    if (k < 0) k += n;
    const double a = 2.0 * M_PI * (double)k / (double)n;
    return cd(std::cos(a), sign * std::sin(a));
}

// MixedRadixPlan.factorization: 2 first (when n / 4^a is even), then the 4s, then the odd primes ascending.
std::vector<int> factorization(int n) {
    std::vector<int> out, fours;
    if (n < 2) return out;
    int rest = n;
    while (rest % 4 == 0) {
        fours.push_back(4);
        rest /= 4;
    }
    if (rest % 2 == 0) {
        out.push_back(2);
        rest /= 2;
    }
    out.insert(out.end(), fours.begin(), fours.end());
    for (int p = 3; p * p <= rest; p += 2)
        while (rest % p == 0) {
            out.push_back(p);
            rest /= p;
        }
    if (rest > 1) out.push_back(rest);
    return out;
}

// The passes of a length the reference hands to vDSP's DFT (f 2^m, f in {1, 3, 5, 15}): radix 8 while it divides,
// then 4, 2 and the odd factors; this file's own choice for that library transform.
std::vector<int> direct_radices(int n) {
    std::vector<int> out;
    int rest = n;
    for (int p : {8, 4, 2, 3, 5})
        while (rest % p == 0) {
            out.push_back(p);
            rest /= p;
        }
    if (rest > 1) {
        const std::vector<int> f = factorization(rest);
        out.insert(out.end(), f.begin(), f.end());
    }
    return out;
}

int bluestein_length(int n) {
    int m = 16;
    while (m < 2 * n - 1) m *= 2;
    return m;
}

bool has_direct_transform(int n) {
    if (n < 8) return false;
    int m = n, power = 0;
    while (m % 2 == 0) {
        m /= 2;
        ++power;
    }
    return (m == 1 || m == 3 || m == 5 || m == 15) && power >= 3;
}

// MixedRadixPlan.prefersBluestein / costGuess.
bool prefers_bluestein(int n) {
    const std::vector<int> f = factorization(n);
    if (f.empty()) return true;
    const int largest = *std::max_element(f.begin(), f.end());
    if (n < 50 || (long long)largest * largest <= n) return false;
    double cost = 0.0;
    for (int p : f) cost += (p == 4) ? 4.0 : (p <= 5 ? (double)p : 1.1 * p);
    cost *= n;
    const double m = bluestein_length(n);
    return 2.5 * m * std::log2(m) < cost;
}

struct Pass {
    int R = 0, ns = 0;            // radix, points already combined
    std::vector<double> wr, wi;   // forward twiddles e^{-2 pi i k r / (ns R)} at k (R - 1) + r - 1
    std::vector<double> cr, ci;   // radix 5 and generic: e^{-2 pi i t / R}, t < R
};

struct Line {
    int n = 0;
    int max_radix = 1;
    std::vector<Pass> passes;
    bool bluestein = false;
    int m = 0;
    std::unique_ptr<Line> inner;  // passes of the power-of-two length m
    std::vector<double> chr, chi; // chirp e^{-i pi k^2 / n}
    std::vector<double> fr, fi;   // FFT_m of the wrapped conjugate chirp
};

// Scratch for one line transform of B lanes: ping-pong buffers and the pass's per-radix arrays.
struct Work {
    std::vector<double> ar, ai, br, bi, ur, ui;
    void fit(int len, int radix) {
        const size_t n = (size_t)len * B;
        if (ar.size() < n) {
            ar.resize(n);
            ai.resize(n);
            br.resize(n);
            bi.resize(n);
        }
        if (ur.size() < (size_t)radix * B) {
            ur.resize((size_t)radix * B);
            ui.resize((size_t)radix * B);
        }
    }
};

std::unique_ptr<Line> make_line(int n, bool allow_bluestein = true);
void run(const Line& L, double* re, double* im, Work& w, int sign);

std::unique_ptr<Line> make_line(int n, bool allow_bluestein) {
    auto L = std::make_unique<Line>();
    L->n = n;
    if (n == 1) return L;
    if (allow_bluestein && !has_direct_transform(n) && prefers_bluestein(n)) {
        L->bluestein = true;
        const int m = bluestein_length(n);
        L->m = m;
        L->inner = make_line(m, false);
        L->chr.resize(n);
        L->chi.resize(n);
        for (long long k = 0; k < n; ++k) {
            const cd w = unit_root(-((k * k) % (2LL * n)), 2LL * n, 1);
            L->chr[k] = w.real();
            L->chi[k] = w.imag();
        }
        std::vector<double> br((size_t)m * B, 0.0), bi((size_t)m * B, 0.0);
        for (int k = 0; k < n; ++k) {
            br[(size_t)k * B] = L->chr[k];
            bi[(size_t)k * B] = -L->chi[k];
            if (k) {
                br[(size_t)(m - k) * B] = L->chr[k];
                bi[(size_t)(m - k) * B] = -L->chi[k];
            }
        }
        Work w;
        run(*L->inner, br.data(), bi.data(), w, -1);
        L->fr.resize(m);
        L->fi.resize(m);
        for (int k = 0; k < m; ++k) {
            L->fr[k] = br[(size_t)k * B];
            L->fi[k] = bi[(size_t)k * B];
        }
        L->max_radix = L->inner->max_radix;
        return L;
    }
    int ns = 1;
    for (int R : has_direct_transform(n) || !allow_bluestein ? direct_radices(n) : factorization(n)) {
        Pass p;
        p.R = R;
        p.ns = ns;
        p.wr.resize((size_t)ns * (R - 1));
        p.wi.resize((size_t)ns * (R - 1));
        for (int k = 0; k < ns; ++k)
            for (int r = 1; r < R; ++r) {
                const cd w = unit_root((long long)k * r, (long long)ns * R, -1);
                p.wr[(size_t)k * (R - 1) + r - 1] = w.real();
                p.wi[(size_t)k * (R - 1) + r - 1] = w.imag();
            }
        if (R != 2 && R != 3 && R != 4) {
            p.cr.resize(R);
            p.ci.resize(R);
            for (int t = 0; t < R; ++t) {
                const cd w = unit_root(t, R, -1);
                p.cr[t] = w.real();
                p.ci[t] = w.imag();
            }
        }
        L->max_radix = std::max(L->max_radix, R);
        L->passes.push_back(std::move(p));
        ns *= R;
    }
    return L;
}

// The small DFTs of one Stockham pass on a lane (v: R values, in place); s = sign of the exponent.
template <int R>
inline void small_dft(double* vr, double* vi, double s);

template <>
inline void small_dft<2>(double* vr, double* vi, double) {
    const double ar = vr[0], ai = vi[0];
    vr[0] = ar + vr[1];
    vi[0] = ai + vi[1];
    vr[1] = ar - vr[1];
    vi[1] = ai - vi[1];
}

template <>
inline void small_dft<3>(double* vr, double* vi, double s) {
    const double s1 = s * 0.86602540378443864676;  // sin(2 pi / 3)
    const double tr = vr[1] + vr[2], ti = vi[1] + vi[2];
    const double dr = vr[1] - vr[2], di = vi[1] - vi[2];
    const double mr = vr[0] - 0.5 * tr, mi = vi[0] - 0.5 * ti;
    vr[0] += tr;
    vi[0] += ti;
    vr[1] = mr - s1 * di;
    vi[1] = mi + s1 * dr;
    vr[2] = mr + s1 * di;
    vi[2] = mi - s1 * dr;
}

template <>
inline void small_dft<4>(double* vr, double* vi, double s) {
    const double ar = vr[0] + vr[2], ai = vi[0] + vi[2];
    const double br = vr[0] - vr[2], bi = vi[0] - vi[2];
    const double cr = vr[1] + vr[3], ci = vi[1] + vi[3];
    const double er = vr[1] - vr[3], ei = vi[1] - vi[3];
    const double dr = -s * ei, di = s * er;  // (v1 - v3) i s
    vr[0] = ar + cr;
    vi[0] = ai + ci;
    vr[2] = ar - cr;
    vi[2] = ai - ci;
    vr[1] = br + dr;
    vi[1] = bi + di;
    vr[3] = br - dr;
    vi[3] = bi - di;
}

template <>
inline void small_dft<8>(double* vr, double* vi, double s) {
    // even outputs: the 4-point DFT of v_t + v_{t+4}; odd: of (v_t - v_{t+4}) e^{s 2 pi i t / 8}
    const double c = 0.70710678118654752440;  // sqrt(1/2)
    double ar[4], ai[4], br[4], bi[4];
    for (int t = 0; t < 4; ++t) {
        ar[t] = vr[t] + vr[t + 4];
        ai[t] = vi[t] + vi[t + 4];
        br[t] = vr[t] - vr[t + 4];
        bi[t] = vi[t] - vi[t + 4];
    }
    double x = br[1], y = bi[1];
    br[1] = c * (x - s * y);
    bi[1] = c * (y + s * x);
    x = br[2];
    y = bi[2];
    br[2] = -s * y;
    bi[2] = s * x;
    x = br[3];
    y = bi[3];
    br[3] = -c * (x + s * y);
    bi[3] = c * (s * x - y);
    small_dft<4>(ar, ai, s);
    small_dft<4>(br, bi, s);
    for (int q = 0; q < 4; ++q) {
        vr[2 * q] = ar[q];
        vi[2 * q] = ai[q];
        vr[2 * q + 1] = br[q];
        vi[2 * q + 1] = bi[q];
    }
}

// One Stockham pass over B interleaved lines, x -> y: output (jb R + k + q ns) = sum_t W_R^{q t} W_{ns R}^{k t} x(j + t m)
// for j = jb + k, k < ns, m = n / R; W = e^{sign 2 pi i / .} (sign -1 forward, +1 inverse: conjugate twiddles).
template <int R>
void pass_fixed(const Pass& P, int n, const double* __restrict xr, const double* __restrict xi,
                double* __restrict yr, double* __restrict yi, int sign) {
    const int ns = P.ns, m = n / R;
    const double s = (double)sign;
    for (int jb = 0; jb < m; jb += ns) {
        for (int k = 0; k < ns; ++k) {
            const int j = jb + k;
            double wr[R], wi[R];
            wr[0] = 1.0;
            wi[0] = 0.0;
            for (int r = 1; r < R; ++r) {
                wr[r] = P.wr[(size_t)k * (R - 1) + r - 1];
                wi[r] = -s * P.wi[(size_t)k * (R - 1) + r - 1];
            }
            const size_t o = (size_t)jb * R + k;
#pragma GCC ivdep
            for (int l = 0; l < B; ++l) {
                double vr[R], vi[R];
                for (int r = 0; r < R; ++r) {
                    const double a = xr[(size_t)(j + r * m) * B + l], b = xi[(size_t)(j + r * m) * B + l];
                    vr[r] = a * wr[r] - b * wi[r];
                    vi[r] = a * wi[r] + b * wr[r];
                }
                small_dft<R>(vr, vi, s);
                for (int q = 0; q < R; ++q) {
                    yr[(o + (size_t)q * ns) * B + l] = vr[q];
                    yi[(o + (size_t)q * ns) * B + l] = vi[q];
                }
            }
        }
    }
}

// Radix 5 and the generic odd radix: twiddled inputs staged in u (R B values), then the R-point DFT by the table
// e^{sign 2 pi i t / R}.
void pass_generic(const Pass& P, int n, const double* __restrict xr, const double* __restrict xi,
                  double* __restrict yr, double* __restrict yi, double* __restrict ur, double* __restrict ui,
                  int sign) {
    const int R = P.R, ns = P.ns, m = n / R;
    const double s = (double)sign;
    for (int jb = 0; jb < m; jb += ns) {
        for (int k = 0; k < ns; ++k) {
            const int j = jb + k;
            for (int r = 0; r < R; ++r) {
                const double* a = xr + (size_t)(j + r * m) * B;
                const double* b = xi + (size_t)(j + r * m) * B;
                const double wr = r ? P.wr[(size_t)k * (R - 1) + r - 1] : 1.0;
                const double wi = r ? -s * P.wi[(size_t)k * (R - 1) + r - 1] : 0.0;
                for (int l = 0; l < B; ++l) {
                    ur[r * B + l] = a[l] * wr - b[l] * wi;
                    ui[r * B + l] = a[l] * wi + b[l] * wr;
                }
            }
            const size_t o = (size_t)jb * R + k;
            for (int q = 0; q < R; ++q) {
                double accr[B], acci[B];
                for (int l = 0; l < B; ++l) {
                    accr[l] = ur[l];
                    acci[l] = ui[l];
                }
                int e = 0;
                for (int t = 1; t < R; ++t) {
                    e += q;
                    if (e >= R) e -= R;
                    const double wr = P.cr[e], wi = -s * P.ci[e];
                    for (int l = 0; l < B; ++l) {
                        accr[l] += ur[t * B + l] * wr - ui[t * B + l] * wi;
                        acci[l] += ur[t * B + l] * wi + ui[t * B + l] * wr;
                    }
                }
                double* yqr = yr + (o + (size_t)q * ns) * B;
                double* yqi = yi + (o + (size_t)q * ns) * B;
                for (int l = 0; l < B; ++l) {
                    yqr[l] = accr[l];
                    yqi[l] = acci[l];
                }
            }
        }
    }
}

void stockham_pass(const Pass& P, int n, const double* xr, const double* xi, double* yr, double* yi, double* ur,
                   double* ui, int sign) {
    switch (P.R) {
    case 2: pass_fixed<2>(P, n, xr, xi, yr, yi, sign); break;
    case 3: pass_fixed<3>(P, n, xr, xi, yr, yi, sign); break;
    case 4: pass_fixed<4>(P, n, xr, xi, yr, yi, sign); break;
    case 8: pass_fixed<8>(P, n, xr, xi, yr, yi, sign); break;
    default: pass_generic(P, n, xr, xi, yr, yi, ur, ui, sign); break;
    }
}

// B interleaved lines of L.n points in place (re, im: n B values). Unnormalised; sign -1 forward, +1 inverse.
void run(const Line& L, double* re, double* im, Work& w, int sign) {
    const int n = L.n;
    if (n == 1) return;
    if (L.bluestein) {
        const int m = L.m;
        w.fit(m, L.max_radix);
        double* br = w.br.data();
        double* bi = w.bi.data();
        // the inverse conjugates on the way in and out of the forward chirp-z transform
        const double c = sign < 0 ? 1.0 : -1.0;
        for (int k = 0; k < n; ++k) {
            const double wr = L.chr[k], wi = L.chi[k];
            for (int l = 0; l < B; ++l) {
                const double xr = re[(size_t)k * B + l], xi = c * im[(size_t)k * B + l];
                br[(size_t)k * B + l] = xr * wr - xi * wi;
                bi[(size_t)k * B + l] = xr * wi + xi * wr;
            }
        }
        std::fill(br + (size_t)n * B, br + (size_t)m * B, 0.0);
        std::fill(bi + (size_t)n * B, bi + (size_t)m * B, 0.0);
        run(*L.inner, br, bi, w, -1);
        for (int k = 0; k < m; ++k) {
            const double fr = L.fr[k], fi = L.fi[k];
            for (int l = 0; l < B; ++l) {
                const double xr = br[(size_t)k * B + l], xi = bi[(size_t)k * B + l];
                br[(size_t)k * B + l] = xr * fr - xi * fi;
                bi[(size_t)k * B + l] = xr * fi + xi * fr;
            }
        }
        run(*L.inner, br, bi, w, +1);
        const double inv_m = 1.0 / (double)m;
        for (int k = 0; k < n; ++k) {
            const double wr = L.chr[k] * inv_m, wi = L.chi[k] * inv_m;
            for (int l = 0; l < B; ++l) {
                const double xr = br[(size_t)k * B + l], xi = bi[(size_t)k * B + l];
                re[(size_t)k * B + l] = xr * wr - xi * wi;
                im[(size_t)k * B + l] = c * (xr * wi + xi * wr);
            }
        }
        return;
    }
    w.fit(n, L.max_radix);
    double* sr = re;
    double* si = im;
    double* dr = w.ar.data();
    double* di = w.ai.data();
    for (const Pass& P : L.passes) {
        stockham_pass(P, n, sr, si, dr, di, w.ur.data(), w.ui.data(), sign);
        std::swap(sr, dr);
        std::swap(si, di);
    }
    if (sr != re) {
        std::memcpy(re, sr, sizeof(double) * (size_t)n * B);
        std::memcpy(im, si, sizeof(double) * (size_t)n * B);
    }
}

struct Plan2 {
    int nx = 0, ny = 0;
    std::unique_ptr<Line> row, col;  // row: length ny (contiguous), col: length nx
};

Plan2 make_plan2(int nx, int ny) {
    Plan2 p;
    p.nx = nx;
    p.ny = ny;
    p.row = make_line(ny);
    p.col = make_line(nx);
    return p;
}

// Per-thread buffers of the 2-D transform.
struct Work2 {
    Work w;
    std::vector<double> lr, li;  // B gathered lines
};

// In place on the split field (re, im: nx ny, row-major [ix][iy]), rows then columns. Optional elementwise factors:
// `pre` multiplies the field before the transform (fused into the row gather) and `post` after it (fused into the
// column scatter); a null imaginary part makes a factor real. `scale` multiplies the result. sign -1: NumPy's fft2;
// +1 with scale 1 / (nx ny): its ifft2.
void fft2(const Plan2& p, double* re, double* im, int sign, Work2& ws, const double* pre_r = nullptr,
          const double* pre_i = nullptr, const double* post_r = nullptr, const double* post_i = nullptr,
          double scale = 1.0) {
    const int nx = p.nx, ny = p.ny;
    const size_t len = (size_t)std::max(nx, ny) * B;
    if (ws.lr.size() < len) {
        ws.lr.resize(len);
        ws.li.resize(len);
    }
    double* lr = ws.lr.data();
    double* li = ws.li.data();
    // rows: B rows at a time, gathered lane-interleaved
    for (int x0 = 0; x0 < nx; x0 += B) {
        const int cnt = std::min(B, nx - x0);
        for (int l = 0; l < B; ++l) {
            if (l < cnt) {
                const size_t base = (size_t)(x0 + l) * ny;
                const double* a = re + base;
                const double* b = im + base;
                if (pre_r && !pre_i) {
                    const double* c = pre_r + base;
                    for (int y = 0; y < ny; ++y) {
                        lr[(size_t)y * B + l] = a[y] * c[y];
                        li[(size_t)y * B + l] = b[y] * c[y];
                    }
                } else if (pre_r) {
                    const double* c = pre_r + base;
                    const double* d = pre_i + base;
                    for (int y = 0; y < ny; ++y) {
                        lr[(size_t)y * B + l] = a[y] * c[y] - b[y] * d[y];
                        li[(size_t)y * B + l] = a[y] * d[y] + b[y] * c[y];
                    }
                } else {
                    for (int y = 0; y < ny; ++y) {
                        lr[(size_t)y * B + l] = a[y];
                        li[(size_t)y * B + l] = b[y];
                    }
                }
            } else {
                for (int y = 0; y < ny; ++y) lr[(size_t)y * B + l] = li[(size_t)y * B + l] = 0.0;
            }
        }
        run(*p.row, lr, li, ws.w, sign);
        for (int l = 0; l < cnt; ++l) {
            double* a = re + (size_t)(x0 + l) * ny;
            double* b = im + (size_t)(x0 + l) * ny;
            for (int y = 0; y < ny; ++y) {
                a[y] = lr[(size_t)y * B + l];
                b[y] = li[(size_t)y * B + l];
            }
        }
    }
    // columns: B neighbouring columns at a time (one contiguous run of B values per row)
    for (int y0 = 0; y0 < ny; y0 += B) {
        const int cnt = std::min(B, ny - y0);
        for (int x = 0; x < nx; ++x) {
            const double* a = re + (size_t)x * ny + y0;
            const double* b = im + (size_t)x * ny + y0;
            for (int l = 0; l < B; ++l) {
                lr[(size_t)x * B + l] = l < cnt ? a[l] : 0.0;
                li[(size_t)x * B + l] = l < cnt ? b[l] : 0.0;
            }
        }
        run(*p.col, lr, li, ws.w, sign);
        for (int x = 0; x < nx; ++x) {
            const size_t base = (size_t)x * ny + y0;
            for (int l = 0; l < cnt; ++l) {
                double vr = lr[(size_t)x * B + l], vi = li[(size_t)x * B + l];
                if (post_r) {
                    const double c = post_r[base + l], d = post_i ? post_i[base + l] : 0.0;
                    const double tr = vr * c - vi * d;
                    vi = vr * d + vi * c;
                    vr = tr;
                }
                re[base + l] = vr * scale;
                im[base + l] = vi * scale;
            }
        }
    }
}

// ---- the per-potential set-up of the scan, restated (each stage follows the float64 NumPy oracle's order) ------------

constexpr double kPlanck = 6.62607004e-34, kMass = 9.10938356e-31, kLight = 299792458.0,
                 kCharge = 1.6021766208e-19, kKappa = 0.0208865737082965, kAseKg = 6.0221408585491615e26,
                 kAseCoulomb = 6.241509125883258e18, kAseSecond = 98226947884640.62,
                 kAseJoule = 6.241509125883258e18;

// ElectronBeam.swift:38-43 and 24-30
double wavelength(double e) {
    const double c2 = kLight * kLight;
    return kPlanck * kLight / std::sqrt(e * (2 * kMass * c2 / kCharge + e)) / kCharge * 1.0e10;
}
double interaction_parameter(double e) {
    const double mass = (1 + kCharge * e / (kMass * (kLight * kLight))) * kMass;
    const double hsj = kPlanck * kAseSecond * kAseJoule;
    return 2 * M_PI * mass * kAseKg * kCharge * kAseCoulomb * wavelength(e) / (hsj * hsj);
}

// Grid.swift:45-86: sampling extent / n, NumPy's fftfreq(n, d) bit for bit.
struct Geo {
    int nx, ny;
    double ex, ey;
    double dx() const { return ex / nx; }
    double dy() const { return ey / ny; }
    size_t count() const { return (size_t)nx * ny; }
};
std::vector<double> fftfreq(int n, double d) {
    const double val = 1.0 / (n * d);
    const int pos = (n - 1) / 2 + 1;
    std::vector<double> f(n);
    for (int i = 0; i < n; ++i) f[i] = (double)(i < pos ? i : i - n) * val;
    return f;
}

// Antialias.swift:18-52
std::vector<double> antialias(const Geo& g) {
    const double dmax = std::max(g.dx(), g.dy());
    const double kc = 0.6666666 / dmax / 2, w = 0.01 / dmax;
    const std::vector<double> kx = fftfreq(g.nx, g.dx()), ky = fftfreq(g.ny, g.dy());
    std::vector<double> out(g.count(), 1.0);
    for (int ix = 0; ix < g.nx; ++ix)
        for (int iy = 0; iy < g.ny; ++iy) {
            const double r = std::sqrt(kx[ix] * kx[ix] + ky[iy] * ky[iy]);
            double& o = out[(size_t)ix * g.ny + iy];
            if (r > kc - w && r <= kc) o = 0.5 * (1 + std::cos(M_PI * (r - kc + w) / w));
            if (r > kc) o = 0.0;
        }
    return out;
}

// Aberrations.swift:39-59 with NumPy's grouping; ab in simk_probe's order (C10 C12 phi12 C21 phi21 C23 phi23 C30 C32
// phi32 C34 phi34 C41 phi41 C43 phi43 C45 phi45 C50 C52 phi52 C54 phi54 C56 phi56).
double chi(double alpha, double phi, const double* ab, double lam) {
    enum { C10, C12, P12, C21, P21, C23, P23, C30, C32, P32, C34, P34, C41, P41, C43, P43, C45, P45, C50, C52, P52,
           C54, P54, C56, P56 };
    double x = 0.0;
    if (ab[C10] || ab[C12] || ab[P12]) x = x + 1.0 / 2 * std::pow(alpha, 2) * (ab[C10] + ab[C12] * std::cos(2 * (phi - ab[P12])));
    if (ab[C21] || ab[P21] || ab[C23] || ab[P23])
        x = x + 1.0 / 3 * std::pow(alpha, 3) * (ab[C21] * std::cos(phi - ab[P21]) + ab[C23] * std::cos(3 * (phi - ab[P23])));
    if (ab[C30] || ab[C32] || ab[P32] || ab[C34] || ab[P34])
        x = x + 1.0 / 4 * std::pow(alpha, 4) *
                    (ab[C30] + ab[C32] * std::cos(2 * (phi - ab[P32])) + ab[C34] * std::cos(4 * (phi - ab[P34])));
    if (ab[C41] || ab[P41] || ab[C43] || ab[P43] || ab[C45] || ab[P45])
        x = x + 1.0 / 5 * std::pow(alpha, 5) *
                    (ab[C41] * std::cos(phi - ab[P41]) + ab[C43] * std::cos(3 * (phi - ab[P43])) +
                     ab[C45] * std::cos(5 * (phi - ab[P45])));
    if (ab[C50] || ab[C52] || ab[P52] || ab[C54] || ab[P54] || ab[C56] || ab[P56])
        x = x + 1.0 / 6 * std::pow(alpha, 6) *
                    (ab[C50] + ab[C52] * std::cos(2 * (phi - ab[P52])) + ab[C54] * std::cos(4 * (phi - ab[P54])) +
                     ab[C56] * std::cos(6 * (phi - ab[P56])));
    return x * (2 * M_PI / lam);
}

}  // namespace

extern "C" {

// The path one axis of length n takes (FFT2D.swift:130-156): 0 the direct transform (vDSP's lengths), 1 the mixed-radix
// passes, 2 Bluestein; -1 for n < 1.
int simk_cpu_fft_path(int n) {
    if (n < 1) return -1;
    if (has_direct_transform(n)) return 0;
    return prefers_bluestein(n) ? 2 : 1;
}

// MixedRadixPlan.factorization into out[0 .. cap); returns the number of factors (0 for n < 2).
int simk_cpu_factorization(int n, int* out, int cap) {
    const std::vector<int> f = factorization(n);
    for (int i = 0; i < (int)f.size() && i < cap; ++i) out[i] = f[i];
    return (int)f.size();
}

// MixedRadixPlan.costGuess.
double simk_cpu_cost_guess(int n) {
    double cost = 0.0;
    for (int p : factorization(n)) cost += (p == 4) ? 4.0 : (p <= 5 ? (double)p : 1.1 * p);
    return cost * n;
}

// In place on `count` arrays of nx x ny (split re / im), NumPy's fft2 (inverse != 0: ifft2).
int simk_cpu_fft2(int nx, int ny, int count, int inverse, double* re, double* im) {
    if (nx < 1 || ny < 1 || count < 0) return 1;
    const Plan2 p = make_plan2(nx, ny);
    const size_t N = (size_t)nx * ny;
    Work2 ws;
    const double scale = inverse ? 1.0 / ((double)nx * (double)ny) : 1.0;
    for (int c = 0; c < count; ++c)
        fft2(p, re + c * N, im + c * N, inverse ? +1 : -1, ws, nullptr, nullptr, nullptr, nullptr, scale);
    return 0;
}

// The STEM scan of one potential: for each position (ux, uy) in pixels, the probe IFFT2(spec r_x r_y) with
// r_x[ix] = e^{-2 pi i fx[ix] ux} (fx: NumPy's fftfreq(nx, 1), Probe.swift:140-156), through every slice
// (psi <- IFFT2(FFT2(psi t_j) P_{prop[j]})), then each detector's sum over its mask of |FFT2(exit)|^2. Arrays are split
// re / im, row-major [ix][iy]; masks: n_det x nx x ny weights; out: n_pos x n_det. `threads` workers take positions
// in turn, each with its own buffers.
int simk_cpu_stem_scan(int nx, int ny, int n_slices, const double* t_re, const double* t_im, const int* prop,
                       const double* p_re, const double* p_im, const double* spec_re, const double* spec_im,
                       const double* fx, const double* fy, int n_pos, const double* pos, int n_det,
                       const double* masks, int threads, double* out) {
    if (nx < 1 || ny < 1 || n_slices < 0 || n_pos < 0 || n_det < 0 || threads < 1) return 1;
    const size_t N = (size_t)nx * ny;
    const Plan2 plan = make_plan2(nx, ny);
    const double inv_n = 1.0 / ((double)nx * (double)ny);
    auto work = [&](int first, int stride) {
        std::vector<double> pr(N), pi(N), rxr(nx), rxi(nx), ryr(ny), ryi(ny);
        Work2 ws;
        for (int q = first; q < n_pos; q += stride) {
            const double x = pos[2 * q], y = pos[2 * q + 1];
            for (int ix = 0; ix < nx; ++ix) {
                const double a = -2.0 * M_PI * fx[ix] * x;
                rxr[ix] = std::cos(a);
                rxi[ix] = std::sin(a);
            }
            for (int iy = 0; iy < ny; ++iy) {
                const double a = -2.0 * M_PI * fy[iy] * y;
                ryr[iy] = std::cos(a);
                ryi[iy] = std::sin(a);
            }
            for (int ix = 0; ix < nx; ++ix)
                for (int iy = 0; iy < ny; ++iy) {
                    const size_t i = (size_t)ix * ny + iy;
                    const double sr = rxr[ix] * ryr[iy] - rxi[ix] * ryi[iy];
                    const double si = rxr[ix] * ryi[iy] + rxi[ix] * ryr[iy];
                    pr[i] = spec_re[i] * sr - spec_im[i] * si;
                    pi[i] = spec_re[i] * si + spec_im[i] * sr;
                }
            fft2(plan, pr.data(), pi.data(), +1, ws, nullptr, nullptr, nullptr, nullptr, inv_n);
            for (int j = 0; j < n_slices; ++j) {
                fft2(plan, pr.data(), pi.data(), -1, ws, t_re + j * N, t_im + j * N, p_re + (size_t)prop[j] * N,
                     p_im + (size_t)prop[j] * N);
                fft2(plan, pr.data(), pi.data(), +1, ws, nullptr, nullptr, nullptr, nullptr, inv_n);
            }
            fft2(plan, pr.data(), pi.data(), -1, ws);
            for (int d = 0; d < n_det; ++d) {
                const double* m = masks + (size_t)d * N;
                double s = 0.0;
                for (size_t i = 0; i < N; ++i)
                    if (m[i] != 0.0) s += m[i] * (pr[i] * pr[i] + pi[i] * pi[i]);
                out[(size_t)q * n_det + d] = s;
            }
        }
    };
    const int T = std::max(1, std::min(threads, n_pos));
    std::vector<std::thread> pool;
    for (int t = 1; t < T; ++t) pool.emplace_back(work, t, T);
    work(0, T);
    for (auto& th : pool) th.join();
    return 0;
}

// ---- the per-potential set-up ----------------------------------------------------------------------------------------

// The infinite-projection Lobato potential (ProjectedPotential.swift:110-201, Slicing.swift:71-104): atoms wrapped into
// the box (top-face rule), sliced at the nudged cumulative edges, then per slice and per element in increasing Z the
// bilinear deltas (weights added atom by atom), FFT2, times f(k^2) / S(k), inverse FFT2, real part, summed. Lobato
// parameters: n_table elements, table_z[e] with a[5 e .. 5 e + 4], b[..]; pi_choice 0 exact, 1 abTEM's float32 pi.
// out: n_slices x nx x ny V [V A]. Returns 1 for bad arguments, 2 for an element missing from the table.
int simk_cpu_potential(int nx, int ny, double ex, double ey, double ez, int n_slices, const double* thickness,
                       int n_atoms, const int* z, const double* xyz, int n_table, const int* table_z,
                       const double* table_a, const double* table_b, int pi_choice, double* out) {
    if (nx < 1 || ny < 1 || n_slices < 1 || n_atoms < 0 || !(ex > 0 && ey > 0 && ez > 0)) return 1;
    const Geo g{nx, ny, ex, ey};
    const size_t N = g.count();
    // wrap (fractional mod 1, ASE's wrap(eps=0)) and the top-face rule
    std::vector<double> p((size_t)n_atoms * 3);
    const double box[3] = {ex, ey, ez};
    for (int a = 0; a < n_atoms; ++a) {
        for (int d = 0; d < 3; ++d) {
            double f = std::fmod(xyz[3 * a + d] / box[d], 1.0);
            if (f < 0) f += 1.0;
            if (f == 1.0) f = 0.0;
            p[3 * a + d] = f * box[d];
        }
        if (p[3 * a + 2] > ez - 1e-10) p[3 * a + 2] = 0.0;
    }
    // slice of each atom: first edge strictly greater than z, edges = running sums - 1e-12; the last slice at most
    std::vector<double> edges(n_slices);
    double acc = 0.0;
    for (int j = 0; j < n_slices; ++j) {
        acc += thickness[j];
        edges[j] = acc - 1e-12;
    }
    std::vector<int> slice_of(n_atoms);
    for (int a = 0; a < n_atoms; ++a) {
        const int k = (int)(std::upper_bound(edges.begin(), edges.end(), p[3 * a + 2]) - edges.begin());
        slice_of[a] = std::min(k, n_slices - 1);
    }
    // kernels f(k^2) / S(k) per element present
    const std::vector<double> kx = fftfreq(nx, g.dx()), ky = fftfreq(ny, g.dy());
    std::vector<double> k2(N), comp(N);
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy) {
            const size_t i = (size_t)ix * ny + iy;
            k2[i] = kx[ix] * kx[ix] + ky[iy] * ky[iy];
            const double a = kx[ix] * g.dx(), b = ky[iy] * g.dy();
            const double k = (ix == 0 && iy == 0) ? 1.0 : std::sqrt(a * a + b * b);
            comp[i] = (ix == 0 && iy == 0) ? g.dx() * g.dy() : std::sin(k) / k * (g.dx() * g.dy());
        }
    const double pi = pi_choice ? (double)(float)M_PI : M_PI;
    const double pi2 = pi_choice ? (double)(float)(M_PI * M_PI) : M_PI * M_PI;
    std::vector<int> elements(z, z + n_atoms);
    std::sort(elements.begin(), elements.end());
    elements.erase(std::unique(elements.begin(), elements.end()), elements.end());
    std::vector<std::vector<double>> kernel(elements.size());
    for (size_t e = 0; e < elements.size(); ++e) {
        int row = -1;
        for (int t = 0; t < n_table; ++t)
            if (table_z[t] == elements[e]) row = t;
        if (row < 0) return 2;
        double A[5], B[5];
        for (int i = 0; i < 5; ++i) {
            const double a = table_a[5 * row + i], b = table_b[5 * row + i];
            A[i] = M_PI * M_PI * a / std::pow(b, 1.5) / kKappa;
            B[i] = 2 * M_PI / std::sqrt(b);
        }
        kernel[e].resize(N);
        for (size_t i = 0; i < N; ++i) {
            const double q = (4 * pi2) * k2[i];
            double sum = 0.0;
            for (int t = 0; t < 5; ++t) {
                const double d = q + B[t] * B[t];
                sum = sum + (A[t] / B[t] / d + A[t] * B[t] / (d * d));
            }
            kernel[e][i] = (8 * pi) * sum / comp[i];
        }
    }
    const Plan2 plan = make_plan2(nx, ny);
    Work2 ws;
    std::vector<double> dr(N), di(N);
    for (int j = 0; j < n_slices; ++j) {
        double* v = out + (size_t)j * N;
        std::fill(v, v + N, 0.0);
        for (size_t e = 0; e < elements.size(); ++e) {
            std::fill(dr.begin(), dr.end(), 0.0);
            std::fill(di.begin(), di.end(), 0.0);
            bool any = false;
            // weights in NumPy's np.add.at order: weight k outer, atoms inner
            for (int k = 0; k < 4; ++k)
                for (int a = 0; a < n_atoms; ++a) {
                    if (slice_of[a] != j || z[a] != elements[e]) continue;
                    any = true;
                    const double px = p[3 * a] / g.dx(), py = p[3 * a + 1] / g.dy();
                    const double rf = std::floor(px), cf = std::floor(py);
                    const double x = px - rf, y = py - cf, xy = x * y;
                    const double w[4] = {1 + xy - y - x, x - xy, y - xy, xy};
                    long long r = (long long)rf + ((k == 1 || k == 3) ? 1 : 0);
                    long long c = (long long)cf + (k >= 2 ? 1 : 0);
                    r %= nx;
                    if (r < 0) r += nx;
                    c %= ny;
                    if (c < 0) c += ny;
                    dr[(size_t)r * ny + c] += w[k];
                }
            if (!any) continue;
            fft2(plan, dr.data(), di.data(), -1, ws, nullptr, nullptr, kernel[e].data(), nullptr);
            fft2(plan, dr.data(), di.data(), +1, ws, nullptr, nullptr, nullptr, nullptr, 1.0 / (double)N);
            for (size_t i = 0; i < N; ++i) v[i] = v[i] + dr[i];
        }
    }
    return 0;
}
// The band-limited transmission of one slice (Multislice.swift:83-103): t = IFFT2(FFT2(e^{i sigma V}) A).
int simk_cpu_transmission(int nx, int ny, double ex, double ey, double energy, const double* v, double* re,
                          double* im) {
    if (nx < 1 || ny < 1 || !(ex > 0 && ey > 0 && energy > 0)) return 1;
    const Geo g{nx, ny, ex, ey};
    const size_t N = g.count();
    const double sigma = interaction_parameter(energy);
    for (size_t i = 0; i < N; ++i) {
        const double x = sigma * v[i];
        re[i] = std::cos(x);
        im[i] = std::sin(x);
    }
    const std::vector<double> a = antialias(g);
    const Plan2 plan = make_plan2(nx, ny);
    Work2 ws;
    fft2(plan, re, im, -1, ws, nullptr, nullptr, a.data(), nullptr);
    fft2(plan, re, im, +1, ws, nullptr, nullptr, nullptr, nullptr, 1.0 / (double)N);
    return 0;
}

// The Fresnel propagator of a slice dz [A] (Multislice.swift:108-130): e^{-i pi lambda dz k^2} A, times the tilt phase
// e^{-2 pi i dz (kx tan tx + ky tan ty)} for a beam tilt (tx, ty) [mrad].
int simk_cpu_propagator(int nx, int ny, double ex, double ey, double energy, double dz, double tilt_x, double tilt_y,
                        double* re, double* im) {
    if (nx < 1 || ny < 1 || !(ex > 0 && ey > 0 && energy > 0)) return 1;
    const Geo g{nx, ny, ex, ey};
    const double lam = wavelength(energy);
    const std::vector<double> kx = fftfreq(nx, g.dx()), ky = fftfreq(ny, g.dy()), a = antialias(g);
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy) {
            const size_t i = (size_t)ix * ny + iy;
            const double k2 = kx[ix] * kx[ix] + ky[iy] * ky[iy];
            const double x = -k2 * M_PI * dz * lam;
            double pr = std::cos(x) * a[i], pi = std::sin(x) * a[i];
            if (tilt_x != 0 || tilt_y != 0) {
                const double t = -2 * M_PI * dz * (kx[ix] * std::tan(tilt_x / 1e3) + ky[iy] * std::tan(tilt_y / 1e3));
                const double c = std::cos(t), sn = std::sin(t);
                const double r2 = pr * c - pi * sn;
                pi = pr * sn + pi * c;
                pr = r2;
            }
            re[i] = pr;
            im[i] = pi;
        }
    return 0;
}

// The probe's centred spectrum (Probe.swift:25-48, 113-136): the aperture (abTEM's soft edge one pixel wide when
// `soft`; semiangle [mrad], INFINITY for none) times e^{-i chi} (25 aberrations in simk_probe's order), divided by its
// norm.
int simk_cpu_probe_spectrum(int nx, int ny, double ex, double ey, double energy, double semiangle, int soft,
                            const double* aberrations, double* re, double* im) {
    if (nx < 1 || ny < 1 || !(ex > 0 && ey > 0 && energy > 0)) return 1;
    const Geo g{nx, ny, ex, ey};
    const double lam = wavelength(energy);
    const std::vector<double> kx = fftfreq(nx, g.dx()), ky = fftfreq(ny, g.dy());
    const double rsx = 1.0 / (nx * g.dx()), rsy = 1.0 / (ny * g.dy());
    const double cutoff = semiangle * 1e-3, dax = rsx * 1e3 * lam * 1e-3, day = rsy * 1e3 * lam * 1e-3;
    double norm2 = 0.0;
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy) {
            const size_t i = (size_t)ix * ny + iy;
            const double alpha = std::sqrt(kx[ix] * kx[ix] + ky[iy] * ky[iy]) * lam;
            const double phi = std::atan2(ky[iy], kx[ix]);
            double ap = 1.0;
            if (!std::isinf(semiangle)) {
                if (!soft) {
                    ap = alpha <= cutoff ? 1.0 : 0.0;
                } else if (ix == 0 && iy == 0) {
                    ap = 1.0;
                } else {
                    const double a = std::cos(phi) * dax, b = std::sin(phi) * day;
                    const double d = std::sqrt(a * a + b * b);
                    ap = std::min(std::max((cutoff - alpha) / d + 0.5, 0.0), 1.0);
                }
            }
            const double c = chi(alpha, phi, aberrations, lam);
            re[i] = ap * std::cos(-c);
            im[i] = ap * std::sin(-c);
            norm2 += re[i] * re[i] + im[i] * im[i];
        }
    const double n = std::sqrt(norm2);
    for (size_t i = 0; i < g.count(); ++i) {
        re[i] /= n;
        im[i] /= n;
    }
    return 0;
}

// An annular detector's mask on the k-space pixels (Detectors.swift:39-44, 119-135): inner^2 <= alpha^2 < outer^2,
// alpha from fftfreq(m, 1 / d / m) with d the angular sampling [mrad / pixel]; out 1 or 0.
int simk_cpu_annular_mask(int nx, int ny, double ex, double ey, double energy, double inner, double outer,
                          double* out) {
    if (nx < 1 || ny < 1 || !(ex > 0 && ey > 0 && energy > 0)) return 1;
    const Geo g{nx, ny, ex, ey};
    const double lam = wavelength(energy);
    const double ax = 1.0 / (nx * g.dx()) * lam * 1e3, ay = 1.0 / (ny * g.dy()) * lam * 1e3;
    const std::vector<double> fx = fftfreq(nx, 1.0 / ax / nx), fy = fftfreq(ny, 1.0 / ay / ny);
    for (int ix = 0; ix < nx; ++ix)
        for (int iy = 0; iy < ny; ++iy) {
            const double a2 = fx[ix] * fx[ix] + fy[iy] * fy[iy];
            out[(size_t)ix * ny + iy] = (a2 >= inner * inner && a2 < outer * outer) ? 1.0 : 0.0;
        }
    return 0;
}

// GaussianGenerator (FrozenPhonons.swift:14-58): SplitMix64 seeding, xoshiro256**, Box-Muller using both outputs.
int simk_cpu_normals(uint64_t seed, int n, double* out) {
    if (n < 0) return 1;
    auto fin = [](uint64_t z) {
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    };
    uint64_t st[4], x = seed;
    for (int i = 0; i < 4; ++i) {
        x += 0x9E3779B97F4A7C15ULL;
        st[i] = fin(x);
    }
    auto rotl = [](uint64_t v, int k) { return (v << k) | (v >> (64 - k)); };
    auto next = [&]() {
        const uint64_t result = rotl(st[1] * 5, 7) * 9;
        const uint64_t t = st[1] << 17;
        st[2] ^= st[0];
        st[3] ^= st[1];
        st[1] ^= st[2];
        st[0] ^= st[3];
        st[2] ^= t;
        st[3] = rotl(st[3], 45);
        return result;
    };
    for (int i = 0; i < n; i += 2) {
        const double u1 = (double)((next() >> 11) + 1) * 0x1p-53;
        const double u2 = (double)(next() >> 11) * 0x1p-53;
        const double r = std::sqrt(-2 * std::log(u1)), th = 2 * M_PI * u2;
        out[i] = r * std::cos(th);
        if (i + 1 < n) out[i + 1] = r * std::sin(th);
    }
    return 0;
}

}  // extern "C"
