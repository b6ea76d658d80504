// fft.cu -- host-side line plans and the generic batched line-FFT kernel (shared-memory Stockham, any length).
#include "fft.cuh"

#include <algorithm>
#include <complex>

namespace simk {

LinePlanDev LinePlan::dev() const {
    LinePlanDev d{};
    d.n = n;
    d.m = m;
    d.nfac = (int)factors.size();
    d.bluestein = bluestein ? 1 : 0;
    for (int i = 0; i < d.nfac; ++i) {
        d.fac[i] = factors[i];
        d.rad_off[i] = rad_off.empty() ? 0 : rad_off[i];
    }
    d.tw = tw.ptr;
    d.chirp = chirp.ptr;
    d.khat = khat.ptr;
    d.rad_cos = rad_cos.as<double>();
    d.rad_sin = rad_sin.as<double>();
    return d;
}

std::vector<int> gpu_factorization(int n) {
    std::vector<int> out;
    int rest = n;
    for (int r : {16, 8, 4, 2}) {
        while (rest % r == 0 && rest > 1) {
            out.push_back(r);
            rest /= r;
        }
    }
    for (int p = 3; p <= kMaxGenericRadix && rest > 1; p += 2) {
        while (rest % p == 0) {
            out.push_back(p);
            rest /= p;
        }
    }
    if (rest != 1) return {};
    // Larger radices first keeps the first passes' twiddle-free work large; the order does not change the result.
    return out;
}

namespace {

// In-place radix-2 FFT in float64 on the host, forward (e^{-}), for the Bluestein kernel spectrum (m a power of two).
void host_fft_pow2(std::vector<std::complex<double>>& a) {
    const size_t m = a.size();
    for (size_t i = 1, j = 0; i < m; ++i) {
        size_t bit = m >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (size_t len = 2; len <= m; len <<= 1) {
        for (size_t i = 0; i < m; i += len) {
            for (size_t k = 0; k < len / 2; ++k) {
                // exact integer phase k / len, reduced to the table of the full length
                double ang = -2.0 * M_PI * (double)k / (double)len;
                std::complex<double> w(std::cos(ang), std::sin(ang));
                auto u = a[i + k], v = a[i + k + len / 2] * w;
                a[i + k] = u + v;
                a[i + k + len / 2] = u - v;
            }
        }
    }
}

template <typename V>
void upload_complex(DeviceBuffer& buf, const std::vector<std::complex<double>>& v) {
    std::vector<V> h(v.size());
    for (size_t i = 0; i < v.size(); ++i) {
        h[i].x = (decltype(V::x))v[i].real();
        h[i].y = (decltype(V::x))v[i].imag();
    }
    buf.alloc(h.size() * sizeof(V));
    SIMK_CUDA(cudaMemcpy(buf.ptr, h.data(), h.size() * sizeof(V), cudaMemcpyHostToDevice));
}

std::vector<std::complex<double>> twiddles(int m) {
    std::vector<std::complex<double>> t(m);
    for (int k = 0; k < m; ++k) {
        // e^{-2 pi i k/m} from the exact ratio k/m
        double s, c;
        host_sincospi(-2.0 * (double)k / (double)m, &s, &c);
        t[k] = {c, s};
    }
    return t;
}

}  // namespace

std::unique_ptr<LinePlan> make_line_plan(int n, int precision) {
    SIMK_REQUIRE(n >= 1, "FFT length must be at least 1");
    auto p = std::make_unique<LinePlan>();
    p->n = n;
    p->precision = precision;
    std::vector<int> f = (n == 1) ? std::vector<int>{} : gpu_factorization(n);
    if (n > 1 && f.empty()) {
        // Bluestein: the smallest power of two >= 2n - 1 and >= 16 (FFT2D.swift:84-88)
        int m = 16;
        while (m < 2 * n - 1) m *= 2;
        p->bluestein = true;
        p->m = m;
        p->factors = gpu_factorization(m);
        std::vector<std::complex<double>> chirp(n), kern(m, {0.0, 0.0});
        for (int j = 0; j < n; ++j) {
            long long r = ((long long)j * j) % (2LL * n);  // j^2 mod 2n keeps the phase exact (FFT2D.swift:65-70)
            double s, c;
            host_sincospi(-(double)r / (double)n, &s, &c);
            chirp[j] = {c, s};
            kern[j] = std::conj(chirp[j]);
            if (j > 0) kern[m - j] = std::conj(chirp[j]);
        }
        host_fft_pow2(kern);
        for (auto& k : kern) k /= (double)m;
        if (precision == 64) {
            upload_complex<double2>(p->chirp, chirp);
            upload_complex<double2>(p->khat, kern);
        } else {
            upload_complex<float2>(p->chirp, chirp);
            upload_complex<float2>(p->khat, kern);
        }
    } else {
        p->m = n;
        p->factors = f;
    }
    SIMK_REQUIRE((int)p->factors.size() <= kMaxFactors, "FFT length has too many factors");
    auto tw = twiddles(p->m);
    if (precision == 64) upload_complex<double2>(p->tw, tw);
    else upload_complex<float2>(p->tw, tw);
    // cos/sin tables of the generic radices
    std::vector<double> rc, rs;
    for (int r : p->factors) {
        p->rad_off.push_back((int)rc.size());
        if (r == 2 || r == 3 || r == 4 || r == 5 || r == 8 || r == 16) continue;
        for (int k = 0; k < r; ++k) {
            double s, c;
            host_sincospi(2.0 * (double)k / (double)r, &s, &c);
            rc.push_back(c);
            rs.push_back(s);
        }
    }
    if (rc.empty()) {
        rc.push_back(1.0);
        rs.push_back(0.0);
    }
    p->rad_cos.alloc(rc.size() * sizeof(double));
    p->rad_sin.alloc(rs.size() * sizeof(double));
    SIMK_CUDA(cudaMemcpy(p->rad_cos.ptr, rc.data(), rc.size() * sizeof(double), cudaMemcpyHostToDevice));
    SIMK_CUDA(cudaMemcpy(p->rad_sin.ptr, rs.data(), rs.size() * sizeof(double), cudaMemcpyHostToDevice));
    return p;
}

// ---- the generic kernel -------------------------------------------------------------------------------------------
template <typename T, int DIR>
__device__ void line_fft_body(c2_t<T>* __restrict__ data, const LinePlanDev& p, long long nlines, int lines_per_batch,
                              long long line_stride, long long elem_stride, long long batch_stride, T scale, int L,
                              int lds) {
    using V = c2_t<T>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* a = reinterpret_cast<V*>(smem_raw);
    V* b = a + (size_t)L * lds;
    const long long first = (long long)blockIdx.x * L;
    const int lines = (int)min((long long)L, nlines - first);
    const int n = p.n, m = p.m;
    const int tid = threadIdx.x, nth = blockDim.x;
    auto base_of = [&](int l) -> long long {
        long long g = first + l;
        return (g / lines_per_batch) * batch_stride + (g % lines_per_batch) * line_stride;
    };
    const V* chirp = static_cast<const V*>(p.chirp);
    // load: consecutive threads read consecutive addresses (along the line for rows, across lines for columns)
    const bool along = (elem_stride == 1);
    for (int idx = tid; idx < lines * n; idx += nth) {
        int l, e;
        if (along) { l = idx / n; e = idx - l * n; }
        else { e = idx / lines; l = idx - e * lines; }
        V x = data[base_of(l) + e * elem_stride];
        if (p.bluestein) {
            if (DIR > 0) x = cconj(x);  // the inverse as conj(DFT(conj x))
            x = cmul(x, chirp[e]);
        }
        a[l * lds + e] = x;
    }
    if (p.bluestein) {
        for (int idx = tid; idx < lines * (m - n); idx += nth) {
            int l = idx / (m - n), e = n + idx % (m - n);
            a[l * lds + e] = mk<V>((T)0, (T)0);
        }
    }
    __syncthreads();
    V* res;
    if (!p.bluestein) {
        res = stockham_lines<DIR>(a, b, p, lines, lds);
    } else {
        res = stockham_lines<-1>(a, b, p, lines, lds);
        V* other = (res == a) ? b : a;
        const V* kh = static_cast<const V*>(p.khat);
        for (int idx = tid; idx < lines * m; idx += nth) {
            int l = idx / m, e = idx - l * m;
            res[l * lds + e] = cmul(res[l * lds + e], kh[e]);
        }
        __syncthreads();
        res = stockham_lines<+1>(res, other, p, lines, lds);
    }
    for (int idx = tid; idx < lines * n; idx += nth) {
        int l, e;
        if (along) { l = idx / n; e = idx - l * n; }
        else { e = idx / lines; l = idx - e * lines; }
        V y = res[l * lds + e];
        if (p.bluestein) {
            y = cmul(y, chirp[e]);
            if (DIR > 0) y = cconj(y);
        }
        data[base_of(l) + e * elem_stride] = y * scale;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) line_fft_kernel(c2_t<T>* data, LinePlanDev p, long long nlines,
                                                       int lines_per_batch, long long line_stride,
                                                       long long elem_stride, long long batch_stride, int dir,
                                                       T scale, int L, int lds) {
    if (dir < 0)
        line_fft_body<T, -1>(data, p, nlines, lines_per_batch, line_stride, elem_stride, batch_stride, scale, L, lds);
    else
        line_fft_body<T, +1>(data, p, nlines, lines_per_batch, line_stride, elem_stride, batch_stride, scale, L, lds);
}

namespace {
template <typename T>
void launch_t(const LinePlan& plan, void* data, long long nlines, int lines_per_batch, long long line_stride,
              long long elem_stride, long long batch_stride, int dir, double scale, cudaStream_t stream,
              int64_t* launches) {
    using V = c2_t<T>;
    const int lds = plan.m + ((plan.m % 2 == 0) ? 1 : 0);
    const size_t budget = 96 * 1024;
    int L = (int)std::max<size_t>(1, std::min<size_t>(16, budget / (2 * (size_t)lds * sizeof(V))));
    if (elem_stride == 1) L = std::min(L, 4);  // rows: a few whole lines per CTA
    const size_t smem = 2 * (size_t)L * lds * sizeof(V);
    static bool attr_set[2] = {false, false};
    const int which = sizeof(T) == 8 ? 1 : 0;
    if (!attr_set[which]) {
        SIMK_CUDA(cudaFuncSetAttribute(line_fft_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr_set[which] = true;
    }
    SIMK_REQUIRE(smem <= 200 * 1024, "FFT line too long for one CTA");
    long long blocks = (nlines + L - 1) / L;
    SIMK_REQUIRE(blocks < (1LL << 31), "too many FFT lines");
    line_fft_kernel<T><<<(unsigned)blocks, 256, smem, stream>>>(static_cast<V*>(data), plan.dev(), nlines,
                                                               lines_per_batch, line_stride, elem_stride, batch_stride,
                                                               dir, (T)scale, L, lds);
    SIMK_CUDA(cudaGetLastError());
    if (launches) ++*launches;
}
}  // namespace

void launch_line_fft(const LinePlan& plan, void* data, long long nlines, int lines_per_batch, long long line_stride,
                     long long elem_stride, long long batch_stride, int dir, double scale, cudaStream_t stream,
                     int64_t* launches) {
    if (nlines <= 0) return;
    if (plan.precision == 64)
        launch_t<double>(plan, data, nlines, lines_per_batch, line_stride, elem_stride, batch_stride, dir, scale,
                         stream, launches);
    else
        launch_t<float>(plan, data, nlines, lines_per_batch, line_stride, elem_stride, batch_stride, dir, scale, stream,
                        launches);
}

void fft2(const LinePlan& row_plan, const LinePlan& col_plan, void* data, int nx, int ny, long long count, int dir,
          double scale, cudaStream_t stream, int64_t* launches) {
    const long long N = (long long)nx * ny;
    // rows: length ny, contiguous
    launch_line_fft(row_plan, data, count * nx, nx, ny, 1, N, dir, 1.0, stream, launches);
    // columns: length nx, stride ny
    launch_line_fft(col_plan, data, count * ny, ny, 1, ny, N, dir, scale, stream, launches);
}

}  // namespace simk
