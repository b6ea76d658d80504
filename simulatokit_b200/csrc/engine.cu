// engine.cu -- the multislice loop on the device: Multislice.run / runBatch and the STEM scan, in the plain form
// (one operation per launch over a batch of waves) and the fused form (fused.cu).
#include <algorithm>
#include <cstring>

#include "context.cuh"
#include "engine.cuh"

namespace simk {

// fft2 with each line pass timed as "line_fft" (algorithmic bytes: one read and one write of every element).
void fft2_timed(Context& ctx, const LinePlan& prow, const LinePlan& pcol, float2* data, int nx, int ny, long long count,
                int dir, double scale) {
    const long long N = (long long)nx * ny;
    const double bytes = 16.0 * (double)N * (double)count;
    {
        KernelTimer t(ctx, "line_fft", bytes);
        launch_line_fft(prow, data, count * nx, nx, ny, 1, N, dir, 1.0, ctx.stream, &ctx.launches);
    }
    {
        KernelTimer t(ctx, "line_fft", bytes);
        launch_line_fft(pcol, data, count * ny, ny, 1, ny, N, dir, scale, ctx.stream, &ctx.launches);
    }
}

void mul_timed(Context& ctx, float2* psi, const float2* f, long long N, int count, float scale) {
    KernelTimer t(ctx, "pointwise", 16.0 * (double)N * (double)count);
    launch_mul_broadcast(ctx, psi, f, N, count, scale);
}

// A kernel whose bounded wait ran out set ctx.err_flag: report it (and clear it) after the stream has drained.
void check_device_error(Context& ctx) {
    if (!ctx.err_flag.ptr) return;
    int flag = 0;
    SIMK_CUDA(cudaMemcpyAsync(&flag, ctx.err_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
    if (flag) {
        SIMK_CUDA(cudaMemsetAsync(ctx.err_flag.ptr, 0, sizeof(int), ctx.stream));
        throw Error(SIMK_ERR_TIMEOUT, "a device wait for an asynchronous copy ran out; the results are invalid");
    }
}

long long batch_size(const Context& ctx, const GridGeom& g, long long count) {
    long long b = ctx.batch;
    if (b <= 0) b = std::max<long long>(1, ctx.batch_bytes / (long long)(g.count() * sizeof(float2)));
    return std::max<long long>(1, std::min(b, count));
}

// psi (count waves, float2, on the device) through every slice of the potential, plain form. After slice j,
// on_slice(j) is called (stream-ordered) so the caller can copy planes out.
void propagate_plain(Context& ctx, PotentialImpl& pot, double energy, double tx, double ty, float2* psi, int count,
                     bool last_inverse, const std::function<void(int)>& on_slice) {
    const GridGeom& g = pot.g;
    const long long N = g.count();
    const LinePlan& prow = ctx.plan(g.ny, 32);
    const LinePlan& pcol = ctx.plan(g.nx, 32);
    const int S = pot.n_slices();
    for (int j = 0; j < S; ++j) {
        const Propagator& P = ctx.propagator(g, energy, pot.dz[j], tx, ty);
        mul_timed(ctx, psi, pot.t.as<float2>() + (long long)j * N, N, count, 1.0f);
        fft2_timed(ctx, prow, pcol, psi, g.nx, g.ny, count, -1, 1.0);
        mul_timed(ctx, psi, P.p.as<float2>(), N, count, 1.0f / (float)N);
        if (j < S - 1 || last_inverse) fft2_timed(ctx, prow, pcol, psi, g.nx, g.ny, count, +1, 1.0);
        if (on_slice) on_slice(j);
    }
}

void run_waves(Context& ctx, PotentialImpl& pot, double energy, double tx, double ty, int count, const double* in_re,
               const double* in_im, const std::vector<int>& planes, double* out_re, double* out_im) {
    const GridGeom& g = pot.g;
    const long long N = g.count();
    prepare_transmissions(ctx, pot, energy);
    const long long B = batch_size(ctx, g, count);
    ctx.work_a.ensure(B * N * sizeof(float2));
    std::vector<float2> host(B * N);
    const int np = (int)planes.size();
    for (long long first = 0; first < count; first += B) {
        const int b = (int)std::min<long long>(B, count - first);
        for (long long i = 0; i < b * N; ++i)
            host[i] = make_float2((float)in_re[first * N + i], (float)in_im[first * N + i]);
        SIMK_CUDA(cudaMemcpyAsync(ctx.work_a.ptr, host.data(), b * N * sizeof(float2), cudaMemcpyHostToDevice,
                                  ctx.stream));
        float2* psi = ctx.work_a.as<float2>();
        const bool fused = (ctx.form != SIMK_FORM_PLAIN) && fused_supported(ctx, g);
        if (fused) ctx.work_b.ensure(B * N * sizeof(float2));
        auto copy_out = [&](int j) {
            for (int q = 0; q < np; ++q) {
                if (planes[q] != j) continue;
                const float2* src = psi;
                if (fused) {  // complete the row inverse transform on a copy
                    SIMK_CUDA(cudaMemcpyAsync(ctx.work_b.ptr, psi, b * N * sizeof(float2), cudaMemcpyDeviceToDevice,
                                              ctx.stream));
                    finish_rows(ctx, g, ctx.work_b.as<float2>(), b);
                    src = ctx.work_b.as<float2>();
                }
                SIMK_CUDA(cudaMemcpyAsync(host.data(), src, b * N * sizeof(float2), cudaMemcpyDeviceToHost, ctx.stream));
                SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
                // output layout: [wave][plane][N] for run (count = 1) and [wave][N] for run_batch (one plane)
                for (int w = 0; w < b; ++w)
                    for (long long i = 0; i < N; ++i) {
                        const long long o = ((first + w) * np + q) * N + i;
                        out_re[o] = host[w * N + i].x;
                        out_im[o] = host[w * N + i].y;
                    }
            }
        };
        if (fused)
            propagate_fused(ctx, pot, energy, tx, ty, psi, b, false, [&](int j, bool) { copy_out(j); }, false);
        else
            propagate_plain(ctx, pot, energy, tx, ty, psi, b, true, copy_out);
    }
    SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
    check_device_error(ctx);
}

namespace {
void scan_plain_batch(Context& ctx, PotentialImpl& pot, const simk_probe& probe, const float2* spectrum,
                      const double* positions_dev, long long first, int b, const DetectorPlan& dplan,
                      double* const* outputs_dev, double weight) {
    const GridGeom& g = pot.g;
    const long long N = g.count();
    const LinePlan& prow = ctx.plan(g.ny, 32);
    const LinePlan& pcol = ctx.plan(g.nx, 32);
    float2* psi = ctx.work_a.as<float2>();
    launch_ramps(ctx, g, positions_dev, first, b, ctx.rx.as<float2>(), ctx.ry.as<float2>());
    launch_probes(ctx, g, spectrum, ctx.rx.as<float2>(), ctx.ry.as<float2>(), b, psi, 1.0f);
    fft2_timed(ctx, prow, pcol, psi, g.nx, g.ny, b, +1, 1.0 / (double)N);
    propagate_plain(ctx, pot, probe.energy, probe.tilt_x, probe.tilt_y, psi, b, true, nullptr);
    // the diffraction intensity |FFT2(exit)|^2 (DiffractionIntensity, Detectors.swift:28-36)
    fft2_timed(ctx, prow, pcol, psi, g.nx, g.ny, b, -1, 1.0);
    {
        KernelTimer t(ctx, "detect", 8.0 * (double)N * b);
        launch_detect(ctx, dplan, g, psi, b, first, outputs_dev, weight, 1.0f);
    }
}
}  // namespace

void scan_device(Context& ctx, const simk_probe& probe, const std::vector<PotentialImpl*>& pots, int n_pos,
                 const double* positions_dev, int n_det, const simk_detector* dets, double* const* outputs_dev) {
    SIMK_REQUIRE(!pots.empty(), "no potential");
    const GridGeom g = pots[0]->g;
    for (auto* p : pots)
        SIMK_REQUIRE(p->g.nx == g.nx && p->g.ny == g.ny &&
                         std::fabs(p->g.ex - g.ex) <= 1e-12 * std::max(std::fabs(p->g.ex), std::fabs(g.ex)) &&
                         std::fabs(p->g.ey - g.ey) <= 1e-12 * std::max(std::fabs(p->g.ey), std::fabs(g.ey)),
                     "the potentials' grids must match the probe's");
    const long long N = g.count();
    // detector maps and the probe spectrum depend only on (grid, energy, detectors) and (grid, probe): built once
    auto key_bytes = [](const void* p, size_t n) { return std::string(static_cast<const char*>(p), n); };
    std::string gkey = key_bytes(&g.nx, sizeof(int) * 2) + key_bytes(&g.ex, sizeof(double)) +
                       key_bytes(&g.ey, sizeof(double));
    std::string dkey = gkey + key_bytes(&probe.energy, sizeof(double)) +
                       key_bytes(dets, sizeof(simk_detector) * (size_t)n_det);
    auto dit = ctx.detector_plans.find(dkey);
    if (dit == ctx.detector_plans.end()) {
        if (ctx.detector_plans.size() > 64) ctx.detector_plans.clear();
        dit = ctx.detector_plans.emplace(dkey, build_detector_plan(ctx, g, probe.energy, dets, n_det)).first;
    }
    DetectorPlan* dplan = dit->second.get();
    std::string skey = gkey + key_bytes(&probe, sizeof(simk_probe));
    auto sit = ctx.spectra.find(skey);
    if (sit == ctx.spectra.end()) {
        if (ctx.spectra.size() > 64) ctx.spectra.clear();
        auto buf = std::make_unique<DeviceBuffer>();
        probe_spectrum_device(ctx, g, probe, *buf, nullptr);
        sit = ctx.spectra.emplace(skey, std::move(buf)).first;
    }
    const DeviceBuffer& spectrum = *sit->second;
    for (int d = 0; d < n_det; ++d)
        SIMK_CUDA(cudaMemsetAsync(outputs_dev[d], 0, (size_t)n_pos * dplan->det_count[d] * sizeof(double), ctx.stream));
    // SIMK_OPT_AUTOTUNE: the tuned column tile, TMA choice and batch wherever the caller left them automatic, for
    // this call only
    struct Restore {
        Context& c;
        int tc, tma;
        long long batch;
        int composite, tcgen05;
        ~Restore() {
            c.col_tile = tc;
            c.tma = tma;
            c.batch = batch;
            c.composite = composite;
            c.tcgen05 = tcgen05;
        }
    } restore{ctx, ctx.col_tile, ctx.tma, ctx.batch, ctx.composite, ctx.tcgen05};
    if (ctx.autotune && ctx.form != SIMK_FORM_PLAIN && fused_supported(ctx, g)) {
        prepare_transmissions(ctx, *pots[0], probe.energy);
        const Context::Tuned t = autotune(ctx, *pots[0], probe.energy, probe.tilt_x, probe.tilt_y, n_pos);
        if (ctx.col_tile == 0) ctx.col_tile = t.col_tile;
        if (ctx.tma) ctx.tma = t.tma;
        if (ctx.batch == 0) ctx.batch = t.batch;
        if (t.engine >= 0) {  // the tuned engine (radix plan) for this scan
            if (ctx.form == SIMK_FORM_FUSED) ctx.composite = t.engine;
            else ctx.tcgen05 = t.engine;
        }
    }
    const long long B = batch_size(ctx, g, n_pos);
    ctx.work_a.ensure(B * N * sizeof(float2));
    ctx.rx.ensure(B * g.nx * sizeof(float2));
    ctx.ry.ensure(B * g.ny * sizeof(float2));
    const double weight = 1.0 / (double)pots.size();
    for (auto* pot : pots) {
        prepare_transmissions(ctx, *pot, probe.energy);
        bool fused = (ctx.form != SIMK_FORM_PLAIN) && fused_supported(ctx, g);
        if (fused) ctx.work_b.ensure(B * N * sizeof(float2));
        for (long long first = 0; first < n_pos; first += B) {
            const int b = (int)std::min<long long>(B, n_pos - first);
            if (fused)
                scan_fused_batch(ctx, *pot, probe, spectrum.as<float2>(), positions_dev, first, b, *dplan, outputs_dev,
                                 weight);
            else
                scan_plain_batch(ctx, *pot, probe, spectrum.as<float2>(), positions_dev, first, b, *dplan, outputs_dev,
                                 weight);
        }
    }
}

// ---- the waves detector --------------------------------------------------------------------------------------------
// Waves.resampled (WavesResample.swift:16-43) on the device: the exit spectrum FFT2(exit) is at hand after the last
// slice (the fused form stops there for the detectors; the plain form too, times 1/N), so resampling is a gather of
// the frequencies kept (Waves.resampleMap: the lowest rows x columns, or all of them zero-padded) into the target
// spectrum followed by one inverse transform of the target size; rows columns / N (abTEM's scaling) times the
// inverse's 1 / (rows columns) leaves 1 / N, applied in the gather. Without resampling the map is the identity.
namespace {
__global__ void k_resample_gather(const float2* __restrict__ S, long long N, int ny, const int* __restrict__ srcx,
                                  const int* __restrict__ srcy, int rows, int cols, int count, float scale,
                                  float2* __restrict__ out) {
    const long long M = (long long)rows * cols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < M * count;
         i += (long long)gridDim.x * blockDim.x) {
        const long long w = i / M, o = i - w * M;
        const int dx = (int)(o / cols), dy = (int)(o - (long long)dx * cols);
        const int sx = srcx[dx], sy = srcy[dy];
        out[i] = (sx >= 0 && sy >= 0) ? S[w * N + (long long)sx * ny + sy] * scale : make_float2(0.0f, 0.0f);
    }
}

// For every destination index of an axis resampled from n to m points, its source frequency or -1 (zero padding).
std::vector<int> resample_sources(int n, int m) {
    std::vector<int> src(m, -1);
    if (m <= n) {
        if (m == 1) {
            src[0] = 0;
            return src;
        }
        // the first m/2 (even m) or floor(m/2) + 1 (odd m) frequencies, then the last floor(m/2)
        const int low = (m % 2) ? m / 2 + 1 : m / 2, high = m / 2;
        for (int d = 0; d < low; ++d) src[d] = d;
        for (int d = 0; d < high; ++d) src[low + d] = n - high + d;
        return src;
    }
    if (n == 1) {
        src[0] = 0;
        return src;
    }
    const int positive = (n % 2 == 0) ? n / 2 : n / 2 + 1;
    for (int i = 0; i < n; ++i) src[i < positive ? i : m - n + i] = i;
    return src;
}
}  // namespace

void scan_waves(Context& ctx, const simk_probe& probe, PotentialImpl& pot, int n_pos, const double* positions_xy,
                int rows, int columns, double* out_re, double* out_im) {
    const GridGeom& g = pot.g;
    const long long N = g.count();
    if (rows == 0 && columns == 0) {
        rows = g.nx;
        columns = g.ny;
    }
    SIMK_REQUIRE(rows >= 2 && columns >= 2, "the waves detector needs at least 2 points per axis");
    const long long M = (long long)rows * columns;
    prepare_transmissions(ctx, pot, probe.energy);
    DeviceBuffer spectrum, pos((size_t)2 * n_pos * sizeof(double));
    probe_spectrum_device(ctx, g, probe, spectrum, nullptr);
    SIMK_CUDA(cudaMemcpyAsync(pos.ptr, positions_xy, (size_t)2 * n_pos * sizeof(double), cudaMemcpyHostToDevice,
                              ctx.stream));
    const std::vector<int> sx = resample_sources(g.nx, rows), sy = resample_sources(g.ny, columns);
    DeviceBuffer dsx(sx.size() * sizeof(int)), dsy(sy.size() * sizeof(int));
    SIMK_CUDA(cudaMemcpyAsync(dsx.ptr, sx.data(), sx.size() * sizeof(int), cudaMemcpyHostToDevice, ctx.stream));
    SIMK_CUDA(cudaMemcpyAsync(dsy.ptr, sy.data(), sy.size() * sizeof(int), cudaMemcpyHostToDevice, ctx.stream));
    const long long B = batch_size(ctx, g, n_pos);
    ctx.work_a.ensure(B * N * sizeof(float2));
    ctx.rx.ensure(B * g.nx * sizeof(float2));
    ctx.ry.ensure(B * g.ny * sizeof(float2));
    const bool fused = (ctx.form != SIMK_FORM_PLAIN) && fused_supported(ctx, g);
    if (fused) ctx.work_b.ensure(B * N * sizeof(float2));
    DeviceBuffer outb((size_t)B * M * sizeof(float2));
    std::vector<float2> h((size_t)B * M);
    const LinePlan& prow = ctx.plan(g.ny, 32);
    const LinePlan& pcol = ctx.plan(g.nx, 32);
    for (long long first = 0; first < n_pos; first += B) {
        const int b = (int)std::min<long long>(B, n_pos - first);
        float2* psi = ctx.work_a.as<float2>();
        float scale;
        if (fused) {
            exit_spectra_fused(ctx, pot, probe, spectrum.as<float2>(), pos.as<double>(), first, b);
            scale = 1.0f / (float)N;
        } else {
            launch_ramps(ctx, g, pos.as<double>(), first, b, ctx.rx.as<float2>(), ctx.ry.as<float2>());
            launch_probes(ctx, g, spectrum.as<float2>(), ctx.rx.as<float2>(), ctx.ry.as<float2>(), b, psi, 1.0f);
            fft2_timed(ctx, prow, pcol, psi, g.nx, g.ny, b, +1, 1.0 / (double)N);
            propagate_plain(ctx, pot, probe.energy, probe.tilt_x, probe.tilt_y, psi, b, false, nullptr);
            scale = 1.0f;  // the last slice already carries the 1 / N of the transform it skipped
        }
        const long long total = M * b;
        k_resample_gather<<<(int)std::max<long long>(1, std::min<long long>((total + 255) / 256, 148LL * 16)), 256, 0,
                            ctx.stream>>>(psi, N, g.ny, dsx.as<int>(), dsy.as<int>(), rows, columns, b, scale,
                                          outb.as<float2>());
        SIMK_CUDA(cudaGetLastError());
        ++ctx.launches;
        fft2(ctx.plan(columns, 32), ctx.plan(rows, 32), outb.ptr, rows, columns, b, +1, 1.0, ctx.stream,
             &ctx.launches);
        SIMK_CUDA(cudaMemcpyAsync(h.data(), outb.ptr, (size_t)total * sizeof(float2), cudaMemcpyDeviceToHost,
                                  ctx.stream));
        SIMK_CUDA(cudaStreamSynchronize(ctx.stream));
        for (long long i = 0; i < total; ++i) {
            out_re[first * M + i] = h[i].x;
            out_im[first * M + i] = h[i].y;
        }
    }
    check_device_error(ctx);
}

}  // namespace simk
