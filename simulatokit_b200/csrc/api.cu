// api.cu -- the extern "C" entry points of libsimulato_cuda.so (declared in include/simulato_cuda.h).
// Every call catches C++ exceptions and turns them into a status code plus a thread-local message.
#include <cstring>
#include <string>

#include "context.cuh"
#include "engine.cuh"
#include "potops.cuh"
#include "scanops.cuh"
#include "surrogate.cuh"

using namespace simk;

struct simk_surrogate {
    std::unique_ptr<simk::SurrogateImpl> impl;
};

namespace simk {
void probe_spectrum_noalloc(const simk_grid* grid, const simk_probe* probe, void* out_device, void* stream);
}

namespace {
thread_local std::string g_last_error;

template <typename F>
int guarded(F&& f) {
    try {
        f();
        g_last_error.clear();
        return SIMK_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.status;
    } catch (const std::bad_alloc&) {
        g_last_error = "host memory exhausted";
        return SIMK_ERR_MEMORY;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return SIMK_ERR_CUDA;
    }
}

GridGeom geom_of(const simk_grid* g) {
    SIMK_REQUIRE(g != nullptr, "grid is null");
    SIMK_REQUIRE(g->nx >= 2 && g->ny >= 2, "grid lengths must be at least 2 (Grid.isSupportedLength)");
    SIMK_REQUIRE(std::isfinite(g->extent_x) && std::isfinite(g->extent_y) && g->extent_x > 0 && g->extent_y > 0,
                 "the extent must be finite and positive");
    SIMK_REQUIRE((long long)g->nx * g->ny <= (1LL << 28), "grid too large");
    GridGeom r;
    r.nx = g->nx;
    r.ny = g->ny;
    r.ex = g->extent_x;
    r.ey = g->extent_y;
    return r;
}

void activate(Context& c) { SIMK_CUDA(cudaSetDevice(c.device)); }

std::vector<double> checked_thickness(int32_t n_slices, const double* thickness) {
    SIMK_REQUIRE(n_slices >= 1 && thickness != nullptr, "a potential needs at least one slice");
    std::vector<double> dz(thickness, thickness + n_slices);
    for (double d : dz) SIMK_REQUIRE(std::isfinite(d) && d > 0, "slice thicknesses must be finite and positive");
    return dz;
}
}  // namespace

extern "C" {

int simk_cuda_available(int32_t* device_count) {
    return guarded([&] {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
        int usable = 0;
        for (int d = 0; d < n; ++d) {
            cudaDeviceProp p;
            if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major >= 10) ++usable;
        }
        if (device_count) *device_count = usable;
        if (usable == 0) throw Error(SIMK_ERR_UNAVAILABLE, "no CUDA device of compute capability 10.x or later");
    });
}

const char* simk_last_error(void) { return g_last_error.c_str(); }

int simk_context_create(int32_t device, simk_context** out) {
    return guarded([&] {
        SIMK_REQUIRE(out != nullptr, "out is null");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) throw Error(SIMK_ERR_UNAVAILABLE, "no CUDA device");
        SIMK_REQUIRE(device >= 0 && device < n, "device index out of range");
        cudaDeviceProp p;
        SIMK_CUDA(cudaGetDeviceProperties(&p, device));
        if (p.major < 10) throw Error(SIMK_ERR_UNAVAILABLE, "the library is built for sm_100a (B200)");
        auto* c = new simk_context();
        c->impl.device = device;
        c->impl.sm_count = p.multiProcessorCount;
        try {
            SIMK_CUDA(cudaSetDevice(device));
            SIMK_CUDA(cudaStreamCreateWithFlags(&c->impl.own_stream, cudaStreamNonBlocking));
        } catch (...) {
            delete c;
            throw;
        }
        c->impl.stream = c->impl.own_stream;
        *out = c;
    });
}

int simk_context_destroy(simk_context* ctx) {
    return guarded([&] {
        if (!ctx) return;
        cudaSetDevice(ctx->impl.device);
        cudaStreamSynchronize(ctx->impl.stream);
        cudaStream_t s = ctx->impl.own_stream;
        delete ctx;
        if (s) cudaStreamDestroy(s);
    });
}

int simk_context_set_stream(simk_context* ctx, void* stream) {
    return guarded([&] {
        SIMK_REQUIRE(ctx, "context is null");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        ctx->impl.stream = stream ? static_cast<cudaStream_t>(stream) : ctx->impl.own_stream;
    });
}

int simk_context_set_option(simk_context* ctx, int32_t option, int64_t value) {
    return guarded([&] {
        SIMK_REQUIRE(ctx, "context is null");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        Context& c = ctx->impl;
        switch (option) {
            case SIMK_OPT_FORM:
                SIMK_REQUIRE(value == SIMK_FORM_PLAIN || value == SIMK_FORM_FUSED || value == SIMK_FORM_BF16X3,
                             "unknown form");
                c.form = (int)value;
                break;
            case SIMK_OPT_BATCH: SIMK_REQUIRE(value >= 0, "batch must be >= 0"); c.batch = value; break;
            case SIMK_OPT_BATCH_BYTES: c.batch_bytes = std::max<int64_t>(1, value); break;
            case SIMK_OPT_GRAPHS:
                c.graphs = value ? 1 : 0;
                if (!c.graphs) c.drop_graphs();
                break;
            case SIMK_OPT_TIMING:
                c.timing = value ? 1 : 0;
                if (c.timing) c.times.reserve(16384);
                break;
            case SIMK_OPT_COL_TILE:
                SIMK_REQUIRE(value == 0 || value == 1 || value == 2 || value == 4 || value == 8 || value == 16,
                             "column tile must be 0, 1, 2, 4, 8 or 16");
                c.col_tile = (int)value;
                break;
            case SIMK_OPT_TMA: c.tma = value ? 1 : 0; break;
            case SIMK_OPT_AUTOTUNE: c.autotune = value ? 1 : 0; break;
            case SIMK_OPT_TCGEN05:
                SIMK_REQUIRE(value >= 0 && value <= 2, "tcgen05 option must be 0, 1 or 2");
                c.tcgen05 = (int)value;
                break;
            case SIMK_OPT_EPILOGUE_DETECT: c.epilogue_detect = value ? 1 : 0; break;
            case SIMK_OPT_POISSON_STREAM:
                SIMK_REQUIRE(value == 0 || value == 1, "Poisson stream must be 0 (per value) or 1 (reference order)");
                c.poisson_stream = (int)value;
                break;
            case SIMK_OPT_COMPOSITE: c.composite = value ? 1 : 0; break;
            case SIMK_OPT_PAIRED: c.paired = value ? 1 : 0; break;
            default: throw Error(SIMK_ERR_INVALID, "unknown option");
        }
    });
}

int simk_context_kernel_time(simk_context* ctx, const char* name, double* total_ms, int64_t* launches,
                             double* algorithmic_bytes, int32_t reset) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && name && total_ms && launches && algorithmic_bytes, "null argument");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        SIMK_CUDA(cudaStreamSynchronize(ctx->impl.stream));
        ctx->impl.times.collect();
        auto it = ctx->impl.times.done.find(name);
        if (it == ctx->impl.times.done.end()) {
            *total_ms = 0;
            *launches = 0;
            *algorithmic_bytes = 0;
        } else {
            *total_ms = std::get<0>(it->second);
            *launches = std::get<1>(it->second);
            *algorithmic_bytes = std::get<2>(it->second);
        }
        if (reset) ctx->impl.times.done.clear();
    });
}

int simk_context_get_option(simk_context* ctx, int32_t option, int64_t* value) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && value, "null argument");
        Context& c = ctx->impl;
        switch (option) {
            case SIMK_OPT_FORM: *value = c.form; break;
            case SIMK_OPT_BATCH: *value = c.batch; break;
            case SIMK_OPT_BATCH_BYTES: *value = c.batch_bytes; break;
            case SIMK_OPT_GRAPHS: *value = c.graphs; break;
            case SIMK_OPT_TIMING: *value = c.timing; break;
            case SIMK_OPT_COL_TILE: *value = c.col_tile; break;
            case SIMK_OPT_TMA: *value = c.tma; break;
            case SIMK_OPT_GRAPHS_CACHED: *value = (int64_t)c.slice_graphs.size(); break;
            case SIMK_OPT_AUTOTUNE: *value = c.autotune; break;
            case SIMK_OPT_TCGEN05: *value = c.tcgen05; break;
            case SIMK_OPT_EPILOGUE_DETECT: *value = c.epilogue_detect; break;
            case SIMK_OPT_POISSON_STREAM: *value = c.poisson_stream; break;
            case SIMK_OPT_COMPOSITE: *value = c.composite; break;
            case SIMK_OPT_PAIRED: *value = c.paired; break;
            case SIMK_OPT_TABLE_LAUNCHES: *value = c.table_launches; break;
            case SIMK_OPT_TABLE_KERNELS: *value = c.table_kernels; break;
            case SIMK_OPT_TABLE_SHAPES: *value = c.table_shapes; break;
            case SIMK_OPT_TUNED_COL_TILE: *value = c.last_tuned.col_tile; break;
            case SIMK_OPT_TUNED_TMA: *value = c.last_tuned.tma; break;
            case SIMK_OPT_TUNED_BATCH: *value = c.last_tuned.batch; break;
            case SIMK_OPT_TUNED_ENGINE: *value = c.last_tuned.engine; break;
            default: throw Error(SIMK_ERR_INVALID, "unknown option");
        }
    });
}

int simk_context_synchronize(simk_context* ctx) {
    return guarded([&] {
        SIMK_REQUIRE(ctx, "context is null");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        SIMK_CUDA(cudaStreamSynchronize(ctx->impl.stream));
        check_device_error(ctx->impl);
    });
}

int simk_context_launch_count(simk_context* ctx, int64_t* count, int32_t reset) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && count, "null argument");
        *count = ctx->impl.launches;
        if (reset) ctx->impl.launches = 0;
    });
}

// ---- potentials ------------------------------------------------------------------------------------------------------
int simk_potential_from_atoms(simk_context* ctx, const simk_grid* grid, int32_t n_slices, const double* thickness,
                              int32_t pi_choice, int32_t n_atoms, const int32_t* atomic_numbers, const double* xyz,
                              const int32_t* slice_of_atom, simk_potential** out) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && out, "null argument");
        SIMK_REQUIRE(n_atoms >= 0, "negative atom count");
        SIMK_REQUIRE(n_atoms == 0 || (atomic_numbers && xyz && slice_of_atom), "null atom arrays");
        SIMK_REQUIRE(pi_choice == SIMK_PI_EXACT || pi_choice == SIMK_PI_ABTEM_FLOAT32, "unknown pi choice");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        auto p = std::make_unique<simk_potential>();
        p->impl.ctx = &ctx->impl;
        p->impl.g = geom_of(grid);
        p->impl.dz = checked_thickness(n_slices, thickness);
        build_potential_from_atoms(ctx->impl, p->impl, pi_choice, n_atoms, atomic_numbers, xyz, slice_of_atom);
        *out = p.release();
    });
}

int simk_potential_from_values(simk_context* ctx, const simk_grid* grid, int32_t n_slices, const double* thickness,
                               const double* values, simk_potential** out) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && out && values, "null argument");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        auto p = std::make_unique<simk_potential>();
        p->impl.ctx = &ctx->impl;
        p->impl.g = geom_of(grid);
        p->impl.dz = checked_thickness(n_slices, thickness);
        const size_t bytes = (size_t)n_slices * p->impl.g.count() * sizeof(double);
        p->impl.V.alloc(bytes);
        SIMK_CUDA(cudaMemcpy(p->impl.V.ptr, values, bytes, cudaMemcpyHostToDevice));
        *out = p.release();
    });
}

int simk_potential_destroy(simk_potential* potential) {
    return guarded([&] {
        if (!potential) return;
        if (potential->impl.ctx) cudaSetDevice(potential->impl.ctx->device);
        delete potential;
    });
}

int simk_potential_slice_count(const simk_potential* potential, int32_t* n_slices) {
    return guarded([&] {
        SIMK_REQUIRE(potential && n_slices, "null argument");
        *n_slices = potential->impl.n_slices();
    });
}

int simk_potential_read_slices(simk_context* ctx, simk_potential* potential, double* values) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && potential && values, "null argument");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        SIMK_CUDA(cudaStreamSynchronize(ctx->impl.stream));
        SIMK_CUDA(cudaMemcpy(values, potential->impl.V.ptr,
                             (size_t)potential->impl.n_slices() * potential->impl.g.count() * sizeof(double),
                             cudaMemcpyDeviceToHost));
    });
}

int simk_potential_tile(simk_context* ctx, const simk_potential* potential, int32_t repetitions_x,
                        int32_t repetitions_y, int32_t repetitions_z, simk_potential** out) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && potential && out, "null argument");
        SIMK_REQUIRE(potential->impl.ctx == &ctx->impl, "the potential belongs to another context");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        auto p = std::make_unique<simk_potential>();
        tile_potential(ctx->impl, potential->impl, repetitions_x, repetitions_y, repetitions_z, p->impl);
        SIMK_CUDA(cudaStreamSynchronize(ctx->impl.stream));
        *out = p.release();
    });
}

int simk_potential_project(simk_context* ctx, const simk_potential* potential, double* out) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && potential && out, "null argument");
        SIMK_REQUIRE(potential->impl.ctx == &ctx->impl, "the potential belongs to another context");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        Context& c = ctx->impl;
        const long long N = potential->impl.g.count();
        DeviceBuffer d(N * sizeof(double));
        project_potential(c, potential->impl, d.as<double>());
        SIMK_CUDA(cudaMemcpyAsync(out, d.ptr, N * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        SIMK_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int simk_potential_grid(const simk_potential* potential, simk_grid* grid) {
    return guarded([&] {
        SIMK_REQUIRE(potential && grid, "null argument");
        grid->nx = potential->impl.g.nx;
        grid->ny = potential->impl.g.ny;
        grid->extent_x = potential->impl.g.ex;
        grid->extent_y = potential->impl.g.ey;
    });
}

int simk_potential_read_transmission(simk_context* ctx, simk_potential* potential, double energy, int32_t slice,
                                     double* re, double* im) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && potential && re && im, "null argument");
        SIMK_REQUIRE(std::isfinite(energy) && energy > 0, "the energy must be finite and positive");
        SIMK_REQUIRE(slice >= 0 && slice < potential->impl.n_slices(), "slice out of range");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        prepare_transmissions(ctx->impl, potential->impl, energy);
        const long long N = potential->impl.g.count();
        std::vector<float2> h(N);
        SIMK_CUDA(cudaStreamSynchronize(ctx->impl.stream));  // the copy below is not ordered after that stream
        SIMK_CUDA(cudaMemcpy(h.data(), potential->impl.t.as<float2>() + slice * N, N * sizeof(float2),
                             cudaMemcpyDeviceToHost));
        for (long long i = 0; i < N; ++i) {
            re[i] = h[i].x;
            im[i] = h[i].y;
        }
    });
}

// ---- multislice ------------------------------------------------------------------------------------------------------
int simk_run(simk_context* ctx, simk_potential* potential, double energy, double tilt_x, double tilt_y,
             const double* in_re, const double* in_im, int32_t n_planes, const int32_t* planes, double* out_re,
             double* out_im) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && potential && in_re && in_im && out_re && out_im && planes, "null argument");
        SIMK_REQUIRE(std::isfinite(energy) && energy > 0, "the energy must be finite and positive");
        SIMK_REQUIRE(std::isfinite(tilt_x) && std::isfinite(tilt_y), "the tilt must be finite");
        const int S = potential->impl.n_slices();
        SIMK_REQUIRE(n_planes >= 1, "at least one exit plane");
        std::vector<int> pl(planes, planes + n_planes);
        for (int q = 0; q < n_planes; ++q) {
            SIMK_REQUIRE(pl[q] >= 0 && pl[q] < S, "exit planes must lie within 0 ..< slice count");
            SIMK_REQUIRE(q == 0 || pl[q] > pl[q - 1], "exit planes must be ascending and distinct");
        }
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        run_waves(ctx->impl, potential->impl, energy, tilt_x, tilt_y, 1, in_re, in_im, pl, out_re, out_im);
    });
}

int simk_run_batch(simk_context* ctx, simk_potential* potential, double energy, double tilt_x, double tilt_y,
                   int32_t count, const double* in_re, const double* in_im, double* out_re, double* out_im) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && potential, "null argument");
        SIMK_REQUIRE(count >= 0, "negative count");
        if (count == 0) return;
        SIMK_REQUIRE(in_re && in_im && out_re && out_im, "null argument");
        SIMK_REQUIRE(std::isfinite(energy) && energy > 0, "the energy must be finite and positive");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        std::vector<int> pl{potential->impl.n_slices() - 1};
        run_waves(ctx->impl, potential->impl, energy, tilt_x, tilt_y, count, in_re, in_im, pl, out_re, out_im);
    });
}

// ---- probes ------------------------------------------------------------------------------------------------------------
int simk_probe_spectrum(simk_context* ctx, const simk_grid* grid, const simk_probe* probe, double* re, double* im) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && probe && re && im, "null argument");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        GridGeom g = geom_of(grid);
        DeviceBuffer f32, f64;
        probe_spectrum_device(ctx->impl, g, *probe, f32, &f64);
        std::vector<double2> h(g.count());
        SIMK_CUDA(cudaStreamSynchronize(ctx->impl.stream));  // the copy below is not ordered after that stream
        SIMK_CUDA(cudaMemcpy(h.data(), f64.ptr, g.count() * sizeof(double2), cudaMemcpyDeviceToHost));
        for (long long i = 0; i < g.count(); ++i) {
            re[i] = h[i].x;
            im[i] = h[i].y;
        }
    });
}

int simk_ctf_kernel(simk_context* ctx, const simk_grid* grid, double energy, const simk_ctf* ctf, double* re,
                    double* im) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && ctf && re && im, "null argument");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        GridGeom g = geom_of(grid);
        DeviceBuffer f64;
        ctf_kernel_device(ctx->impl, g, energy, *ctf, f64);
        std::vector<double2> h(g.count());
        SIMK_CUDA(cudaMemcpyAsync(h.data(), f64.ptr, g.count() * sizeof(double2), cudaMemcpyDeviceToHost,
                                  ctx->impl.stream));
        SIMK_CUDA(cudaStreamSynchronize(ctx->impl.stream));
        for (long long i = 0; i < g.count(); ++i) {
            re[i] = h[i].x;
            im[i] = h[i].y;
        }
    });
}

int simk_apply_ctf(simk_context* ctx, const simk_grid* grid, double energy, const simk_ctf* ctf, int32_t count,
                   const double* in_re, const double* in_im, double* out_re, double* out_im, double* out_intensity) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && ctf, "null argument");
        SIMK_REQUIRE(count >= 0, "negative count");
        if (count == 0) return;
        SIMK_REQUIRE(in_re && in_im, "null input");
        SIMK_REQUIRE((out_re == nullptr) == (out_im == nullptr), "give both out_re and out_im, or neither");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        apply_ctf_device(ctx->impl, geom_of(grid), energy, *ctf, count, in_re, in_im, out_re, out_im, out_intensity);
    });
}

// ---- scan post-processing ------------------------------------------------------------------------------------------

int simk_gaussian_source_size_device(simk_context* ctx, int32_t nx, int32_t ny, int64_t value_count, double sigma_x,
                                     double sigma_y, double sampling_x, double sampling_y, const double* in_device,
                                     double* out_device) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && in_device && out_device, "null argument");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        gaussian_source_size_device(ctx->impl, nx, ny, value_count, sigma_x, sigma_y, sampling_x, sampling_y,
                                    in_device, out_device);
    });
}

int simk_gaussian_source_size(simk_context* ctx, int32_t nx, int32_t ny, int64_t value_count, double sigma_x,
                              double sigma_y, double sampling_x, double sampling_y, const double* in, double* out) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && in && out, "null argument");
        SIMK_REQUIRE(nx >= 1 && ny >= 1 && value_count >= 1, "the scan needs at least one position and one value");
        SIMK_REQUIRE(value_count <= (1LL << 40) / ((long long)nx * ny), "the scan holds more than 2^40 values");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        Context& c = ctx->impl;
        const size_t bytes = (size_t)nx * ny * value_count * sizeof(double);
        DeviceBuffer d(bytes);
        SIMK_CUDA(cudaMemcpyAsync(d.ptr, in, bytes, cudaMemcpyHostToDevice, c.stream));
        gaussian_source_size_device(c, nx, ny, value_count, sigma_x, sigma_y, sampling_x, sampling_y, d.as<double>(),
                                    d.as<double>());
        SIMK_CUDA(cudaMemcpyAsync(out, d.ptr, bytes, cudaMemcpyDeviceToHost, c.stream));
        SIMK_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int simk_poisson_noise_device(simk_context* ctx, int64_t count, const double* in_device, double dose, int32_t samples,
                              uint64_t seed, double* out_device) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && (count == 0 || (in_device && out_device)), "null argument");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        poisson_noise_device(ctx->impl, count, in_device, dose, samples, seed, out_device);
    });
}

int simk_poisson_noise(simk_context* ctx, int64_t count, const double* in, double dose, int32_t samples, uint64_t seed,
                       double* out) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && (count == 0 || (in && out)), "null argument");
        SIMK_REQUIRE(count >= 0, "negative value count");
        SIMK_REQUIRE(samples >= 1, "samples must be at least 1, got " + std::to_string(samples));
        SIMK_REQUIRE(count <= (1LL << 40) / samples, "more than 2^40 values and samples");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        Context& c = ctx->impl;
        if (count == 0) {
            poisson_noise_device(c, 0, nullptr, dose, samples, seed, nullptr);  // argument checks only
            return;
        }
        DeviceBuffer din(count * sizeof(double)), dout((size_t)count * samples * sizeof(double));
        SIMK_CUDA(cudaMemcpyAsync(din.ptr, in, count * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        poisson_noise_device(c, count, din.as<double>(), dose, samples, seed, dout.as<double>());
        SIMK_CUDA(cudaMemcpyAsync(out, dout.ptr, (size_t)count * samples * sizeof(double), cudaMemcpyDeviceToHost,
                                  c.stream));
        SIMK_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int simk_integrate_gradient_device(simk_context* ctx, int32_t nx, int32_t ny, double sampling_x, double sampling_y,
                                   const double* gx_device, const double* gy_device, int64_t stride,
                                   double* out_device) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && gx_device && gy_device && out_device, "null argument");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        integrate_gradient_device(ctx->impl, nx, ny, sampling_x, sampling_y, gx_device, gy_device, stride, out_device);
    });
}

int simk_integrate_gradient(simk_context* ctx, int32_t nx, int32_t ny, double sampling_x, double sampling_y,
                            const double* gx, const double* gy, int64_t stride, double* out) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && gx && gy && out, "null argument");
        SIMK_REQUIRE(nx >= 2 && ny >= 2, "the gradient's images need at least 2 points per axis, got " +
                                             std::to_string(nx) + " x " + std::to_string(ny));
        SIMK_REQUIRE(stride >= 1, "the component stride must be at least 1");
        SIMK_REQUIRE((long long)nx * ny <= (1LL << 28), "the gradient's images hold more than 2^28 pixels");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        Context& c = ctx->impl;
        const long long n = (long long)nx * ny;
        std::vector<double> h(2 * n);
        for (long long i = 0; i < n; ++i) {
            h[i] = gx[i * stride];
            h[n + i] = gy[i * stride];
        }
        DeviceBuffer d(2 * n * sizeof(double)), o(n * sizeof(double));
        SIMK_CUDA(cudaMemcpyAsync(d.ptr, h.data(), 2 * n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        integrate_gradient_device(c, nx, ny, sampling_x, sampling_y, d.as<double>(), d.as<double>() + n, 1,
                                  o.as<double>());
        SIMK_CUDA(cudaMemcpyAsync(out, o.ptr, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        SIMK_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int simk_build_probes(simk_context* ctx, const simk_grid* grid, const simk_probe* probe, int32_t count,
                      const double* positions_xy, double* out_re, double* out_im) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && probe, "null argument");
        SIMK_REQUIRE(count >= 0, "negative count");
        if (count == 0) return;
        SIMK_REQUIRE(positions_xy && out_re && out_im, "null argument");
        for (int i = 0; i < 2 * count; ++i)
            SIMK_REQUIRE(std::isfinite(positions_xy[i]), "invalid position " + std::to_string(i / 2));
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        Context& c = ctx->impl;
        GridGeom g = geom_of(grid);
        const long long N = g.count();
        DeviceBuffer spectrum, pos(2 * count * sizeof(double)), rx(count * g.nx * sizeof(float2)),
            ry(count * g.ny * sizeof(float2)), psi(count * N * sizeof(float2));
        probe_spectrum_device(c, g, *probe, spectrum, nullptr);
        SIMK_CUDA(cudaMemcpyAsync(pos.ptr, positions_xy, 2 * count * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        launch_ramps(c, g, pos.as<double>(), 0, count, rx.as<float2>(), ry.as<float2>());
        launch_probes(c, g, spectrum.as<float2>(), rx.as<float2>(), ry.as<float2>(), count, psi.as<float2>(), 1.0f);
        fft2(c.plan(g.ny, 32), c.plan(g.nx, 32), psi.ptr, g.nx, g.ny, count, +1, 1.0 / (double)N, c.stream,
             &c.launches);
        std::vector<float2> h(count * N);
        SIMK_CUDA(cudaMemcpyAsync(h.data(), psi.ptr, count * N * sizeof(float2), cudaMemcpyDeviceToHost, c.stream));
        SIMK_CUDA(cudaStreamSynchronize(c.stream));
        for (long long i = 0; i < count * N; ++i) {
            out_re[i] = h[i].x;
            out_im[i] = h[i].y;
        }
    });
}

// ---- detectors and scans ---------------------------------------------------------------------------------------------
int simk_detector_shape(const simk_grid* grid, double energy, const simk_detector* detector, int32_t* ndim,
                        int32_t* shape) {
    return guarded([&] {
        SIMK_REQUIRE(detector && ndim && shape, "null argument");
        GridGeom g = geom_of(grid);
        int nd = 0, sh[2] = {0, 0};
        detector_shape(g, energy, *detector, &nd, sh);
        *ndim = nd;
        shape[0] = sh[0];
        shape[1] = sh[1];
    });
}

namespace {
std::vector<PotentialImpl*> potentials_of(int32_t n, simk_potential* const* p) {
    SIMK_REQUIRE(n >= 1 && p, "no potential");
    std::vector<PotentialImpl*> v;
    for (int i = 0; i < n; ++i) {
        SIMK_REQUIRE(p[i] != nullptr, "null potential");
        v.push_back(&p[i]->impl);
    }
    return v;
}
}  // namespace

int simk_scan(simk_context* ctx, const simk_probe* probe, int32_t n_potentials, simk_potential* const* potentials,
              int32_t n_positions, const double* positions_xy, int32_t n_detectors, const simk_detector* detectors,
              double* const* outputs) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && probe, "null argument");
        SIMK_REQUIRE(n_positions >= 1 && positions_xy, "no scan position");
        SIMK_REQUIRE(n_detectors >= 0 && n_detectors <= 16 && (n_detectors == 0 || (detectors && outputs)),
                     "0 to 16 detectors");
        for (int i = 0; i < 2 * n_positions; ++i)
            SIMK_REQUIRE(std::isfinite(positions_xy[i]), "invalid position " + std::to_string(i / 2));
        auto pots = potentials_of(n_potentials, potentials);
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        Context& c = ctx->impl;
        const GridGeom& g = pots[0]->g;
        std::vector<long long> counts(n_detectors);
        for (int d = 0; d < n_detectors; ++d) {
            int nd, sh[2] = {1, 1};
            detector_shape(g, probe->energy, detectors[d], &nd, sh);
            counts[d] = nd == 0 ? 1 : nd == 1 ? sh[0] : (long long)sh[0] * sh[1];
        }
        c.positions.ensure(2 * n_positions * sizeof(double));
        SIMK_CUDA(cudaMemcpyAsync(c.positions.ptr, positions_xy, 2 * n_positions * sizeof(double),
                                  cudaMemcpyHostToDevice, c.stream));
        if ((int)c.outputs.size() < n_detectors) c.outputs.resize(n_detectors);
        std::vector<double*> dev_out(n_detectors);
        for (int d = 0; d < n_detectors; ++d) {
            c.outputs[d].ensure(n_positions * counts[d] * sizeof(double));
            dev_out[d] = c.outputs[d].as<double>();
        }
        scan_device(c, *probe, pots, n_positions, c.positions.as<double>(), n_detectors, detectors, dev_out.data());
        for (int d = 0; d < n_detectors; ++d)
            SIMK_CUDA(cudaMemcpyAsync(outputs[d], dev_out[d], n_positions * counts[d] * sizeof(double),
                                      cudaMemcpyDeviceToHost, c.stream));
        SIMK_CUDA(cudaStreamSynchronize(c.stream));
        check_device_error(c);
    });
}

int simk_scan_device(simk_context* ctx, const simk_probe* probe, int32_t n_potentials,
                     simk_potential* const* potentials, int32_t n_positions, const double* positions_xy_device,
                     int32_t n_detectors, const simk_detector* detectors, double* const* outputs_device) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && probe, "null argument");
        SIMK_REQUIRE(n_positions >= 1 && positions_xy_device, "no scan position");
        SIMK_REQUIRE(n_detectors >= 0 && n_detectors <= 16 && (n_detectors == 0 || (detectors && outputs_device)),
                     "0 to 16 detectors");
        auto pots = potentials_of(n_potentials, potentials);
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        scan_device(ctx->impl, *probe, pots, n_positions, positions_xy_device, n_detectors, detectors, outputs_device);
    });
}

int simk_scan_waves(simk_context* ctx, const simk_probe* probe, simk_potential* potential, int32_t n_positions,
                    const double* positions_xy, int32_t rows, int32_t columns, double* out_re, double* out_im) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && probe && potential, "null argument");
        SIMK_REQUIRE(n_positions >= 1 && positions_xy && out_re && out_im, "no scan position or output");
        SIMK_REQUIRE((rows == 0 && columns == 0) || (rows >= 2 && columns >= 2),
                     "the waves detector needs at least 2 points per axis (or 0, 0 for the simulation grid)");
        for (int i = 0; i < 2 * n_positions; ++i)
            SIMK_REQUIRE(std::isfinite(positions_xy[i]), "invalid position " + std::to_string(i / 2));
        SIMK_REQUIRE(potential->impl.ctx == &ctx->impl, "the potential belongs to another context");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        scan_waves(ctx->impl, *probe, potential->impl, n_positions, positions_xy, rows, columns, out_re, out_im);
    });
}

int simk_job_table_run(simk_context* ctx, int32_t n_jobs, const simk_job* jobs, double* done_ms) {
    return guarded([&] {
        SIMK_REQUIRE(ctx, "context is null");
        SIMK_REQUIRE(n_jobs >= 0 && (n_jobs == 0 || jobs), "no job table");
        std::vector<JobSpec> js(n_jobs);
        for (int i = 0; i < n_jobs; ++i) {
            const simk_job& j = jobs[i];
            SIMK_REQUIRE(j.potential, "job " + std::to_string(i) + ": null potential");
            SIMK_REQUIRE(j.incident == SIMK_JOB_PLANE_WAVE || j.incident == SIMK_JOB_PROBE,
                         "job " + std::to_string(i) + ": unknown incident wave");
            SIMK_REQUIRE(j.potential->impl.ctx == &ctx->impl,
                         "job " + std::to_string(i) + ": the potential belongs to another context");
            js[i].pot = &j.potential->impl;
            js[i].energy = j.energy;
            js[i].probe = (j.incident == SIMK_JOB_PROBE);
            js[i].probe_spec = j.probe;
            js[i].x = j.x;
            js[i].y = j.y;
            js[i].intensity = j.intensity;
        }
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        run_job_table(ctx->impl, js, done_ms);
    });
}

int simk_fft2(simk_context* ctx, int32_t nx, int32_t ny, int32_t count, int32_t inverse, int32_t precision,
              const double* in_re, const double* in_im, double* out_re, double* out_im) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && in_re && in_im && out_re && out_im, "null argument");
        SIMK_REQUIRE(nx >= 1 && ny >= 1 && count >= 1, "sizes must be positive");
        SIMK_REQUIRE(precision == 32 || precision == 64, "precision is 32 or 64");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        Context& c = ctx->impl;
        const long long N = (long long)nx * ny, total = N * count;
        const double scale = inverse ? 1.0 / (double)N : 1.0;
        if (precision == 64) {
            std::vector<double2> h(total);
            for (long long i = 0; i < total; ++i) h[i] = make_double2(in_re[i], in_im[i]);
            DeviceBuffer d(total * sizeof(double2));
            SIMK_CUDA(cudaMemcpy(d.ptr, h.data(), total * sizeof(double2), cudaMemcpyHostToDevice));
            fft2(c.plan(ny, 64), c.plan(nx, 64), d.ptr, nx, ny, count, inverse ? +1 : -1, scale, c.stream, &c.launches);
            SIMK_CUDA(cudaStreamSynchronize(c.stream));
            SIMK_CUDA(cudaMemcpy(h.data(), d.ptr, total * sizeof(double2), cudaMemcpyDeviceToHost));
            for (long long i = 0; i < total; ++i) {
                out_re[i] = h[i].x;
                out_im[i] = h[i].y;
            }
        } else {
            std::vector<float2> h(total);
            for (long long i = 0; i < total; ++i) h[i] = make_float2((float)in_re[i], (float)in_im[i]);
            DeviceBuffer d(total * sizeof(float2));
            SIMK_CUDA(cudaMemcpy(d.ptr, h.data(), total * sizeof(float2), cudaMemcpyHostToDevice));
            fft2(c.plan(ny, 32), c.plan(nx, 32), d.ptr, nx, ny, count, inverse ? +1 : -1, scale, c.stream, &c.launches);
            SIMK_CUDA(cudaStreamSynchronize(c.stream));
            SIMK_CUDA(cudaMemcpy(h.data(), d.ptr, total * sizeof(float2), cudaMemcpyDeviceToHost));
            for (long long i = 0; i < total; ++i) {
                out_re[i] = h[i].x;
                out_im[i] = h[i].y;
            }
        }
    });
}

int simk_probe_spectrum_noalloc(const simk_grid* grid, const simk_probe* probe, void* out_device, void* stream) {
    return guarded([&] { probe_spectrum_noalloc(grid, probe, out_device, stream); });
}

// ---- finite projection and the surrogate ------------------------------------------------------------------------------
int simk_finite_profile(simk_context* ctx, int32_t n, const int32_t* atomic_numbers, const double* rho,
                        const double* zl, const double* zu, double* out) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && n >= 0, "bad argument");
        if (n == 0) return;
        SIMK_REQUIRE(atomic_numbers && rho && zl && zu && out, "null argument");
        for (int i = 0; i < n; ++i) {
            SIMK_REQUIRE(atomic_numbers[i] >= 1 && atomic_numbers[i] <= 103, "unsupported element");
            SIMK_REQUIRE(std::isfinite(rho[i]) && rho[i] > 0 && std::isfinite(zl[i]) && std::isfinite(zu[i]),
                         "rho must be positive and the limits finite");
        }
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        std::vector<int> z(atomic_numbers, atomic_numbers + n);
        std::vector<double> r(rho, rho + n), l(zl, zl + n), u(zu, zu + n);
        DeviceBuffer d(n * sizeof(double));
        surrogate_quadrature_points(ctx->impl, z, r, l, u, d.as<double>());
        SIMK_CUDA(cudaStreamSynchronize(ctx->impl.stream));  // the copy below is not ordered after that stream
        SIMK_CUDA(cudaMemcpy(out, d.ptr, n * sizeof(double), cudaMemcpyDeviceToHost));
    });
}

int simk_potential_from_atoms_finite(simk_context* ctx, const simk_grid* grid, int32_t n_slices, const double* thickness,
                                     int32_t n_atoms, const int32_t* atomic_numbers, const double* xyz,
                                     simk_surrogate* surrogate, double error_bound, int32_t* used_surrogate,
                                     double* judged_max_rel, simk_potential** out) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && out && used_surrogate && judged_max_rel, "null argument");
        SIMK_REQUIRE(n_atoms >= 0 && (n_atoms == 0 || (atomic_numbers && xyz)), "null atom arrays");
        SIMK_REQUIRE(std::isfinite(error_bound) && error_bound > 0, "the error bound must be positive");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        auto p = std::make_unique<simk_potential>();
        p->impl.ctx = &ctx->impl;
        p->impl.g = geom_of(grid);
        p->impl.dz = checked_thickness(n_slices, thickness);
        int used = 0;
        double judged = 0.0;
        build_potential_finite(ctx->impl, p->impl, n_atoms, atomic_numbers, xyz,
                               surrogate ? surrogate->impl.get() : nullptr, error_bound, &used, &judged);
        *used_surrogate = used;
        *judged_max_rel = judged;
        *out = p.release();
    });
}

int simk_surrogate_train(simk_context* ctx, int32_t n_elements, const int32_t* atomic_numbers, int64_t n_samples,
                         int32_t steps, int32_t batch, double learning_rate, uint64_t seed, double max_thickness,
                         double rho_min, simk_surrogate** out) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && out && atomic_numbers && n_elements >= 1, "null argument");
        SIMK_REQUIRE(std::isfinite(learning_rate) && learning_rate > 0, "bad learning rate");
        SIMK_REQUIRE(std::isfinite(max_thickness) && max_thickness > 0 && std::isfinite(rho_min) && rho_min > 0,
                     "bad domain");
        SIMK_REQUIRE(n_samples <= (1LL << 27), "at most 2^27 training samples");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        std::vector<int> els(atomic_numbers, atomic_numbers + n_elements);
        auto s = std::make_unique<simk_surrogate>();
        s->impl = surrogate_train(ctx->impl, els, n_samples, steps, batch, learning_rate, seed, max_thickness, rho_min);
        *out = s.release();
    });
}

int simk_surrogate_destroy(simk_surrogate* surrogate) {
    return guarded([&] { delete surrogate; });
}

int simk_surrogate_info(const simk_surrogate* surrogate, double* info) {
    return guarded([&] {
        SIMK_REQUIRE(surrogate && info, "null argument");
        const SurrogateImpl& s = *surrogate->impl;
        info[0] = s.train_loss;
        info[1] = s.val_max_rel;
        info[2] = s.val_rms_rel;
        info[3] = s.y_mean;
        info[4] = s.y_std;
        info[5] = s.steps;
        info[6] = (double)s.samples;
        info[7] = s.max_thickness;
    });
}

int simk_surrogate_evaluate(simk_context* ctx, simk_surrogate* surrogate, int32_t n, const int32_t* atomic_numbers,
                            const double* rho, const double* zl, const double* zu, double* out) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && surrogate && n >= 0, "bad argument");
        if (n == 0) return;
        SIMK_REQUIRE(atomic_numbers && rho && zl && zu && out, "null argument");
        for (int i = 0; i < n; ++i)
            SIMK_REQUIRE(atomic_numbers[i] >= 1 && atomic_numbers[i] <= 103 && rho[i] > 0, "bad query");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        std::vector<int> z(atomic_numbers, atomic_numbers + n);
        std::vector<double> r(rho, rho + n), l(zl, zl + n), u(zu, zu + n);
        surrogate_evaluate(ctx->impl, *surrogate->impl, z, r, l, u, out);
    });
}

int simk_surrogate_parameters(simk_context* ctx, simk_surrogate* surrogate, float* get, const float* set, double* ms) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && surrogate, "null argument");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        SurrogateImpl& s = *surrogate->impl;
        if (get) {
            SIMK_CUDA(cudaMemcpy(get, s.params.ptr, kSurrogateParams * sizeof(float), cudaMemcpyDeviceToHost));
            if (ms) {
                ms[0] = s.y_mean;
                ms[1] = s.y_std;
            }
        }
        if (set) {
            SIMK_CUDA(cudaStreamSynchronize(ctx->impl.stream));  // no launch in flight still reads the old values
            SIMK_CUDA(cudaMemcpy(s.params.ptr, set, kSurrogateParams * sizeof(float), cudaMemcpyHostToDevice));
            if (ms && !get) {
                s.y_mean = ms[0];
                s.y_std = ms[1];
            }
            SIMK_CUDA(cudaStreamSynchronize(ctx->impl.stream));
        }
    });
}

int simk_surrogate_gradients(simk_context* ctx, simk_surrogate* surrogate, int32_t n, const int32_t* atomic_numbers,
                             const double* rho, const double* zl, const double* zu, const double* target,
                             float* gradients, double* loss) {
    return guarded([&] {
        SIMK_REQUIRE(ctx && surrogate && n >= 1 && atomic_numbers && rho && zl && zu && target && gradients && loss,
                     "null argument");
        std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
        activate(ctx->impl);
        std::vector<int> z(atomic_numbers, atomic_numbers + n);
        std::vector<double> r(rho, rho + n), l(zl, zl + n), u(zu, zu + n), t(target, target + n);
        *loss = surrogate_gradients(ctx->impl, *surrogate->impl, z, r, l, u, t, gradients);
    });
}

}  // extern "C"
