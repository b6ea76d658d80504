// context.cuh -- the library's context (stream, options, plan and table caches) and its potential handle.
#pragma once

#include <map>
#include <set>
#include <string>

#include "common.cuh"
#include "fft.cuh"

struct simk_context;
struct simk_potential;

namespace simk {

// Device view of a grid for kernels.
struct GridDev {
    int nx, ny;
    double dx, dy;
};
inline GridDev grid_dev(const GridGeom& g) { return GridDev{g.nx, g.ny, g.dx(), g.dy()}; }

// One reduction channel set of a detector (annular: 1, COM: 2, segmented: nr * nphi): the pixels of every channel as a
// CSR list (pixel index, weight), channels of all detectors concatenated.
struct DetectorPlan {
    int n_channels = 0;
    std::vector<int> det_first_channel;    // per detector: its first reduction channel (-1: pixelated)
    std::vector<int> det_count;            // per detector: values per position
    std::vector<int> det_pixelated_offset; // per detector: offset of its crop map (pixelated), -1 otherwise
    DeviceBuffer chan_ptr;   // int32 [n_channels + 1]
    DeviceBuffer chan_pix;   // int32 [total]
    DeviceBuffer chan_w;     // float [total]
    DeviceBuffer crop_src;   // int32, concatenated crop maps of the pixelated detectors
    long long total_entries = 0;
    long long total_crop = 0;
    std::vector<int> host_chan_ptr;
    // binned detectors: per axis, each bin's (pixel, overlap weight) list in CSR form
    struct Binned {
        int det = 0, nbx = 0, nby = 0;
        DeviceBuffer xp, xi, xw, yp, yi, yw;  // int32 ptr [nb + 1], int32 pixel, float64 weight
    };
    std::vector<std::unique_ptr<Binned>> binned;
    // Pixelated or binned detectors are present: they read the k-space waves the last column pass stores.
    bool has_pixel_outputs = false;
    int grid_ny = 0;
    std::vector<int> host_chan_pix;
    std::vector<float> host_chan_w;
    // The channel lists regrouped for detection inside the fused form's last column pass, for column tiles of `tc`
    // columns: the entries of column group g (columns g tc .. g tc + tc - 1) and channel ch, in increasing local index
    // ix tc + (iy - g tc), at ent[ptr[g C + ch] .. ptr[g C + ch + 1]) as (local index, float bits of the weight).
    struct TileChannels {
        int tc = 0, groups = 0;
        DeviceBuffer ptr;  // int32 [groups C + 1]
        DeviceBuffer ent;  // int2 [total]
    };
    std::vector<std::unique_ptr<TileChannels>> tile_channels;
    // Built on first use per tile width (allocates and copies: not inside a stream capture).
    const TileChannels& tiles(int tc);
};

// Detection inside the fused form's last column pass (MODE 3): the plan, the per-(wave, column group, channel)
// float64 partial sums it writes, and whether the pass must also store the k-space waves (pixelated / binned).
struct FusedDetect {
    DetectorPlan* plan = nullptr;
    double* partial = nullptr;
    int store = 0;
};

struct Propagator {
    DeviceBuffer p;  // float2 [N]: exp(-i pi lambda dz k^2) A (x tilt phase)
};

struct Context;

struct PotentialImpl {
    Context* ctx = nullptr;
    GridGeom g;
    std::vector<double> dz;
    DeviceBuffer V;          // double [S][N], as built
    double t_energy = -1.0;  // energy the transmissions below were built for
    DeviceBuffer t;          // float2 [S][N]
    int n_slices() const { return (int)dz.size(); }
};

// Per-kernel CUDA-event timing (SIMK_OPT_TIMING): events recorded around each launch of a named kernel, with the
// launch's algorithmic bytes, summed when queried.
struct KernelTimes {
    struct Rec {
        cudaEvent_t a, b;
        double bytes;
    };
    std::map<std::string, std::vector<Rec>> pending;
    std::map<std::string, std::tuple<double, long long, double>> done;  // ms, launches, bytes
    std::vector<cudaEvent_t> pool;
    // Creates `n` events up front so that recording them in the hot loop costs no cudaEventCreate.
    void reserve(size_t n) {
        while (pool.size() < n) {
            cudaEvent_t e;
            SIMK_CUDA(cudaEventCreate(&e));
            pool.push_back(e);
        }
    }
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        SIMK_CUDA(cudaEventCreate(&e));
        return e;
    }
    void collect() {
        for (auto& kv : pending) {
            auto& d = done[kv.first];
            for (auto& r : kv.second) {
                float ms = 0;
                SIMK_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
                std::get<0>(d) += ms;
                std::get<1>(d) += 1;
                std::get<2>(d) += r.bytes;
                pool.push_back(r.a);
                pool.push_back(r.b);
            }
        }
        pending.clear();
    }
    ~KernelTimes() {
        for (auto& kv : pending)
            for (auto& r : kv.second) {
                cudaEventDestroy(r.a);
                cudaEventDestroy(r.b);
            }
        for (auto e : pool) cudaEventDestroy(e);
    }
};

struct Context {
    int device = 0;
    int timing = 0;
    KernelTimes times;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    std::recursive_mutex mu;
    int form = SIMK_FORM_FUSED;
    long long batch = 0;
    long long batch_bytes = 1LL << 30;
    int graphs = 1;
    int col_tile = 0;
    int tma = 1;            // TMA-pipelined persistent column pass where available
    int tcgen05 = 2;        // the bf16x3 form's DFT stages on tcgen05 where its tiles fit (else mma.sync): 2 stacked
    int epilogue_detect = 1;  // channel detectors summed in the last column pass (TMA passes)
    int poisson_stream = 0;   // Poisson noise: 0 = a generator per value and sample, 1 = the reference's one stream
    int composite = 1;        // fused passes at 3 or 5 times a power of two: the composite register engine
    int paired = 1;           // fused column passes at 256 and 512 on column pairs (engine 5)
    // the last fused job table: host launch calls for its slice steps (1 when captured as one graph), the kernels in
    // them, and the grid shapes they covered
    long long table_launches = 0, table_kernels = 0;
    int table_shapes = 0;
    // the last fused job table captured as a graph (its buffers, graph and events), kept for a repeat of the same jobs
    std::shared_ptr<void> table_cache;
    std::string table_cache_key;
    int autotune = 0;       // time the launch configurations on first use of a (grid, form)
    struct Tuned {
        int col_tile = -1, tma = -1;
        long long batch = -1;
        // the line-FFT engine (radix plan) where there is a choice: the composite option at lengths 3 or 5 times a
        // power of two (fused form), the tcgen05 option at 256 and 512 (bf16x3 form); -1 where there is none
        int engine = -1;
    };
    std::map<std::string, Tuned> tuned;
    Tuned last_tuned;
    int sm_count = 0;
    int64_t launches = 0;
    DeviceBuffer err_flag;  // int: set by a kernel whose bounded wait ran out
    // Set by a job-table run for the duration of one slice step: wave b of the fused passes multiplies by the
    // transmission slice wave_t[b] and by the propagator wave_p[b] among wave_p_blocks stacked ones (device arrays).
    const float2* const* wave_t = nullptr;
    const int* wave_p = nullptr;
    int wave_p_blocks = 0;
    std::map<std::pair<int, int>, std::unique_ptr<LinePlan>> plans;
    std::map<std::tuple<int, int, double, double, double, double, double, double>, std::unique_ptr<Propagator>> props;
    // workspaces
    DeviceBuffer work_a, work_b, work_c, rx, ry, positions, partial;
    // float64 channel partial sums of the detection fused into the last column pass: [wave][column group][channel]
    DeviceBuffer det_partial;
    // scan post-processing: the Gaussian passes' intermediate, their weights, the Poisson sampler's status word, the
    // gradient integration's two spectra and its minimum
    DeviceBuffer post_work, post_weights, post_flag, post_spectra, post_min;
    // the potential builder's scratch, kept across builds (grown on demand): the atoms' merged pixels and weights, the
    // elements' Lobato kernels and parameters, the present-element lists, the group's spectra and the delta images
    // (which the transmissions reuse as their float64 fields)
    DeviceBuffer pot_pix, pot_w, pot_kern, pot_ab, pot_elem, pot_spec, pot_delta;
    std::vector<DeviceBuffer> outputs;
    // per-scan set-up kept across calls: detector maps by (grid, energy, detectors), spectra by (grid, probe)
    std::map<std::string, std::unique_ptr<DetectorPlan>> detector_plans;
    std::map<std::string, std::unique_ptr<DeviceBuffer>> spectra;
    // The fused form's slice loop of a batch, captured as a CUDA graph on its second use (the first runs eagerly and
    // creates what the launches need), keyed by every pointer and setting the recorded launches read.
    struct SliceGraph {
        cudaGraphExec_t exec = nullptr;
        int64_t launches = 0;
        int det_groups = 0;  // column groups of the detection fused into the last pass (0: none)
    };
    std::map<std::string, SliceGraph> slice_graphs;
    std::set<std::string> slice_seen;
    void drop_graphs() {
        for (auto& kv : slice_graphs)
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        slice_graphs.clear();
        slice_seen.clear();
        table_cache.reset();
        table_cache_key.clear();
    }
    ~Context() { drop_graphs(); }

    const LinePlan& plan(int n, int precision) {
        auto key = std::make_pair(n, precision);
        auto it = plans.find(key);
        if (it != plans.end()) return *it->second;
        auto p = make_line_plan(n, precision);
        auto& ref = *p;
        plans[key] = std::move(p);
        return ref;
    }
    const Propagator& propagator(const GridGeom& g, double energy, double dz, double tx, double ty);
};

// Records events around one launch of kernel `name` when the context's timing is on.
struct KernelTimer {
    Context& c;
    const char* name;
    double bytes;
    cudaEvent_t a = nullptr;
    KernelTimer(Context& ctx, const char* n, double algorithmic_bytes) : c(ctx), name(n), bytes(algorithmic_bytes) {
        if (c.timing) {
            a = c.times.get();
            SIMK_CUDA(cudaEventRecord(a, c.stream));
        }
    }
    ~KernelTimer() {
        if (a) {
            cudaEvent_t b = c.times.get();
            cudaEventRecord(b, c.stream);
            c.times.pending[name].push_back({a, b, bytes});
        }
    }
};

// kernels and helpers of physics.cu
void build_potential_from_atoms(Context& ctx, PotentialImpl& pot, int pi_choice, int n_atoms, const int* Z,
                                const double* xyz, const int* slice_of_atom);
void prepare_transmissions(Context& ctx, PotentialImpl& pot, double energy);
void ctf_kernel_device(Context& ctx, const GridGeom& g, double energy, const simk_ctf& ctf, DeviceBuffer& out_f64);
void apply_ctf_device(Context& ctx, const GridGeom& g, double energy, const simk_ctf& ctf, int count,
                      const double* in_re, const double* in_im, double* out_re, double* out_im, double* out_intensity);
void probe_spectrum_device(Context& ctx, const GridGeom& g, const simk_probe& probe, DeviceBuffer& out_f32,
                           DeviceBuffer* out_f64);
// The same spectrum into buffers the caller keeps (grown when too small), with no allocation when they are large
// enough and no synchronisation: for many probes in a row on one stream.
void probe_spectrum_into(Context& ctx, const GridGeom& g, const simk_probe& probe, DeviceBuffer& out_f32,
                         DeviceBuffer& tmp, DeviceBuffer& norm);
void launch_ramps(Context& ctx, const GridGeom& g, const double* positions_dev, long long first, int count,
                  float2* rx, float2* ry);
void launch_probes(Context& ctx, const GridGeom& g, const float2* spectrum, const float2* rx, const float2* ry,
                   int count, float2* out, float scale);
void launch_mul_broadcast(Context& ctx, float2* psi, const float2* factor, long long n, int count, float scale);
std::unique_ptr<DetectorPlan> build_detector_plan(Context& ctx, const GridGeom& g, double energy,
                                                  const simk_detector* dets, int n_dets);
void detector_shape(const GridGeom& g, double energy, const simk_detector& d, int* ndim, int* shape);
// Every detector of the plan on the k-space waves phi; with channels = false only the pixelated and binned ones (the
// channel detectors were summed inside the last column pass).
void launch_detect(Context& ctx, const DetectorPlan& plan, const GridGeom& g, const float2* phi, int count,
                   long long first_position, double* const* outputs_dev, double weight, float intensity_scale,
                   bool channels = true);
// The channel detectors from the fused pass's partial sums: per (wave, channel) the sum over the `groups` column
// groups in order, times weight, added to the detector's output.
void launch_detect_fold(Context& ctx, const DetectorPlan& plan, const double* partial, int groups, int count,
                        long long first_position, double* const* outputs_dev, double weight);

}  // namespace simk

struct simk_context {
    simk::Context impl;
};
struct simk_potential {
    simk::PotentialImpl impl;
};
