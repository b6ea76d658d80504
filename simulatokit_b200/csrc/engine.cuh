// engine.cuh -- entry points of the multislice engine (engine.cu) and of its fused form (fused.cu).
#pragma once

#include <functional>

#include "context.cuh"

namespace simk {

long long batch_size(const Context& ctx, const GridGeom& g, long long count);
void check_device_error(Context& ctx);
void run_waves(Context& ctx, PotentialImpl& pot, double energy, double tx, double ty, int count, const double* in_re,
               const double* in_im, const std::vector<int>& planes, double* out_re, double* out_im);
void scan_device(Context& ctx, const simk_probe& probe, const std::vector<PotentialImpl*>& pots, int n_pos,
                 const double* positions_dev, int n_det, const simk_detector* dets, double* const* outputs_dev);

void propagate_plain(Context& ctx, PotentialImpl& pot, double energy, double tx, double ty, float2* psi, int count,
                     bool last_inverse, const std::function<void(int)>& on_slice);

// One job of a job table: an incident plane wave (probe == false) or probe at (x, y) through `pot` at `energy`;
// `intensity` (host, nx ny float64) receives |exit wave|^2.
struct JobSpec {
    PotentialImpl* pot = nullptr;
    double energy = 0.0;
    bool probe = false;
    simk_probe probe_spec{};
    double x = 0.0, y = 0.0;
    double* intensity = nullptr;
};
// Every job of the table; done_ms[j] = device time from the start of the run to job j's exit intensity.
void run_job_table(Context& ctx, const std::vector<JobSpec>& jobs, double* done_ms);

// The launch configuration for fused scans of pot's grid with the context's form: the cached choice, or one made
// by timing a slice step of pot's first transmission and propagator (SIMK_OPT_AUTOTUNE). The batch is chosen per grid
// (up to 1024 waves within half the free memory), not per call; max_waves is unused.
Context::Tuned autotune(Context& ctx, PotentialImpl& pot, double energy, double tx, double ty, long long max_waves);

// fused form (fused.cu)
bool fused_supported(Context& ctx, const GridGeom& g);
// Every slice on `count` waves in place. probe_rows_pending: the waves come from the probe's column IFFT and still
// need the row IFFT (and 1/N). After slice j the waves are in row-spectrum form (finish_rows completes them);
// kspace_last: the last slice ends in k-space (P Phi) for the detectors. on_slice(j, kspace) after each slice. With
// `det` (and kspace_last) the last column pass sums the channel detectors in its epilogue where a TMA pass runs it:
// returns the column groups of det->partial then, else 0.
int propagate_fused(Context& ctx, PotentialImpl& pot, double energy, double tx, double ty, float2* psi, int count,
                    bool probe_rows_pending, const std::function<void(int, bool)>& on_slice, bool kspace_last,
                    const FusedDetect* det = nullptr);
void finish_rows(Context& ctx, const GridGeom& g, float2* psi, int count);
// The probes of positions [first, first + b) through every slice, left as FFT2(exit wave) in ctx.work_a (unless `det`
// took the channel detectors in the last pass and no pixelated or binned detector wants the waves; the return value is
// propagate_fused's).
int exit_spectra_fused(Context& ctx, PotentialImpl& pot, const simk_probe& probe, const float2* spectrum,
                       const double* positions_dev, long long first, int b, const FusedDetect* det = nullptr);
// STEM.scan with a WavesDetector: the exit wave at every position (host positions), resampled in Fourier space to
// rows x columns points (0, 0: the simulation grid), into host float64 arrays [position][row][column].
void scan_waves(Context& ctx, const simk_probe& probe, PotentialImpl& pot, int n_pos, const double* positions_xy,
                int rows, int columns, double* out_re, double* out_im);
void scan_fused_batch(Context& ctx, PotentialImpl& pot, const simk_probe& probe, const float2* spectrum,
                      const double* positions_dev, long long first, int b, DetectorPlan& dplan,
                      double* const* outputs_dev, double weight);

}  // namespace simk
