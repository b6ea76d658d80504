/*
 * simulato_cuda.h -- the C ABI of libsimulato_cuda.so, the `.cuda` backend of SimulatoKit's multislice hot path.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and returns an `int` status (SIMK_OK = 0);
 * `simk_last_error()` gives the message of the calling thread's last failure. Host buffers are owned by the caller and
 * are not retained. Device memory is owned by the context and by the potential handles. One context serialises its
 * calls with a mutex (the analogue of MetalEngine's `runLock`, Sources/SimulatoMultislice/MetalEngine.swift:51).
 *
 * Complex arrays cross the boundary as split float64 real / imaginary arrays, row-major [ix * ny + iy], the layout of
 * SimulatoKit's `ComplexField` (Sources/SimulatoCore/Fields.swift:8-49), so a Swift caller passes `field.real` and
 * `field.imaginary` directly. Inside, waves are interleaved complex64 [batch][ix][iy] in HBM.
 *
 * Each function names the reference interface it replaces.
 */
#ifndef SIMULATO_CUDA_H
#define SIMULATO_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (mapped by the Swift side onto SimulatoError, Sources/SimulatoCore/SimulatoError.swift:7-57) ---- */
#define SIMK_OK 0
#define SIMK_ERR_INVALID 1       /* a refused argument: SimulatoError.invalid* / unsupported* */
#define SIMK_ERR_CUDA 2          /* a CUDA failure: the .metalFailure(String) analogue */
#define SIMK_ERR_UNAVAILABLE 3   /* no usable sm_100 device: the .metalUnavailable analogue */
#define SIMK_ERR_MEMORY 4        /* device memory refused */
#define SIMK_ERR_TIMEOUT 5       /* a bounded device wait ran out */

/* ---- execution forms (the metric's A/B pair) ---- */
#define SIMK_FORM_PLAIN 0   /* one operation per launch, FP32 Stockham FFT in shared memory */
#define SIMK_FORM_FUSED 1   /* batched: transmission/propagator fused into register-resident FFT passes, FP32 */
#define SIMK_FORM_BF16X3 2  /* FUSED with radix-16 DFT stages on tensor cores: split BF16 (data hi+lo, DFT matrix
                               hi+lo+lo2), FP32 accumulate; grid sides 256, 512, 768, 1024, 2048 */

/* ---- context options (the ExecutionOptions analogue, Sources/SimulatoMultislice/ExecutionOptions.swift:21-49) ---- */
#define SIMK_OPT_FORM 0         /* one of SIMK_FORM_* (default SIMK_FORM_FUSED) */
#define SIMK_OPT_BATCH 1        /* waves per batch, 0 = from SIMK_OPT_BATCH_BYTES (default 0) */
#define SIMK_OPT_BATCH_BYTES 2  /* device bytes of waves one batch may hold (default 1 GiB) */
#define SIMK_OPT_GRAPHS 3       /* capture the slice loop of a batch in a CUDA graph (default 1) */
#define SIMK_OPT_TIMING 4       /* record CUDA events around every hot-path launch (default 0) */
#define SIMK_OPT_COL_TILE 5     /* columns per CTA in the fused column pass, 0 = automatic (default 0) */
#define SIMK_OPT_TMA 6          /* TMA-pipelined persistent column pass where the grid allows it (default 1) */
#define SIMK_OPT_GRAPHS_CACHED 7 /* read-only: slice loops held as instantiated CUDA graphs */
/* On the first fused scan of a grid shape and form, time one slice step of the actual transmission and propagator
 * for each column tile (2, 4, 8, and 16 at 256 x 256 with SIMK_OPT_PAIRED), with and without the TMA passes, then for
 * batch sizes up to what half of the free device memory holds, and use the fastest wherever SIMK_OPT_COL_TILE /
 * SIMK_OPT_BATCH are 0 (automatic) and TMA is allowed. The choice is kept per (grid, form) in the context. Default 0 (off). */
#define SIMK_OPT_AUTOTUNE 8
#define SIMK_OPT_TUNED_COL_TILE 9 /* read-only: the last tuning's choice (-1 before any) */
#define SIMK_OPT_TUNED_TMA 10
#define SIMK_OPT_TUNED_BATCH 11
/* read-only: the last tuning's line-FFT engine where the grid offers a choice (-1: none): the SIMK_OPT_COMPOSITE value
 * (fused form at lengths 3 or 5 times a power of two) or the SIMK_OPT_TCGEN05 value (bf16x3 form at 256 and 512); the
 * tuned scan runs with it */
#define SIMK_OPT_TUNED_ENGINE 19
/* The bf16x3 form's radix-16 DFT stages on the fifth-generation tensor cores (tcgen05.mma, accumulators in tensor
 * memory) for grid sides 256 and 512, with the data split in three BF16 terms: 2 (default) = six products of N = 96,
 * 64 and 32 per block of 128 vectors (the B terms stacked) into three accumulator blocks, hi x hi alone in one, which
 * the threads add; 1 = the same terms as twelve products of N = 32 into one accumulator; 0 = the warp-level mma.sync
 * stages (data in two terms) everywhere. */
#define SIMK_OPT_TCGEN05 12
/* Sum the annular, centre-of-mass and segmented detectors inside the fused form's last column pass (TMA passes), so
 * the k-space waves are neither written nor read back unless a pixelated or binned detector wants them; 0 = detect
 * from the stored waves with separate kernels. Default 1. */
#define SIMK_OPT_EPILOGUE_DETECT 13
/* The generator of simk_poisson_noise[_device]: 0 (default) = a generator of its own for every value and sample (the
 * work splits over the GPU; a seed gives the same noise on every run, not the reference's draws); 1 = the reference's
 * single GaussianGenerator stream over the samples and values in order (ScanOperations.swift:80-117), walked by one
 * device thread, so a seed gives the reference's draws. */
#define SIMK_OPT_POISSON_STREAM 14
/* The fused form's passes at lengths 3 or 5 times a power of two (384, 640, 768, 1536): 1 (default) = the composite
 * register engine (each line as 3 or 5 register-resident power-of-two transforms of its decimated sub-lines); 0 = the
 * shared-memory Stockham engine. */
#define SIMK_OPT_COMPOSITE 15
/* The fused form's column passes at grid sides 256, 512 and 1024: 1 (default) = tiles of 16 (256) or 8 columns, one
 * thread transforming the same rows of two adjacent columns, so that every global row segment is 128 or 64 bytes wide
 * (the pass then moves its bytes at close to the device's copy rate), where SIMK_OPT_COL_TILE is 0 or that width;
 * 0 = one column a thread, SIMK_OPT_COL_TILE (default 4) columns a tile. */
#define SIMK_OPT_PAIRED 20
/* read-only, the last fused simk_job_table_run: host launch calls that ran its slice steps (1: one CUDA graph launch,
 * with SIMK_OPT_GRAPHS on and SIMK_OPT_TIMING off), the kernels inside them, and the grid shapes they covered */
#define SIMK_OPT_TABLE_LAUNCHES 16
#define SIMK_OPT_TABLE_KERNELS 17
#define SIMK_OPT_TABLE_SHAPES 18

/* ---- Lobato pi choice (LobatoParameterization.PiConstant, LobatoParameterization.swift:15-24) ---- */
#define SIMK_PI_EXACT 0
#define SIMK_PI_ABTEM_FLOAT32 1

/* ---- detector kinds (Sources/SimulatoDetector/Detectors.swift:91-263) ---- */
#define SIMK_DET_ANNULAR 0
#define SIMK_DET_PIXELATED 1
#define SIMK_DET_COM 2
#define SIMK_DET_SEGMENTED 3
/* No reference counterpart (its PixelatedDetector offers cutoff / valid / full only, Detectors.swift:140-168): the
 * pattern on a uniform nr x nphi grid of angles over [-outer, outer) mrad in x and y (bin 0 at -outer). Each k-space
 * pixel is a square of one angular sample centred on its angle; its intensity goes to the bins it overlaps in
 * proportion to the overlap area, so the total inside the window is conserved. outer must not exceed the largest
 * simulated angle along either axis. */
#define SIMK_DET_BINNED 4
#define SIMK_MAXANGLE_CUTOFF 0   /* PixelatedDetector.MaxAngle */
#define SIMK_MAXANGLE_VALID 1
#define SIMK_MAXANGLE_FULL 2
#define SIMK_UNITS_MRAD 0        /* CenterOfMassDetector.Units */
#define SIMK_UNITS_INV_ANGSTROM 1

typedef struct simk_context simk_context;
typedef struct simk_potential simk_potential;
typedef struct simk_surrogate simk_surrogate;

/* Parameters of the finite-projection surrogate network (float32): emb[103][16] | W1[64][18] b1[64] |
 * W2[64][64] b2[64] | W3[64][64] b3[64] | W4[64] b4[1]. The network is a cumulative profile C(Z, rho, z); a slab's
 * profile is P_inf(rho) (C(Z, rho, zu) - C(Z, rho, zl)). */
#define SIMK_SURROGATE_PARAMS 11249

/* Grid (Sources/SimulatoCore/Grid.swift:8-91): nx x ny points over extent_x x extent_y [A]. */
typedef struct {
    int32_t nx, ny;
    double extent_x, extent_y;
} simk_grid;

/* Probe (Sources/SimulatoProbe/Probe.swift:51-70) with its Aberrations (Aberrations.swift:8-15), in the order
 * C10 C12 phi12 C21 phi21 C23 phi23 C30 C32 phi32 C34 phi34 C41 phi41 C43 phi43 C45 phi45 C50 C52 phi52 C54 phi54
 * C56 phi56 [A, rad]. semiangle_mrad = INFINITY for no aperture. */
typedef struct {
    double energy;
    double semiangle_mrad;
    int32_t soft;
    int32_t reserved;
    double aberrations[25];
    double tilt_x, tilt_y;  /* [mrad] */
} simk_probe;

/* One detector (Detectors.swift:91-263). annular: inner, outer (has_outer = 0: the default outer angle);
 * pixelated: max_angle; com: max_angle, units; segmented: nr, nphi, inner, outer, rotation [rad]; binned: nr x nphi
 * bins (x, y), outer = the window's half-width [mrad]. */
typedef struct {
    int32_t kind;
    int32_t max_angle;
    int32_t units;
    int32_t has_outer;
    int32_t nr, nphi;
    double inner, outer, rotation;
} simk_detector;

/* ---- availability, context (Multislice.metalIsAvailable, MetalMultislice.swift:20; MetalEngine.require :72-77) --- */
int simk_cuda_available(int32_t* device_count);
const char* simk_last_error(void);
int simk_context_create(int32_t device, simk_context** out);
int simk_context_destroy(simk_context* ctx);
/* Runs every later call of this context on `stream` (a cudaStream_t; NULL = the context's own stream). */
int simk_context_set_stream(simk_context* ctx, void* stream);
int simk_context_set_option(simk_context* ctx, int32_t option, int64_t value);
int simk_context_get_option(simk_context* ctx, int32_t option, int64_t* value);
int simk_context_synchronize(simk_context* ctx);
/* Kernels this context launched since the last reset (the bench's launch count). */
int simk_context_launch_count(simk_context* ctx, int64_t* count, int32_t reset);
/* With SIMK_OPT_TIMING on: the summed CUDA-event time [ms], launch count and algorithmic bytes of the hot-path kernel
 * `name` ("line_fft", "pointwise", "detect", "fused_rows", "fused_cols") since the last reset. Synchronises. */
int simk_context_kernel_time(simk_context* ctx, const char* name, double* total_ms, int64_t* launches,
                             double* algorithmic_bytes, int32_t reset);

/* ---- potentials ---------------------------------------------------------------------------------------------------
 * From atoms: replaces MetalMultislice.prepare(Potential) (MetalEngine.swift:277-308) and Potential.build
 * (Potential.swift:83-91, ProjectedPotential.swift:109-202). `xyz` are the wrapped positions (n_atoms x 3) and
 * `slice_of_atom` the slice of each (Potential.init, Potential.swift:49-63); V is built on the device in float64
 * (bilinear deltas, FFT, x f(k^2)/S(k), IFFT, summed over elements in increasing Z). */
int simk_potential_from_atoms(simk_context* ctx, const simk_grid* grid, int32_t n_slices, const double* thickness,
                              int32_t pi_choice, int32_t n_atoms, const int32_t* atomic_numbers, const double* xyz,
                              const int32_t* slice_of_atom, simk_potential** out);
/* From values: replaces MetalMultislice.prepare(ProjectedPotential) (MetalEngine.swift:310-321); values are
 * n_slices x nx x ny float64 V [V A]. */
int simk_potential_from_values(simk_context* ctx, const simk_grid* grid, int32_t n_slices, const double* thickness,
                               const double* values, simk_potential** out);
int simk_potential_destroy(simk_potential* potential);
int simk_potential_slice_count(const simk_potential* potential, int32_t* n_slices);
/* V of every slice as the device built it (n_slices x nx x ny): the gpuPotentialSlices test hook
 * (MetalMultislice.swift:107-110). */
int simk_potential_read_slices(simk_context* ctx, simk_potential* potential, double* values);
/* The bandlimited transmission t of one slice for a beam energy (Multislice.transmissionFunctions,
 * Multislice.swift:83-103), as stored on the device (complex64 widened). */
int simk_potential_read_transmission(simk_context* ctx, simk_potential* potential, double energy, int32_t slice,
                                     double* re, double* im);
/* ProjectedPotential.tiled(repetitionsX:repetitionsY:repetitionsZ:) (Sources/SimulatoMultislice/ProjectedPotential.swift:
 * 76-105), on the device: `*out` is a new potential whose slices are `potential`'s tiled repetitions_x x repetitions_y
 * times in the plane (extent multiplied, sampling kept), the whole stack repeated repetitions_z times. A periodic
 * crystal built as one cell and tiled equals the crystal built atom by atom. Counts below 1, a tiled slice of more
 * than 2^28 values, more than 1,000,000 slices or more than 2^31 values in all: SIMK_ERR_INVALID, before anything is
 * allocated. Destroy the result with simk_potential_destroy. */
int simk_potential_tile(simk_context* ctx, const simk_potential* potential, int32_t repetitions_x,
                        int32_t repetitions_y, int32_t repetitions_z, simk_potential** out);
/* ProjectedPotential.project() (ProjectedPotential.swift:64-73): the sum of the slices [V A], added in slice order in
 * float64, into host out[nx ny]. */
int simk_potential_project(simk_context* ctx, const simk_potential* potential, double* out);
/* The grid a potential lives on (a tiled potential's is its source's times the repetitions). */
int simk_potential_grid(const simk_potential* potential, simk_grid* grid);

/* ---- finite projection and its learned surrogate -------------------------------------------------------------------
 * No reference implementation: SimulatoKit lists Potential(projection="finite") as not ported (docs/parity.md:58,251).
 * P(rho; zl, zu) = int_zl^zu V(sqrt(rho^2 + z^2)) dz of the Lobato potential V(r) = sum A_i (2/(B_i r) + 1) e^{-B_i r}
 * (A, B of LobatoParameterization.swift:38-44), by float64 Gauss-Legendre quadrature on the device, at n points. */
int simk_finite_profile(simk_context* ctx, int32_t n, const int32_t* atomic_numbers, const double* rho,
                        const double* zl, const double* zu, double* out);
/* V of every slice by finite projection (each atom reaches R_c(Z) in the plane and along the beam; xyz wrapped in
 * x, y). With `surrogate` (may be NULL) the profiles of the pairs inside its trained domain come from the network,
 * judged on a sample by the quadrature: above `error_bound` (max relative) the quadrature replaces it.
 * *used_surrogate and *judged_max_rel report what happened. */
int simk_potential_from_atoms_finite(simk_context* ctx, const simk_grid* grid, int32_t n_slices, const double* thickness,
                                     int32_t n_atoms, const int32_t* atomic_numbers, const double* xyz,
                                     simk_surrogate* surrogate, double error_bound, int32_t* used_surrogate,
                                     double* judged_max_rel, simk_potential** out);
/* Trains the surrogate on the device: n_samples quadrature-labelled samples of the elements, `steps` Adam steps of
 * `batch` samples, slabs up to max_thickness A, radii from rho_min A. */
int simk_surrogate_train(simk_context* ctx, int32_t n_elements, const int32_t* atomic_numbers, int64_t n_samples,
                         int32_t steps, int32_t batch, double learning_rate, uint64_t seed, double max_thickness,
                         double rho_min, simk_surrogate** out);
int simk_surrogate_destroy(simk_surrogate* surrogate);
/* info[8] = train loss, held-out max and rms error of P in units of P_inf(rho) (|dF|), 0, 1, steps, samples, max
 * thickness. */
int simk_surrogate_info(const simk_surrogate* surrogate, double* info);
int simk_surrogate_evaluate(simk_context* ctx, simk_surrogate* surrogate, int32_t n, const int32_t* atomic_numbers,
                            const double* rho, const double* zl, const double* zu, double* out);
/* Reads (get != NULL) and/or replaces (set != NULL) the SIMK_SURROGATE_PARAMS float32 parameters; the target
 * standardisation (mean, spread) is read into / set from ms[2] when ms != NULL. */
int simk_surrogate_parameters(simk_context* ctx, simk_surrogate* surrogate, float* get, const float* set, double* ms);
/* One forward + backward pass on the given batch against targets F = P / P_inf(rho): the loss and the gradient of every
 * parameter (the training kernels, exposed for gradient checks). */
int simk_surrogate_gradients(simk_context* ctx, simk_surrogate* surrogate, int32_t n, const int32_t* atomic_numbers,
                             const double* rho, const double* zl, const double* zu, const double* target,
                             float* gradients, double* loss);

/* ---- multislice -----------------------------------------------------------------------------------------------------
 * Multislice.run (Multislice.swift:52-80 -> MetalMultislice.run, MetalEngine.swift:458-474): one incident wave through
 * the potential; returns the waves after the slices in `planes` (ascending, >= 0; the caller adds the incident for -1),
 * n_planes x nx x ny. `normalization_values` = 1 for a plane-wave-normalised wave (ignored here; kept for symmetry). */
int simk_run(simk_context* ctx, simk_potential* potential, double energy, double tilt_x, double tilt_y,
             const double* in_re, const double* in_im, int32_t n_planes, const int32_t* planes,
             double* out_re, double* out_im);
/* Multislice.runBatch (MetalMultislice.swift:52-83 -> MetalEngine.swift:476-501): `count` incident waves, the exit
 * wave of each after the last slice. */
int simk_run_batch(simk_context* ctx, simk_potential* potential, double energy, double tilt_x, double tilt_y,
                   int32_t count, const double* in_re, const double* in_im, double* out_re, double* out_im);

/* ---- probes -------------------------------------------------------------------------------------------------------
 * Probe.centredSpectrum (Probe.swift:113-136) computed on the device in float64. */
int simk_probe_spectrum(simk_context* ctx, const simk_grid* grid, const simk_probe* probe, double* re, double* im);
/* The probes IFFT(Psi0 . r_x (x) r_y) at `count` positions (x, y) [A]: the gpuProbes test hook
 * (MetalMultislice.swift:113-117); equals Probe.build(at:) (Probe.swift:72-109). */
int simk_build_probes(simk_context* ctx, const simk_grid* grid, const simk_probe* probe, int32_t count,
                      const double* positions_xy, double* out_re, double* out_im);

/* ---- detectors and the STEM scan -----------------------------------------------------------------------------------
 * The value shape of one position for a detector (Detector.shape(for:beam:), Detectors.swift:84-88): writes ndim
 * (0, 1 or 2) and the sizes. */
int simk_detector_shape(const simk_grid* grid, double energy, const simk_detector* detector, int32_t* ndim,
                        int32_t* shape);
/* STEM.scan (STEM.swift:49-80, 95-150; Metal arm MetalEngine.swift:583-677): the probe at every position through every
 * potential (one per frozen-phonon configuration), every detector on |FFT2(exit)|^2 on the device, the mean over
 * potentials. outputs[d] holds n_positions x (the detector's value count) float64, row-major. */
int simk_scan(simk_context* ctx, const simk_probe* probe, int32_t n_potentials, simk_potential* const* potentials,
              int32_t n_positions, const double* positions_xy, int32_t n_detectors, const simk_detector* detectors,
              double* const* outputs);
/* The same with every buffer already on the device: positions_xy is a device pointer (n_positions x 2 float64) and
 * outputs[d] are device pointers; nothing is copied to or from the host and the call does not synchronise. */
int simk_scan_device(simk_context* ctx, const simk_probe* probe, int32_t n_potentials,
                     simk_potential* const* potentials, int32_t n_positions, const double* positions_xy_device,
                     int32_t n_detectors, const simk_detector* detectors, double* const* outputs_device);

/* STEM.scan(probe:potentials:scan:detector:) with a WavesDetector (Sources/SimulatoDetector/WavesDetector.swift:115-137,
 * collect :191-216): the complex exit wave at every position through one potential, resampled in Fourier space to
 * rows x columns points over the same extent (Waves.resampled, Sources/SimulatoCore/WavesResample.swift:16-43:
 * the lowest frequencies kept, or all of them zero-padded, values' amplitude kept); rows = columns = 0 keeps the
 * simulation grid. out_re / out_im: host, n_positions x rows x columns float64, positions in the given order.
 * STEM.scanFrozenPhonons with a WavesDetector is this call once per configuration. */
int simk_scan_waves(simk_context* ctx, const simk_probe* probe, simk_potential* potential, int32_t n_positions,
                    const double* positions_xy, int32_t rows, int32_t columns, double* out_re, double* out_im);

/* ---- contrast transfer function (Sources/SimulatoProbe/ContrastTransferFunction.swift) -----------------------------
 * An objective lens: aberrations (the simk_probe order), aperture semiangle [mrad] (INFINITY: none) with abTEM's soft
 * edge when `soft`, focal spread Delta [A] (temporal envelope) and angular spread beta [mrad] (spatial envelope). */
typedef struct {
    double aberrations[25];
    double semiangle_mrad;
    int32_t soft;
    int32_t reserved;
    double focal_spread;
    double angular_spread;
} simk_ctf;
/* ContrastTransferFunction.kernel (ContrastTransferFunction.swift:85-115), float64 on the device, FFT order. */
int simk_ctf_kernel(simk_context* ctx, const simk_grid* grid, double energy, const simk_ctf* ctf, double* re,
                    double* im);
/* Waves.applying (ContrastTransferFunction.swift:146-161) on `count` waves: IFFT(FFT(psi) H) in float32 with the
 * float64-computed kernel; out_re / out_im (the waves) and out_intensity (|.|^2, the HRTEM image) are optional (NULL). */
int simk_apply_ctf(simk_context* ctx, const simk_grid* grid, double energy, const simk_ctf* ctf, int32_t count,
                   const double* in_re, const double* in_im, double* out_re, double* out_im, double* out_intensity);

/* ---- scan post-processing (Sources/SimulatoDetector/ScanOperations.swift, IntegratedCenterOfMass.swift,
 * Sources/SimulatoCore/ImageOperations.swift) ------------------------------------------------------------------------
 * On a finished scan's float64 values, row-major [scan x][scan y][value_count] (a ScanMeasurement's layout). Each call
 * has a host form (host arrays, copied in and out) and a _device form (device pointers, e.g. simk_scan_device's
 * outputs, which stay on the device); both return when the result is written. */

/* ScanMeasurement.gaussianSourceSize(sigmaX:sigmaY:samplingX:samplingY:) (ScanOperations.swift:19-36): every value
 * filtered over the nx x ny scan with scipy's periodic Gaussian (radius floor(4 s + 1/2) pixels, s = sigma / sampling,
 * weights normalised), along y then x; sigma 0 leaves an axis alone. sigma [A] finite and >= 0, sampling [A] finite
 * and > 0, else SIMK_ERR_INVALID. Bit-equal to the reference's float64 loop. `out` may equal `in`. */
int simk_gaussian_source_size(simk_context* ctx, int32_t nx, int32_t ny, int64_t value_count, double sigma_x,
                              double sigma_y, double sampling_x, double sampling_y, const double* in, double* out);
int simk_gaussian_source_size_device(simk_context* ctx, int32_t nx, int32_t ny, int64_t value_count, double sigma_x,
                                     double sigma_y, double sampling_x, double sampling_y, const double* in_device,
                                     double* out_device);

/* ScanMeasurement.poissonNoise(dose:samples:seed:) (ScanOperations.swift:80-117): `samples` draws of the `count` values,
 * out[s count + i] ~ Poisson(max(in[i] dose, 0)), by the reference's sampler (Knuth below a mean of 10, PTRS above).
 * poissonNoise(dosePerArea:samplingX:samplingY:...) is dose = samplingX samplingY dosePerArea. The generator differs
 * from the reference's single stream: every value and sample has its own xoshiro256** seeded by
 * mix(mix(seed) + s count + i), so a seed gives the same noise on every run, not the reference's draws (with
 * SIMK_OPT_POISSON_STREAM = 1 the reference's stream instead, drawn in order by one device thread). dose finite
 * and >= 0, samples >= 1, finite values, else SIMK_ERR_INVALID. `out` (samples x count) may equal `in` when samples is
 * 1. */
int simk_poisson_noise(simk_context* ctx, int64_t count, const double* in, double dose, int32_t samples, uint64_t seed,
                       double* out);
int simk_poisson_noise_device(simk_context* ctx, int64_t count, const double* in_device, double dose, int32_t samples,
                              uint64_t seed, double* out_device);

/* RealField.integratingGradient (ImageOperations.swift:39-48, 140-167) and ScanMeasurement.integratedCenterOfMass
 * (IntegratedCenterOfMass.swift:36-40): the nx x ny gradient field gx[i stride], gy[i stride] (pixel i = ix ny + iy)
 * integrated in Fourier space, T^ = (kx g^x + ky g^y) / (2 pi i |k|^2) (|k|^2 = 1e-12 at zero frequency), the real
 * part of the inverse transform less its minimum, into out[nx ny]. A centre-of-mass measurement's interleaved (x, y)
 * pairs are gx = values, gy = values + 1, stride 2. nx, ny >= 2 and sampling finite and > 0, else SIMK_ERR_INVALID. */
int simk_integrate_gradient(simk_context* ctx, int32_t nx, int32_t ny, double sampling_x, double sampling_y,
                            const double* gx, const double* gy, int64_t stride, double* out);
int simk_integrate_gradient_device(simk_context* ctx, int32_t nx, int32_t ny, double sampling_x, double sampling_y,
                                   const double* gx_device, const double* gy_device, int64_t stride,
                                   double* out_device);

/* ---- job tables ----------------------------------------------------------------------------------------------------
 * No reference counterpart as one call (the reference runs such jobs one Multislice.run at a time, Multislice.swift:52-80
 * -> MetalEngine.swift:458-474); proposed as simk_job_table_run for uneven batches. Each job: an incident plane wave
 * (incident = SIMK_JOB_PLANE_WAVE, ones) or a probe (SIMK_JOB_PROBE: aperture, aberrations and tilt from `probe`, its
 * energy replaced by the job's) at (x, y) [A] through its own potential at its own energy; `intensity` (host,
 * nx x ny float64 of that potential's grid) receives |exit wave|^2 after the last slice. Jobs of one grid shape advance
 * together, one row and one column pass per slice step over the jobs still running, each shape on its own stream;
 * with SIMK_OPT_GRAPHS on (and SIMK_OPT_TIMING off) that whole schedule is captured as one CUDA graph and run by one
 * launch (SIMK_OPT_TABLE_LAUNCHES / _KERNELS / _SHAPES report it); the context keeps the last such graph with its
 * device buffers, and a call with the same jobs (potentials, energies, incident waves, positions, settings) only
 * recomputes the incident waves and launches it again. Turning SIMK_OPT_GRAPHS off releases it. With SIMK_FORM_PLAIN they run one after another
 * through the plain path (the sequential baseline). done_ms (optional, n_jobs) receives each job's
 * completion time on the device from the start of the call. A potential may serve several jobs of one energy. */
#define SIMK_JOB_PLANE_WAVE 0
#define SIMK_JOB_PROBE 1
typedef struct {
    simk_potential* potential;
    double energy;        /* [eV] */
    int32_t incident;     /* SIMK_JOB_PLANE_WAVE or SIMK_JOB_PROBE */
    int32_t reserved;
    simk_probe probe;     /* probe jobs */
    double x, y;          /* probe jobs: position [A] */
    double* intensity;    /* out (host): nx x ny */
} simk_job;
int simk_job_table_run(simk_context* ctx, int32_t n_jobs, const simk_job* jobs, double* done_ms);

/* ---- no-allocation variant ---------------------------------------------------------------------------------------
 * No counterpart in the reference: an addition for callers that cannot let the library allocate device memory
 * (a host framework that owns all device memory through its own allocator, such as PyTorch's caching allocator or an
 * XLA custom call, where a cudaMalloc inside the call would bypass its accounting and may synchronise the device).
 * Writes the same values as simk_probe_spectrum, rounded to complex64 (interleaved re, im, nx x ny), into the
 * caller's device buffer `out_device`, on `stream` (a cudaStream_t; NULL = the default stream), without
 * synchronising. It allocates nothing: its scratch is a fixed 32 KiB float64 array in the library's device image, so
 * grids above 2048 x 2048 pixels (4,194,304) are refused with SIMK_ERR_INVALID. The first call on a device (with that
 * device current) looks up the array's address; make it before any stream capture. Calls that are not captured look
 * the address up again (it belongs to the current context). A CUDA error already pending on the calling thread is
 * returned as SIMK_ERR_CUDA and left pending; nothing is launched then. Every call shares the array: calls that
 * overlap on the GPU race and must be serialised by the caller. */
int simk_probe_spectrum_noalloc(const simk_grid* grid, const simk_probe* probe, void* out_device, void* stream);

/* ---- the transform itself (FFT2D, Sources/SimulatoCore/FFT2D.swift:169-265) ----------------------------------------
 * `count` nx x ny fields, forward (unnormalised, e^{-2 pi i}) or inverse (x 1/(nx ny)), in float32 (precision 32) or
 * float64 (precision 64) on the device. A test hook: the hot path calls the transforms internally. */
int simk_fft2(simk_context* ctx, int32_t nx, int32_t ny, int32_t count, int32_t inverse, int32_t precision,
              const double* in_re, const double* in_im, double* out_re, double* out_im);

#ifdef __cplusplus
}
#endif

#endif /* SIMULATO_CUDA_H */
