/*
 * cubo_ptycho.h — C ABI of the B200 (sm_100a) single-slice ptychography gradient-descent engine.
 *
 * This is the drop-in boundary for CuboKit's CuboPtycho hot path.  A SwiftPM system-library target (the way CuboKit
 * already declares CStrainLAPACK and CEmbeddingLAPACK, Package.swift:48,50, with their headers in include/) exposes these
 * functions to Swift; the Swift shim converts [Double]/[Float] to pointers and maps the int status to the reference's
 * throws (status 1 -> PtychographyError.invalidInput, 2 -> CancellationError).  Conventions follow the reference's C shims
 * (Sources/CStrainLAPACK/include/CStrainLAPACK.h:1-2, Sources/CStrainLAPACK/LeastSquares.c:4-14): functions named
 * cubo_<module>_<verb>, an int status (0 = ok), caller-owned buffers, plain pointers and sizes.
 *
 * Layouts are the reference's: every complex field is split into a real and an imaginary plane of doubles, row-major
 * (PtychographyArray, Sources/CuboPtycho/Ptychography.swift:5-21); amplitudes are corner-centred
 * [position][row][column] (Ptychography.swift:189); positions are in object pixels, row then column
 * (PtychographyPosition, Ptychography.swift:88-93).
 *
 * Threading: every call is synchronous and blocking on the calling thread.  A context belongs to one host thread at a
 * time; different contexts (also on the same device) are independent.  There is no global mutable state.
 */
#ifndef CUBO_PTYCHO_H
#define CUBO_PTYCHO_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUBO_PTYCHO_ABI_VERSION 1

#if defined(__GNUC__)
#define CUBO_PTYCHO_API __attribute__((visibility("default")))
#else
#define CUBO_PTYCHO_API
#endif

/* Status codes.  Positive values are the reference's own throws; negative ones are device failures the CPU path cannot
 * have (a Swift shim maps them to a new error case).  The device never traps: a device-side wait that runs out reports
 * CUBO_PTYCHO_DEVICE_TIMEOUT and leaves the context usable. */
enum {
    CUBO_PTYCHO_OK = 0,
    CUBO_PTYCHO_INVALID_INPUT = 1,   /* PtychographyError.invalidInput (Ptychography.swift:24-27, :247-259) */
    CUBO_PTYCHO_CANCELLED = 2,       /* CancellationError (PtychographySingle.swift:222-224) */
    CUBO_PTYCHO_CUDA_ERROR = -1,
    CUBO_PTYCHO_OUT_OF_MEMORY = -2,
    CUBO_PTYCHO_DEVICE_TIMEOUT = -3,
    CUBO_PTYCHO_NO_DEVICE = -4,
    CUBO_PTYCHO_UNSUPPORTED = -5     /* a size or form this build has no kernel for (the message names it) */
};

/* Arithmetic of the per-position transforms.  FP32: complex64 state and shared-memory FFTs.  SPLIT_BF16: the 128 x 128
 * detector transforms as DFT-matrix products on the tensor cores with hi/lo BF16 operands and FP32 accumulation.  FP64:
 * complex128 everywhere (the adjoint check's form).  In every form the loss, the normalisation maxima and the probe
 * constraints are FP64. */
enum { CUBO_PTYCHO_FORM_FP32 = 0, CUBO_PTYCHO_FORM_SPLIT_BF16 = 1, CUBO_PTYCHO_FORM_FP64 = 2 };

/* PtychographyErrorNormalization (Ptychography.swift:30-48). */
enum { CUBO_PTYCHO_ERRORS_SUPPLIED_AMPLITUDE_ENERGY = 0, CUBO_PTYCHO_ERRORS_MEAN_INTENSITY = 1 };

typedef struct cubo_ptycho_context cubo_ptycho_context;
typedef struct cubo_ptycho_plan cubo_ptycho_plan;

/* The measured data and the geometry: SingleslicePtychography.reconstruct's amplitudes, positions and the shapes of its
 * object and probe (Ptychography.swift:218-219).  Amplitudes are Float32 on the host, as reconstructSingle takes them
 * (PtychographySingle.swift:40-41); the Swift shim converts the Double path's [Double] exactly as the reference's
 * .single branch does (Ptychography.swift:237-239). */
typedef struct {
    int rows, columns;                 /* detector = probe shape */
    int object_rows, object_columns;
    int count;                         /* number of scan positions */
    const float *amplitudes;           /* count * rows * columns */
    const double *position_rows;       /* count */
    const double *position_columns;    /* count */
    int amplitudes_on_device;          /* nonzero: `amplitudes` is device memory on the context's device (for example
                                        * the output of cubo_ptycho_prepare_amplitudes_device), copied on the device
                                        * instead of uploaded */
} cubo_ptycho_problem;

typedef void (*cubo_ptycho_progress_fn)(int completed, int total, void *user);

/* Every parameter of SingleslicePtychography.reconstruct (Ptychography.swift:218-234).  Booleans are ints
 * (0 / nonzero).  cubo_ptycho_params_default fills in the reference's defaults. */
typedef struct {
    int iterations;                    /* 8 */
    double step_size;                  /* 0.5 */
    double normalization_minimum;      /* 1 */
    int fix_probe;                     /* false */
    int pure_phase_object;             /* false */
    int constrain_object_amplitude;    /* true */
    int fix_probe_center_of_mass;      /* false */
    int constrain_probe_amplitude;     /* false */
    double probe_amplitude_relative_radius;  /* 0.5 */
    double probe_amplitude_relative_width;   /* 0.05 */
    int fix_probe_aperture;            /* false */
    const unsigned char *probe_support_mask; /* NULL, or rows * columns bytes, nonzero = kept */
    int error_normalization;           /* CUBO_PTYCHO_ERRORS_SUPPLIED_AMPLITUDE_ENERGY */
    double mean_intensity;             /* for CUBO_PTYCHO_ERRORS_MEAN_INTENSITY */
    int has_position_correction;       /* nonzero: positionCorrection is given (its settings at the end of this struct) */
    int form;                          /* CUBO_PTYCHO_FORM_FP32 */
    /* isCancelled: read before every iteration; nonzero stops the call with CUBO_PTYCHO_CANCELLED and leaves the
     * caller's object and probe untouched.  NULL: never cancelled. */
    const volatile int *cancel;
    /* progress(completed, total) after each iteration, on the calling thread.  NULL: none. */
    cubo_ptycho_progress_fn progress;
    void *progress_user;
    /* Kernel choice: CUBO_PTYCHO_VARIANT_AUTO picks the specialised kernel for the detector size when there is one;
     * CUBO_PTYCHO_VARIANT_GENERIC forces the any-size transforms (for cross-checks): the shared-memory one, and for
     * FP64 planes larger than one CTA the batched line transform through global memory instead of the clustered
     * 128 x 128 plane launch;
     * CUBO_PTYCHO_VARIANT_GLOBAL (FP64 and FP32 forms) forces the position pass through global memory that detectors
     * too large for one CTA's plane use (FP64: above 12,288 pixels; FP32: above 16,384, sides up to 4096) (for
     * cross-checks). */
    int variant;
    /* Object-gather tile (pixels per CTA, 256 in all): 0 = default (16 x 16), 1 = 32 x 8, 2 = 16 x 16, 3 = 64 x 4
     * (width x height along the residual's contiguous axis).  A performance choice only: every pixel sums the same
     * positions in the same order whatever the tile, so results are bitwise the same. */
    int gather_tile;
    /* positionCorrection (PtychographyPositionCorrection, Ptychography.swift:53-85), read when has_position_correction
     * is nonzero.  The reference runs it on its Double path only (its .single path refuses it, Ptychography.swift:236):
     * here the FP64 form; the FP32 and split-BF16 forms refuse it with CUBO_PTYCHO_INVALID_INPUT, and so do batches.
     * Distances in Å with has_* = 0 for nil (unlimited); samplings in Å per pixel, NaN for nil, needed (finite,
     * positive) when a distance is given; invalid settings are refused as pixelDistances refuses them (:74-84). */
    double position_step_size;                  /* 0.5 */
    int has_max_position_update_distance;       /* false */
    double max_position_update_distance;
    int has_max_position_total_distance;        /* false */
    double max_position_total_distance;
    double position_row_sampling;               /* NaN */
    double position_column_sampling;            /* NaN */
    int constrain_positions_center_of_mass;     /* false */
    /* Result.positions: when both are non-NULL, cubo_ptycho_reconstruct writes the positions after the last iteration
     * (count values each; the given positions when nothing corrected them). */
    double *position_rows_out, *position_columns_out;
    /* Position-pass kernel at 64 x 64 and 96 x 96 detectors: 0 = default (FP32: register-resident line transforms,
     * four steps per line; FP64: the shared-memory pass with the compile-time radix plan at 256 threads for 64 x 64 and
     * 512 for 96 x 96); 1, 2, 3 = the shared-memory pass with the compile-time plan at 128, 256, 512 threads per CTA
     * (as many CTAs per SM as registers and shared memory allow; a shape that would spill falls back to the nearest one
     * that does not).  Other detector sizes ignore it.  A performance choice: the shared-memory shapes give the same
     * object and probe bit for bit (every butterfly computes the same values; the per-position error is summed over the
     * CTA's threads and agrees to round-off); the register-line kernel factors the transform differently and agrees
     * with them to FP32 round-off.  Appended last so that the fields before it keep their offsets. */
    int pass_shape;
} cubo_ptycho_params;

enum { CUBO_PTYCHO_VARIANT_AUTO = 0, CUBO_PTYCHO_VARIANT_GENERIC = 1, CUBO_PTYCHO_VARIANT_GLOBAL = 2 };

/* Replaces the default arguments of SingleslicePtychography.reconstruct (Ptychography.swift:220-232). */
CUBO_PTYCHO_API void cubo_ptycho_params_default(cubo_ptycho_params *params);

/* A context owns a CUDA stream and device scratch on one device.  Replaces nothing in the reference (its CPU path has no
 * device state); it is the handle the Swift shim keeps. */
CUBO_PTYCHO_API int cubo_ptycho_create(int device, cubo_ptycho_context **out);
CUBO_PTYCHO_API int cubo_ptycho_destroy(cubo_ptycho_context *context);
/* Human-readable reason of the last non-zero status returned on this context (never NULL). */
CUBO_PTYCHO_API const char *cubo_ptycho_last_error(const cubo_ptycho_context *context);

/* SingleslicePtychography.reconstruct (Ptychography.swift:218-406).
 * object_re/object_im (object_rows * object_columns) and probe_re/probe_im (rows * columns) hold the start on entry and
 * the result on return (Result.object, Result.probe, Ptychography.swift:179-188); errors receives params->iterations
 * values (Result.errors); params->position_rows_out / _columns_out, when given, Result.positions.  Validation is the
 * reference's (Ptychography.swift:247-264): CUBO_PTYCHO_INVALID_INPUT and nothing written on a refusal. */
CUBO_PTYCHO_API int cubo_ptycho_reconstruct(cubo_ptycho_context *context, const cubo_ptycho_problem *problem,
                            const cubo_ptycho_params *params, double *object_re, double *object_im, double *probe_re,
                            double *probe_im, double *errors);

/* ---- The mixed-state engine: MixedstatePtychography.reconstruct (PtychographyEngines.swift:121-262).  Several mutually
 * incoherent probe states share one object; the detector intensity is the sum of the states' far-field intensities.
 * Runs in the FP64 form (params->form must be CUBO_PTYCHO_FORM_FP64: the reference's engine is Double) with the shared
 * params: iterations, step_size, normalization_minimum, fix_probe, pure_phase_object, fix_probe_center_of_mass (the
 * centre of mass of state 0 shifts every state), constrain_probe_amplitude (every state), fix_probe_aperture (state 0),
 * probe_support_mask (every state), error_normalization; the object threshold |O| <= 1 always applies (no
 * constrain_object_amplitude switch in this engine); position correction is refused.  Probes are `states` complex
 * grids, [state][row][column]. */
enum { CUBO_PTYCHO_ZERO_PIXEL_REFERENCE = 0, CUBO_PTYCHO_ZERO_PIXEL_FINITE = 1 };  /* MixedstateZeroPixelError */
typedef struct {
    int states;                /* probe states, 1 to 16 */
    int orthogonalize_probes;  /* true: after every iteration the states become the eigenvectors of their Gram matrix,
                                * by decreasing intensity (also with fix_probe, as py4DSTEM) */
    int zero_pixel_error;      /* a far-field pixel of zero summed intensity adds an infinite error term
                                * (CUBO_PTYCHO_ZERO_PIXEL_REFERENCE, py4DSTEM) or measured^2 (_FINITE) */
} cubo_ptycho_mixed_params;
CUBO_PTYCHO_API void cubo_ptycho_mixed_params_default(cubo_ptycho_mixed_params *mixed);
/* object_re/_im hold the start and receive Result.object; probes_re/_im (states * rows * columns) hold the starting
 * states and receive Result.probes; errors receives params->iterations values. */
CUBO_PTYCHO_API int cubo_ptycho_mixed_reconstruct(cubo_ptycho_context *context, const cubo_ptycho_problem *problem,
                                                  const cubo_ptycho_params *params,
                                                  const cubo_ptycho_mixed_params *mixed, double *object_re,
                                                  double *object_im, double *probes_re, double *probes_im,
                                                  double *errors);
/* MixedstatePtychography.orthogonalize (PtychographyEngines.swift:265-269,300-330) on the device, in place: the states
 * become the eigenvectors of their Gram matrix G[i][j] = sum conj(p_i) p_j, new_i = sum_j V[j][i] p_j, by decreasing
 * eigenvalue.  Each state's overall phase is an eigenvector convention (free). */
CUBO_PTYCHO_API int cubo_ptycho_orthogonalize(cubo_ptycho_context *context, int states, int rows, int columns,
                                              double *re, double *im);
/* A device-resident mixed-state plan: the cubo_ptycho_plan_* calls then take and return every state (set_state /
 * get_state probes of states * rows * columns values); forward / backward are single-slice only. */
CUBO_PTYCHO_API int cubo_ptycho_mixed_plan_create(cubo_ptycho_context *context, const cubo_ptycho_problem *problem,
                                                  const cubo_ptycho_params *params,
                                                  const cubo_ptycho_mixed_params *mixed, cubo_ptycho_plan **out);

/* ---- The multislice engine: MultislicePtychography.reconstruct (PtychographyEngines.swift:458-588).  The object is a
 * stack of `slices` transmission functions (entrance first) with a Fresnel propagation between neighbours; the
 * problem's object_rows x object_columns is one slice.  Runs in the FP64 form (the reference's engine is Double) with
 * the shared params: iterations, step_size, normalization_minimum, fix_probe, pure_phase_object, fix_probe_center_of_mass,
 * constrain_probe_amplitude, fix_probe_aperture, probe_support_mask, error_normalization; the object threshold
 * |O| <= 1 always applies; position correction is refused.  Objects are [slice][row][column]. */
typedef struct {
    int slices;                       /* object slices, 1 to 1024 */
    const double *slice_thicknesses;  /* slices - 1 gaps (length units of the samplings); may be NULL for one slice */
    double wavelength;                /* same units */
    double row_sampling, column_sampling;  /* object pixel sizes, same units */
    int identical_slices;             /* true: after each update every slice becomes the slices' mean */
} cubo_ptycho_multislice_params;
/* MultislicePtychography.propagators (PtychographyEngines.swift:427-442), on the host: count grids of rows x columns,
 * exp(-i pi wavelength dz (kr^2 + kc^2)) with k = fftfreq / sampling, into re / im ([thickness][row][column]). */
CUBO_PTYCHO_API int cubo_ptycho_propagators(int rows, int columns, double row_sampling, double column_sampling,
                                            double wavelength, int count, const double *thicknesses, double *re,
                                            double *im);
/* object_re/_im (slices * object_rows * object_columns) hold the start and receive Result.object; probe_re/_im the
 * probe; errors receives params->iterations values. */
CUBO_PTYCHO_API int cubo_ptycho_multislice_reconstruct(cubo_ptycho_context *context, const cubo_ptycho_problem *problem,
                                                       const cubo_ptycho_params *params,
                                                       const cubo_ptycho_multislice_params *multislice,
                                                       double *object_re, double *object_im, double *probe_re,
                                                       double *probe_im, double *errors);
/* A device-resident multislice plan: set_state / get_state take and return every slice; forward / backward are
 * single-slice only. */
CUBO_PTYCHO_API int cubo_ptycho_multislice_plan_create(cubo_ptycho_context *context, const cubo_ptycho_problem *problem,
                                                       const cubo_ptycho_params *params,
                                                       const cubo_ptycho_multislice_params *multislice,
                                                       cubo_ptycho_plan **out);

/* ---- Device-resident plans: the same reconstruction split into its upload, iterations and download, so data stays in
 * HBM across calls (resume = more iterations on the same plan).  No counterpart in the reference, whose arrays are
 * Swift values; reconstruct() is create + set_state + iterate + get_state + destroy. */
CUBO_PTYCHO_API int cubo_ptycho_plan_create(cubo_ptycho_context *context, const cubo_ptycho_problem *problem,
                            const cubo_ptycho_params *params, cubo_ptycho_plan **out);
CUBO_PTYCHO_API int cubo_ptycho_plan_destroy(cubo_ptycho_plan *plan);
CUBO_PTYCHO_API int cubo_ptycho_plan_set_state(cubo_ptycho_plan *plan, const double *object_re, const double *object_im,
                               const double *probe_re, const double *probe_im);
CUBO_PTYCHO_API int cubo_ptycho_plan_get_state(cubo_ptycho_plan *plan, double *object_re, double *object_im, double *probe_re,
                               double *probe_im);
/* The plan's current scan positions (count values each): the given ones, moved by position correction when it is on. */
CUBO_PTYCHO_API int cubo_ptycho_plan_get_positions(cubo_ptycho_plan *plan, double *rows, double *columns);
/* ---- Sharded iterations: one reconstruction's positions split into bands, one plan per band (per GPU), each holding
 * the whole object and probe.  An iteration is enqueue_gradients on every band; the sum over the bands of the buffers
 * gradient_buffers names (on the device; an NCCL all-reduce, say); apply_gradients on every band, which updates the
 * object and probe from the sums exactly as one plan over all positions does (the maxima are taken of the summed
 * weights).  No counterpart in the reference (its engine runs on one CPU thread).  The buffers: the object gradient
 * sum (complex, real_bytes per part: 4 in the FP32 and split-BF16 forms, 8 in FP64) and weights (one real per object
 * pixel), the probe gradient sums (complex double, states x rows x columns) and weights (double, rows x columns), and
 * the band's summed squared amplitude error (one double; the iteration's error is its sum over the bands divided by
 * the error normalisation of all positions).  Single-slice and mixed-state plans without position correction. */
CUBO_PTYCHO_API int cubo_ptycho_plan_enqueue_gradients(cubo_ptycho_plan *plan);
CUBO_PTYCHO_API int cubo_ptycho_plan_gradient_buffers(cubo_ptycho_plan *plan, void **grad_object, void **weight_object,
                                                      void **grad_probe, void **weight_probe, void **loss,
                                                      int *real_bytes);
CUBO_PTYCHO_API int cubo_ptycho_plan_apply_gradients(cubo_ptycho_plan *plan);

/* Runs `iterations` GD iterations on the resident state; errors (may be NULL) receives one value per iteration.
 * Honours params->cancel and params->progress. */
CUBO_PTYCHO_API int cubo_ptycho_plan_iterate(cubo_ptycho_plan *plan, int iterations, double *errors);
/* Enqueues `iterations` iterations on the context's stream and returns without waiting (no cancel, no progress; the
 * errors stay on the device, read them with cubo_ptycho_plan_errors after a synchronize).  For timing.  With position
 * correction each iteration after the first waits for the previous one: the positions it moved are read back to
 * rebuild the scan tables. */
CUBO_PTYCHO_API int cubo_ptycho_plan_enqueue(cubo_ptycho_plan *plan, int iterations);
CUBO_PTYCHO_API int cubo_ptycho_plan_errors(cubo_ptycho_plan *plan, int count, double *errors);
/* The context's cudaStream_t, as an opaque pointer. */
CUBO_PTYCHO_API void *cubo_ptycho_stream(cubo_ptycho_context *context);
CUBO_PTYCHO_API int cubo_ptycho_synchronize(cubo_ptycho_context *context);

/* ---- Adjoint pair on a plan's current state (no update is applied).  No counterpart function in the reference: its
 * reconstruct() computes these quantities inside the loop (Ptychography.swift:337-358); the pair exposes them.
 * forward: loss = sum over positions and detector pixels of (|F_k| - A_k)^2, F = fft2(S * O[patch]) unnormalised (the
 *   unnormalised residual of Ptychography.swift:342).  It keeps the inverse-transformed projection residuals of every
 *   position on the device (the tape) for backward.
 * backward: gradients of that loss, dL/dRe + i dL/dIm: object -2n sum_p conj(S_p) dpsi_p scattered to the patches, probe
 *   -2n sum_p conj(O[patch_p]) dpsi_p (the accumulations of Ptychography.swift:351-358 scaled to the loss; for
 *   fractional positions the probe term is the reference's, which does not undo each shift).  recompute_exit_waves != 0
 *   recomputes the exit waves and residuals instead of reading the tape (also done when no valid tape exists).  loss
 *   may be NULL.  Gradient buffers have the object's and the probe's sizes; any of them may be NULL. */
CUBO_PTYCHO_API int cubo_ptycho_plan_forward(cubo_ptycho_plan *plan, double *loss);
CUBO_PTYCHO_API int cubo_ptycho_plan_backward(cubo_ptycho_plan *plan, int recompute_exit_waves, double *loss,
                                              double *grad_object_re, double *grad_object_im, double *grad_probe_re,
                                              double *grad_probe_im);

/* ---- Batches: many independent reconstructions (each its own problem and parameters: scan, detector and object sizes
 * may differ) advanced together.  One iteration of every reconstruction of the batch is captured once into a CUDA graph
 * and replayed, so a run of the whole batch costs one graph launch per iteration.  No counterpart in the reference,
 * which reconstructs one dataset per call.  Cancellation and progress hooks of the params are not used by batch runs. */
typedef struct cubo_ptycho_batch cubo_ptycho_batch;
CUBO_PTYCHO_API int cubo_ptycho_batch_create(cubo_ptycho_context *context, int count,
                                             const cubo_ptycho_problem *problems, const cubo_ptycho_params *params,
                                             cubo_ptycho_batch **out);
CUBO_PTYCHO_API int cubo_ptycho_batch_destroy(cubo_ptycho_batch *batch);
CUBO_PTYCHO_API int cubo_ptycho_batch_set_state(cubo_ptycho_batch *batch, int index, const double *object_re,
                                                const double *object_im, const double *probe_re,
                                                const double *probe_im);
CUBO_PTYCHO_API int cubo_ptycho_batch_get_state(cubo_ptycho_batch *batch, int index, double *object_re,
                                                double *object_im, double *probe_re, double *probe_im);
/* Enqueues `iterations` replays of the captured iteration on the context stream; synchronize = 0 returns at once. */
CUBO_PTYCHO_API int cubo_ptycho_batch_run(cubo_ptycho_batch *batch, int iterations, int synchronize);
CUBO_PTYCHO_API int cubo_ptycho_batch_errors(cubo_ptycho_batch *batch, int index, int count, double *errors);
/* Kernel launches one replay of the captured iteration contains. */
CUBO_PTYCHO_API long long cubo_ptycho_batch_launches_per_iteration(const cubo_ptycho_batch *batch);

/* Launch accounting of a plan: kernels launched since the plan was created, and, when timing is on, the device time of
 * each kernel kind summed over its launches (CUDA events on the context stream).  kinds/ms/launches have room for
 * `capacity` entries; *count receives the number of kinds filled in.  names are static strings. */
CUBO_PTYCHO_API int cubo_ptycho_plan_set_timing(cubo_ptycho_plan *plan, int enabled);
CUBO_PTYCHO_API int cubo_ptycho_plan_kernel_stats(cubo_ptycho_plan *plan, int capacity, const char **names, double *ms,
                                  long long *launches, int *count);
CUBO_PTYCHO_API long long cubo_ptycho_plan_launch_count(const cubo_ptycho_plan *plan);

/* PtychographyProbe.build (Ptychography.swift:142-172) evaluated on the device in FP64 (the inverse transform is this
 * library's FP64 FFT).  terms: term_count rows of {radialOrder, angularOrder, sine (0/1), coefficient}
 * (PtychographyAberrationTerm, Ptychography.swift:101-133).  Writes rows * columns samples to re and im. */
CUBO_PTYCHO_API int cubo_ptycho_probe_build(cubo_ptycho_context *context, int rows, int columns, double row_sampling,
                            double column_sampling, double wavelength, double cutoff, double rolloff, double defocus,
                            double astigmatism, double astigmatism_angle, double spherical_aberration, int term_count,
                            const double *terms, double *re, double *im);

/* PtychographyShift (PtychographyPreparation.swift:56-62). */
enum { CUBO_PTYCHO_SHIFT_BILINEAR = 0, CUBO_PTYCHO_SHIFT_CUBIC_SPLINE = 1 };

/* PtychographyPreparation.amplitudes(from:origins:shift:) (PtychographyPreparation.swift:142-183) on the device: every
 * pattern of `cube` (count patterns of rows * columns Float32 values, [position][row][column], host memory) is shifted
 * so that its origin (origin_rows[p], origin_columns[p], detector pixels; a uniform origin is repeated) sits on the
 * corner pixel, out[i][j] = pattern[i + origin_row][j + origin_column] interpolated (bilinear or periodic cubic
 * B-spline, with wrap-around) in FP64, and amplitudes (host, same layout, Float32: the engine's input) receives
 * sqrt(max(out, 0)).  mean_intensity = the mean over patterns of the summed shifted intensity (negatives included,
 * py4DSTEM's mean_intensity and the .meanIntensity error normalisation); clipped_mean_intensity = the same with the
 * negative values set to zero first.  Invalid input (empty cube, an axis of one pixel, an origin not finite or beyond
 * 1e9, a cube value not finite) returns CUBO_PTYCHO_INVALID_INPUT; cubic-spline patterns whose FP64 copy does not fit
 * the shared memory of one CTA (above about 26,000 pixels, 160 x 160) return CUBO_PTYCHO_UNSUPPORTED. */
CUBO_PTYCHO_API int cubo_ptycho_prepare_amplitudes(cubo_ptycho_context *context, int count, int rows, int columns,
                                                   const float *cube, const double *origin_rows,
                                                   const double *origin_columns, int shift, float *amplitudes,
                                                   double *mean_intensity, double *clipped_mean_intensity);

/* The same with `cube` and `amplitudes` in device memory on the context's device (the origins stay on the host);
 * enqueued on the context's stream and completed before it returns.  The amplitudes can be handed to
 * cubo_ptycho_plan_create with problem.amplitudes_on_device set, so the prepared data never leaves the GPU. */
CUBO_PTYCHO_API int cubo_ptycho_prepare_amplitudes_device(cubo_ptycho_context *context, int count, int rows,
                                                          int columns, const float *cube_device,
                                                          const double *origin_rows, const double *origin_columns,
                                                          int shift, float *amplitudes_device, double *mean_intensity,
                                                          double *clipped_mean_intensity);

/* Kernel timing of the preprocessing calls on a context: when enabled (which also clears the totals), each launch of
 * the preprocessing kernel is bracketed by CUDA events on its stream, and the device time is summed once the call has
 * synchronised.  No counterpart in the reference (CPU code); for measurement. */
CUBO_PTYCHO_API int cubo_ptycho_set_timing(cubo_ptycho_context *context, int enabled);
CUBO_PTYCHO_API int cubo_ptycho_prepare_kernel_stats(cubo_ptycho_context *context, double *ms, long long *launches);

/* The device's FP32 and FP64 CUDA-core FMA rates in TFLOP/s (eight independent multiply-add chains per thread, best of
 * three timed launches): the denominators of the compute fractions reported for the FP32 and FP64 forms.  No
 * counterpart in the reference; for measurement. */
CUBO_PTYCHO_API int cubo_ptycho_measure_peaks(cubo_ptycho_context *context, double *fp32_tflops, double *fp64_tflops);

/* ---- Loss without allocating.  No counterpart in the reference: CuboPtycho computes on the CPU and never allocates
 * device memory.  For callers that cannot call cudaMalloc: a host application whose device memory belongs to its own
 * pool allocator, or a latency-critical loop that must not allocate (cudaMalloc can synchronise the device).
 * Computes loss[0] = sum over positions and detector pixels of (A - |fft2(P * O[patch])|)^2 in FP32 with FP64 sums
 * (the squared amplitude residual of Ptychography.swift:338-342, before any normalisation) for integer scan centres.
 * All pointers are the caller's device memory: amplitudes (count * rows * columns floats, [position][row][column],
 * 4-byte aligned), centre_rows / centre_columns (count ints, the rounded scan centres; any value, wrapped periodically),
 * object and probe as interleaved complex64 (2 floats per sample, row-major, 8-byte aligned), loss (one double, 8-byte
 * aligned); a misaligned pointer is refused with CUBO_PTYCHO_INVALID_INPUT.  Enqueued on `stream` (a cudaStream_t,
 * NULL = the default stream); returns without waiting.  Allocates nothing: the per-position scratch is a fixed device
 * array of CUBO_PTYCHO_NOALLOC_MAX_POSITIONS doubles inside the library, held on every GPU that loads it until the
 * process exits; count above that maximum is refused with CUBO_PTYCHO_INVALID_INPUT, detectors of more than 16384
 * pixels (rows * columns; 128 x 128 is the largest square) with CUBO_PTYCHO_UNSUPPORTED.  The first call on a device
 * resolves that array's device address (set-up done once per device, with the device current) and keeps it for the
 * life of the process: make that first call before any stream capture, and do not call this entry point on a device
 * after cudaDeviceReset of that device.  Every call shares the array, so calls that overlap on the GPU race: order
 * them on one stream. */
#define CUBO_PTYCHO_NOALLOC_MAX_POSITIONS (1 << 20)
CUBO_PTYCHO_API int cubo_ptycho_loss_fp32_noalloc(int rows, int columns, int object_rows, int object_columns, int count,
                                                  const float *amplitudes, const int *centre_rows,
                                                  const int *centre_columns, const float *object, const float *probe,
                                                  double *loss, void *stream);

#ifdef __cplusplus
}
#endif
#endif
