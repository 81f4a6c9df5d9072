/*
 * FP64 C restatement of CuboPtycho's single-slice gradient descent — TEST INFRASTRUCTURE ONLY.
 *
 * This library is the oracle and the timed CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline / reference legs may load it.  The product library (cubokit_b200/libcuboptycho.so) never links it and
 * has no CPU fallback.
 *
 * Restated from (paths inside the CuboKit project):
 *   Sources/CuboPtycho/Ptychography.swift:142-172     PtychographyProbe.build
 *   Sources/CuboPtycho/Ptychography.swift:218-406     SingleslicePtychography.reconstruct, Double path
 *   Sources/CuboPtycho/PtychographySingle.swift:40-220 reconstructSingle, Float32 path (oracle_reconstruct_single)
 *   Sources/CuboPtycho/PtychographyConstraints.swift:9-83 probe constraints
 *   Sources/CuboCore/DoubleFFT.swift:3-6              transform convention: NumPy fft (e^-2pi i kn/N, unnormalised) and
 *                                                     ifft (e^+2pi i kn/N, divided by N), any length
 * The FFT is written here from the DFT definition: iterative radix-2 Cooley-Tukey for powers of two and Bluestein's
 * chirp-z (1968) through a radix-2 transform for every other length.
 *
 * Pinned against the py4DSTEM fixtures of CuboKit's own tests by tests/test_oracle.py.
 */
#ifndef CUBO_PTYCHO_ORACLE_H
#define CUBO_PTYCHO_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int iterations;
    double step_size;
    double normalization_minimum;
    int fix_probe;
    int pure_phase_object;
    int constrain_object_amplitude;
    int fix_probe_center_of_mass;
    int constrain_probe_amplitude;
    double probe_amplitude_relative_radius;
    double probe_amplitude_relative_width;
    int fix_probe_aperture;
    const unsigned char *probe_support_mask; /* NULL, or rows*columns bytes, nonzero = kept */
    int error_normalization;                 /* 0 = supplied amplitude energy, 1 = mean intensity */
    double mean_intensity;
    int threads;                             /* <= 1: the reference's single-threaded order; > 1: OpenMP over positions */
    int single_shift_fft;                    /* 1: one shifted-probe transform per position, as the reference does */
} oracle_params;

/* 0 ok, 1 invalid input (PtychographyError.invalidInput). */
int oracle_probe_build(int rows, int columns, double row_sampling, double column_sampling, double wavelength,
                       double cutoff, double rolloff, double defocus, double astigmatism, double astigmatism_angle,
                       double spherical_aberration, int term_count, const double *terms /* term_count x {n, m, sine, c} */,
                       double *re, double *im);

int oracle_reconstruct(const oracle_params *params, int rows, int columns, int object_rows, int object_columns,
                       int count, const double *amplitudes, const double *position_rows, const double *position_columns,
                       double *object_re, double *object_im, double *probe_re, double *probe_im, double *errors);

/* The Float32 path (amplitudes already Float; probe spectrum and constraints in Double once per iteration). */
int oracle_reconstruct_single(const oracle_params *params, int rows, int columns, int object_rows, int object_columns,
                              int count, const float *amplitudes, const double *position_rows,
                              const double *position_columns, double *object_re, double *object_im, double *probe_re,
                              double *probe_im, double *errors);

/* NumPy fft2 / ifft2 of a split complex rows x columns field, in place. */
void oracle_fft2(int rows, int columns, double *re, double *im, int inverse);

#ifdef __cplusplus
}
#endif
#endif
