// Internal interface between the host orchestration (plan.cu) and the kernels (engine_kernels.cu, probe_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "fft_smem.cuh"

namespace cubo {

// Per-position data of the scan, on the device.
struct ScanTables {
    const int *rr;    // ties-to-even rounded row centre, wrapped into [0, object_rows)
    const int *cc;    // same for columns
    const int *cls;   // shift class (index into the shifted-probe table)
};

template <typename T>
struct PositionPassArgs {
    int rows, columns, object_rows, object_columns, n;
    int first, count;          // positions [first, first + count)
    ScanTables scan;
    const C2<T> *shifted;      // [classes][n] shifted probes
    const C2<T> *object;       // [object_rows * object_columns]
    const float *amplitudes;   // [positions][n]
    C2<T> *dpsi;               // [positions][n] the inverse transform of the projection residual
    double *error;             // [positions] squared amplitude residual
    const C2<T> *tw_rows, *tw_columns;  // W_rows^t, W_columns^t
    Radices rad_rows, rad_columns;
    T inv_n;
};

template <typename T>
struct ObjectGatherArgs {
    int rows, columns, object_rows, object_columns, n;
    int tiles_x;               // tiles per object row
    int tile_w, tile_h;        // tile shape, tile_w x tile_h = kGatherThreads pixels
    const int *tile_start;     // CSR offsets, [tiles + 1]
    const int *tile_list;      // position indices, ascending within each tile
    ScanTables scan;
    const C2<T> *shifted;
    const C2<T> *dpsi;
    C2<T> *grad;               // object gradient sum conj(S) dpsi
    T *weight;                 // sum |S|^2
    double *tile_max;          // per-tile max of weight
    int states = 1;            // mixed state (FP64): dpsi and shifted hold one block per state, these strides apart
    long long dpsi_state_stride = 0, shifted_state_stride = 0;
    // One band of the positions ([band_first, band_end), single state): block b takes tile band_tiles[b] and only its
    // candidates inside the band, whose residuals dpsi holds from position band_first on.  A tile's sums start from
    // the values grad / weight hold unless the band holds its first candidate, and its tile_max is written by the
    // band that holds its last one (or by the band that lists it with no candidates at all).  nullptr: every tile,
    // every candidate, dpsi from position 0.
    const int *band_tiles = nullptr;
    int band_first = 0, band_end = 0;
};

template <typename T>
struct ProbeGatherArgs {
    int rows, columns, object_rows, object_columns, n;
    int count, groups;         // positions, position groups (one partial sum each)
    ScanTables scan;
    const C2<T> *object;
    const C2<T> *dpsi;
    C2<T> *partial_grad;       // [groups][n]
    T *partial_weight;         // [groups][n]
    // One band: the positions [first, first + count), their residuals in dpsi from position `first` on, split into the
    // same `groups`; with `accumulate` each group's sums continue from the partials the earlier bands left.
    int first = 0;
    int accumulate = 0;
};

// The 128 x 128 FP32 position pass (fast128.cu); amplitudes in its register order, 32 residual partials per position.
struct Fast128Args {
    int object_rows, object_columns;
    int first, count;
    ScanTables scan;
    const float2 *shifted;
    const float2 *object;
    const float *amplitudes;   // [positions][column][h][t][e] (fast128.cu)
    float2 *dpsi;              // [positions - dpsi_first][row][column]
    int dpsi_first;            // the position whose residual dpsi[0] holds (a band's first, or 0)
    double *error;             // [positions][fast128_partials_per_position()]
    const float2 *tw128;       // W_128^t
    float2 *partial_grad;      // [fast128_ctas()][n] probe-gradient partials, one per CTA
    float *partial_weight;     // [fast128_ctas()][n]
    int accumulate;            // 1: each CTA's partial continues from the one it left (an earlier band), 0: from zero
    int *fault;                // set when the amplitude prefetch wait ran out
};
int fast128_ctas();
bool fast128_applicable(int rows, int columns);
int fast128_partials_per_position();
size_t fast128_smem();
cudaError_t configure_fast128();
cudaError_t launch_fast128(const Fast128Args &a, int ctas, cudaStream_t s);
cudaError_t launch_permute_amplitudes(const float *in, float *out, long long positions, cudaStream_t s);

// The 128 x 128 split-BF16 position pass (bf16dense.cu): DFT-matrix products on the tensor cores.
struct Bf16Args {
    int object_rows, object_columns;
    int first, count;
    ScanTables scan;
    const float2 *shifted;
    const float2 *object;
    const float *amplitudes;   // permuted into the order the kernel's threads consume them (permute_bf16_amplitudes)
    float2 *dpsi;              // [positions - dpsi_first][row][column]
    int dpsi_first;            // the position whose residual dpsi[0] holds (a band's first, or 0)
    double *error;             // [positions][bf16_partials_per_position()]
    const uint16_t *c_planes;  // [4][128][128] bf16 bits: C hi, C lo, C_sigma hi, C_sigma lo (rows m, columns k)
    int *fault;                // set when a device wait ran out
};
bool bf16_applicable(int rows, int columns);
int bf16_partials_per_position();
int bf16_sigma(int pos);  // the frequency at contraction position pos of the kernel's stage 4
cudaError_t configure_bf16();
cudaError_t launch_bf16(const Bf16Args &a, int ctas, cudaStream_t s);
cudaError_t launch_permute_bf16_amplitudes(const float *in, float *out, long long positions, cudaStream_t s);

// prepare.cu: amplitude preprocessing (pattern shift, square root, mean intensities)
// dynamic shared memory of one CTA: cubic, the coefficients in FP64 and the prefilter's carries; when `staged`, one
// (cubic) or two (bilinear) Float32 patterns copied in ahead of use
size_t prepare_smem(int rows, int columns, bool cubic, bool staged);
int prepare_max_line();         // the longest line the cubic prefilter takes (either axis)
int prepare_scratch_doubles();  // scratch of launch_prepare_means; the two means are its last two values
int prepare_sums_per_pattern();  // values launch_prepare writes per pattern into `sums`
cudaError_t configure_prepare();
// patterns [count][rows][columns] (Float32) -> amplitudes (same layout); sums[p * prepare_sums_per_pattern() ..] = the
// partial sums (of the shifted pattern p, of its positive part) of each of the CTA's warps, in pairs. *bad gains bit 1 if a value is not finite (*bad is not cleared). Patterns
// are staged in shared memory ahead of use when that fits in smem_limit bytes and the copy's alignment allows it.
struct PatternShift {  // one pattern's origin: its whole part wrapped into [0, rows) x [0, columns), and its fraction
    double row_fraction, column_fraction;
    int row, column;
};
cudaError_t launch_prepare(const float *cube, int count, int rows, int columns, const PatternShift *shifts, bool cubic,
                           float *amplitudes, double *sums, int *bad, int ctas, size_t smem_limit, cudaStream_t s);
// the mean intensities over `count` patterns' partial sums, in a fixed order
cudaError_t launch_prepare_means(const double *sums, int count, double *scratch, cudaStream_t s);

constexpr int kTileW = 16, kTileH = 16;  // default object-gather tile (one pixel per thread)
constexpr int kGatherThreads = kTileW * kTileH;

// engine_kernels.cu
template <typename T> cudaError_t launch_position_pass(const PositionPassArgs<T> &a, int shape, cudaStream_t s);
// linepass.cu: the FP32 position pass for 64 x 64 and 96 x 96 detectors with register-resident line transforms (four
// steps: R-point DFTs in registers, one in-group exchange, G-point DFTs), one CTA per position; the default FP32 pass
// at those sizes (cubo_ptycho_params.pass_shape 0).
bool line_pass_applicable(int rows, int columns);
cudaError_t configure_line_pass();
cudaError_t launch_line_pass(const PositionPassArgs<float> &a, cudaStream_t s);
cudaError_t launch_line_pass_grouped(const PositionPassArgs<float> *args, const int *prefix, int items, int total, int N,
                                     cudaStream_t s);

// Grouped launches (batches of independent reconstructions): every item's units in one persistent launch.  prefix holds
// items + 1 offsets (item i owns units prefix[i] .. prefix[i + 1] - 1); args one structure per item, in device memory.
// The position pass groups items of one square detector with a compile-time plan (position_pass_groupable), units =
// positions; the object gather's units are tiles; the probe gather's are (pixel block, position group) pairs.
bool position_pass_groupable(int rows, int columns, bool fp64);
template <typename T> cudaError_t launch_position_pass_grouped(const PositionPassArgs<T> *args, const int *prefix,
                                                               int items, int total, int N, int shape, cudaStream_t s);
template <typename T> cudaError_t launch_object_gather_grouped(const ObjectGatherArgs<T> *args, const int *prefix,
                                                               int items, int total, cudaStream_t s);
template <typename T> cudaError_t launch_probe_gather_grouped(const ProbeGatherArgs<T> *args, const int *prefix,
                                                              int items, int total, cudaStream_t s);
template <typename T> cudaError_t launch_object_gather(const ObjectGatherArgs<T> &a, int tiles, cudaStream_t s);
template <typename T> cudaError_t launch_probe_gather(const ProbeGatherArgs<T> &a, cudaStream_t s);
template <typename T> int probe_gather_resident_ctas();  // CTAs of the probe gather resident on one SM (at least 1)
template <typename T>
cudaError_t launch_probe_reduce(const C2<T> *partial_grad, const T *partial_weight, int groups, int n,
                                double2 *grad, double *weight, double *block_max, cudaStream_t s);
cudaError_t launch_max_reduce(const double *values, int count, double *out, cudaStream_t s);
// The maximum of count values (float or double) into *out, one CTA in a fixed order.
template <typename V> cudaError_t launch_max_values(const V *values, long long count, double *out, cudaStream_t s);
template <typename T>
cudaError_t launch_object_update(C2<T> *object, const C2<T> *grad, const T *weight, int count, const double *max_weight,
                                 double step, double minimum, int cap, int pure_phase, cudaStream_t s);
// Fixed-order FP64 sum of error[0, count) divided by `divisor` into errors[*iteration], then ++*iteration.
cudaError_t launch_error_reduce(const double *error, long long count, double divisor, double *errors, int *iteration,
                                double *scratch, cudaStream_t s);
int error_reduce_scratch();  // doubles of scratch launch_error_reduce needs
// object-gather candidate lists on the device: without `list`, counts[tile] = the number of positions whose window
// touches the tile; with it (and starts = exclusive sums of the counts), those positions in ascending order
template <typename T>
cudaError_t launch_object_cap(C2<T> *object, int count, int pure_phase, cudaStream_t s);

// position_kernels.cu: position correction (Ptychography.swift:411-472), FP64.  Positions are [rows | columns].
// Exit waves of positions first .. first + m - 1: out[(i * 3 + v) * n + k] = shifted probe x object patch, v = 0 the
// object before the update at the centre, v = 1 / 2 the updated object one row / one column further.
cudaError_t launch_position_exit_waves(const double2 *shifted, ScanTables scan, const double2 *before,
                                       const double2 *after, int first, int m, int rows, int columns, int object_rows,
                                       int object_columns, double2 *out, cudaStream_t s);
// From their far fields: per position the 2 x 2 normal equations over the detector, the step and its limits, the new
// position (limit_update / limit_total in pixels, infinite = none); *bad = 1 for a position beyond 2^61.
cudaError_t launch_position_solve(const double2 *far, const float *amplitudes, int first, int m, int n, double *positions,
                                  const double *initial, int count, double step, double limit_update,
                                  double limit_total, int *bad, cudaStream_t s);
// Scan tables of the positions on the device ([rows | columns]): wrapped ties-to-even centres, class p + 1 for position
// p (0 for a whole-pixel position) and its fractional shift (for the ramp table).
cudaError_t launch_scan_tables(const double *positions, int count, int object_rows, int object_columns, int *rr,
                               int *cc, int *cls, double2 *fractions, cudaStream_t s);
// starts[t] = sum of counts[0 .. t) for t <= tiles (one CTA, fixed order); *bad gains bit 2 if the total exceeds
// capacity.
cudaError_t launch_exclusive_scan(const int *counts, int tiles, int *starts, long long capacity, int *bad,
                                  cudaStream_t s);
// Ptychography.swift:398-401: every position shifted so that their mean is the initial mean again.
cudaError_t launch_position_center(double *positions, int count, double initial_mean_row, double initial_mean_column,
                                   cudaStream_t s);
cudaError_t launch_tile_lists(const int *rr, const int *cc, int count, int rows, int columns, int object_rows,
                              int object_columns, int tile_w, int tile_h, int tiles_x, int tiles, int *counts,
                              const int *starts, int *list, int capacity, cudaStream_t s);
// sum A^2 of `count` amplitudes into scratch[amplitude_check_scratch() - 1] (FP64, fixed order); *bad = 1 if any is not
// finite and non-negative (*bad is not cleared)
cudaError_t launch_amplitude_check(const float *amplitudes, long long count, double *scratch, int *bad, cudaStream_t s);
int amplitude_check_scratch();
bool position_pass_supported(int n, bool fp64);
size_t position_pass_smem(int n, int rows, int columns, bool fp64);

// probe_kernels.cu — FP64, probe-sized work
struct Fft2Plan64 {
    int rows, columns;
    Radices rad_rows, rad_columns;
    const double2 *tw_rows, *tw_columns;
};
cudaError_t launch_fft2_f64(const Fft2Plan64 &p, double2 *data, int batch, bool inverse, cudaStream_t s);
// global32.cu: the FP32 position pass through global memory (detectors above one CTA's shared memory, sides at most
// 4096): exit wave + row transforms, column transforms around the projection, inverse row transforms; its squared
// residual as global32_partials_per_position partials per position.  *launches receives the kernels it enqueued.
bool global32_applicable(int rows, int columns);
int global32_partials_per_position(int rows, int columns);
cudaError_t configure_global32();
cudaError_t launch_position_pass_global32(const PositionPassArgs<float> &a, int *launches, cudaStream_t s);
// The FP64 position pass through global memory (any detector whose sides are at most 4096): exit waves into dpsi,
// batched FFT, projection with the per-position error, inverse FFT.  *launches receives the kernels it enqueued.
cudaError_t launch_position_pass_global(const PositionPassArgs<double> &a, const Fft2Plan64 &fft, int *launches,
                                       cudaStream_t s);
bool line_fft_supported(int rows, int columns);
// The projection alone, in place on dpsi of positions first .. first + count - 1 (their far fields): the inverse
// transform's 1/n folded in, the per-position squared error written.
cudaError_t launch_project_global(const PositionPassArgs<double> &a, cudaStream_t s);

// multislice_kernels.cu: the multislice engine (MultislicePtychography, PtychographyEngines.swift:458-588), FP64.
// out[p][k] = in[class][k] x O[patch(p)][k] (conj(O) when conj_object; no object factor when object is null), class =
// scan.cls[p] when by_class, else p; in and out may be the same buffer.
cudaError_t launch_patch_multiply(const double2 *in, bool by_class, const double2 *object, bool conj_object,
                                  ScanTables scan, int first, int m, int rows, int columns, int object_rows,
                                  int object_columns, double2 *out, cudaStream_t s);
// data[plane][k] *= scale x prop[k] (or its conjugate) for `planes` planes of n values.
cudaError_t launch_spectrum_multiply(double2 *data, long long planes, int n, const double2 *prop, bool conj_prop,
                                     double scale, cudaStream_t s);
// identicalSlices: every slice becomes the mean of the slices.
cudaError_t launch_average_slices(double2 *object, int slices, long long plane, cudaStream_t s);

// plane128.cu: the 128 x 128 FP64 plane transform of positions first .. first + count - 1 in one launch, one cluster
// of plane128_cluster() CTAs per plane.  kPlaneFull: the input plane (times the object patch) -> FFT -> the pointwise
// step -> inverse FFT (unscaled) -> out; kPlaneForward: the input (times the patch) -> FFT -> out, unscaled;
// kPlaneInverse: a spectrum -> the pointwise step -> inverse FFT (unscaled) -> out.
enum { kPlaneFull = 0, kPlaneForward = 1, kPlaneInverse = 2 };
enum { kInputByPosition = 0, kInputByClass = 1, kInputSingle = 2 };
enum { kPointwiseNone = 0, kPointwiseFactors = 1, kPointwiseProjection = 2, kPointwiseSolve = 3,
       kPointwiseFactorPlane = 4 };
struct Plane128Args {
    int mode;
    int first, count;
    const double2 *in;              // input plane of position p: in + (p, scan.cls[p] or 0 by in_kind) * 16384
    int in_kind;
    const double2 *object;          // full / forward: the object patch factor, conjugated when conj_object; null: none
    int conj_object;
    int object_row_offset, object_column_offset;  // the patch one row / column further (position correction)
    ScanTables scan;
    int object_rows, object_columns;
    int pointwise;                  // kPointwiseFactors: x prop_rows[kr] prop_columns[kc] x scale; kPointwiseProjection
                                    // (full mode): modulus projection with amplitudes (x inv_n) and error[p]
    const double2 *prop_rows;       // 128 factors of the row frequency, then prop_stride further per position
    const double2 *prop_columns;    // 128 of the column frequency; both conjugated when conj_prop
    long long prop_stride;          // (a Fresnel kernel and the Fourier-shift ramps both factor so)
    int conj_prop;
    double scale;
    const float *amplitudes;        // [positions][128 x 128]
    double *error;                  // [positions] squared amplitude residual
    double inv_n;
    const double2 *tw;              // W_128^k, k = 0..127 (forward sign)
    double2 *out;                   // output plane of position p: out + (p * out_stride + out_offset) * 16384
    long long out_stride, out_offset;
    int *fault;                     // set when a bulk copy's wait ran out
    int ahead;                      // L2 prefetch distance in planes (0: the clusters resident at once)
    // forward mode with kPointwiseSolve (position correction): the spectrum is the far field of the updated object one
    // column further; with the forward model's far field and the one of the updated object one row further
    // (far + ((p - first) * 2 + 0 or 1) * 16384) and the amplitudes, position p's 2 x 2 normal equations are summed and
    // the position moved (positions / initial [rows | columns] of position_count); nothing is written to out
    const double2 *far;
    double *positions;
    const double *initial;
    int position_count;
    double position_step_size, limit_update, limit_total;
    int *position_bad;
    const double *factors;          // inverse mode with kPointwiseFactorPlane: [positions][128 x 128] real scales
};
int plane128_cluster();
cudaError_t configure_plane128();
cudaError_t launch_plane128(const Plane128Args &a, int cluster, cudaStream_t s);

// peaks.cu: the FP32 and FP64 FMA rates of the device (TFLOP/s, best of three timed launches on stream s).
cudaError_t measure_fma_peaks(cudaStream_t s, int sms, double *fp32_tflops, double *fp64_tflops);

// mixed_kernels.cu: the mixed-state engine (MixedstatePtychography, PtychographyEngines.swift:121-267), FP64.
constexpr int kMaxStates = 16;
struct MixedPassArgs {
    int rows, columns, object_rows, object_columns, count, states;
    ScanTables scan;
    const double2 *shifted;          // [state][class][pixel]
    long long shifted_state_stride;  // classes * n
    const double2 *object;
    const float *amplitudes;
    double2 *dpsi;                   // [state][position][pixel]
    double *error;                   // per position
    int zero_pixel_infinite;         // a pixel whose summed intensity is 0 adds an infinite error term (else A^2)
};
// Exit waves of every state, their far fields, the summed-intensity projection, the inverse transforms.
cudaError_t launch_mixed_position_pass(const MixedPassArgs &a, const Fft2Plan64 &fft, int *launches, cudaStream_t s);
// The summed-intensity projection's common factor of every pixel of the states' far fields dpsi[state][position][pixel]
// into factors[position][pixel] (the inverse transform's 1/n folded in), the states left as they are, the per-position
// error written.
cudaError_t launch_mixed_factors(const double2 *dpsi, const float *amplitudes, int count, int states, int n,
                                 bool zero_pixel_infinite, double *error, double *factors, cudaStream_t s);
// The states become the eigenvectors of their Gram matrix, by decreasing intensity (gram, mixing: states^2 values;
// scratch: states * n).
cudaError_t launch_orthogonalize(double2 *probes, int states, int n, double2 *gram, double2 *mixing, double2 *scratch,
                                 cudaStream_t s);

cudaError_t configure_fft_lines();
cudaError_t launch_scale_f64(double2 *data, int count, double scale, cudaStream_t s);
cudaError_t launch_probe_update(double2 *probe, const double2 *grad, const double *weight, int n, const double *max_weight,
                                double step, double minimum, cudaStream_t s);
// sums[0] = sum |p|^2, sums[1] = sum fr*R*w, sums[2] = sum fc*C*w (fixed order, one CTA)
cudaError_t launch_probe_moments(const double2 *probe, int rows, int columns, double *sums, cudaStream_t s);
cudaError_t launch_energy(const double2 *data, int n, double *sum, cudaStream_t s);
cudaError_t launch_com_ramp(double2 *spectrum, int rows, int columns, const double *sums, cudaStream_t s);
cudaError_t launch_commit_if_valid(double2 *probe, const double2 *candidate, int n, const double *sums,
                                   cudaStream_t s);
cudaError_t launch_aperture_phase(double2 *spectrum, const double *aperture, int n, cudaStream_t s);
cudaError_t launch_amplitude_mask(double2 *probe, int rows, int columns, double radius, double width,
                                  cudaStream_t s);
// dst = src * sqrt(before / after) when both are positive, else dst = src
cudaError_t launch_renormalise(double2 *dst, const double2 *src, int n, const double *before, const double *after,
                               cudaStream_t s);
cudaError_t launch_support_mask(double2 *probe, const unsigned char *mask, int n, cudaStream_t s);
cudaError_t launch_magnitude(const double2 *data, double *out, int n, cudaStream_t s);
cudaError_t launch_shift_ramps(const double2 *spectrum, const double2 *ramps_rows, const double2 *ramps_columns,
                               int rows, int columns, int classes, double2 *out, cudaStream_t s);
// The phase ramps of `classes` fractional shifts (dr, dc) = fractions[f]: exp(-2 pi i frequency(k) d) per row and column.
cudaError_t launch_ramp_table(const double2 *fractions, int classes, int rows, int columns, double2 *ramps_rows,
                              double2 *ramps_columns, cudaStream_t s);
template <typename T>
cudaError_t launch_convert(const double2 *in, C2<T> *out, long long count, cudaStream_t s);
cudaError_t configure_kernels();
cudaError_t launch_probe_spectrum(double2 *out, int rows, int columns, double row_sampling, double column_sampling,
                                  double wavelength, double cutoff, double rolloff, double defocus, double astigmatism,
                                  double astigmatism_angle, double spherical, int term_count, const double *terms,
                                  cudaStream_t s);

}  // namespace cubo
