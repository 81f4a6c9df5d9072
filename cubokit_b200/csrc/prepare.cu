// Amplitude preprocessing on the device: PtychographyPreparation.amplitudes(from:origins:shift:)
// (PtychographyPreparation.swift:142-183, pattern shifts :296-344).
//
// Each diffraction pattern (Float32) is shifted so that its origin sits on the corner pixel,
// out[i][j] = pattern[i + origin_row][j + origin_column] interpolated with wrap-around, and the result is
// sqrt(max(out, 0)) (Float32, the engine's input) with the sums of out and of max(out, 0) over the pattern (FP64).
//
//   bilinear      four taps (Swift :301-315)
//   cubic spline  periodic cubic B-spline: coefficients c with (c[k-1] + 4 c[k] + c[k+1]) / 6 = pattern[k] along each
//                 axis, then 4 x 4 taps with the B-spline weights (Swift :317-342).  The reference divides by the
//                 kernel's DFT; here each line is solved exactly by the two-pass recursive filter with the pole
//                 z = sqrt(3) - 2 (Unser, Aldroubi & Eden, IEEE Trans. Signal Process. 41(2), 1993) with periodic
//                 states, O(n) per line in FP64, no transform needed.
//
// One CTA of 1024 threads per pattern at a time (grid-stride over patterns, one CTA per SM).  While a pattern is
// computed, the next one is copied into shared memory with cp.async.  The arithmetic is FP64 up to the square root of
// the Float32 output.  Every output pixel has the pattern's own fractional offsets, so the 2-D weights are a product
// of per-axis weights and the interpolation is separable: each thread walks down one column with the last few
// row-interpolated values in registers.  Each warp writes its sums of a pattern (fixed order), and a fixed-order sum
// runs over them afterwards: the same inputs give the same bits, however the patterns are split into launches.
#include <cfloat>

#include "engine.h"
#include "umma.cuh"

namespace cubo {

namespace {

constexpr int kPrepThreads = 1024;
constexpr int kPrepSumBlocks = 256;
constexpr int kSegMax = 16;  // values of one line segment that a thread holds in registers in the prefilter
constexpr int kPrepWarps = kPrepThreads / 32;

// the prefilter's pole z = sqrt(3) - 2 and its powers z^0 .. z^kSegMax
constexpr double kPole = -0.26794919243112270647;
struct PolePowers {
    double v[kSegMax + 1];
};
constexpr PolePowers pole_powers() {
    PolePowers p{};
    p.v[0] = 1.0;
    for (int k = 1; k <= kSegMax; k++) p.v[k] = p.v[k - 1] * kPole;
    return p;
}
__constant__ PolePowers kZ = pole_powers();

// Wraps v into [0, n) for v in [-n, 2n).
__device__ __forceinline__ int wrap_index(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__device__ __forceinline__ double int_power(double x, int e) {
    double r = 1.0;
    while (e) {
        if (e & 1) r *= x;
        x *= x;
        e >>= 1;
    }
    return r;
}

// The prefilter's constants for lines of n values: segments of kSegMax values (the last one `last`), the gains z^kSegMax
// and z^last across a segment, and the periodic factor 1 / (1 - z^n).
struct AxisFilter {
    int segs, last;
    double gain_full, gain_last, wrap;
};
__device__ __forceinline__ AxisFilter axis_filter(int n) {
    AxisFilter f;
    f.segs = (n + kSegMax - 1) / kSegMax;
    f.last = n - (f.segs - 1) * kSegMax;
    f.gain_full = int_power(kPole, kSegMax);
    f.gain_last = int_power(kPole, f.last);
    f.wrap = 1.0 / (1.0 - int_power(kPole, n));
    return f;
}

// One axis of the prefilter, with every thread of the CTA: for each of `lines` lines (line l reads src + l * src_line,
// values src_step apart, and writes dst + l * dst_line, values dst_step apart) the periodic cubic B-spline coefficients
// c, (c[k-1] + 4 c[k] + c[k+1]) / 6 = x[k].  The factorisation: the causal y[k] = x[k] + z y[k-1] with y[-1] = y[n-1],
// then the anticausal u[k] = z (u[k+1] - y[k]) with u[n] = u[0], c = 6 u.  The factor 6 is left out here: the pattern's
// interpolation weights carry it (36 for the two axes).
//
// A line is cut into segments of kSegMax values, one per thread, held in registers.  Each segment runs the recurrence
// from a zero state and publishes its end value; every thread then folds its line's end values itself into the true
// state entering its segment (the state after the segments before it, plus the periodic state carried across them),
// and adds z^d times that state to its values (d = the distance from the segment's entry).  The periodic state is
// exact: running a whole line from a zero state gives Y, and y[-1] = Y / (1 - z^n) (likewise u[n]).  Lines are taken
// in rounds of as many whole lines as there are threads for their segments.  `ends_causal` and `ends_anticausal` hold
// kPrepThreads values each.  Returns with the CTA synchronised and dst written.
template <typename S>
__device__ __forceinline__ void prefilter_axis(const S *src, int src_line, int src_step, double *dst, int dst_line,
                                               int dst_step, int lines, const AxisFilter &f, double *ends_causal,
                                               double *ends_anticausal) {
    const double z = kPole;
    const int segs = f.segs, last = f.last;
    const int per_round = kPrepThreads / segs;
    for (int first = 0; first < lines; first += per_round) {
        const int lr = min(per_round, lines - first);
        const int t = threadIdx.x;
        const bool active = t < lr * segs;
        const int g = active ? t / lr : 0, q = active ? t - g * lr : 0;  // adjacent threads: adjacent lines
        const int cnt = active ? (g == segs - 1 ? last : kSegMax) : 0;
        const S *in = src + ((first + q) * src_line + g * kSegMax * src_step);  // offsets within one pattern: int
        double v[kSegMax];
        double y = 0.0;
#pragma unroll
        for (int k = 0; k < kSegMax; k++) {
            if (k < cnt) {
                y = (double)in[k * src_step] + z * y;
                v[k] = y;
            } else {
                v[k] = 0.0;
            }
        }
        if (active) ends_causal[t] = y;
        __syncthreads();
        double u = 0.0;
        if (active) {
            // causal: s after segments 0 .. g-1 from a zero state, plus z^(16 g) y[-1]
            double s = 0.0, before = 0.0;
#pragma unroll 4
            for (int h = 0; h < segs; h++) {
                if (h == g) before = s;
                s = ends_causal[h * lr + q] + (h == segs - 1 ? f.gain_last : f.gain_full) * s;
            }
            const double e = before + int_power(f.gain_full, g) * (f.wrap * s);
#pragma unroll
            for (int k = 0; k < kSegMax; k++) v[k] += kZ.v[k + 1] * e;
#pragma unroll
            for (int k = kSegMax - 1; k >= 0; k--)
                if (k < cnt) {
                    u = z * (u - v[k]);
                    v[k] = u;
                }
            ends_anticausal[t] = u;
        }
        __syncthreads();
        if (active) {
            // anticausal: s after segments segs-1 .. g+1 from a zero state, plus z^(n - end of segment g) u[n]
            double s = 0.0, after = 0.0;
#pragma unroll 4
            for (int h = segs - 1; h >= 0; h--) {
                if (h == g) after = s;
                s = ends_anticausal[h * lr + q] + (h == segs - 1 ? f.gain_last : f.gain_full) * s;
            }
            const double span = g == segs - 1 ? 1.0 : f.gain_last * int_power(f.gain_full, segs - 2 - g);
            const double e = after + span * (f.wrap * s);
            double *out = dst + ((first + q) * dst_line + g * kSegMax * dst_step);
#pragma unroll
            for (int k = 0; k < kSegMax; k++)
                if (k < cnt) out[k * dst_step] = v[k] + kZ.v[cnt - k] * e;
        }
        // the next round writes `ends_causal` only after every thread has passed the barrier above, that is after its
        // reads of them; it writes `ends_anticausal` after its own first barrier, after these reads
    }
    __syncthreads();
}

// Cubic B-spline weights of the fraction t for the taps floor - 1 .. floor + 2 (Swift :330-334).
__device__ __forceinline__ void cubic_weights(double t, double (&w)[4]) {
    constexpr double kSixth = 1.0 / 6.0;
    w[0] = (1 - t) * (1 - t) * (1 - t) * kSixth;
    w[1] = (3 * t * t * t - 6 * t * t + 4) * kSixth;
    w[2] = (-3 * t * t * t + 3 * t * t + 3 * t + 1) * kSixth;
    w[3] = t * t * t * kSixth;
}

// One source row's taps along the columns: sum_b wc[b] row[ci[b]].
template <int kTaps, typename S>
__device__ __forceinline__ double row_taps(const S *row, const int (&ci)[kTaps], const double (&wc)[4]) {
    double s = 0.0;
#pragma unroll
    for (int b = 0; b < kTaps; b++) s += wc[b] * (double)row[ci[b]];
    return s;
}

// out[r][c] = sum_a wr[a] sum_b wc[b] P[r + dr + a][c + dc + b] (indices wrapped) for the whole pattern; each thread
// takes one column and a run of rows, keeping the last kTaps row sums in registers (a ring, renamed by unrolling).
// Accumulates the sums of the values and of their positive parts and writes sqrt(max(value, 0)) as Float32 (the
// correctly rounded Float32 square root of the value rounded to Float32).
template <int kTaps, typename S>
__device__ __forceinline__ void shift_pattern(const S *P, int pitch, int rows, int columns, int dr, int dc,
                                              const double (&wr)[4], const double (&wc)[4], float *out, double &total,
                                              double &clipped) {
    int runs = kPrepThreads / columns;
    runs = runs < 1 ? 1 : (runs > rows ? rows : runs);
    const int per = (rows + runs - 1) / runs;
    runs = (rows + per - 1) / per;
    for (int t = threadIdx.x; t < runs * columns; t += kPrepThreads) {
        const int g = t / columns, c = t - g * columns;  // adjacent threads: adjacent columns
        const int r0 = g * per, r1 = min(rows, r0 + per);
        int ci[kTaps];
        ci[0] = wrap_index(c + dc, columns);
#pragma unroll
        for (int b = 1; b < kTaps; b++) ci[b] = ci[b - 1] + 1 == columns ? 0 : ci[b - 1] + 1;
        int i = wrap_index(r0 + dr, rows);
        double h[kTaps];
#pragma unroll
        for (int a = 0; a < kTaps - 1; a++) {
            h[a] = row_taps<kTaps>(P + i * pitch, ci, wc);
            i = i + 1 == rows ? 0 : i + 1;
        }
        for (int r = r0; r < r1; r += kTaps) {
#pragma unroll
            for (int j = 0; j < kTaps; j++) {
                if (r + j < r1) {
                    h[(j + kTaps - 1) % kTaps] = row_taps<kTaps>(P + i * pitch, ci, wc);
                    i = i + 1 == rows ? 0 : i + 1;
                    double v = 0.0;
#pragma unroll
                    for (int a = 0; a < kTaps; a++) v += wr[a] * h[(j + a) % kTaps];
                    total += v;
                    const double pos = v > 0.0 ? v : 0.0;
                    clipped += pos;
                    out[(r + j) * columns + c] = sqrtf((float)pos);
                }
            }
        }
    }
}

// Bilinear, from a pattern in shared memory whose rows are whole 16-byte units (columns a multiple of 4): a thread
// takes four adjacent output columns c0 .. c0 + 3 (one aligned 16-byte store per row) and a run of rows; their taps
// are the five source columns c0 + dc .. c0 + dc + 4 (wrapped), so a source row costs five loads and four row sums.
__device__ __forceinline__ void shift_bilinear_x4(const float *P, int rows, int columns, int dr, int dc, double wr0,
                                                  double wr1, double wc0, double wc1, float *out, double &total,
                                                  double &clipped) {
    const int groups = columns / 4;
    int runs = kPrepThreads / groups;
    runs = runs < 1 ? 1 : (runs > rows ? rows : runs);
    const int per = (rows + runs - 1) / runs;
    runs = (rows + per - 1) / per;
    for (int t = threadIdx.x; t < runs * groups; t += kPrepThreads) {
        const int g = t / groups, c0 = 4 * (t - g * groups);  // adjacent threads: adjacent column groups
        const int r0 = g * per, r1 = min(rows, r0 + per);
        int sc[5];
        sc[0] = wrap_index(c0 + dc, columns);
#pragma unroll
        for (int b = 1; b < 5; b++) sc[b] = sc[b - 1] + 1 == columns ? 0 : sc[b - 1] + 1;
        int i = wrap_index(r0 + dr, rows);
        double h0[4], h1[4];
        auto row_sums = [&](int row, double (&h)[4]) {
            const float *q = P + row * columns;
            double x[5];
#pragma unroll
            for (int b = 0; b < 5; b++) x[b] = (double)q[sc[b]];
#pragma unroll
            for (int j = 0; j < 4; j++) h[j] = wc0 * x[j] + wc1 * x[j + 1];
        };
        auto emit = [&](int r, const double (&ha)[4], const double (&hb)[4]) {
            float4 o;
            float *ov = reinterpret_cast<float *>(&o);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const double v = wr0 * ha[j] + wr1 * hb[j];
                total += v;
                const double pos = v > 0.0 ? v : 0.0;
                clipped += pos;
                ov[j] = sqrtf((float)pos);
            }
            *reinterpret_cast<float4 *>(out + (r * columns + c0)) = o;
        };
        row_sums(i, h0);
        i = i + 1 == rows ? 0 : i + 1;
        for (int r = r0; r < r1; r += 2) {  // the two row-sum sets alternate roles (no copies)
            row_sums(i, h1);
            i = i + 1 == rows ? 0 : i + 1;
            emit(r, h0, h1);
            if (r + 1 < r1) {
                row_sums(i, h0);
                i = i + 1 == rows ? 0 : i + 1;
                emit(r + 1, h1, h0);
            }
        }
    }
}

template <int NT>
__device__ double block_sum_f64(double v, double *scratch) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    v = threadIdx.x < NT / 32 ? scratch[threadIdx.x] : 0.0;
    if (warp == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;  // thread 0 holds the sum
}

// Starts copying one pattern (n values, n a multiple of 4, both addresses 16-byte aligned) into shared memory, 16 bytes
// per cp.async, spread over the CTA's threads; every thread commits one group.
__device__ __forceinline__ void copy_pattern_async(float *dst, const float *src, int n) {
    const uint32_t d = umma::smem_u32(dst);
    for (int i = threadIdx.x; i < n / 4; i += kPrepThreads)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d + 16u * (uint32_t)i), "l"(src + 4 * (size_t)i)
                     : "memory");
    asm volatile("cp.async.commit_group;" ::: "memory");
}

// Waits for this thread's copies, then for the CTA's.
__device__ __forceinline__ void copy_pattern_wait() {
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
}

// Shared memory (dynamic), in doubles from the start:
//   cubic     the FP64 coefficients (rows x pitch, pitch = columns | 1), the segments' end values of the two
//             recurrences (kPrepThreads each),
//             then, when staged, one Float32 pattern (the next one, copied in behind the column pass)
//   bilinear  when staged, two Float32 patterns (the current one and the next); nothing otherwise (taps read from
//             global memory)
// staged_at: where the staging area starts (in doubles), or -1 for none.  aligned_rows: the bilinear taps may take
// whole 16-byte units of a staged row and store 16-byte units of the output.  *bad gains bit 1 when a pattern holds a
// value that is not finite.
// kRows, kColumns: the pattern's size when it is known at compile time (0: the arguments give it).
template <bool kCubic, int kRows, int kColumns>
__global__ void __launch_bounds__(kPrepThreads) prepare_kernel(const float *cube, int count, int rows_arg,
                                                              int columns_arg, const PatternShift *shifts,
                                                              float *amplitudes, double *sums, int *bad, int staged_at,
                                                              int aligned_rows) {
    extern __shared__ __align__(16) double smem[];
    const int rows = kRows ? kRows : rows_arg, columns = kColumns ? kColumns : columns_arg;
    const int n = rows * columns;
    const int pitch = columns | 1;  // rows an odd number of doubles apart: a warp walking 32 rows hits 32 bank pairs
    double *coef = smem, *ends_causal = smem + rows * pitch, *ends_anticausal = ends_causal + kPrepThreads;
    const bool staged = staged_at >= 0;
    float *const buffer = reinterpret_cast<float *>(smem + (staged ? staged_at : 0));  // bilinear: two, n values apart
    AxisFilter along_columns, along_rows;  // lines of `rows` values (one per column), lines of `columns` values
    if (kCubic) {
        along_columns = axis_filter(rows);
        along_rows = axis_filter(columns);
    }
    int k = 0;  // bilinear: the buffer holding pattern p
    if (staged && blockIdx.x < count) copy_pattern_async(buffer, cube + (size_t)blockIdx.x * n, n);
    for (int p = blockIdx.x; p < count; p += gridDim.x) {
        const bool next = p + (int)gridDim.x < count;
        const float *raw = cube + (size_t)p * n;
        const float *here = buffer + k * n;  // the staged copy of pattern p (shared memory)
        if (staged) {
            copy_pattern_wait();
            if (!kCubic && next) copy_pattern_async(buffer + (k ^ 1) * n, cube + (size_t)(p + gridDim.x) * n, n);
        }
        const PatternShift sh = shifts[p];
        double total = 0.0, clipped = 0.0;
        float *out = amplitudes + (size_t)p * n;
        if (kCubic) {
            // columns first (reading the raw pattern, coalesced), then rows in place; the order of the two axes
            // changes only the roundoff
            if (staged)
                prefilter_axis(here, 1, columns, coef, 1, pitch, columns, along_columns, ends_causal, ends_anticausal);
            else
                prefilter_axis(raw, 1, columns, coef, 1, pitch, columns, along_columns, ends_causal, ends_anticausal);
            if (staged && next) copy_pattern_async(buffer, cube + (size_t)(p + gridDim.x) * n, n);
            prefilter_axis(static_cast<const double *>(coef), pitch, 1, coef, pitch, 1, rows, along_rows, ends_causal,
                           ends_anticausal);
            double wr[4], wc[4];
            cubic_weights(sh.row_fraction, wr);
            cubic_weights(sh.column_fraction, wc);
#pragma unroll
            for (int a = 0; a < 4; a++) wr[a] *= 36.0;  // the factor 6 of both axes' coefficients
            shift_pattern<4>(static_cast<const double *>(coef), pitch, rows, columns, sh.row - 1, sh.column - 1, wr,
                             wc, out, total, clipped);
        } else {
            // Swift :311-312, p00 (1-fr)(1-fc) + p10 fr (1-fc) + p01 (1-fr) fc + p11 fr fc, as (1-fr) (p00 (1-fc) +
            // p01 fc) + fr (p10 (1-fc) + p11 fc)
            const double tr = sh.row_fraction, tc = sh.column_fraction;
            if (staged && aligned_rows) {
                shift_bilinear_x4(here, rows, columns, sh.row, sh.column, 1 - tr, tr, 1 - tc, tc, out, total, clipped);
            } else {
                const double wr[4] = {1 - tr, tr, 0.0, 0.0}, wc[4] = {1 - tc, tc, 0.0, 0.0};
                if (staged)
                    shift_pattern<2>(here, columns, rows, columns, sh.row, sh.column, wr, wc, out, total, clipped);
                else
                    shift_pattern<2>(raw, columns, rows, columns, sh.row, sh.column, wr, wc, out, total, clipped);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            total += __shfl_down_sync(0xffffffffu, total, o);
            clipped += __shfl_down_sync(0xffffffffu, clipped, o);
        }
        if ((threadIdx.x & 31) == 0) {
            // every raw value reaches some warp's sum with a weight (a NaN or an infinity makes it NaN or infinite,
            // 0 x infinity included); finite values cannot overflow it
            if (!(fabs(total) <= DBL_MAX)) atomicOr(bad, 1);
            double *w = sums + ((size_t)p * kPrepWarps + (threadIdx.x >> 5)) * 2;
            w[0] = total;
            w[1] = clipped;
        }
        // Staged, the next pattern starts with a barrier (after its copy wait) before anything in shared memory is
        // written.  Unstaged, the cubic column pass would write the coefficients at once: this barrier keeps it from
        // overwriting what a slower warp still interpolates.  (Unstaged bilinear uses no shared memory.)
        if (kCubic && !staged) __syncthreads();
        if (!kCubic) k ^= 1;
    }
}

// Fixed-order sums over the patterns: block b sums its slice of patterns (each pattern's warp sums in warp order), then
// one block sums the blocks.
__global__ void __launch_bounds__(1024) prepare_partial_kernel(const double *sums, int count, double *block_sums) {
    __shared__ double scratch[32];
    const long long b = (long long)count * blockIdx.x / kPrepSumBlocks, e = (long long)count * (blockIdx.x + 1) / kPrepSumBlocks;
    double t = 0, c = 0;
    for (long long i = b + threadIdx.x; i < e; i += 1024) {
        const double *w = sums + i * 2 * kPrepWarps;
        double pt = 0, pc = 0;
#pragma unroll 8
        for (int k = 0; k < kPrepWarps; k++) {
            pt += w[2 * k];
            pc += w[2 * k + 1];
        }
        t += pt;
        c += pc;
    }
    t = block_sum_f64<1024>(t, scratch);
    c = block_sum_f64<1024>(c, scratch);
    if (threadIdx.x == 0) {
        block_sums[2 * blockIdx.x] = t;
        block_sums[2 * blockIdx.x + 1] = c;
    }
}

__global__ void __launch_bounds__(kPrepSumBlocks) prepare_final_kernel(const double *block_sums, int count,
                                                                      double *means) {
    __shared__ double scratch[32];
    const double t = block_sum_f64<kPrepSumBlocks>(block_sums[2 * threadIdx.x], scratch);
    const double c = block_sum_f64<kPrepSumBlocks>(block_sums[2 * threadIdx.x + 1], scratch);
    if (threadIdx.x == 0) {
        means[0] = t / (double)count;
        means[1] = c / (double)count;
    }
}

// doubles before the staging area: cubic, the coefficients and the prefilter's carries (rounded up to 16 bytes);
// bilinear, none
size_t prepare_base_doubles(int rows, int columns, bool cubic) {
    if (!cubic) return 0;
    const size_t d = (size_t)rows * (columns | 1) + 2 * kPrepThreads;
    return (d + 1) & ~(size_t)1;
}

}  // namespace

size_t prepare_smem(int rows, int columns, bool cubic, bool staged) {
    const size_t n = (size_t)rows * columns;
    return prepare_base_doubles(rows, columns, cubic) * sizeof(double) +
           (staged ? (cubic ? 1 : 2) * n * sizeof(float) : 0);
}

namespace {
bool prepare_can_stage(const float *cube, int rows, int columns, bool cubic, size_t smem_limit) {
    // cp.async of 16-byte units from a 16-byte-aligned address
    const size_t n = (size_t)rows * columns;
    return n % 4 == 0 && ((uintptr_t)cube & 15) == 0 && prepare_smem(rows, columns, cubic, true) <= smem_limit;
}
}  // namespace

int prepare_max_line() { return kSegMax * kPrepThreads; }
int prepare_scratch_doubles() { return 2 * kPrepSumBlocks + 2; }
int prepare_sums_per_pattern() { return 2 * kPrepWarps; }

cudaError_t configure_prepare() {
    int device = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    const int limit = optin - 1024;
    for (auto f : {prepare_kernel<false, 0, 0>, prepare_kernel<false, 128, 128>, prepare_kernel<true, 0, 0>,
                   prepare_kernel<true, 128, 128>}) {
        e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_prepare(const float *cube, int count, int rows, int columns, const PatternShift *shifts, bool cubic,
                           float *amplitudes, double *sums, int *bad, int ctas, size_t smem_limit, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const int grid = count < ctas ? count : ctas;
    const bool staged = prepare_can_stage(cube, rows, columns, cubic, smem_limit);
    const int staged_at = staged ? (int)prepare_base_doubles(rows, columns, cubic) : -1;
    const int aligned_rows = columns % 4 == 0 && ((uintptr_t)amplitudes & 15) == 0;
    const size_t smem = prepare_smem(rows, columns, cubic, staged);
    // 128 x 128 patterns (the usual detector) have their own instantiation: constant strides and trip counts
    const bool square128 = rows == 128 && columns == 128;
    auto kernel = cubic ? (square128 ? prepare_kernel<true, 128, 128> : prepare_kernel<true, 0, 0>)
                        : (square128 ? prepare_kernel<false, 128, 128> : prepare_kernel<false, 0, 0>);
    kernel<<<grid, kPrepThreads, smem, s>>>(cube, count, rows, columns, shifts, amplitudes, sums, bad, staged_at,
                                            aligned_rows);
    return cudaGetLastError();
}

cudaError_t launch_prepare_means(const double *sums, int count, double *scratch, cudaStream_t s) {
    prepare_partial_kernel<<<kPrepSumBlocks, 1024, 0, s>>>(sums, count, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    prepare_final_kernel<<<1, kPrepSumBlocks, 0, s>>>(scratch, count, scratch + 2 * kPrepSumBlocks);
    return cudaGetLastError();
}

}  // namespace cubo
