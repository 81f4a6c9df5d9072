// Position correction of the single-slice engine on the device: py4DSTEM's `_position_correction` as CuboPtycho states
// it (Ptychography.swift:371-377 in the iteration, the update :411-472, the centre-of-mass constraint :398-401), FP64.
//
// Per position p (rounded centre rr, cc; shifted probe s, the one the forward model used this iteration):
//   f   = FFT(s x O_before[patch at (rr, cc)])        the forward model's far field
//   fdx = FFT(s x O_after [patch at (rr + 1, cc)])    the updated object read one row further
//   fdy = FFT(s x O_after [patch at (rr, cc + 1)])    ... one column further
//   dx = 2 Re((f - fdx) conj f), dy likewise, difference = A^2 - |f|^2, over the detector pixels
//   [sum dx dx, sum dx dy; sum dx dy, sum dy dy] u = [sum dx difference, sum dy difference] (Cramer's rule), u *= step
//   |u| clipped to the update limit; dropped when the new position would be further than the total limit from its
//   start; position -= u.  A singular or non-finite system keeps the position.
// The three exit waves of a chunk of positions are formed by one kernel, transformed by the engine's batched FP64 FFT,
// and reduced by one CTA per position (fixed-order FP64 sums: the same inputs give the same bits).
#include "engine.h"
#include "position_step.cuh"

namespace cubo {

namespace {

constexpr int kSolveThreads = 256;

__device__ __forceinline__ int wrap_once(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__global__ void __launch_bounds__(256) exit_waves_kernel(const double2 *shifted, ScanTables scan, const double2 *before,
                                                         const double2 *after, int first, int m, int rows, int columns,
                                                         int object_rows, int object_columns, double2 *out) {
    const int n = rows * columns;
    const long long t = (long long)blockIdx.x * 256 + threadIdx.x;
    if (t >= (long long)m * n) return;
    const int i = (int)(t / n), k = (int)(t - (long long)i * n);
    const int r = k / columns, c = k - r * columns;
    const int p = first + i;
    // corner-centred patch offsets (Ptychography.swift:321-328, :426-430); rr, cc are wrapped and the object is at
    // least as large as the detector, so one wrap brings every index (one row or column further included) back
    const int ro = r < (rows + 1) / 2 ? r : r - rows, co = c < (columns + 1) / 2 ? c : c - columns;
    const int r0 = wrap_once(scan.rr[p] + ro, object_rows), c0 = wrap_once(scan.cc[p] + co, object_columns);
    const int r1 = r0 + 1 == object_rows ? 0 : r0 + 1, c1 = c0 + 1 == object_columns ? 0 : c0 + 1;
    const double2 sv = shifted[(size_t)scan.cls[p] * n + k];
    const double2 o0 = before[(size_t)r0 * object_columns + c0];
    const double2 ox = after[(size_t)r1 * object_columns + c0];
    const double2 oy = after[(size_t)r0 * object_columns + c1];
    double2 *w = out + (size_t)i * 3 * n + k;
    w[0] = make_double2(sv.x * o0.x - sv.y * o0.y, sv.x * o0.y + sv.y * o0.x);
    w[n] = make_double2(sv.x * ox.x - sv.y * ox.y, sv.x * ox.y + sv.y * ox.x);
    w[2 * n] = make_double2(sv.x * oy.x - sv.y * oy.y, sv.x * oy.y + sv.y * oy.x);
}

// Sums of v[0..4] over the CTA in a fixed order; thread 0 holds them.
__device__ __forceinline__ void block_sum5(double (&v)[5], double (*scratch)[kSolveThreads / 32]) {
#pragma unroll
    for (int j = 0; j < 5; j++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < 5; j++) scratch[j][warp] = v[j];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int j = 0; j < 5; j++) {
            double s = 0.0;
            for (int w = 0; w < kSolveThreads / 32; w++) s += scratch[j][w];
            v[j] = s;
        }
}

__global__ void __launch_bounds__(kSolveThreads) solve_kernel(const double2 *far, const float *amplitudes, int first,
                                                              int n, double *positions, const double *initial, int count,
                                                              double step, double limit_update, double limit_total,
                                                              int *bad) {
    __shared__ double scratch[5][kSolveThreads / 32];
    const int i = blockIdx.x, p = first + i;
    const double2 *f0 = far + (size_t)i * 3 * n, *fx = f0 + n, *fy = f0 + 2 * n;
    const float *a = amplitudes + (size_t)p * n;
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // axx, axy, ayy, bx, by
    for (int k = threadIdx.x; k < n; k += kSolveThreads) position_terms(f0[k], fx[k], fy[k], (double)a[k], v);
    block_sum5(v, scratch);
    if (threadIdx.x != 0) return;
    position_step(v, p, positions, initial, count, step, limit_update, limit_total, bad);
}

__global__ void __launch_bounds__(1024) center_kernel(double *positions, int count, double initial_mean_row,
                                                      double initial_mean_column) {
    __shared__ double scratch[2][32];
    __shared__ double shift[2];
    double s[2] = {0.0, 0.0};
    for (int i = threadIdx.x; i < count; i += 1024) {
        s[0] += positions[i];
        s[1] += positions[count + i];
    }
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s[j] += __shfl_down_sync(0xffffffffu, s[j], o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        scratch[0][warp] = s[0];
        scratch[1][warp] = s[1];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[2] = {0.0, 0.0};
        for (int w = 0; w < 32; w++) {
            t[0] += scratch[0][w];
            t[1] += scratch[1][w];
        }
        shift[0] = t[0] / (double)count - initial_mean_row;
        shift[1] = t[1] / (double)count - initial_mean_column;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < count; i += 1024) {
        positions[i] -= shift[0];
        positions[count + i] -= shift[1];
    }
}

// Scan tables of moved positions: ties-to-even centres wrapped into the object, one shift class per position (class
// p + 1 with its fraction for the ramp table; class 0, the unshifted probe, for a whole-pixel position), as the host
// builds them for a plan with position correction.
__global__ void __launch_bounds__(256) scan_kernel(const double *positions, int count, int object_rows,
                                                   int object_columns, int *rr, int *cc, int *cls, double2 *fractions) {
    const int p = blockIdx.x * 256 + threadIdx.x;
    if (p >= count) return;
    const double r = positions[p], c = positions[count + p];
    const double rn = rint(r), cn = rint(c);  // rint rounds half to even
    long long wr = (long long)rn % object_rows, wc = (long long)cn % object_columns;
    rr[p] = (int)(wr < 0 ? wr + object_rows : wr);
    cc[p] = (int)(wc < 0 ? wc + object_columns : wc);
    const double dr = r - rn, dc = c - cn;
    cls[p] = dr == 0.0 && dc == 0.0 ? 0 : p + 1;  // class 0: the probe itself, as without position correction
    fractions[p] = make_double2(dr, dc);
}

// Exclusive prefix sums of counts[0 .. tiles) into starts (starts[tiles] = the total), one CTA in a fixed order;
// *bad gains bit 2 when the total exceeds `capacity` (the starts are then clamped to it).
__global__ void __launch_bounds__(1024) exclusive_scan_kernel(const int *counts, int tiles, int *starts,
                                                              long long capacity, int *bad) {
    __shared__ long long part[1024];
    const int per = (tiles + 1023) / 1024, begin = threadIdx.x * per, end = min(tiles, begin + per);
    long long s = 0;
    for (int t = begin; t < end; t++) s += counts[t];
    part[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        long long run = 0;
        for (int i = 0; i < 1024; i++) {
            const long long v = part[i];
            part[i] = run;
            run += v;
        }
        starts[tiles] = (int)(run > capacity ? capacity : run);
        if (run > capacity) *bad |= 2;
    }
    __syncthreads();
    long long run = part[threadIdx.x];
    for (int t = begin; t < end; t++) {
        starts[t] = (int)(run > capacity ? capacity : run);
        run += counts[t];
    }
}

}  // namespace

cudaError_t launch_scan_tables(const double *positions, int count, int object_rows, int object_columns, int *rr,
                               int *cc, int *cls, double2 *fractions, cudaStream_t s) {
    scan_kernel<<<(count + 255) / 256, 256, 0, s>>>(positions, count, object_rows, object_columns, rr, cc, cls,
                                                    fractions);
    return cudaGetLastError();
}

cudaError_t launch_exclusive_scan(const int *counts, int tiles, int *starts, long long capacity, int *bad,
                                  cudaStream_t s) {
    exclusive_scan_kernel<<<1, 1024, 0, s>>>(counts, tiles, starts, capacity, bad);
    return cudaGetLastError();
}

cudaError_t launch_position_exit_waves(const double2 *shifted, ScanTables scan, const double2 *before,
                                       const double2 *after, int first, int m, int rows, int columns, int object_rows,
                                       int object_columns, double2 *out, cudaStream_t s) {
    const long long total = (long long)m * rows * columns;
    if (total <= 0) return cudaSuccess;
    exit_waves_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(shifted, scan, before, after, first, m, rows,
                                                                       columns, object_rows, object_columns, out);
    return cudaGetLastError();
}

cudaError_t launch_position_solve(const double2 *far, const float *amplitudes, int first, int m, int n, double *positions,
                                  const double *initial, int count, double step, double limit_update,
                                  double limit_total, int *bad, cudaStream_t s) {
    if (m <= 0) return cudaSuccess;
    solve_kernel<<<m, kSolveThreads, 0, s>>>(far, amplitudes, first, n, positions, initial, count, step, limit_update,
                                              limit_total, bad);
    return cudaGetLastError();
}

cudaError_t launch_position_center(double *positions, int count, double initial_mean_row, double initial_mean_column,
                                   cudaStream_t s) {
    center_kernel<<<1, 1024, 0, s>>>(positions, count, initial_mean_row, initial_mean_column);
    return cudaGetLastError();
}

}  // namespace cubo
