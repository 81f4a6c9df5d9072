// The arithmetic of one position's update (Ptychography.swift:411-472), shared by the solve kernel and the fused
// 128 x 128 plane launch: the per-pixel terms of the 2 x 2 normal equations and the step with its limits.
#pragma once

#include <cuda_runtime.h>

namespace cubo {

// Adds one detector pixel's terms to v = [sum dx dx, sum dx dy, sum dy dy, sum dx difference, sum dy difference]:
// f the forward model's far field, gx / gy the far fields of the updated object one row / one column further,
// measured the amplitude.
__device__ __forceinline__ void position_terms(double2 f, double2 gx, double2 gy, double measured, double (&v)[5]) {
    const double difference = measured * measured - (f.x * f.x + f.y * f.y);
    const double dx = 2 * ((f.x - gx.x) * f.x + (f.y - gx.y) * f.y);
    const double dy = 2 * ((f.x - gy.x) * f.x + (f.y - gy.y) * f.y);
    v[0] += dx * dx;
    v[1] += dx * dy;
    v[2] += dy * dy;
    v[3] += dx * difference;
    v[4] += dy * difference;
}

// Cramer's rule on the summed terms, the step, the per-update and total limits (in pixels; infinite = none), then the
// move of position p (positions and initial are [rows | columns] of `count`).  A singular or non-finite system keeps
// the position; a position beyond 2^61 sets *bad.
__device__ __forceinline__ void position_step(const double (&v)[5], int p, double *positions, const double *initial,
                                              int count, double step, double limit_update, double limit_total,
                                              int *bad) {
    const double axx = v[0], axy = v[1], ayy = v[2], bx = v[3], by = v[4];
    const double determinant = axx * ayy - axy * axy;
    double u0 = 0.0, u1 = 0.0;
    if (determinant != 0 && isfinite(determinant)) {
        u0 = (ayy * bx - axy * by) / determinant * step;
        u1 = (axx * by - axy * bx) / determinant * step;
    }
    if (!isfinite(u0) || !isfinite(u1)) return;  // the position stays
    const double norm = hypot(u0, u1);
    if (norm > limit_update) {
        u0 /= norm / limit_update;
        u1 /= norm / limit_update;
    }
    const double row = positions[p], column = positions[count + p];
    if (isfinite(limit_total) && hypot(row - initial[p] - u0, column - initial[count + p] - u1) > limit_total) {
        u0 = 0.0;
        u1 = 0.0;
    }
    const double moved_row = row - u0, moved_column = column - u1;
    const double bound = 2305843009213693951.0;  // Int.max / 4 (Ptychography.swift:469)
    if (!(fabs(moved_row) < bound && fabs(moved_column) < bound)) {
        *bad = 1;
        return;
    }
    positions[p] = moved_row;
    positions[count + p] = moved_column;
}

}  // namespace cubo
