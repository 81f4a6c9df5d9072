// The mixed-state engine's own kernels (MixedstatePtychography, PtychographyEngines.swift:121-267), FP64: several
// mutually incoherent probe states share one object and the detector sees the sum of their intensities.
//
//   exit waves     dpsi[s][p][k] = S_s(p)[k] x O[patch(p)][k] for every state s (the residual buffer doubles as the far
//                  fields: the engine's batched FFT transforms it in place)
//   projection     one CTA per position: I = sum_s |F_s|^2, factor = A / sqrt(I) - 1 (0 where I = 0), every state's far
//                  field times factor / n (the inverse transform's 1/n), the squared amplitude error; a pixel with I = 0
//                  adds an infinite term (py4DSTEM's behaviour) or, on request, A^2 (:188-195)
//   Gram matrix    G[i][j] = sum_k conj(p_i[k]) p_j[k], one CTA per pair, fixed-order FP64 sums (:303-313)
//   eigenvectors   one thread: cyclic complex Jacobi rotations on the (tiny) Hermitian G, eigenvalues sorted in
//                  decreasing order, ties with the later index first (NumPy's ascending argsort reversed, :325-326)
//   mixing         new_i = sum_j V[j][order(i)] p_j
#include <algorithm>
#include <cfloat>

#include "engine.h"

namespace cubo {

namespace {

constexpr int kProjectThreads = 512;
constexpr int kGramThreads = 256;

__device__ __forceinline__ int wrap_once(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__global__ void __launch_bounds__(256) mixed_exit_kernel(const double2 *shifted, long long shifted_state_stride,
                                                         ScanTables scan, const double2 *object, int first, int m,
                                                         int count, int states, int rows, int columns,
                                                         int object_rows, int object_columns, double2 *dpsi) {
    const int n = rows * columns;
    const long long t = (long long)blockIdx.x * 256 + threadIdx.x;
    if (t >= (long long)m * n) return;
    const int i = (int)(t / n), k = (int)(t - (long long)i * n);
    const int p = first + i;
    const int kr = k / columns, kc = k - kr * columns;
    const int y = wrap_once(scan.rr[p] + corner_offset(kr, rows), object_rows);
    const int x = wrap_once(scan.cc[p] + corner_offset(kc, columns), object_columns);
    const double2 o = object[(size_t)y * object_columns + x];
    const size_t cls_off = (size_t)scan.cls[p] * n + k;
    for (int s = 0; s < states; s++)
        dpsi[((size_t)s * count + p) * n + k] = cmul(shifted[(size_t)s * shifted_state_stride + cls_off], o);
}

__device__ double block_sum_project(double v, double *scratch) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kProjectThreads / 32; w++) s += scratch[w];
    return s;
}

// With `factors` the common factor of each pixel is written there and the states are left as they are (the inverse
// plane launches apply it); without, the states are scaled in place.
__global__ void __launch_bounds__(kProjectThreads) mixed_project_kernel(double2 *dpsi, const float *amplitudes, int first,
                                                                        int count, int states, int n, double inv_n,
                                                                        int zero_infinite, double *error,
                                                                        double *factors) {
    __shared__ double scratch[kProjectThreads / 32];
    const int p = first + blockIdx.x;
    const float *A = amplitudes + (size_t)p * n;
    double err = 0.0;
    for (int k = threadIdx.x; k < n; k += kProjectThreads) {
        double intensity = 0.0;
        for (int s = 0; s < states; s++) {
            const double2 f = dpsi[((size_t)s * count + p) * n + k];
            intensity += f.x * f.x + f.y * f.y;
        }
        const double amplitude = sqrt(intensity), measured = (double)A[k];
        double factor;
        if (amplitude == 0.0) {
            err += zero_infinite ? (double)INFINITY : measured * measured;
            factor = 0.0;
        } else {
            err += (measured - amplitude) * (measured - amplitude);
            factor = (measured / amplitude - 1.0) * inv_n;
        }
        if (factors) {
            factors[(size_t)p * n + k] = factor;
            continue;
        }
        for (int s = 0; s < states; s++) {
            double2 *f = dpsi + ((size_t)s * count + p) * n + k;
            f->x *= factor;
            f->y *= factor;
        }
    }
    const double total = block_sum_project(err, scratch);
    if (threadIdx.x == 0) error[p] = total;
}

// G[i][j] for i <= j (blockIdx.x enumerates the pairs row by row), and its Hermitian mirror.
__global__ void __launch_bounds__(kGramThreads) gram_kernel(const double2 *probes, int states, int n, double2 *gram) {
    __shared__ double sr[kGramThreads / 32], si[kGramThreads / 32];
    int pair = blockIdx.x, i = 0;
    while (pair >= states - i) {
        pair -= states - i;
        i++;
    }
    const int j = i + pair;
    const double2 *a = probes + (size_t)i * n, *b = probes + (size_t)j * n;
    double re = 0.0, im = 0.0;
    for (int k = threadIdx.x; k < n; k += kGramThreads) {
        const double2 x = a[k], y = b[k];
        re += x.x * y.x + x.y * y.y;  // conj(x) y
        im += x.x * y.y - x.y * y.x;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_down_sync(0xffffffffu, re, o);
        im += __shfl_down_sync(0xffffffffu, im, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sr[warp] = re;
        si[warp] = im;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tr = 0.0, ti = 0.0;
        for (int w = 0; w < kGramThreads / 32; w++) {
            tr += sr[w];
            ti += si[w];
        }
        if (i == j) ti = 0.0;  // the diagonal of a Gram matrix is real
        gram[i * states + j] = make_double2(tr, ti);
        gram[j * states + i] = make_double2(tr, -ti);
    }
}

__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cadd2(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }

// Eigen-decomposition of the Hermitian states x states matrix `gram` by cyclic Jacobi rotations.  Each rotation on
// (p, q) first turns a_pq real with D = diag(1, e^{-i phi}) (phi = arg a_pq), then zeroes it with the real rotation
// [c s; -s c] of Rutishauser's formula, t = sgn(z) / (|z| + sqrt(z^2 + 1)), z = (a_qq - a_pp) / (2 |a_pq|); the
// eigenvector matrix accumulates U = D R.  Writes mixing[i][j] = V[j][order(i)] with the eigenvalues in decreasing order
// (ties: the later index first).  One thread; states <= kMaxStates.
__global__ void eigen_kernel(const double2 *gram, int states, double2 *mixing) {
    double2 a[kMaxStates][kMaxStates], v[kMaxStates][kMaxStates];
    const int S = states;
    double scale = 0.0;
    for (int i = 0; i < S; i++)
        for (int j = 0; j < S; j++) {
            a[i][j] = gram[i * S + j];
            v[i][j] = make_double2(i == j ? 1.0 : 0.0, 0.0);
            scale += a[i][j].x * a[i][j].x + a[i][j].y * a[i][j].y;
        }
    scale = sqrt(scale);
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0;
        for (int i = 0; i < S; i++)
            for (int j = 0; j < S; j++)
                if (i != j) off += a[i][j].x * a[i][j].x + a[i][j].y * a[i][j].y;
        if (scale == 0.0 || sqrt(off) <= 1e-15 * scale) break;
        for (int p = 0; p < S - 1; p++)
            for (int q = p + 1; q < S; q++) {
                const double r = hypot(a[p][q].x, a[p][q].y);
                if (r <= 1e-300) continue;
                const double2 e = make_double2(a[p][q].x / r, -a[p][q].y / r);  // e^{-i phi}
                const double z = (a[q][q].x - a[p][p].x) / (2.0 * r);
                const double t = (z >= 0.0 ? 1.0 : -1.0) / (fabs(z) + sqrt(z * z + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                // U columns: u_p = (c, -s e) on rows (p, q); u_q = (s, c e)
                const double2 upp = make_double2(c, 0.0), uqp = make_double2(-s * e.x, -s * e.y);
                const double2 upq = make_double2(s, 0.0), uqq = make_double2(c * e.x, c * e.y);
                for (int row = 0; row < S; row++) {  // A <- A U and V <- V U
                    const double2 xp = a[row][p], xq = a[row][q];
                    a[row][p] = cadd2(cmul(xp, upp), cmul(xq, uqp));
                    a[row][q] = cadd2(cmul(xp, upq), cmul(xq, uqq));
                    const double2 yp = v[row][p], yq = v[row][q];
                    v[row][p] = cadd2(cmul(yp, upp), cmul(yq, uqp));
                    v[row][q] = cadd2(cmul(yp, upq), cmul(yq, uqq));
                }
                for (int col = 0; col < S; col++) {  // A <- U^H A
                    const double2 xp = a[p][col], xq = a[q][col];
                    a[p][col] = cadd2(cmul(cconj(upp), xp), cmul(cconj(uqp), xq));
                    a[q][col] = cadd2(cmul(cconj(upq), xp), cmul(cconj(uqq), xq));
                }
                a[p][q] = make_double2(0.0, 0.0);
                a[q][p] = make_double2(0.0, 0.0);
            }
    }
    int order[kMaxStates];
    for (int i = 0; i < S; i++) order[i] = i;
    for (int i = 1; i < S; i++) {  // insertion sort: decreasing eigenvalue, ties the later index first
        const int x = order[i];
        int j = i - 1;
        while (j >= 0 && (a[order[j]][order[j]].x < a[x][x].x ||
                          (a[order[j]][order[j]].x == a[x][x].x && order[j] < x))) {
            order[j + 1] = order[j];
            j--;
        }
        order[j + 1] = x;
    }
    for (int i = 0; i < S; i++)
        for (int j = 0; j < S; j++) mixing[i * S + j] = v[j][order[i]];
}

__global__ void __launch_bounds__(256) mix_kernel(const double2 *probes, const double2 *mixing, int states, int n,
                                                  double2 *out) {
    const long long t = (long long)blockIdx.x * 256 + threadIdx.x;
    if (t >= (long long)states * n) return;
    const int i = (int)(t / n), k = (int)(t - (long long)i * n);
    double2 acc = make_double2(0.0, 0.0);
    for (int j = 0; j < states; j++) acc = cadd2(acc, cmul(mixing[i * states + j], probes[(size_t)j * n + k]));
    out[(size_t)i * n + k] = acc;
}

}  // namespace

cudaError_t launch_mixed_position_pass(const MixedPassArgs &a, const Fft2Plan64 &fft, int *launches, cudaStream_t s) {
    const int n = a.rows * a.columns;
    const int chunk = (int)std::max<long long>(1, (1LL << 28) / ((long long)n * a.states));
    int count = 0;
    for (int first = 0; first < a.count; first += chunk) {
        const int m = std::min(chunk, a.count - first);
        const long long total = (long long)m * n;
        mixed_exit_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(
            a.shifted, a.shifted_state_stride, a.scan, a.object, first, m, a.count, a.states, a.rows, a.columns,
            a.object_rows, a.object_columns, a.dpsi);
        cudaError_t e = cudaGetLastError();
        count++;
        for (int st = 0; st < a.states && e == cudaSuccess; st++, count += 2)
            e = launch_fft2_f64(fft, a.dpsi + ((size_t)st * a.count + first) * n, m, false, s);
        if (e == cudaSuccess) {
            mixed_project_kernel<<<m, kProjectThreads, 0, s>>>(a.dpsi, a.amplitudes, first, a.count, a.states, n,
                                                               1.0 / n, a.zero_pixel_infinite, a.error, nullptr);
            e = cudaGetLastError();
            count++;
        }
        for (int st = 0; st < a.states && e == cudaSuccess; st++, count += 2)
            e = launch_fft2_f64(fft, a.dpsi + ((size_t)st * a.count + first) * n, m, true, s);
        if (e != cudaSuccess) return e;
    }
    if (launches) *launches = count;
    return cudaSuccess;
}

cudaError_t launch_mixed_factors(const double2 *dpsi, const float *amplitudes, int count, int states, int n,
                                 bool zero_pixel_infinite, double *error, double *factors, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    mixed_project_kernel<<<count, kProjectThreads, 0, s>>>(const_cast<double2 *>(dpsi), amplitudes, 0, count, states, n,
                                                           1.0 / n, zero_pixel_infinite ? 1 : 0, error, factors);
    return cudaGetLastError();
}

cudaError_t launch_orthogonalize(double2 *probes, int states, int n, double2 *gram, double2 *mixing, double2 *scratch,
                                 cudaStream_t s) {
    if (states < 2 || states > kMaxStates) return states < 2 ? cudaSuccess : cudaErrorInvalidValue;
    gram_kernel<<<states * (states + 1) / 2, kGramThreads, 0, s>>>(probes, states, n, gram);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    eigen_kernel<<<1, 1, 0, s>>>(gram, states, mixing);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const long long total = (long long)states * n;
    mix_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(probes, mixing, states, n, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(probes, scratch, (size_t)total * sizeof(double2), cudaMemcpyDeviceToDevice, s);
}

}  // namespace cubo
