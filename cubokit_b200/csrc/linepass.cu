// The FP32 position pass for 64 x 64 and 96 x 96 detectors with register-resident line transforms (sm_100a).
//
// Same arithmetic as the shared-memory position pass (exit wave, forward 2-D FFT, Fourier-modulus projection with the
// 1/n of ifft2 folded in, inverse 2-D FFT; Ptychography.swift:321-350), laid out as the 128 x 128 register kernel is:
//
//  * One CTA per position; a line of length N = G R (N = 96: G = 4, R = 24; N = 64: G = 8, R = 8) belongs to a group of
//    G consecutive threads of one warp, thread t holding the samples n = t + G m (m < R) in registers.
//  * Four-step transform of a line (with k = q + R s, q < R, s < G):
//      X[q + R s] = sum_t W_G^{t s} W_N^{t q} sum_m W_R^{m q} x[t + G m],
//    i.e. an R-point DFT in registers, the twiddle W_N^{t q}, one exchange inside the group through the line's own row
//    of the shared-memory tile (__syncwarp only), and G-point DFTs of the R / G frequencies q the thread keeps.  The
//    24-point DFT is 8 x 3 (three 8-point DFTs, the twiddle W_24^{b c}, eight 3-point DFTs).  The inverse runs the same
//    steps mirrored with conjugate twiddles.  Every twiddle is read from the line's FP64-evaluated table W_N^k.
//  * The 2-D transform: rows (group g owns row g), the spectrum rows written into an N x (N + 1) tile, columns (group g
//    reads column g); the projection on the registers of the column pass; the inverse column pass written back into
//    the tile; the inverse row pass; dpsi written [row][column].
//  * The squared residual is summed per thread in FP64 and over the CTA in a fixed order: one partial per position,
//    as the shared-memory pass writes it.  No atomics: bitwise reproducible.
#include "engine.h"

namespace cubo {

namespace {

__device__ __forceinline__ float2 lmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 ladd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 lsub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// W_N^k (forward) or its conjugate (inverse) from the table of W_N^0 .. W_N^{N-1}.
template <bool INV>
__device__ __forceinline__ float2 twiddle(const float2 *tw, int k) {
    const float2 w = tw[k];
    return INV ? make_float2(w.x, -w.y) : w;
}

// (-i) a forward, (+i) a inverse: the W_4^1 of the direction.
template <bool INV>
__device__ __forceinline__ float2 mul_w4(float2 a) { return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x); }

template <bool INV>
__device__ __forceinline__ void ldft4(float2 &x0, float2 &x1, float2 &x2, float2 &x3) {
    const float2 t0 = ladd(x0, x2), t1 = lsub(x0, x2), t2 = ladd(x1, x3), t3 = mul_w4<INV>(lsub(x1, x3));
    x0 = ladd(t0, t2); x2 = lsub(t0, t2); x1 = ladd(t1, t3); x3 = lsub(t1, t3);
}

// 8-point DFT, natural order in and out: the 4-point DFTs of the even and odd samples joined by W_8^k (W_8^1 =
// tw[N / 8] of an N-point table).
template <bool INV, int N>
__device__ __forceinline__ void ldft8(float2 (&v)[8], const float2 *tw) {
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    ldft4<INV>(e0, e1, e2, e3);
    ldft4<INV>(o0, o1, o2, o3);
    o1 = lmul(o1, twiddle<INV>(tw, N / 8));
    o2 = mul_w4<INV>(o2);
    o3 = lmul(o3, twiddle<INV>(tw, 3 * N / 8));
    v[0] = ladd(e0, o0); v[4] = lsub(e0, o0);
    v[1] = ladd(e1, o1); v[5] = lsub(e1, o1);
    v[2] = ladd(e2, o2); v[6] = lsub(e2, o2);
    v[3] = ladd(e3, o3); v[7] = lsub(e3, o3);
}

// 3-point DFT with W_3 = tw[N / 3]: X0 = a + b + c, X1 = a + W b + W^2 c, X2 = a + W^2 b + W c.
template <bool INV, int N>
__device__ __forceinline__ void ldft3(float2 &a, float2 &b, float2 &c, const float2 *tw) {
    const float2 w1 = twiddle<INV>(tw, N / 3), w2 = twiddle<INV>(tw, 2 * N / 3);
    const float2 x0 = ladd(a, ladd(b, c));
    const float2 x1 = ladd(a, ladd(lmul(b, w1), lmul(c, w2)));
    const float2 x2 = ladd(a, ladd(lmul(b, w2), lmul(c, w1)));
    a = x0; b = x1; c = x2;
}

// 24-point DFT, natural order in and out, as 8 x 3: with m = 3 a + b and k = c + 8 d,
// X[c + 8 d] = sum_b W_3^{b d} W_24^{b c} sum_a W_8^{a c} x[3 a + b].
template <bool INV, int N>
__device__ __forceinline__ void ldft24(float2 (&x)[24], const float2 *tw) {
    float2 y[3][8];
#pragma unroll
    for (int b = 0; b < 3; b++) {
#pragma unroll
        for (int a = 0; a < 8; a++) y[b][a] = x[3 * a + b];
        ldft8<INV, N>(y[b], tw);
    }
#pragma unroll
    for (int c = 1; c < 8; c++) {
        y[1][c] = lmul(y[1][c], twiddle<INV>(tw, c * (N / 24)));
        y[2][c] = lmul(y[2][c], twiddle<INV>(tw, 2 * c * (N / 24)));
    }
#pragma unroll
    for (int c = 0; c < 8; c++) {
        ldft3<INV, N>(y[0][c], y[1][c], y[2][c], tw);
        x[c] = y[0][c];
        x[c + 8] = y[1][c];
        x[c + 16] = y[2][c];
    }
}

template <bool INV, int N, int L>
__device__ __forceinline__ void ldft(float2 (&x)[L], const float2 *tw) {
    if constexpr (L == 24) ldft24<INV, N>(x, tw);
    else if constexpr (L == 8) ldft8<INV, N>(x, tw);
    else {
        static_assert(L == 4, "line radix");
        ldft4<INV>(x[0], x[1], x[2], x[3]);
    }
}

template <int N, int G>
struct LineShape {
    static constexpr int kR = N / G;        // samples per thread and line
    static constexpr int kQ = kR / G;       // frequencies q a thread keeps after the exchange
    static constexpr int kThreads = N * G;  // one line per group of G threads
    static constexpr int kPitch = N + 1;    // tile row pitch (complex64)
    static_assert(kR % G == 0, "the four-step split needs G | R");
};

// Forward transform of the thread's line: x[m] = line[t + G m] in; out[j G + s] = X[q_j + R s], q_j = t kQ + j.
// `row` is the line's scratch row of the tile (only this group touches it during the call).
template <int N, int G>
__device__ __forceinline__ void line_forward(float2 (&x)[N / G], int t, const float2 *tw, float2 *row) {
    using S = LineShape<N, G>;
    constexpr int R = S::kR, Q = S::kQ;
    ldft<false, N, R>(x, tw);
#pragma unroll
    for (int q = 1; q < R; q++) x[q] = lmul(x[q], twiddle<false>(tw, (t * q) % N));
#pragma unroll
    for (int q = 0; q < R; q++) row[t * R + q] = x[q];
    __syncwarp();
#pragma unroll
    for (int j = 0; j < Q; j++) {
        float2 z[G];
#pragma unroll
        for (int tp = 0; tp < G; tp++) z[tp] = row[tp * R + t * Q + j];
        ldft<false, N, G>(z, tw);
#pragma unroll
        for (int s = 0; s < G; s++) x[j * G + s] = z[s];
    }
    __syncwarp();
}

// Inverse of line_forward (unnormalised): x[j G + s] = X[q_j + R s] in, x[m] = line[t + G m] out.
template <int N, int G>
__device__ __forceinline__ void line_inverse(float2 (&x)[N / G], int t, const float2 *tw, float2 *row) {
    using S = LineShape<N, G>;
    constexpr int R = S::kR, Q = S::kQ;
#pragma unroll
    for (int j = 0; j < Q; j++) {
        float2 z[G];
#pragma unroll
        for (int s = 0; s < G; s++) z[s] = x[j * G + s];
        ldft<true, N, G>(z, tw);
#pragma unroll
        for (int tp = 0; tp < G; tp++) row[tp * R + t * Q + j] = z[tp];
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < R; q++) x[q] = row[t * R + q];
    __syncwarp();
#pragma unroll
    for (int q = 1; q < R; q++) x[q] = lmul(x[q], twiddle<true>(tw, (t * q) % N));
    ldft<true, N, R>(x, tw);
}

__device__ __forceinline__ int lwrap(int v, int size) { return v < 0 ? v + size : (v >= size ? v - size : v); }

// One position: group g (threads G g .. G g + G - 1) owns row g in the row passes and column g in the column passes.
template <int N, int G>
__device__ __forceinline__ void line_pass_body(const PositionPassArgs<float> &a, int p) {
    using S = LineShape<N, G>;
    constexpr int R = S::kR, Q = S::kQ, NT = S::kThreads, P = S::kPitch;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *tile = reinterpret_cast<float2 *>(smem_raw);
    float2 *tw = tile + N * P;
    double *scratch = reinterpret_cast<double *>(tw + N);
    const int tid = threadIdx.x, g = tid / G, t = tid - g * G;
    for (int i = tid; i < N; i += NT) tw[i] = a.tw_rows[i];
    const int rr = a.scan.rr[p], cc = a.scan.cc[p], cls = a.scan.cls[p];
    const float2 *Sp = a.shifted + (size_t)cls * (N * N) + g * N;
    float2 x[R];
    {  // exit wave of row g, columns t + G m (Ptychography.swift:321-336)
        const float2 *orow = a.object + (size_t)lwrap(rr + corner_offset(g, N), a.object_rows) * a.object_columns;
#pragma unroll
        for (int m = 0; m < R; m++) {
            const int col = t + G * m;
            x[m] = lmul(Sp[col], orow[lwrap(cc + corner_offset(col, N), a.object_columns)]);
        }
    }
    __syncthreads();  // the twiddle table
    float2 *own = tile + g * P;
    line_forward<N, G>(x, t, tw, own);
#pragma unroll
    for (int j = 0; j < Q; j++)
#pragma unroll
        for (int s = 0; s < G; s++) own[t * Q + j + R * s] = x[j * G + s];
    __syncthreads();
#pragma unroll
    for (int m = 0; m < R; m++) x[m] = tile[(t + G * m) * P + g];
    __syncthreads();  // every column is read before the rows serve as scratch
    line_forward<N, G>(x, t, tw, own);
    // projection (Ptychography.swift:338-349): x[j G + s] = F[kr = t Q + j + R s][kc = g]; the 1/n of ifft2 folded in
    const float *A = a.amplitudes + (size_t)p * (N * N) + g;
    const float inv_n = a.inv_n;
    double err = 0;
#pragma unroll
    for (int j = 0; j < Q; j++)
#pragma unroll
        for (int s = 0; s < G; s++) {
            float2 &f = x[j * G + s];
            const float measured = A[(t * Q + j + R * s) * N];
            const float mag = sqrtf(f.x * f.x + f.y * f.y);
            const float miss = measured - mag;
            err += (double)(miss * miss);
            if (mag > 0.f) {
                const float sc = (measured / mag - 1.0f) * inv_n;
                f = make_float2(f.x * sc, f.y * sc);
            } else {
                f = make_float2(measured * inv_n, 0.f);
            }
        }
    line_inverse<N, G>(x, t, tw, own);
    __syncthreads();  // every group is done with its scratch row
#pragma unroll
    for (int m = 0; m < R; m++) tile[(t + G * m) * P + g] = x[m];
    __syncthreads();
#pragma unroll
    for (int j = 0; j < Q; j++)
#pragma unroll
        for (int s = 0; s < G; s++) x[j * G + s] = own[t * Q + j + R * s];
    __syncwarp();  // the group's row is read before it serves as scratch
    line_inverse<N, G>(x, t, tw, own);
    float2 *out = a.dpsi + (size_t)p * (N * N) + g * N;
#pragma unroll
    for (int m = 0; m < R; m++) out[t + G * m] = x[m];
    // the per-position squared residual, summed over the CTA in a fixed order
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) err += __shfl_down_sync(0xffffffffu, err, o);
    if ((tid & 31) == 0) scratch[tid >> 5] = err;
    __syncthreads();
    if (tid == 0) {
        double total = 0;
        for (int w = 0; w < NT / 32; w++) total += scratch[w];
        a.error[p] = total;
    }
}

template <int N, int G, int MINB>
__global__ void __launch_bounds__(N * G, MINB) line_pass_kernel(PositionPassArgs<float> a) {
    line_pass_body<N, G>(a, a.first + blockIdx.x);
}

// The item of a grouped launch that unit u belongs to: prefix[i] .. prefix[i + 1] - 1 are item i's units.
__device__ __forceinline__ int line_group_item(const int *prefix, int items, int u) {
    int lo = 0, hi = items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= u) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Grouped form (batches): one CTA per (item, position) unit over every item with this detector.
template <int N, int G, int MINB>
__global__ void __launch_bounds__(N * G, MINB) line_pass_grouped_kernel(const PositionPassArgs<float> *args,
                                                                        const int *prefix, int items, int total) {
    const int u = blockIdx.x;
    const int it = line_group_item(prefix, items, u);
    const PositionPassArgs<float> a = args[it];
    line_pass_body<N, G>(a, a.first + (u - prefix[it]));
}

// The instances: 96 x 96 (G = 4, R = 24, 384 threads), 64 x 64 (G = 8, R = 8, 512 threads), two CTAs per SM each.
// 96 x 96 at one CTA per SM (115 registers, no spill) took 0.83 ms per pass of 3,600 positions; at two (80 registers,
// ~200 bytes of spill) 0.58 ms, against 0.78 ms for the best shared-memory shape.
struct Line96 {
    static constexpr int N = 96, G = 4, MINB = 2;
};
struct Line64 {
    static constexpr int N = 64, G = 8, MINB = 2;
};

template <typename L>
size_t line_smem() {
    return (size_t)(L::N * LineShape<L::N, L::G>::kPitch + L::N) * sizeof(float2) + 32 * sizeof(double);
}

template <typename L>
cudaError_t launch_line(const PositionPassArgs<float> &a, cudaStream_t s) {
    line_pass_kernel<L::N, L::G, L::MINB><<<a.count, L::N * L::G, line_smem<L>(), s>>>(a);
    return cudaGetLastError();
}

template <typename L>
cudaError_t launch_line_grouped(const PositionPassArgs<float> *args, const int *prefix, int items, int total,
                                cudaStream_t s) {
    line_pass_grouped_kernel<L::N, L::G, L::MINB><<<total, L::N * L::G, line_smem<L>(), s>>>(args, prefix, items,
                                                                                            total);
    return cudaGetLastError();
}

}  // namespace

bool line_pass_applicable(int rows, int columns) { return rows == columns && (rows == 64 || rows == 96); }

cudaError_t configure_line_pass() {
    cudaError_t e = cudaFuncSetAttribute(line_pass_kernel<96, 4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)line_smem<Line96>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(line_pass_grouped_kernel<96, 4, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)line_smem<Line96>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(line_pass_kernel<64, 8, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)line_smem<Line64>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(line_pass_grouped_kernel<64, 8, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)line_smem<Line64>());
    return e;
}

cudaError_t launch_line_pass(const PositionPassArgs<float> &a, cudaStream_t s) {
    if (a.count <= 0) return cudaSuccess;
    if (a.rows == 96 && a.columns == 96) return launch_line<Line96>(a, s);
    if (a.rows == 64 && a.columns == 64) return launch_line<Line64>(a, s);
    return cudaErrorInvalidValue;
}

cudaError_t launch_line_pass_grouped(const PositionPassArgs<float> *args, const int *prefix, int items, int total, int N,
                                     cudaStream_t s) {
    if (total <= 0) return cudaSuccess;
    if (N == 96) return launch_line_grouped<Line96>(args, prefix, items, total, s);
    if (N == 64) return launch_line_grouped<Line64>(args, prefix, items, total, s);
    return cudaErrorInvalidValue;
}

}  // namespace cubo
