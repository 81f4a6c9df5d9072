// The FP32 position pass for detectors whose plane does not fit one CTA's shared memory (more than 16,384 pixels, sides
// up to 4096, e.g. 256 x 256), or any detector with CUBO_PTYCHO_VARIANT_GLOBAL.
//
// Same arithmetic as the shared-memory pass (exit wave, forward 2-D FFT, Fourier-modulus projection with the 1/n of
// ifft2 folded in, inverse 2-D FFT; Ptychography.swift:321-350, the Float path PtychographySingle.swift:137-176), in
// three launches per batch of positions, each reading and writing the residual plane once:
//
//  1. rows:    the exit wave X = S O[patch] of nl rows of one position, formed on the way into shared memory, and their
//              forward row transforms, into dpsi;
//  2. columns: nl columns of one position: forward column transforms, the projection and its squared residual (one
//              FP64 partial per CTA, summed over the CTA in a fixed order), inverse column transforms;
//  3. rows:    the inverse row transforms.
//
// The line transforms are the shared-memory Stockham stages of the any-size pass (radices 8/4/2/3/5/7, direct DFT for
// other primes), nl lines of a CTA at a time; nl is the largest divisor of the line count that keeps nl lines within
// kG32MaxN elements, so a CTA never straddles two positions and every partial belongs to one position.  Where the
// lengths keep every address on a 16-byte boundary, the column launch brings its residual columns and amplitudes and
// the inverse row launch its rows into shared memory by asynchronous 16-byte copies, all in flight at once.  The FP64
// form has its own global-memory pass (launch_position_pass_global).
#include "engine.h"

namespace cubo {

namespace {

constexpr int kG32Threads = 256;
constexpr int kG32MaxN = 4096;  // complex64 elements of the lines one CTA holds (32 KB)
// CTAs per SM: 4 for the compile-time plans (64 registers, no spills), 2 for the run-time plan (its per-stage arrays
// spill at either count)

__device__ __forceinline__ int g32_wrap(int v, int size) { return v < 0 ? v + size : (v >= size ? v - size : v); }

// 16-byte asynchronous copy global -> shared (both addresses 16-byte aligned); completes at g32_copies_wait.
__device__ __forceinline__ void g32_copy16(uint32_t smem_dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_dst), "l"(src) : "memory");
}
__device__ __forceinline__ void g32_copies_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// Waits until at most `pending` of this thread's committed groups are still in flight.
template <int pending>
__device__ __forceinline__ void g32_copies_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(pending) : "memory"); }

// Fixed-order sum over the CTA: warps by shuffles, then thread 0 adds the warp sums in warp order.
__device__ double g32_block_sum(double v, double *scratch) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = v;
    __syncthreads();
    double total = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kG32Threads / 32; w++) total += scratch[w];
    __syncthreads();
    return total;  // valid in thread 0
}

// The line transform of the CTA's lines: the radix plan R0 x R1 x R2 fixed at compile time (R1, R2 = 0: no stage; it
// must be the plan factor_length gives the line length), or read at run time (R0 = 0).
template <int R0, int R1, int R2>
__device__ __forceinline__ void g32_lines_fft(float2 *D, const LineGeom &g, const Radices &rad, const float2 *tw,
                                              bool inv) {
    if constexpr (R0 == 0) line_fft<float, kG32Threads, kG32MaxN>(D, g, rad, tw, inv);
    else line_fft_fixed<float, kG32Threads, kG32MaxN, R0, R1, R2>(D, g, tw, inv);
}

// Rows r0 .. r0 + nl - 1 of position p = first + block / (rows / nl): with exit_wave the rows of X = S O[patch] (the
// window corner-centred and periodic in the object), else the rows dpsi holds; transformed along the row (forward, or
// inverse with inv) and written to dpsi.
// NL > 0 (compile-time plans only): nl == NL and the line length is R0 R1 R2, so the line geometry is a compile-time
// constant and the transform's index arithmetic folds.
template <int R0, int R1, int R2, int NL>
__global__ void __launch_bounds__(kG32Threads, R0 ? 4 : 2)
    g32_rows_kernel(PositionPassArgs<float> a, int nl_arg, int exit_wave, int inv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2 *D = reinterpret_cast<float2 *>(smem_raw);
    const int L = NL ? R0 * (R1 ? R1 : 1) * (R2 ? R2 : 1) : a.columns;
    const int nl = NL ? NL : nl_arg;
    float2 *tw = D + (size_t)nl * L;
    for (int i = threadIdx.x; i < L; i += kG32Threads) tw[i] = a.tw_columns[i];
    const int per = a.rows / nl;
    const int p = a.first + (int)(blockIdx.x / per), r0 = (int)(blockIdx.x % per) * nl;
    float2 *rows = a.dpsi + (size_t)p * a.n + (size_t)r0 * L;
    if (exit_wave) {
        const int rr = a.scan.rr[p], cc = a.scan.cc[p], cls = a.scan.cls[p];
        const float2 *S = a.shifted + (size_t)cls * a.n + (size_t)r0 * L;
        for (int i = threadIdx.x; i < nl * L; i += kG32Threads) {
            const int j = i / L, e = i - j * L;
            const int y = g32_wrap(rr + corner_offset(r0 + j, a.rows), a.object_rows);
            const int x = g32_wrap(cc + corner_offset(e, a.columns), a.object_columns);
            D[i] = cmul(S[i], a.object[(size_t)y * a.object_columns + x]);
        }
    } else if ((L & 1) == 0) {  // the rows are contiguous and start on a 16-byte boundary: every copy in flight at once
        const uint32_t d0 = (uint32_t)__cvta_generic_to_shared(D);
        for (int i = threadIdx.x; i < nl * L / 2; i += kG32Threads) g32_copy16(d0 + 16u * (uint32_t)i, rows + 2 * i);
        g32_copies_commit();
        g32_copies_wait<0>();
    } else {
        for (int i = threadIdx.x; i < nl * L; i += kG32Threads) D[i] = rows[i];
    }
    __syncthreads();
    g32_lines_fft<R0, R1, R2>(D, LineGeom{L, nl, 1, L}, a.rad_columns, tw, inv != 0);
    for (int i = threadIdx.x; i < nl * L; i += kG32Threads) rows[i] = D[i];
}

// Columns c0 .. c0 + nl - 1 of position p = first + block / (columns / nl), staged with element e of column j at
// D[e nl + j] (consecutive threads read consecutive columns of one row): forward column transforms, the Fourier-modulus
// projection (Ptychography.swift:338-349) with the inverse's 1/n folded in and its squared residual, inverse column
// transforms.  The residual of the CTA's pixels goes to error[p (columns / nl) + c0 / nl].
template <int R0, int R1, int R2, int NL>
__global__ void __launch_bounds__(kG32Threads, R0 ? 4 : 2) g32_columns_kernel(PositionPassArgs<float> a, int nl_arg) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double scratch[kG32Threads / 32];
    float2 *D = reinterpret_cast<float2 *>(smem_raw);
    const int L = NL ? R0 * (R1 ? R1 : 1) * (R2 ? R2 : 1) : a.rows;
    const int nl = NL ? NL : nl_arg;
    float2 *tw = D + (size_t)nl * L;
    float *As = reinterpret_cast<float *>(tw + L);  // the CTA's amplitudes, staged like D
    for (int i = threadIdx.x; i < L; i += kG32Threads) tw[i] = a.tw_rows[i];
    const int per = a.columns / nl;
    const int p = a.first + (int)(blockIdx.x / per), c0 = (int)(blockIdx.x % per) * nl;
    float2 *base = a.dpsi + (size_t)p * a.n + c0;
    const float *A = a.amplitudes + (size_t)p * a.n + c0;
    // nl and the row length multiples of 4 and the column length even (so every copy's source and destination, the
    // amplitude area As included, start on 16-byte boundaries): the residual columns in pairs and the amplitudes in
    // fours by asynchronous copies, every copy in flight at once; the amplitudes land while the forward transforms run
    const bool staged = (nl & 3) == 0 && (a.columns & 3) == 0 && (L & 1) == 0;
    if (staged) {
        const uint32_t d0 = (uint32_t)__cvta_generic_to_shared(D), a0 = (uint32_t)__cvta_generic_to_shared(As);
        const int pairs = nl / 2, quads = nl / 4;
        for (int i = threadIdx.x; i < pairs * L; i += kG32Threads) {
            const int e = i / pairs, j = 2 * (i - e * pairs);
            g32_copy16(d0 + 8u * (uint32_t)(e * nl + j), base + (size_t)e * a.columns + j);
        }
        g32_copies_commit();
        for (int i = threadIdx.x; i < quads * L; i += kG32Threads) {
            const int e = i / quads, j = 4 * (i - e * quads);
            g32_copy16(a0 + 4u * (uint32_t)(e * nl + j), A + (size_t)e * a.columns + j);
        }
        g32_copies_commit();
        g32_copies_wait<1>();  // the residual columns; the amplitudes may still be in flight
    } else {
        for (int i = threadIdx.x; i < nl * L; i += kG32Threads) {
            const int e = i / nl, j = i - e * nl;
            D[i] = base[(size_t)e * a.columns + j];
            As[i] = A[(size_t)e * a.columns + j];
        }
    }
    __syncthreads();
    const LineGeom geom{L, nl, nl, 1};
    g32_lines_fft<R0, R1, R2>(D, geom, a.rad_rows, tw, false);
    if (staged) {
        g32_copies_wait<0>();
        __syncthreads();
    }
    double err = 0;
    for (int i = threadIdx.x; i < nl * L; i += kG32Threads) {
        const float2 f = D[i];
        const float mag = sqrtf(f.x * f.x + f.y * f.y);
        const float measured = As[i];
        const float miss = measured - mag;
        err += (double)(miss * miss);
        if (mag > 0.f) {
            const float s = (measured / mag - 1.f) * a.inv_n;
            D[i] = make_float2(f.x * s, f.y * s);
        } else {
            D[i] = make_float2(measured * a.inv_n, 0.f);
        }
    }
    const double total = g32_block_sum(err, scratch);  // its barriers also order the projection before the inverse
    if (threadIdx.x == 0) a.error[(size_t)p * per + c0 / nl] = total;
    g32_lines_fft<R0, R1, R2>(D, geom, a.rad_rows, tw, true);
    for (int i = threadIdx.x; i < nl * L; i += kG32Threads) {
        const int e = i / nl, j = i - e * nl;
        base[(size_t)e * a.columns + j] = D[i];
    }
}

// The largest divisor d of `lines` with d line_length <= kG32MaxN: lines per CTA.
int g32_lines(int line_length, int lines) {
    int best = 1;
    for (int d = 1; d <= lines && (long long)d * line_length <= kG32MaxN; d++)
        if (lines % d == 0) best = d;
    return best;
}

// Dynamic shared memory: nl lines and the twiddle table (complex64), and for the columns launch the amplitudes (Float32).
size_t g32_smem(int nl, int line_length, bool amplitudes) {
    return ((size_t)nl * line_length + line_length) * sizeof(float2) +
           (amplitudes ? (size_t)nl * line_length * sizeof(float) : 0);
}

using RowsKernel = void (*)(PositionPassArgs<float>, int, int, int);
using ColumnsKernel = void (*)(PositionPassArgs<float>, int);

// Which compile-time plan `rad` is: 1..4 for lines of 128 (8 8 2), 192 (8 8 3), 256 (8 8 4), 512 (8 8 8), else 0 (the
// run-time plan).
int g32_plan_index(const Radices &rad) {
    auto is = [&](int a, int b, int c) {
        const int want[3] = {a, b, c};
        if (rad.count != 3) return false;
        for (int i = 0; i < 3; i++)
            if (rad.r[i] != want[i]) return false;
        return true;
    };
    return is(8, 8, 2) ? 1 : is(8, 8, 3) ? 2 : is(8, 8, 4) ? 3 : is(8, 8, 8) ? 4 : 0;
}
// The lines per CTA of each plan's folded instance (the largest power of two within kG32MaxN elements).
constexpr int kFoldLines[5] = {0, 32, 16, 16, 8};
RowsKernel rows_instance(int i, bool folded) {
    constexpr RowsKernel k[5] = {g32_rows_kernel<0, 0, 0, 0>, g32_rows_kernel<8, 8, 2, 0>, g32_rows_kernel<8, 8, 3, 0>,
                                 g32_rows_kernel<8, 8, 4, 0>, g32_rows_kernel<8, 8, 8, 0>};
    constexpr RowsKernel f[5] = {g32_rows_kernel<0, 0, 0, 0>, g32_rows_kernel<8, 8, 2, 32>,
                                 g32_rows_kernel<8, 8, 3, 16>, g32_rows_kernel<8, 8, 4, 16>,
                                 g32_rows_kernel<8, 8, 8, 8>};
    return folded ? f[i] : k[i];
}
ColumnsKernel columns_instance(int i, bool folded) {
    constexpr ColumnsKernel k[5] = {g32_columns_kernel<0, 0, 0, 0>, g32_columns_kernel<8, 8, 2, 0>,
                                    g32_columns_kernel<8, 8, 3, 0>, g32_columns_kernel<8, 8, 4, 0>,
                                    g32_columns_kernel<8, 8, 8, 0>};
    constexpr ColumnsKernel f[5] = {g32_columns_kernel<0, 0, 0, 0>, g32_columns_kernel<8, 8, 2, 32>,
                                    g32_columns_kernel<8, 8, 3, 16>, g32_columns_kernel<8, 8, 4, 16>,
                                    g32_columns_kernel<8, 8, 8, 8>};
    return folded ? f[i] : k[i];
}

}  // namespace

bool global32_applicable(int rows, int columns) {
    return rows >= 1 && columns >= 1 && rows <= kG32MaxN && columns <= kG32MaxN;
}

int global32_partials_per_position(int rows, int columns) { return columns / g32_lines(rows, columns); }

cudaError_t configure_global32() {
    // at most kG32MaxN elements and their amplitudes, a twiddle table of at most kG32MaxN
    const int bytes = (int)((kG32MaxN + kG32MaxN) * sizeof(float2) + kG32MaxN * sizeof(float));
    for (int i = 0; i < 5; i++)
        for (bool folded : {false, true}) {
            cudaError_t e = cudaFuncSetAttribute(rows_instance(i, folded), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 bytes);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(columns_instance(i, folded), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         bytes);
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}

cudaError_t launch_position_pass_global32(const PositionPassArgs<float> &a, int *launches, cudaStream_t s) {
    if (launches) *launches = 0;
    if (a.count <= 0) return cudaSuccess;
    if (!global32_applicable(a.rows, a.columns)) return cudaErrorInvalidValue;
    const int nr = g32_lines(a.columns, a.rows), nc = g32_lines(a.rows, a.columns);
    const int per_r = a.rows / nr, per_c = a.columns / nc;
    const size_t smem_r = g32_smem(nr, a.columns, false), smem_c = g32_smem(nc, a.rows, true);
    const int ir = g32_plan_index(a.rad_columns), ic = g32_plan_index(a.rad_rows);  // row lines: length columns
    const RowsKernel rows_k = rows_instance(ir, ir > 0 && nr == kFoldLines[ir]);
    const ColumnsKernel columns_k = columns_instance(ic, ic > 0 && nc == kFoldLines[ic]);
    // batches of positions whose CTAs fit one grid dimension
    const int chunk = (int)std::max<long long>(1, (1LL << 30) / std::max(per_r, per_c));
    int count = 0;
    for (int first = 0; first < a.count; first += chunk) {
        PositionPassArgs<float> b = a;
        b.first = a.first + first;
        const int m = std::min(chunk, a.count - first);
        rows_k<<<(unsigned)((long long)m * per_r), kG32Threads, smem_r, s>>>(b, nr, 1, 0);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) {
            columns_k<<<(unsigned)((long long)m * per_c), kG32Threads, smem_c, s>>>(b, nc);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) {
            rows_k<<<(unsigned)((long long)m * per_r), kG32Threads, smem_r, s>>>(b, nr, 0, 1);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) return e;
        count += 3;
    }
    if (launches) *launches = count;
    return cudaSuccess;
}

}  // namespace cubo
