// Generic per-iteration kernels of the single-slice gradient descent, for any detector size (FP32 and FP64 forms).
//
// One iteration of SingleslicePtychography.reconstruct (Sources/CuboPtycho/Ptychography.swift:280-402) becomes:
//   position pass   one CTA per scan position: exit wave S * O[patch] (:321-336), forward FFT (:337), Fourier-modulus
//                   projection and squared residual (:338-349), inverse FFT with its 1/n folded into the projection
//                   (:350); writes dpsi and the position's residual.
//   object gather   one thread per object pixel: the sum over the positions whose window covers the pixel, in ascending
//                   position order, of conj(S) dpsi and |S|^2 (the scatter-add of :351-355 turned into a gather, so
//                   no atomics and a fixed summation order: bitwise reproducible).
//   probe gather    per detector pixel and position group: sum of conj(O[patch]) dpsi and |O|^2 (:356-357); the groups
//                   are summed in a fixed order by probe reduce (FP64).
//   max / update    the global maxima (:362) and the normalised object update with the amplitude cap (:363-382).
//   error reduce    FP64 fixed-order sum of the per-position residuals divided by the normalisation (:400).
#include <cfloat>

#include <algorithm>
#include <type_traits>

#include "engine.h"

namespace cubo {

namespace {

constexpr int kPassThreads = 512;
constexpr int kMaxNFloat = 16384;   // 128 x 128 complex64 = 128 KB of shared memory
constexpr int kMaxNDouble = 12288;  // 12288 complex128 = 192 KB

template <typename T> struct PassConfig;
template <> struct PassConfig<float> { static constexpr int maxn = kMaxNFloat; };
template <> struct PassConfig<double> { static constexpr int maxn = kMaxNDouble; };

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Fixed-order CTA sum: warps reduce by shuffles, then thread 0 adds the warp sums in warp order.
template <int NT>
__device__ double block_sum(double v, double *scratch) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double total = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < NT / 32; w++) total += scratch[w];
    __syncthreads();
    return total;  // valid in thread 0
}

template <int NT>
__device__ double block_max(double v, double *scratch) {
    v = warp_max(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double m = -DBL_MAX;
    if (threadIdx.x == 0)
        for (int w = 0; w < NT / 32; w++) m = fmax(m, scratch[w]);
    __syncthreads();
    return m;
}

__device__ __forceinline__ int wrap_once(int v, int size) { return v < 0 ? v + size : (v >= size ? v - size : v); }

// ------------------------------------------------------------------------------------------------ position pass

// N > 0: an N x N detector with the radix plan (R0, R1, R2) fixed at compile time (the plan factor_length gives N, so the
// stages and their arithmetic are the run-time plan's), sized for N x N: no run-time dispatch, no stack frame, and
// MINB CTAs of NT threads per SM.  N = 0: any size up to MAXN, the plan read at run time.
template <typename T, int NT, int MAXN, int N, int R0, int R1, int R2>
__device__ __forceinline__ void position_pass_body(const PositionPassArgs<T> &a, int p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C2<T> *D = reinterpret_cast<C2<T> *>(smem_raw);
    C2<T> *twr = D + a.n;
    C2<T> *twc = twr + a.rows;
    double *scratch = reinterpret_cast<double *>(twc + a.columns);
    const int tid = threadIdx.x;
    for (int i = tid; i < a.rows; i += NT) twr[i] = a.tw_rows[i];
    for (int i = tid; i < a.columns; i += NT) twc[i] = a.tw_columns[i];
    const int rr = a.scan.rr[p], cc = a.scan.cc[p], cls = a.scan.cls[p];
    const C2<T> *S = a.shifted + (size_t)cls * a.n;
    // exit wave psi = S * O[patch] (Ptychography.swift:321-336)
    for (int k = tid; k < a.n; k += NT) {
        const int kr = k / a.columns, kc = k - kr * a.columns;
        const int y = wrap_once(rr + corner_offset(kr, a.rows), a.object_rows);
        const int x = wrap_once(cc + corner_offset(kc, a.columns), a.object_columns);
        D[k] = cmul(S[k], a.object[(size_t)y * a.object_columns + x]);
    }
    __syncthreads();
    if constexpr (N > 0) {
        line_fft_fixed<T, NT, MAXN, R0, R1, R2>(D, LineGeom{N, N, 1, N}, twc, false);
        line_fft_fixed<T, NT, MAXN, R0, R1, R2>(D, LineGeom{N, N, N, 1}, twr, false);
    } else {
        fft2_smem<T, NT, MAXN>(D, a.rows, a.columns, a.rad_rows, a.rad_columns, twr, twc, false);
    }
    // Fourier-modulus projection (Ptychography.swift:338-349), the inverse's 1/n folded in
    const float *A = a.amplitudes + (size_t)p * a.n;
    double err = 0;
    for (int k = tid; k < a.n; k += NT) {
        const C2<T> f = D[k];
        const T mag = sqrt(f.x * f.x + f.y * f.y);
        const T measured = (T)A[k];
        const T miss = measured - mag;
        err += (double)(miss * miss);
        if (mag > (T)0) {
            const T s = (measured / mag - (T)1) * a.inv_n;
            D[k] = mk<T>(f.x * s, f.y * s);
        } else {
            D[k] = mk<T>(measured * a.inv_n, (T)0);
        }
    }
    const double total = block_sum<NT>(err, scratch);
    if (tid == 0) a.error[p] = total;
    __syncthreads();
    if constexpr (N > 0) {
        line_fft_fixed<T, NT, MAXN, R0, R1, R2>(D, LineGeom{N, N, 1, N}, twc, true);
        line_fft_fixed<T, NT, MAXN, R0, R1, R2>(D, LineGeom{N, N, N, 1}, twr, true);
    } else {
        fft2_smem<T, NT, MAXN>(D, a.rows, a.columns, a.rad_rows, a.rad_columns, twr, twc, true);
    }
    C2<T> *out = a.dpsi + (size_t)p * a.n;
    for (int k = tid; k < a.n; k += NT) out[k] = D[k];
}

template <typename T, int NT, int MAXN, int MINB = 1, int N = 0, int R0 = 0, int R1 = 0, int R2 = 0>
__global__ void __launch_bounds__(NT, MINB) position_pass_kernel(PositionPassArgs<T> a) {
    position_pass_body<T, NT, MAXN, N, R0, R1, R2>(a, a.first + blockIdx.x);
}

// The item of a grouped launch that work unit u belongs to: prefix[i] .. prefix[i + 1] - 1 are item i's units.
__device__ __forceinline__ int group_item(const int *prefix, int items, int u) {
    int lo = 0, hi = items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= u) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Grouped position pass: the positions of every item (independent reconstructions with the same detector) in one
// launch, one CTA per (item, position) unit.  Every position's arithmetic is the one-launch kernel's.  (A persistent
// form, CTAs walking the work list in a fixed stride, kept the FFT stages' register arrays in local memory: 0.7-1.9 KB
// of stack per thread; one unit per CTA compiles like the one-launch kernel.)
template <typename T, int NT, int MAXN, int MINB, int N, int R0, int R1, int R2>
__global__ void __launch_bounds__(NT, MINB) position_pass_grouped_kernel(const PositionPassArgs<T> *args,
                                                                         const int *prefix, int items, int total) {
    const int u = blockIdx.x;
    const int it = group_item(prefix, items, u);
    const PositionPassArgs<T> a = args[it];
    position_pass_body<T, NT, MAXN, N, R0, R1, R2>(a, a.first + (u - prefix[it]));
}

// FP64 position pass through global memory, for detectors whose FP64 plane does not fit one CTA's shared memory (above
// 12,288 pixels, e.g. 128 x 128): the exit waves are written into dpsi, transformed by the batched line FFT, projected
// in place (the same arithmetic and the same per-position error sum as the shared-memory pass) and transformed back.
__global__ void __launch_bounds__(256) exit_wave_global_kernel(PositionPassArgs<double> a, int m) {
    const long long t = (long long)blockIdx.x * 256 + threadIdx.x;
    if (t >= (long long)m * a.n) return;
    const int i = (int)(t / a.n), k = (int)(t - (long long)i * a.n);
    const int p = a.first + i;
    const int rr = a.scan.rr[p], cc = a.scan.cc[p], cls = a.scan.cls[p];
    const int kr = k / a.columns, kc = k - kr * a.columns;
    const int y = wrap_once(rr + corner_offset(kr, a.rows), a.object_rows);
    const int x = wrap_once(cc + corner_offset(kc, a.columns), a.object_columns);
    a.dpsi[(size_t)p * a.n + k] = cmul(a.shifted[(size_t)cls * a.n + k], a.object[(size_t)y * a.object_columns + x]);
}

template <int NT>
__global__ void __launch_bounds__(NT) project_global_kernel(PositionPassArgs<double> a) {
    __shared__ double scratch[NT / 32];
    const int p = a.first + blockIdx.x;
    double2 *D = a.dpsi + (size_t)p * a.n;
    const float *A = a.amplitudes + (size_t)p * a.n;
    double err = 0;
    for (int k = threadIdx.x; k < a.n; k += NT) {
        const double2 f = D[k];
        const double mag = sqrt(f.x * f.x + f.y * f.y);
        const double measured = (double)A[k];
        const double miss = measured - mag;
        err += miss * miss;
        if (mag > 0.0) {
            const double sc = (measured / mag - 1.0) * a.inv_n;
            D[k] = make_double2(f.x * sc, f.y * sc);
        } else {
            D[k] = make_double2(measured * a.inv_n, 0.0);
        }
    }
    const double total = block_sum<NT>(err, scratch);
    if (threadIdx.x == 0) a.error[p] = total;
}

// ------------------------------------------------------------------------------------------------ object gather

constexpr int kChunk = 256;

constexpr int kGatherChunk = 128;   // candidates whose window offsets are staged at a time
constexpr int kMaxTileSide = 64;    // the longest tile side (tiles are 32 x 8, 16 x 16 or 64 x 4)

// Per object pixel, the sum over the positions covering it (ascending, as listed for its tile) of conj(S) dpsi and
// |S|^2 (Ptychography.swift:351-358 as a gather).  For each chunk of candidates the tile's window offsets are staged
// first: per candidate, the residual row offset kr * columns of each tile row and the residual column kc of each tile
// column (corner-centred, periodic; negative where the window does not reach), so a pixel's residual index is one sum.
// MIXED: the mixed-state form (FP64, several states per candidate), its own instance so that its registers do not
// bound the single-state forms' occupancy.
// The first index in list[lo, hi) (ascending) whose value is at least v (hi if none).
__device__ __forceinline__ int lower_bound_index(const int *list, int lo, int hi, int v) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (list[mid] < v) lo = mid + 1; else hi = mid;
    }
    return lo;
}

template <typename T, bool MIXED>
__device__ __forceinline__ void object_gather_body(const ObjectGatherArgs<T> &a, int unit) {
    __shared__ int s_p[kGatherChunk], s_cls[kGatherChunk];
    __shared__ int s_off[kGatherChunk][kMaxTileSide + kGatherThreads / kMaxTileSide + 4];  // rows, then columns
    __shared__ double scratch[32];
    const int tile = a.band_tiles ? a.band_tiles[unit] : unit;
    const int tx = tile % a.tiles_x, ty = tile / a.tiles_x;
    const int x0 = tx * a.tile_w, y0 = ty * a.tile_h;
    // consecutive threads take consecutive object columns, hence consecutive addresses of each [row][column] residual
    const int lx = threadIdx.x % a.tile_w, ly = threadIdx.x / a.tile_w;
    const int x = x0 + lx, y = y0 + ly;
    const bool inside = x < a.object_columns && y < a.object_rows;
    constexpr int kInvalid = -(1 << 30);
    C2<T> g = mk<T>(0, 0);
    T w = 0;
    const int list_begin = a.tile_start[tile], list_end = a.tile_start[tile + 1];
    int begin = list_begin, end = list_end;
    if (a.band_tiles) {  // this band's candidates only; the running sums continue from memory after the first band
        begin = lower_bound_index(a.tile_list, list_begin, list_end, a.band_first);
        end = lower_bound_index(a.tile_list, begin, list_end, a.band_end);
        if (begin != list_begin && inside) {
            const size_t j = (size_t)y * a.object_columns + x;
            g = a.grad[j];
            w = a.weight[j];
        }
    }
    for (int base = begin; base < end; base += kGatherChunk) {
        const int cnt = min(kGatherChunk, end - base);
        __syncthreads();
        // one candidate per thread: its centre once, then the tile's row and column offsets from it
        for (int i = threadIdx.x; i < cnt; i += kGatherThreads) {
            const int p = a.tile_list[base + i];
            const int rr = a.scan.rr[p], cc = a.scan.cc[p];
            s_p[i] = p;
            s_cls[i] = a.scan.cls[p];
            for (int f = 0; f < a.tile_h; f++) {  // tile row y0 + f
                int dy = y0 + f - rr;
                dy = dy < 0 ? dy + a.object_rows : (dy >= a.object_rows ? dy - a.object_rows : dy);
                const int kr = window_index(dy, a.rows, a.object_rows);
                s_off[i][f] = kr >= 0 ? kr * a.columns : kInvalid;
            }
            for (int f = 0; f < a.tile_w; f++) {  // tile column x0 + f
                int dx = x0 + f - cc;
                dx = dx < 0 ? dx + a.object_columns : (dx >= a.object_columns ? dx - a.object_columns : dx);
                const int kc = window_index(dx, a.columns, a.object_columns);
                s_off[i][a.tile_h + f] = kc >= 0 ? kc : kInvalid;
            }
        }
        __syncthreads();
        if constexpr (MIXED) {
            if (!inside) continue;
            // mixed state: for each candidate in order, its states in order (PtychographyEngines.swift:197-205), four
            // (candidate, state) pairs at a time so that their loads are independent
            const int total = cnt * a.states;
            int i0 = 0, st0 = 0;  // the pair q0 = i0 * states + st0
            for (int q0 = 0; q0 < total; q0 += 4) {
                int k[4], off_d[4], off_s[4];
                int i = i0, st = st0;
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    k[u] = q0 + u < total ? s_off[i][ly] + s_off[i][a.tile_h + lx] : -1;
                    off_d[u] = st;
                    off_s[u] = i;
                    if (++st == a.states) { st = 0; i++; }
                }
                i0 = i;
                st0 = st;
                C2<T> d[4], sv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (k[u] >= 0) {
                        d[u] = a.dpsi[(size_t)off_d[u] * a.dpsi_state_stride + (size_t)s_p[off_s[u]] * a.n + k[u]];
                        sv[u] = a.shifted[(size_t)off_d[u] * a.shifted_state_stride + (size_t)s_cls[off_s[u]] * a.n + k[u]];
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (k[u] >= 0) {
                        g = cadd(g, cmulc(sv[u], d[u]));
                        w += sv[u].x * sv[u].x + sv[u].y * sv[u].y;
                    }
                }
            }
        } else if (inside) {
            // four candidates at a time: their loads are independent, the sums stay in candidate order
            for (int i = 0; i < cnt; i += 4) {
                int k[4];
#pragma unroll
                for (int u = 0; u < 4; u++) k[u] = i + u < cnt ? s_off[i + u][ly] + s_off[i + u][a.tile_h + lx] : -1;
                C2<T> d[4], sv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (k[u] >= 0) {
                        d[u] = a.dpsi[(size_t)(s_p[i + u] - a.band_first) * a.n + k[u]];
                        sv[u] = a.shifted[(size_t)s_cls[i + u] * a.n + k[u]];
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (k[u] >= 0) {
                        g = cadd(g, cmulc(sv[u], d[u]));
                        w += sv[u].x * sv[u].x + sv[u].y * sv[u].y;
                    }
                }
            }
        }
    }
    if (inside) {
        const size_t j = (size_t)y * a.object_columns + x;
        a.grad[j] = g;
        a.weight[j] = w;
    }
    if (end != list_end) return;  // a later band still adds to this tile (uniform over the block)
    const double m = block_max<kGatherThreads>(inside ? (double)w : -DBL_MAX, scratch);
    if (threadIdx.x == 0) a.tile_max[tile] = m;
}

template <typename T, bool MIXED>
__global__ void __launch_bounds__(kGatherThreads) object_gather_kernel(ObjectGatherArgs<T> a) {
    object_gather_body<T, MIXED>(a, blockIdx.x);
}

// Grouped object gather: the tiles of every item in one launch, one CTA per (item, tile) unit.
template <typename T>
__global__ void __launch_bounds__(kGatherThreads) object_gather_grouped_kernel(const ObjectGatherArgs<T> *args,
                                                                               const int *prefix, int items, int total) {
    const int u = blockIdx.x;
    const int it = group_item(prefix, items, u);
    const ObjectGatherArgs<T> a = args[it];
    object_gather_body<T, false>(a, u - prefix[it]);
}

// ------------------------------------------------------------------------------------------------ candidate lists

// Whether the cyclic window [start, start + length) of a periodic axis of `size` meets [t0, t0 + len).
__device__ __forceinline__ bool cyclic_overlap(int start, int length, int t0, int len, int size) {
    int d = (t0 - start) % size;
    if (d < 0) d += size;
    return d < length || d + len > size;
}

// One warp per object-gather tile: the positions whose window touches the tile, in ascending order.  Without `list`
// it counts them into counts[tile]; with it, it writes them from starts[tile] on.  A window covers the object rows
// rr - rows/2 .. rr + (rows+1)/2 - 1 and the columns likewise, wrapped.
__global__ void __launch_bounds__(256) tile_lists_kernel(const int *rr, const int *cc, int count, int rows, int columns,
                                                         int object_rows, int object_columns, int tile_w, int tile_h,
                                                         int tiles_x, int tiles, int *counts, const int *starts,
                                                         int *list, int capacity) {
    const int tile = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (tile >= tiles) return;
    const int ty = tile / tiles_x, tx = tile - ty * tiles_x;
    const int y0 = ty * tile_h, x0 = tx * tile_w;
    const int hy = min(tile_h, object_rows - y0), hx = min(tile_w, object_columns - x0);
    int n = 0;
    const int base = list ? starts[tile] : 0;
    for (int i0 = 0; i0 < count; i0 += 32) {
        const int i = i0 + lane;
        const bool hit = i < count && cyclic_overlap(rr[i] - rows / 2, rows, y0, hy, object_rows) &&
                         cyclic_overlap(cc[i] - columns / 2, columns, x0, hx, object_columns);
        const unsigned ballot = __ballot_sync(0xffffffffu, hit);
        if (list && hit) {
            const int at = base + n + __popc(ballot & ((1u << lane) - 1u));
            if (at < capacity) list[at] = i;  // never past the list (a count beyond it is reported by the scan)
        }
        n += __popc(ballot);
    }
    if (!list && lane == 0) counts[tile] = n;
}

// ------------------------------------------------------------------------------------------------ probe gather

constexpr int kProbeThreads = 256;

// Per detector pixel k and position group, the sum over the group's positions (in order) of conj(O[window]) dpsi and
// |O|^2.  Per chunk of positions the window's object base rr * OC + cc is staged, or -1 where the window wraps around
// the object's edge; an interior window's pixel is then base + (offr * OC + offc), the wrapped ones are computed in full.
template <typename T>
__device__ __forceinline__ void probe_gather_body(const ProbeGatherArgs<T> &a, int block, int group) {
    __shared__ int s_rr[kChunk], s_cc[kChunk];
    __shared__ long long s_base[kChunk];
    const int k = block * kProbeThreads + threadIdx.x;  // pixel index, [row][column]
    const int p0 = a.first + (int)((long long)a.count * group / a.groups);
    const int p1 = a.first + (int)((long long)a.count * (group + 1) / a.groups);
    const bool valid = k < a.n;
    const int kr = valid ? k / a.columns : 0, kc = valid ? k - kr * a.columns : 0;
    const int offr = corner_offset(kr, a.rows), offc = corner_offset(kc, a.columns);
    const long long shift = (long long)offr * a.object_columns + offc;
    // the window [rr - low_r, rr + high_r) x [cc - low_c, cc + high_c) stays inside the object
    const int low_r = a.rows / 2, high_r = (a.rows + 1) / 2, low_c = a.columns / 2, high_c = (a.columns + 1) / 2;
    C2<T> g = mk<T>(0, 0);
    T w = 0;
    if (a.accumulate && valid) {  // continue the group's sums over the earlier bands
        g = a.partial_grad[(size_t)group * a.n + k];
        w = a.partial_weight[(size_t)group * a.n + k];
    }
    for (int base = p0; base < p1; base += kChunk) {
        const int cnt = min(kChunk, p1 - base);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += kProbeThreads) {
            const int rr = a.scan.rr[base + i], cc = a.scan.cc[base + i];
            s_rr[i] = rr;
            s_cc[i] = cc;
            const bool interior = rr >= low_r && rr + high_r <= a.object_rows && cc >= low_c && cc + high_c <= a.object_columns;
            s_base[i] = interior ? (long long)rr * a.object_columns + cc : -1;
        }
        __syncthreads();
        if (valid) {
            const C2<T> *dp = a.dpsi + (size_t)(base - a.first) * a.n + k;
            // four positions at a time: independent loads, sums in position order
            for (int i = 0; i < cnt; i += 4) {
                C2<T> o[4], d[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (i + u < cnt) {
                        const long long b0 = s_base[i + u];
                        long long idx;
                        if (b0 >= 0) {
                            idx = b0 + shift;
                        } else {
                            const int y = wrap_once(s_rr[i + u] + offr, a.object_rows);
                            const int x = wrap_once(s_cc[i + u] + offc, a.object_columns);
                            idx = (long long)y * a.object_columns + x;
                        }
                        o[u] = a.object[idx];
                        d[u] = dp[(size_t)(i + u) * a.n];
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (i + u < cnt) {
                        g = cadd(g, cmulc(o[u], d[u]));
                        w += o[u].x * o[u].x + o[u].y * o[u].y;
                    }
                }
            }
        }
    }
    if (valid) {
        a.partial_grad[(size_t)group * a.n + k] = g;
        a.partial_weight[(size_t)group * a.n + k] = w;
    }
}

template <typename T>
__global__ void __launch_bounds__(kProbeThreads) probe_gather_kernel(ProbeGatherArgs<T> a) {
    probe_gather_body<T>(a, blockIdx.x, blockIdx.y);
}

// Grouped probe gather: every item's (pixel block, position group) units in one launch, one CTA per unit.
template <typename T>
__global__ void __launch_bounds__(kProbeThreads) probe_gather_grouped_kernel(const ProbeGatherArgs<T> *args,
                                                                             const int *prefix, int items, int total) {
    const int u = blockIdx.x;
    const int it = group_item(prefix, items, u);
    const ProbeGatherArgs<T> a = args[it];
    const int blocks = (a.n + kProbeThreads - 1) / kProbeThreads, v = u - prefix[it];
    probe_gather_body<T>(a, v % blocks, v / blocks);
}

template <typename T>
__global__ void __launch_bounds__(256) probe_reduce_kernel(const C2<T> *pg, const T *pw, int groups, int n,
                                                           double2 *grad, double *weight, double *block_max_out) {
    __shared__ double scratch[32];
    const int k = blockIdx.x * 256 + threadIdx.x;
    double gx = 0, gy = 0, w = 0;
    if (k < n) {
        for (int g = 0; g < groups; g++) {
            const C2<T> v = pg[(size_t)g * n + k];
            gx += (double)v.x; gy += (double)v.y; w += (double)pw[(size_t)g * n + k];
        }
        grad[k] = make_double2(gx, gy);
        weight[k] = w;
    }
    const double m = block_max<256>(k < n ? w : -DBL_MAX, scratch);
    if (threadIdx.x == 0) block_max_out[blockIdx.x] = m;
}

template <typename V>
__global__ void __launch_bounds__(1024) max_reduce_kernel(const V *v, long long count, double *out) {
    __shared__ double scratch[32];
    double m = -DBL_MAX;
    for (long long i = threadIdx.x; i < count; i += 1024) m = fmax(m, (double)v[i]);
    m = block_max<1024>(m, scratch);
    if (threadIdx.x == 0) *out = m;
}

// Ptychography.swift:362-370,378-382: O += step / sqrt(1e-16 + ((1 - m) w)^2 + (m max w)^2) * grad, then the cap.
// Ptychography.swift:378-381: |object| <= 1 (or = 1 for a pure-phase object); a zero sample becomes the target.
template <typename T>
__device__ __forceinline__ void object_cap(C2<T> &o, int pure_phase) {
    const T amp = sqrt(o.x * o.x + o.y * o.y);
    const T target = pure_phase ? (T)1 : (amp < (T)1 ? amp : (T)1);
    if (amp > (T)0) { const T r = target / amp; o.x *= r; o.y *= r; }
    else { o.x = target; o.y = 0; }
}

template <typename T>
__global__ void __launch_bounds__(256) object_update_kernel(C2<T> *object, const C2<T> *grad, const T *weight,
                                                            int count, const double *max_weight, double step,
                                                            double minimum, int cap, int pure_phase) {
    const int j = blockIdx.x * 256 + threadIdx.x;
    if (j >= count) return;
    const double l = (1 - minimum) * (double)weight[j], x = minimum * *max_weight;
    const T s = (T)(step * (1 / sqrt(1e-16 + l * l + x * x)));
    C2<T> o = object[j];
    const C2<T> g = grad[j];
    o.x += s * g.x; o.y += s * g.y;
    if (cap || pure_phase) object_cap<T>(o, pure_phase);
    object[j] = o;
}

// The cap alone, for position correction, which reads the updated object before it is capped (Ptychography.swift:371-381).
template <typename T>
__global__ void __launch_bounds__(256) object_cap_kernel(C2<T> *object, int count, int pure_phase) {
    const int j = blockIdx.x * 256 + threadIdx.x;
    if (j >= count) return;
    C2<T> o = object[j];
    object_cap<T>(o, pure_phase);
    object[j] = o;
}

constexpr int kErrorBlocks = 256;

// Stage 1: block b sums the fixed slice [b*count/B, (b+1)*count/B) (thread t takes every 1024th element of it, then a
// fixed tree); stage 2 sums the B block sums in order.  No atomics: the same inputs give the same bits.
__global__ void __launch_bounds__(1024) error_partial_kernel(const double *error, long long count, double *block_sums) {
    __shared__ double scratch[32];
    const long long b = count * blockIdx.x / kErrorBlocks, e = count * (blockIdx.x + 1) / kErrorBlocks;
    double s = 0;
    for (long long i = b + threadIdx.x; i < e; i += 1024) s += error[i];
    s = block_sum<1024>(s, scratch);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kErrorBlocks) error_final_kernel(const double *block_sums, double divisor,
                                                                  double *errors, int *iteration) {
    __shared__ double scratch[32];
    const double s = block_sum<kErrorBlocks>(block_sums[threadIdx.x], scratch);
    if (threadIdx.x == 0) {
        const int it = *iteration;
        errors[it] = s / divisor;
        *iteration = it + 1;
    }
}

constexpr int kAmplitudeBlocks = 1024;

// The supplied-amplitude checks of Ptychography.swift:247-259 on the device: every amplitude finite and non-negative
// (*bad = 1 otherwise), and their energy sum A^2 in FP64 (the errors' divisor, :257-259), in the fixed two-level order
// of the error sums: block b takes the slice [b*count/B, (b+1)*count/B), four consecutive values per thread and step.
__global__ void __launch_bounds__(1024) amplitude_partial_kernel(const float *a, long long count, double *block_sums,
                                                                int *bad) {
    __shared__ double scratch[32];
    const long long b = count * blockIdx.x / kAmplitudeBlocks, e = count * (blockIdx.x + 1) / kAmplitudeBlocks;
    double s = 0;
    int flag = 0;
    for (long long i = b + 4 * (long long)threadIdx.x; i < e; i += 4 * 1024) {
        float v[4];
        if (i + 4 <= e && (((uintptr_t)(a + i)) & 15) == 0) {
            const float4 q = *reinterpret_cast<const float4 *>(a + i);
            v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
        } else {
#pragma unroll
            for (int k = 0; k < 4; k++) v[k] = i + k < e ? a[i + k] : 0.f;
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (!(v[k] >= 0.f && v[k] <= FLT_MAX)) flag = 1;
            s += (double)v[k] * (double)v[k];
        }
    }
    s = block_sum<1024>(s, scratch);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = s;
    if (flag) *bad = 1;
}

__global__ void __launch_bounds__(1024) amplitude_final_kernel(const double *block_sums, double *energy) {
    __shared__ double scratch[32];
    const double s = block_sum<1024>(block_sums[threadIdx.x], scratch);
    if (threadIdx.x == 0) *energy = s;
}

template <typename T>
size_t pass_smem(int n, int rows, int columns) {
    return (size_t)(n + rows + columns) * sizeof(C2<T>) + 32 * sizeof(double);
}

// The fixed-plan instances of the shared-memory position pass: 64 x 64 (8 * 8) and 96 x 96 (8 * 4 * 3), the square
// detectors below 128 x 128 that the run-time plan serves with one 512-thread CTA per SM and a local-memory stack frame
// (its per-stage register arrays are sized for 128 x 128).  Each comes in CTA shapes (cubo_ptycho_params.pass_shape:
// 1 = 128, 2 = 256, 3 = 512 threads; 0 = the default) with as many CTAs per SM as registers and shared memory allow.
// 96 x 96 at 128 threads would spill its stage arrays and takes 256; the FP64 96 x 96 plane (147 KB) fits one CTA per
// SM and takes 512 threads whatever the shape.
template <typename T, int N, int NT> struct FixedShape;
template <typename T> struct FixedShape<T, 64, 128> {
    static auto kernel() { return position_pass_kernel<T, 128, 64 * 64, sizeof(T) == 8 ? 3 : 6, 64, 8, 8, 0>; }
    static auto grouped() { return position_pass_grouped_kernel<T, 128, 64 * 64, sizeof(T) == 8 ? 3 : 6, 64, 8, 8, 0>; }
};
template <typename T> struct FixedShape<T, 64, 256> {
    static auto kernel() { return position_pass_kernel<T, 256, 64 * 64, 3, 64, 8, 8, 0>; }
    static auto grouped() { return position_pass_grouped_kernel<T, 256, 64 * 64, 3, 64, 8, 8, 0>; }
};
template <typename T> struct FixedShape<T, 64, 512> {
    static auto kernel() { return position_pass_kernel<T, 512, 64 * 64, 1, 64, 8, 8, 0>; }
    static auto grouped() { return position_pass_grouped_kernel<T, 512, 64 * 64, 1, 64, 8, 8, 0>; }
};
template <typename T> struct FixedShape<T, 96, 256> {
    static auto kernel() { return position_pass_kernel<T, 256, 96 * 96, 2, 96, 8, 4, 3>; }
    static auto grouped() { return position_pass_grouped_kernel<T, 256, 96 * 96, 2, 96, 8, 4, 3>; }
};
template <typename T> struct FixedShape<T, 96, 512> {
    static auto kernel() { return position_pass_kernel<T, 512, 96 * 96, 1, 96, 8, 4, 3>; }
    static auto grouped() { return position_pass_grouped_kernel<T, 512, 96 * 96, 1, 96, 8, 4, 3>; }
};

// The threads per CTA of the fixed-plan pass for detector side N and shape (0: default), or 0 when N has none.
template <typename T>
int fixed_threads(int N, int shape) {
    if (N == 64) return shape == 1 ? 128 : shape == 3 ? 512 : 256;
    if (N == 96) return sizeof(T) == 8 || shape == 3 ? 512 : 256;
    return 0;
}

template <typename T>
void (*fixed_kernel(int N, int threads))(PositionPassArgs<T>) {
    if (N == 64) return threads == 128 ? FixedShape<T, 64, 128>::kernel()
                      : threads == 512 ? FixedShape<T, 64, 512>::kernel() : FixedShape<T, 64, 256>::kernel();
    return threads == 512 ? FixedShape<T, 96, 512>::kernel() : FixedShape<T, 96, 256>::kernel();
}

template <typename T>
void (*fixed_grouped_kernel(int N, int threads))(const PositionPassArgs<T> *, const int *, int, int) {
    if (N == 64) return threads == 128 ? FixedShape<T, 64, 128>::grouped()
                      : threads == 512 ? FixedShape<T, 64, 512>::grouped() : FixedShape<T, 64, 256>::grouped();
    return threads == 512 ? FixedShape<T, 96, 512>::grouped() : FixedShape<T, 96, 256>::grouped();
}

}  // namespace

bool position_pass_supported(int n, bool fp64) {
    return fp64 ? n <= kMaxNDouble : n <= kMaxNFloat;
}

// Raises the dynamic shared-memory limit of the position-pass kernels to the device's opt-in maximum.  Per device: the
// plan calls it with its device current.
cudaError_t configure_kernels() {
    int device = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(position_pass_kernel<float, kPassThreads, kMaxNFloat>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(position_pass_kernel<double, kPassThreads, kMaxNDouble>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    if (e != cudaSuccess) return e;
    for (int N : {64, 96})
        for (int threads : {128, 256, 512}) {
            e = cudaFuncSetAttribute(fixed_kernel<float>(N, threads), cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(fixed_kernel<double>(N, threads), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         optin);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(fixed_grouped_kernel<float>(N, threads),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(fixed_grouped_kernel<double>(N, threads),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
            if (e != cudaSuccess) return e;
        }
    return configure_line_pass();
}

size_t position_pass_smem(int n, int rows, int columns, bool fp64) {
    return fp64 ? pass_smem<double>(n, rows, columns) : pass_smem<float>(n, rows, columns);
}

cudaError_t launch_project_global(const PositionPassArgs<double> &a, cudaStream_t s) {
    if (a.count <= 0) return cudaSuccess;
    project_global_kernel<kPassThreads><<<a.count, kPassThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_position_pass_global(const PositionPassArgs<double> &a, const Fft2Plan64 &fft, int *launches,
                                       cudaStream_t s) {
    const int chunk = (int)std::max<long long>(1, (1LL << 28) / a.n);  // at most 4 GiB of exit waves per round
    int count = 0;
    for (int first = 0; first < a.count; first += chunk) {
        PositionPassArgs<double> b = a;
        b.first = a.first + first;
        const int m = std::min(chunk, a.count - first);
        const long long total = (long long)m * a.n;
        exit_wave_global_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(b, m);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = launch_fft2_f64(fft, b.dpsi + (size_t)b.first * a.n, m, false, s);
        if (e == cudaSuccess) {
            project_global_kernel<kPassThreads><<<m, kPassThreads, 0, s>>>(b);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = launch_fft2_f64(fft, b.dpsi + (size_t)b.first * a.n, m, true, s);
        if (e != cudaSuccess) return e;
        count += 6;
    }
    if (launches) *launches = count;
    return cudaSuccess;
}

template <typename T>
cudaError_t launch_position_pass(const PositionPassArgs<T> &a, int shape, cudaStream_t s) {
    constexpr int maxn = PassConfig<T>::maxn;
    if (a.count <= 0) return cudaSuccess;
    if constexpr (std::is_same<T, float>::value)
        if (shape == 0 && line_pass_applicable(a.rows, a.columns)) return launch_line_pass(a, s);
    const size_t smem = pass_smem<T>(a.n, a.rows, a.columns);
    const int threads = a.rows == a.columns ? fixed_threads<T>(a.rows, shape) : 0;
    if (threads > 0)
        fixed_kernel<T>(a.rows, threads)<<<a.count, threads, smem, s>>>(a);
    else
        position_pass_kernel<T, kPassThreads, maxn><<<a.count, kPassThreads, smem, s>>>(a);
    return cudaGetLastError();
}

bool position_pass_groupable(int rows, int columns, bool fp64) {
    return rows == columns && (fp64 ? fixed_threads<double>(rows, 0) : fixed_threads<float>(rows, 0)) > 0;
}

template <typename T>
cudaError_t launch_position_pass_grouped(const PositionPassArgs<T> *args, const int *prefix, int items, int total,
                                         int N, int shape, cudaStream_t s) {
    if (total <= 0) return cudaSuccess;
    if constexpr (std::is_same<T, float>::value)
        if (shape == 0 && line_pass_applicable(N, N)) return launch_line_pass_grouped(args, prefix, items, total, N, s);
    const int threads = fixed_threads<T>(N, shape);
    if (threads == 0) return cudaErrorInvalidValue;
    const size_t smem = pass_smem<T>(N * N, N, N);
    fixed_grouped_kernel<T>(N, threads)<<<total, threads, smem, s>>>(args, prefix, items, total);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_object_gather_grouped(const ObjectGatherArgs<T> *args, const int *prefix, int items, int total,
                                         cudaStream_t s) {
    if (total <= 0) return cudaSuccess;
    object_gather_grouped_kernel<T><<<total, kGatherThreads, 0, s>>>(args, prefix, items, total);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_probe_gather_grouped(const ProbeGatherArgs<T> *args, const int *prefix, int items, int total,
                                        cudaStream_t s) {
    if (total <= 0) return cudaSuccess;
    probe_gather_grouped_kernel<T><<<total, kProbeThreads, 0, s>>>(args, prefix, items, total);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_object_gather(const ObjectGatherArgs<T> &a, int tiles, cudaStream_t s) {
    if constexpr (std::is_same<T, double>::value) {
        if (a.states > 1) {  // the mixed-state form exists in FP64 only
            object_gather_kernel<T, true><<<tiles, kGatherThreads, 0, s>>>(a);
            return cudaGetLastError();
        }
    }
    object_gather_kernel<T, false><<<tiles, kGatherThreads, 0, s>>>(a);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_probe_gather(const ProbeGatherArgs<T> &a, cudaStream_t s) {
    dim3 grid((a.n + kProbeThreads - 1) / kProbeThreads, a.groups);
    probe_gather_kernel<T><<<grid, kProbeThreads, 0, s>>>(a);
    return cudaGetLastError();
}

template <typename T>
int probe_gather_resident_ctas() {
    int ctas = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ctas, probe_gather_kernel<T>, kProbeThreads, 0) != cudaSuccess) {
        (void)cudaGetLastError();
        ctas = 0;
    }
    return ctas > 0 ? ctas : 1;
}

template <typename T>
cudaError_t launch_probe_reduce(const C2<T> *pg, const T *pw, int groups, int n, double2 *grad, double *weight,
                                double *block_max_out, cudaStream_t s) {
    probe_reduce_kernel<T><<<(n + 255) / 256, 256, 0, s>>>(pg, pw, groups, n, grad, weight, block_max_out);
    return cudaGetLastError();
}

cudaError_t launch_max_reduce(const double *values, int count, double *out, cudaStream_t s) {
    max_reduce_kernel<double><<<1, 1024, 0, s>>>(values, count, out);
    return cudaGetLastError();
}

template <typename V>
cudaError_t launch_max_values(const V *values, long long count, double *out, cudaStream_t s) {
    max_reduce_kernel<V><<<1, 1024, 0, s>>>(values, count, out);
    return cudaGetLastError();
}
template cudaError_t launch_max_values<float>(const float *, long long, double *, cudaStream_t);
template cudaError_t launch_max_values<double>(const double *, long long, double *, cudaStream_t);

template <typename T>
cudaError_t launch_object_update(C2<T> *object, const C2<T> *grad, const T *weight, int count, const double *max_weight,
                                 double step, double minimum, int cap, int pure_phase, cudaStream_t s) {
    object_update_kernel<T><<<(count + 255) / 256, 256, 0, s>>>(object, grad, weight, count, max_weight, step, minimum,
                                                                 cap, pure_phase);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_object_cap(C2<T> *object, int count, int pure_phase, cudaStream_t s) {
    object_cap_kernel<T><<<(count + 255) / 256, 256, 0, s>>>(object, count, pure_phase);
    return cudaGetLastError();
}

int error_reduce_scratch() { return kErrorBlocks; }

cudaError_t launch_tile_lists(const int *rr, const int *cc, int count, int rows, int columns, int object_rows,
                              int object_columns, int tile_w, int tile_h, int tiles_x, int tiles, int *counts,
                              const int *starts, int *list, int capacity, cudaStream_t s) {
    tile_lists_kernel<<<(tiles + 7) / 8, 256, 0, s>>>(rr, cc, count, rows, columns, object_rows, object_columns, tile_w,
                                                      tile_h, tiles_x, tiles, counts, starts, list, capacity);
    return cudaGetLastError();
}

int amplitude_check_scratch() { return kAmplitudeBlocks + 1; }

cudaError_t launch_amplitude_check(const float *amplitudes, long long count, double *scratch, int *bad, cudaStream_t s) {
    amplitude_partial_kernel<<<kAmplitudeBlocks, 1024, 0, s>>>(amplitudes, count, scratch, bad);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    amplitude_final_kernel<<<1, kAmplitudeBlocks, 0, s>>>(scratch, scratch + kAmplitudeBlocks);
    return cudaGetLastError();
}

cudaError_t launch_error_reduce(const double *error, long long count, double divisor, double *errors, int *iteration,
                                double *scratch, cudaStream_t s) {
    error_partial_kernel<<<kErrorBlocks, 1024, 0, s>>>(error, count, scratch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    error_final_kernel<<<1, kErrorBlocks, 0, s>>>(scratch, divisor, errors, iteration);
    return cudaGetLastError();
}

#define INSTANTIATE(T)                                                                                                 \
    template cudaError_t launch_position_pass<T>(const PositionPassArgs<T> &, int, cudaStream_t);                      \
    template cudaError_t launch_position_pass_grouped<T>(const PositionPassArgs<T> *, const int *, int, int, int, int,   \
                                                         cudaStream_t);                                              \
    template cudaError_t launch_object_gather_grouped<T>(const ObjectGatherArgs<T> *, const int *, int, int,          \
                                                         cudaStream_t);                                              \
    template cudaError_t launch_probe_gather_grouped<T>(const ProbeGatherArgs<T> *, const int *, int, int,            \
                                                        cudaStream_t);                                               \
    template cudaError_t launch_object_gather<T>(const ObjectGatherArgs<T> &, int, cudaStream_t);                      \
    template cudaError_t launch_probe_gather<T>(const ProbeGatherArgs<T> &, cudaStream_t);                             \
    template int probe_gather_resident_ctas<T>();                                                                      \
    template cudaError_t launch_probe_reduce<T>(const C2<T> *, const T *, int, int, double2 *, double *, double *,     \
                                                cudaStream_t);                                                         \
    template cudaError_t launch_object_update<T>(C2<T> *, const C2<T> *, const T *, int, const double *, double,       \
                                                 double, int, int, cudaStream_t);                                      \
    template cudaError_t launch_object_cap<T>(C2<T> *, int, int, cudaStream_t);
INSTANTIATE(float)
INSTANTIATE(double)

}  // namespace cubo
