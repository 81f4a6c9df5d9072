// The 128 x 128 FP64 plane transform: one position's plane through FFT -> a pointwise step -> inverse FFT in ONE
// launch, read once from HBM and written once (or the forward FFT alone, or a pointwise step and the inverse alone).  An FP64 plane of 128 x 128 (256 KB) is larger than one SM's shared
// memory, so a cluster of Q CTAs holds it: each CTA keeps 128 / Q rows in registers (16 complex values per thread,
// eight threads per line), and the row / column redistributions go through distributed shared memory.
//
// Per line of 128 = 16 x 8 (n = j + 8 m, k = k1 + 16 k2), the eight threads j of a line each hold x[j + 8 m]:
//   1. a 16-point DFT over m in registers, then the twiddle W_128^(j k1);
//   2. an 8 x 8 transpose of pairs across the line's eight lanes, through a swizzled per-warp shared-memory scratch;
//   3. 8-point DFTs over j: thread j' then holds X[2 j' + c + 16 k2], c = 0, 1, k2 = 0 .. 7.
// The inverse runs the same steps in the opposite order (from that distribution back to x[j + 8 m]), so the spectrum
// never needs reordering: rows -> columns -> pointwise -> inverse columns -> inverse rows.
//
// The CTA's input rows (contiguous in HBM) arrive by bulk asynchronous copies on an mbarrier; its output rows leave
// the same way.  The pointwise step is either the Fresnel propagator times a scale (multislice propagation, MultislicePtychography,
// PtychographyEngines.swift:503-545) or the modulus projection with the per-position squared error
// (Ptychography.swift:327-349 and PtychographyEngines.swift:516-524).  The input can be multiplied by the object patch
// of the position (or its conjugate) as it is read: the exit wave of the forward model, or chi x conj(O) of the
// backward one.
#include <cooperative_groups.h>

#include <cstdlib>

#include "engine.h"
#include "position_step.cuh"

namespace cg = cooperative_groups;

namespace cubo {

namespace {

constexpr int kSide = 128, kPlane = kSide * kSide;

template <int Q>
struct PlaneGeometry {
    static constexpr int kLines = kSide / Q;            // rows (row passes) or columns (column passes) per CTA
    static constexpr int kThreads = 8 * kLines;         // eight threads per line
    static constexpr int kStrideA = kLines + 1;          // [128 rows][kLines columns] + 1 (conflict-free columns)
    static constexpr int kStrideB = kSide + 1;           // [kLines rows][128 columns] + 1
    static constexpr int kBuffer = (kSide * kStrideA > kLines * kStrideB) ? kSide * kStrideA : kLines * kStrideB;
    static constexpr int kTables = 512;                  // twiddles [k1][j] and [i][c][j], propagator factors
    // staged rows of the CTA's columns, 16-byte rows: amplitudes (floats; full and forward modes) or per-pixel factors
    // (doubles; inverse mode), one region sized for the mode
    static constexpr int kAmpStride = kLines + 4;        // in floats
    static constexpr int kFactorStride = kLines + 2;     // in doubles
    __host__ __device__ static constexpr size_t stage_bytes(int mode) {
        return mode == kPlaneInverse ? (size_t)kSide * kFactorStride * sizeof(double)
                                     : (size_t)kSide * kAmpStride * sizeof(float);
    }
    __host__ __device__ static constexpr size_t smem(int mode) {
        return (size_t)(kBuffer + kTables) * sizeof(double2) + stage_bytes(mode) + (32 + 8 + 2) * sizeof(double);
    }
};

__device__ __forceinline__ int wrap_once(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// 4-point DFT in place (sign -1 forward, +1 when INV, unscaled).
template <bool INV>
__device__ __forceinline__ void dft4(double2 &x0, double2 &x1, double2 &x2, double2 &x3) {
    const double2 a0 = cadd(x0, x2), a1 = csub(x0, x2), b0 = cadd(x1, x3), b1 = cmul_mi(csub(x1, x3), INV);
    x0 = cadd(a0, b0);
    x2 = csub(a0, b0);
    x1 = cadd(a1, b1);
    x3 = csub(a1, b1);
}

// 8-point DFT of x[0..7] in place (radix 2 over two 4-point DFTs).
template <bool INV>
__device__ __forceinline__ void dft8(double2 (&x)[8]) {
    constexpr double h = 0.70710678118654752440;  // 1 / sqrt(2)
    double2 e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6], o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    // W_8^k o_k: k = 1 -> (1 -/+ i) h, k = 2 -> -/+ i, k = 3 -> (-1 -/+ i) h
    const double s = INV ? 1.0 : -1.0;
    const double2 t1 = make_double2((o1.x - s * o1.y) * h, (o1.y + s * o1.x) * h);
    const double2 t2 = cmul_mi(o2, INV);
    const double2 t3 = make_double2((-o3.x - s * o3.y) * h, (-o3.y + s * o3.x) * h);
    x[0] = cadd(e0, o0);
    x[4] = csub(e0, o0);
    x[1] = cadd(e1, t1);
    x[5] = csub(e1, t1);
    x[2] = cadd(e2, t2);
    x[6] = csub(e2, t2);
    x[3] = cadd(e3, t3);
    x[7] = csub(e3, t3);
}

// 16-point DFT of v[0..15] in place (radix 4 x 4).
template <bool INV>
__device__ __forceinline__ void dft16(double2 (&v)[16]) {
    constexpr double c1 = 0.92387953251128675613, s1 = 0.38268343236508977173, h = 0.70710678118654752440;
    const double s = INV ? 1.0 : -1.0;  // sign of the exponent
#pragma unroll
    for (int m1 = 0; m1 < 4; m1++) dft4<INV>(v[m1], v[m1 + 4], v[m1 + 8], v[m1 + 12]);
    // v[m1 + 4 a] *= W_16^(m1 a)
    const double2 w1 = make_double2(c1, s * s1), w2 = make_double2(h, s * h), w3 = make_double2(s1, s * c1);
    const double2 w6 = make_double2(-h, s * h), w9 = make_double2(-c1, -s * s1);
    v[5] = cmul(v[5], w1);
    v[9] = cmul(v[9], w2);
    v[13] = cmul(v[13], w3);
    v[6] = cmul(v[6], w2);
    v[10] = cmul_mi(v[10], INV);
    v[14] = cmul(v[14], w6);
    v[7] = cmul(v[7], w3);
    v[11] = cmul(v[11], w6);
    v[15] = cmul(v[15], w9);
#pragma unroll
    for (int a = 0; a < 4; a++) dft4<INV>(v[4 * a], v[4 * a + 1], v[4 * a + 2], v[4 * a + 3]);
    // X[a + 4 b] sits at v[4 a + b]: transpose the 4 x 4 index
    double2 t[16];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) t[a + 4 * b] = v[4 * a + b];
#pragma unroll
    for (int k = 0; k < 16; k++) v[k] = t[k];
}

// Thread j of line lw (of the warp's four) holds blocks b = 0..7 (pairs v[2b], v[2b+1]); afterwards thread b holds
// what thread j had in block b, in block j.  Through the warp's 512-entry scratch: row lw * 8 + j, column k stored at
// k ^ (j ^ lw) (both the writes and the pair reads take the minimum four wavefronts).
__device__ __forceinline__ void pair_transpose(double2 (&v)[16], int j, int lw, double2 *scratch) {
    double2 *mine = scratch + (lw * 8 + j) * 16;
    const int sw = j ^ lw;
#pragma unroll
    for (int k = 0; k < 16; k++) mine[k ^ sw] = v[k];
    __syncwarp();
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const double2 *row = scratch + (lw * 8 + i) * 16;
        const int si = i ^ lw;
#pragma unroll
        for (int c = 0; c < 2; c++) v[2 * i + c] = row[(2 * j + c) ^ si];
    }
    __syncwarp();
}

// Forward line transform: thread j holds x[j + 8 m] in v[m]; afterwards thread j holds X[2 j + c + 16 k2] in
// v[2 k2 + c].  tf[k1 * 8 + j] = W_128^(j k1).
__device__ __forceinline__ void line_forward(double2 (&v)[16], int j, int lw, const double2 *tf, double2 *scratch) {
    dft16<false>(v);
#pragma unroll
    for (int k1 = 1; k1 < 16; k1++) v[k1] = cmul(v[k1], tf[k1 * 8 + j]);
    pair_transpose(v, j, lw, scratch);
#pragma unroll
    for (int c = 0; c < 2; c++) {
        double2 x[8];
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = v[2 * i + c];
        dft8<false>(x);
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) v[2 * k2 + c] = x[k2];
    }
}

// Inverse line transform (unscaled) from the forward's output distribution back to x[j + 8 m] in v[m].
// ti[(i * 2 + c) * 8 + j] = W_128^(-i (2 j + c)).
__device__ __forceinline__ void line_inverse(double2 (&v)[16], int j, int lw, const double2 *ti, double2 *scratch) {
#pragma unroll
    for (int c = 0; c < 2; c++) {
        double2 x[8];
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) x[k2] = v[2 * k2 + c];
        dft8<true>(x);
        v[c] = x[0];
#pragma unroll
        for (int i = 1; i < 8; i++) v[2 * i + c] = cmul(x[i], ti[(i * 2 + c) * 8 + j]);
    }
    pair_transpose(v, j, lw, scratch);
    dft16<true>(v);
}

__device__ __forceinline__ uint32_t smem_address(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool mbarrier_try_wait(uint64_t *bar, uint32_t phase) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_address(bar)), "r"(phase) : "memory");
    return ok != 0;
}

// The shared::cluster address of `local` (this CTA's shared memory) in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_address(uint32_t local, int rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(local), "r"(rank));
    return out;
}

__device__ __forceinline__ void store_cluster(uint32_t address, double2 v) {
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(address), "d"(v.x), "d"(v.y) : "memory");
}

// Waits for phase 0 of `bar` a bounded number of times; false if it did not complete.
__device__ __forceinline__ bool mbarrier_wait_bounded(uint64_t *bar) {
    for (int i = 0; i < (1 << 22); i++)
        if (mbarrier_try_wait(bar, 0)) return true;
    return false;
}

template <int Q, int MODE>
__global__ void __cluster_dims__(Q, 1, 1) __launch_bounds__(PlaneGeometry<Q>::kThreads, Q / 2)
    plane128_kernel(Plane128Args a) {
    using G = PlaneGeometry<Q>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2 *buf = reinterpret_cast<double2 *>(smem_raw);
    double2 *tf = buf + G::kBuffer;       // [k1][j] W_128^(j k1)
    double2 *ti = tf + 128;               // [i][c][j] W_128^(-i (2 j + c))
    double2 *pr = ti + 128;               // factor of the row frequency (conjugated when asked)
    double2 *pc = pr + 128;               // of the column frequency
    float *amp = reinterpret_cast<float *>(pc + 128);  // [frequency row][kAmpStride]: the CTA's columns
    double *factor = reinterpret_cast<double *>(amp);  // [frequency row][kFactorStride], the same region
    double *warp_err = reinterpret_cast<double *>(reinterpret_cast<char *>(amp) + G::stage_bytes(MODE));  // [32]
    double *cluster_err = warp_err + 32;                                          // [8], rank 0's copy is read
    uint64_t *input_ready = reinterpret_cast<uint64_t *>(cluster_err + 8);
    uint64_t *amp_ready = input_ready + 1;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int p = a.first + (int)(blockIdx.x / Q);
    const int t = threadIdx.x, line = t >> 3, j = t & 7, lw = (t >> 3) & 3;
    double2 *scratch = buf + (t >> 5) * 512;  // the warp's four lines of 128 = its transpose scratch
    const int row = rank * G::kLines + line, column = rank * G::kLines + line;
    const bool project = MODE == kPlaneFull && a.pointwise == kPointwiseProjection;
    const bool solve = MODE == kPlaneForward && a.pointwise == kPointwiseSolve;
    const bool stage_amp = project || solve;  // the amplitudes of the CTA's columns are bulk-copied into amp
    const bool stage_factor = MODE == kPlaneInverse && a.pointwise == kPointwiseFactorPlane;  // or the factors
    const bool factors = MODE != kPlaneForward && a.pointwise == kPointwiseFactors;
    constexpr uint32_t kHalfBytes = G::kLines * kSide * sizeof(double2), kChunk = 16384;
    constexpr uint32_t kAmpRowBytes = G::kLines * sizeof(float), kSpanBytes = G::kLines * sizeof(double2);
    // the input and output planes of position p (computed where used: they would hold registers across the kernel)
    auto in_plane = [&]() -> size_t {
        return (size_t)(a.in_kind == kInputByClass ? a.scan.cls[p] : a.in_kind == kInputSingle ? 0 : p) * kPlane;
    };
    auto out_plane = [&]() -> double2 * { return a.out + (size_t)((long long)p * a.out_stride + a.out_offset) * kPlane; };

    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_address(input_ready)) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_address(amp_ready)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = t; i < 128; i += G::kThreads) {
        const int k1 = i >> 3, jj = i & 7;
        tf[i] = a.tw[(jj * k1) & (kSide - 1)];
        const int ii = i >> 4, c = (i >> 3) & 1;
        ti[i] = cconj(a.tw[(ii * (2 * jj + c)) & (kSide - 1)]);
        if (factors) {
            const size_t off = (size_t)((long long)(p - a.first) * a.prop_stride);
            double2 r = a.prop_rows[off + i], q = a.prop_columns[off + i];
            if (a.conj_prop) { r.y = -r.y; q.y = -q.y; }
            pr[i] = r;
            pc[i] = q;
        }
    }
    __syncthreads();  // the mbarriers are initialised

    // ---- bulk copies.  Full / forward: the CTA's kLines input rows (contiguous) into buf[line][128]; inverse: the
    // spectrum's rows restricted to the CTA's columns into buf[row][kStrideA], one row per thread of the first 128.
    // For the projection, the amplitudes of the CTA's columns into amp, likewise.  An L2 prefetch of what the cluster
    // `ahead` planes further will read.  The expected bytes are set before any copy is issued.
    if (t == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                     ::"r"(smem_address(input_ready)), "r"(kHalfBytes) : "memory");
        if (stage_amp || stage_factor)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                         ::"r"(smem_address(amp_ready)), "r"(kSide * (stage_amp ? kAmpRowBytes : kSpanBytes / 2))
                         : "memory");
    }
    __syncthreads();
    static_assert(PlaneGeometry<Q>::kThreads >= kSide, "one row copy per thread");
    if (MODE != kPlaneInverse) {
        if (t == 0) {
            const char *src = reinterpret_cast<const char *>(a.in + in_plane() + (size_t)rank * G::kLines * kSide);
            for (uint32_t off = 0; off < kHalfBytes; off += kChunk)
                asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                             ::"r"(smem_address(buf) + off), "l"(src + off), "r"(kChunk), "r"(smem_address(input_ready))
                             : "memory");
        }
    } else if (t < kSide) {
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(smem_address(buf + t * G::kStrideA)),
                     "l"(a.in + in_plane() + (size_t)t * kSide + rank * G::kLines), "r"(kSpanBytes),
                     "r"(smem_address(input_ready))
                     : "memory");
    }
    if (stage_factor && t < kSide)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(smem_address(factor + t * G::kFactorStride)),
                     "l"(a.factors + (size_t)p * kPlane + (size_t)t * kSide + rank * G::kLines), "r"(kSpanBytes / 2),
                     "r"(smem_address(amp_ready))
                     : "memory");
    if (stage_amp && t < kSide)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(smem_address(amp + t * G::kAmpStride)),
                     "l"(a.amplitudes + (size_t)p * kPlane + (size_t)t * kSide + rank * G::kLines),
                     "r"(kAmpRowBytes), "r"(smem_address(amp_ready))
                     : "memory");
    if (t == 32) {  // another warp than the input copies
        const int next = p + a.ahead;
        if (a.ahead > 0 && next < a.first + a.count) {
            if (a.in_kind == kInputByPosition)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                             ::"l"(a.in + (size_t)next * kPlane + (size_t)rank * G::kLines * kSide), "r"(kHalfBytes)
                             : "memory");
            if (stage_amp && rank == 0)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                             ::"l"(a.amplitudes + (size_t)next * kPlane), "r"((uint32_t)(kPlane * sizeof(float)))
                             : "memory");
            if (stage_factor && rank == 0)
                asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                             ::"l"(a.factors + (size_t)next * kPlane), "r"((uint32_t)(kPlane * sizeof(double)))
                             : "memory");
        }
    }

    double2 v[16];
    const uint32_t buf_local = smem_address(buf);
    if constexpr (MODE != kPlaneInverse) {
        // ---- the object patch (from L2) while the rows arrive, then the input times the patch
        double2 o[16];
        if (a.object) {
            const int oy = wrap_once(a.scan.rr[p] + a.object_row_offset + corner_offset(row, kSide), a.object_rows);
            const double2 *orow = a.object + (size_t)oy * a.object_columns;
            const int cc = a.scan.cc[p] + a.object_column_offset;
#pragma unroll
            for (int m = 0; m < 16; m++) {
                o[m] = orow[wrap_once(cc + corner_offset(j + 8 * m, kSide), a.object_columns)];
                if (a.conj_object) o[m].y = -o[m].y;
            }
        }
        bool arrived = mbarrier_wait_bounded(input_ready);
        if (!arrived) {
            atomicOr(a.fault, 1);
            arrived = mbarrier_wait_bounded(input_ready);  // the copies land before the buffer is reused, or give up
        }
#pragma unroll
        for (int m = 0; m < 16; m++) v[m] = buf[line * kSide + j + 8 * m];
        if (a.object) {
#pragma unroll
            for (int m = 0; m < 16; m++) v[m] = cmul(v[m], o[m]);
        }
        __syncwarp();  // the warp's input rows are read: the same region is its scratch
        line_forward(v, j, lw, tf, scratch);

        // ---- rows -> columns: X[row][k] to the CTA holding column k, buffer [row][k mod kLines]
        cluster.sync();  // every CTA has finished with its input and scratch (and runs): the buffers take the exchange
        constexpr int kPerRank = G::kLines / 16;  // k2 values per destination CTA
#pragma unroll
        for (int q = 0; q < Q; q++) {
            const uint32_t dest = cluster_address(buf_local, q) + (uint32_t)(row * G::kStrideA + 2 * j) * 16u;
#pragma unroll
            for (int k2 = q * kPerRank; k2 < (q + 1) * kPerRank; k2++)
#pragma unroll
                for (int c = 0; c < 2; c++)
                    store_cluster(dest + (uint32_t)(c + 16 * (k2 % kPerRank)) * 16u, v[2 * k2 + c]);
        }
        cluster.sync();
#pragma unroll
        for (int m = 0; m < 16; m++) v[m] = buf[(j + 8 * m) * G::kStrideA + line];
        __syncthreads();  // the columns are read: buf is scratch until the next exchange
        line_forward(v, j, lw, tf, scratch);  // v[2 k2 + c] = F[2 j + c + 16 k2][column]
    } else {
        // ---- the spectrum's values of the CTA's columns: F[2 j + c + 16 k2][column]
        bool arrived = mbarrier_wait_bounded(input_ready);
        if (!arrived) {
            atomicOr(a.fault, 1);
            arrived = mbarrier_wait_bounded(input_ready);
        }
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++)
#pragma unroll
            for (int c = 0; c < 2; c++) v[2 * k2 + c] = buf[(2 * j + c + 16 * k2) * G::kStrideA + line];
        __syncthreads();  // the spectrum is read: buf is scratch until the exchange
    }

    if constexpr (MODE == kPlaneForward) {
        // ---- the spectrum out: buf[row][kStrideA] as the columns' exchange buffer, then one bulk copy per row
        __syncthreads();  // every warp is done with its scratch
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++)
#pragma unroll
            for (int c = 0; c < 2; c++) buf[(2 * j + c + 16 * k2) * G::kStrideA + line] = v[2 * k2 + c];
        if (solve) {
            // ---- position correction: this CTA's columns of the normal equations, summed thread -> warp -> CTA ->
            // cluster in a fixed order, then rank 0 moves the position (Ptychography.swift:411-472)
            __syncthreads();
            bool landed = mbarrier_wait_bounded(amp_ready);
            if (!landed) {
                atomicOr(a.fault, 1);
                landed = mbarrier_wait_bounded(amp_ready);
            }
            const double2 *f0 = a.far + (size_t)(p - a.first) * 2 * kPlane, *fx = f0 + kPlane;
            double terms[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            for (int e = 0; e < 16; e++) {
                const int kr = 2 * j + (e & 1) + 16 * (e >> 1);
                const size_t k = (size_t)kr * kSide + column;
                position_terms(f0[k], fx[k], buf[kr * G::kStrideA + line], (double)amp[kr * G::kAmpStride + line],
                               terms);
            }
            double *warp_terms = reinterpret_cast<double *>(ti);            // [5][warps], ti is unused here
            double *cluster_terms = reinterpret_cast<double *>(ti) + 128;   // [Q][5], rank 0's copy is read
#pragma unroll
            for (int q = 0; q < 5; q++)
#pragma unroll
                for (int o2 = 16; o2 > 0; o2 >>= 1) terms[q] += __shfl_down_sync(0xffffffffu, terms[q], o2);
            if ((t & 31) == 0)
#pragma unroll
                for (int q = 0; q < 5; q++) warp_terms[q * (G::kThreads / 32) + (t >> 5)] = terms[q];
            __syncthreads();
            if (t == 0) {
                double *dest = cluster.map_shared_rank(cluster_terms + 5 * rank, 0);
                for (int q = 0; q < 5; q++) {
                    double total = 0.0;
                    for (int w = 0; w < G::kThreads / 32; w++) total += warp_terms[q * (G::kThreads / 32) + w];
                    dest[q] = total;
                }
            }
            cluster.sync();  // every rank's sums are in rank 0
            if (rank == 0 && t == 0) {
                double sums[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
                for (int r = 0; r < Q; r++)
                    for (int q = 0; q < 5; q++) sums[q] += cluster_terms[5 * r + q];
                position_step(sums, p, a.positions, a.initial, a.position_count, a.position_step_size, a.limit_update,
                              a.limit_total, a.position_bad);
            }
            return;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (t < 32) {
            for (int r = t; r < kSide; r += 32)
                asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                             ::"l"(out_plane() + (size_t)r * kSide + rank * G::kLines),
                             "r"(smem_address(buf + r * G::kStrideA)), "r"(kSpanBytes)
                             : "memory");
            asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        }
        return;
    }

    // ---- the pointwise step on F[2 j + c + 16 k2][column]
    double err = 0.0;
    if (project) {
        bool landed = mbarrier_wait_bounded(amp_ready);
        if (!landed) {
            atomicOr(a.fault, 1);
            landed = mbarrier_wait_bounded(amp_ready);
        }
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const int kr = 2 * j + c + 16 * k2;
                const double2 f = v[2 * k2 + c];
                const double mag = sqrt(f.x * f.x + f.y * f.y);
                const double measured = (double)amp[kr * G::kAmpStride + line];
                const double miss = measured - mag;
                err += miss * miss;
                if (mag > 0.0) {
                    const double sc = (measured / mag - 1.0) * a.inv_n;
                    v[2 * k2 + c] = make_double2(f.x * sc, f.y * sc);
                } else {
                    v[2 * k2 + c] = make_double2(measured * a.inv_n, 0.0);
                }
            }
    } else if (stage_factor) {  // the mixed states' common factor of each pixel (a real scale)
        bool landed = mbarrier_wait_bounded(amp_ready);
        if (!landed) {
            atomicOr(a.fault, 1);
            landed = mbarrier_wait_bounded(amp_ready);
        }
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const double sc = factor[(2 * j + c + 16 * k2) * G::kFactorStride + line];
                v[2 * k2 + c] = make_double2(v[2 * k2 + c].x * sc, v[2 * k2 + c].y * sc);
            }
    } else if (factors) {
        const double2 wc = pc[column];
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++)
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const double2 u = cmul(v[2 * k2 + c], cmul(pr[2 * j + c + 16 * k2], wc));
                v[2 * k2 + c] = make_double2(u.x * a.scale, u.y * a.scale);
            }
    }
    line_inverse(v, j, lw, ti, scratch);  // v[m] = column's value at row j + 8 m

    if (project) {  // the position's squared error: warps, then the CTA in warp order, then ranks in order
#pragma unroll
        for (int o2 = 16; o2 > 0; o2 >>= 1) err += __shfl_down_sync(0xffffffffu, err, o2);
        if ((t & 31) == 0) warp_err[t >> 5] = err;
        __syncthreads();
        if (t == 0) {
            double total = 0.0;
            for (int w = 0; w < G::kThreads / 32; w++) total += warp_err[w];
            *cluster.map_shared_rank(cluster_err + rank, 0) = total;
        }
    }
    cluster.sync();  // every CTA is done with its buffer (and runs): the buffers take the second exchange

    // ---- columns -> rows: G[r][column] to the CTA holding row r, buffer [r mod kLines][column]
    constexpr int kRowsPerRank = G::kLines / 8;  // m values per destination CTA
#pragma unroll
    for (int q = 0; q < Q; q++) {
        const uint32_t dest = cluster_address(buf_local, q) + (uint32_t)(j * G::kStrideB + column) * 16u;
#pragma unroll
        for (int m = q * kRowsPerRank; m < (q + 1) * kRowsPerRank; m++)
            store_cluster(dest + (uint32_t)(8 * (m % kRowsPerRank) * G::kStrideB) * 16u, v[m]);
    }
    cluster.sync();
#pragma unroll
    for (int k2 = 0; k2 < 8; k2++)
#pragma unroll
        for (int c = 0; c < 2; c++) v[2 * k2 + c] = buf[line * G::kStrideB + 2 * j + c + 16 * k2];
    __syncthreads();  // the rows are read: buf is scratch, then the output rows
    line_inverse(v, j, lw, ti, scratch);

    // ---- the output rows: buf[line][128] (the warp's own region), then bulk copies to HBM
#pragma unroll
    for (int m = 0; m < 16; m++) buf[line * kSide + j + 8 * m] = v[m];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (t == 0) {
        char *dst = reinterpret_cast<char *>(out_plane() + (size_t)rank * G::kLines * kSide);
        for (uint32_t off = 0; off < kHalfBytes; off += kChunk)
            asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;"
                         ::"l"(dst + off), "r"(smem_address(buf) + off), "r"(kChunk) : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        if (project && rank == 0) {
            double total = 0.0;
            for (int q = 0; q < Q; q++) total += cluster_err[q];
            a.error[p] = total;
        }
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
    }
}

template <int Q, int MODE>
cudaError_t launch_q(Plane128Args a, cudaStream_t s) {
    using G = PlaneGeometry<Q>;
    if (a.ahead == 0) {  // the clusters resident at once: the L2 prefetch distance
        int device = 0, sms = 0;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        a.ahead = sms / 2;  // Q / 2 CTAs per SM, Q per cluster
    }
    plane128_kernel<Q, MODE><<<(unsigned)a.count * Q, G::kThreads, G::smem(MODE), s>>>(a);
    return cudaGetLastError();
}

template <int Q>
cudaError_t set_smem() {
    using G = PlaneGeometry<Q>;
    cudaError_t e = cudaFuncSetAttribute(plane128_kernel<Q, kPlaneFull>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)G::smem(kPlaneFull));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(plane128_kernel<Q, kPlaneForward>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)G::smem(kPlaneForward));
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(plane128_kernel<Q, kPlaneInverse>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)G::smem(kPlaneInverse));
    return e;
}

template <int Q>
cudaError_t launch_mode(const Plane128Args &a, cudaStream_t s) {
    if (a.mode == kPlaneFull) return launch_q<Q, kPlaneFull>(a, s);
    if (a.mode == kPlaneForward) return launch_q<Q, kPlaneForward>(a, s);
    if (a.mode == kPlaneInverse) return launch_q<Q, kPlaneInverse>(a, s);
    return cudaErrorInvalidValue;
}

}  // namespace

// CTAs per plane: 2 (512 threads each, one CTA per SM) by default; CUBO_PTYCHO_PLANE_CLUSTER=4 or 8 selects four CTAs
// of 256 threads (two per SM) or eight of 128 (four per SM).  Every size gives the same results bit for bit.
int plane128_cluster() {
    static const int q = [] {
        const char *v = std::getenv("CUBO_PTYCHO_PLANE_CLUSTER");
        const int want = v ? std::atoi(v) : 2;
        return want == 4 || want == 8 ? want : 2;
    }();
    return q;
}

cudaError_t configure_plane128() {
    cudaError_t e = set_smem<2>();
    if (e == cudaSuccess) e = set_smem<4>();
    if (e == cudaSuccess) e = set_smem<8>();
    return e;
}

cudaError_t launch_plane128(const Plane128Args &a, int cluster, cudaStream_t s) {
    if (a.count <= 0) return cudaSuccess;
    if (cluster == 8) return launch_mode<8>(a, s);
    if (cluster == 4) return launch_mode<4>(a, s);
    if (cluster == 2) return launch_mode<2>(a, s);
    return cudaErrorInvalidValue;
}

}  // namespace cubo
