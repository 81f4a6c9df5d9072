// The FP32 position pass for a 128 x 128 detector: register-resident 2-D FFT pair (sm_100a).
//
// Same arithmetic as the generic position pass (exit wave, forward 2-D FFT, Fourier-modulus projection with the 1/n of
// ifft2 folded in, inverse 2-D FFT; Ptychography.swift:321-350), laid out for the hardware:
//
//  * Persistent CTAs of 512 threads (one per SM) walk the positions in a fixed stride; each 8-thread group owns two
//    lines (rows g and g + 64 in the row pass, columns in the column pass) and each thread holds 2 x 16 complex
//    samples in registers, so every phase has two independent instruction streams and nothing spills.
//  * A 128-point line transform is 128 = 16 x 8 (four-step): with c = t + 8m and k = q + 16s,
//      X[q + 16s] = sum_t W8^{ts} W128^{tq} sum_m W16^{mq} x[t + 8m],
//    i.e. a 16-point DFT in registers, a twiddle, one exchange inside the 8-thread group (shared memory, __syncwarp
//    only) and two 8-point DFTs in registers.  The inverse runs the same steps mirrored with conjugate twiddles.
//  * The spectrum is never put back in natural order: the projection is pointwise, so each thread projects the 16
//    frequencies it holds and the inverse starts from the same registers.  The amplitudes are stored once per plan
//    in that register order ([position][column][t][parity][s]), so each thread reads 64 contiguous bytes.
//  * Shared memory holds one 128 x 132 complex64 tile (pitch 132: row-major float4 writes and 8-row column reads
//    are free of bank conflicts); the group exchanges use a rotated slot order for the same reason.
//  * The squared residual is summed per warp and written as 16 FP64 partials per position (reduced in a fixed order
//    by the error kernels): no atomics, bitwise reproducible.
//  * The next position's amplitudes are prefetched into shared memory by a bulk copy into this CTA alone while the
//    current one is transformed.
//  * The probe gradient (conj(O[patch]) dpsi and |O|^2, Ptychography.swift:356-357) is accumulated here, in tensor
//    memory: every thread owns 32 fixed detector pixels, so each CTA sums its positions in order and writes one
//    partial; a fixed-order FP64 reduction over the 148 partials follows.  This replaces a second pass over dpsi.
#include "engine.h"
#include "umma.cuh"

namespace cubo {

namespace {

constexpr int kN = 128;          // detector side
constexpr int kPitch = 132;      // shared-memory row pitch (complex64)
constexpr int kThreads = 512;
constexpr int kLines = kThreads / 8;    // lines per pass handled at once; each group owns two (g, g + kLines)
constexpr int kWarps = kThreads / 32;   // residual partials per position

__device__ __forceinline__ float2 fm(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 fmc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// Complex add / subtract as one packed FP32x2 instruction each (sm_100 add.rn.f32x2 / sub.rn.f32x2), same rounding as
// two scalar FP32 operations.
__device__ __forceinline__ float2 fadd(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 fsub(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {  // * (-i) forward, * (+i) inverse
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ void f4(float2 &x0, float2 &x1, float2 &x2, float2 &x3) {
    const float2 t0 = fadd(x0, x2), t1 = fsub(x0, x2), t2 = fadd(x1, x3), t3 = mul_mi<INV>(fsub(x1, x3));
    x0 = fadd(t0, t2); x2 = fsub(t0, t2); x1 = fadd(t1, t3); x3 = fsub(t1, t3);
}

// W16^k (forward e^{-2 pi i k / 16}); cos(pi/8), sin(pi/8), cos(pi/4) written out.
template <bool INV, int K>
__device__ __forceinline__ float2 tw16(float2 a) {
    constexpr float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f, h = 0.70710678118654752440f;
    constexpr float sg = INV ? 1.f : -1.f;  // sign of the imaginary part of the twiddle
    if (K == 0) return a;
    if (K == 1) return fm(a, make_float2(c1, sg * s1));
    if (K == 2) return make_float2(h * (a.x - sg * a.y), h * (a.y + sg * a.x));
    if (K == 3) return fm(a, make_float2(s1, sg * c1));
    if (K == 4) return mul_mi<INV>(a);
    if (K == 6) return make_float2(h * (-a.x - sg * a.y), h * (-a.y + sg * a.x));
    if (K == 9) return fm(a, make_float2(-c1, -sg * s1));
    return a;
}

// 16-point DFT in registers, natural order in and out (4 x 4 with W16 twiddles).
template <bool INV>
__device__ __forceinline__ void dft16(float2 (&x)[16]) {
#pragma unroll
    for (int b = 0; b < 4; b++) f4<INV>(x[b], x[4 + b], x[8 + b], x[12 + b]);  // x[4c + b] = y_b[c]
    x[5] = tw16<INV, 1>(x[5]); x[9] = tw16<INV, 2>(x[9]); x[13] = tw16<INV, 3>(x[13]);
    x[6] = tw16<INV, 2>(x[6]); x[10] = tw16<INV, 4>(x[10]); x[14] = tw16<INV, 6>(x[14]);
    x[7] = tw16<INV, 3>(x[7]); x[11] = tw16<INV, 6>(x[11]); x[15] = tw16<INV, 9>(x[15]);
#pragma unroll
    for (int c = 0; c < 4; c++) f4<INV>(x[4 * c], x[4 * c + 1], x[4 * c + 2], x[4 * c + 3]);  // x[4c + d] = X[c + 4d]
    float2 y[16];
#pragma unroll
    for (int q = 0; q < 16; q++) y[q] = x[4 * (q & 3) + (q >> 2)];
#pragma unroll
    for (int q = 0; q < 16; q++) x[q] = y[q];
}

// 8-point DFT in registers, natural order in and out.
template <bool INV>
__device__ __forceinline__ void dft8(float2 (&v)[8]) {
    float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    f4<INV>(e0, e1, e2, e3);
    f4<INV>(o0, o1, o2, o3);
    o1 = tw16<INV, 2>(o1);
    o2 = mul_mi<INV>(o2);
    o3 = tw16<INV, 6>(o3);
    v[0] = fadd(e0, o0); v[4] = fsub(e0, o0);
    v[1] = fadd(e1, o1); v[5] = fsub(e1, o1);
    v[2] = fadd(e2, o2); v[6] = fsub(e2, o2);
    v[3] = fadd(e3, o3); v[7] = fsub(e3, o3);
}

// Group exchange (inside lines_forward / lines_inverse): Y[t][q] of a line sits at slot t * 16 + ((q + 2t) & 15) of
// that line's scratch row, so the float4 writes and reads of the 8 threads of a group cover all 32 banks.

// Forward transform of two lines at once (independent work for the scheduler): for each line l, the 16 samples
// x[l][m] = line[t + 8m]; on return u0[l][s] = X[2t + 16s], u1[l][s] = X[2t+1+16s].
__device__ __forceinline__ void lines_forward(float2 (&x)[2][16], int t, const float2 *tw, float2 *const (&scratch)[2],
                                              float2 (&u0)[2][8], float2 (&u1)[2][8]) {
    dft16<false>(x[0]);
    dft16<false>(x[1]);
#pragma unroll
    for (int q = 1; q < 16; q++) {
        const float2 w = tw[(t * q) & 127];
        x[0][q] = fm(x[0][q], w);
        x[1][q] = fm(x[1][q], w);
    }
    // group exchange for both lines: thread t then holds u0[l][t'] = Y_l[t'][2t], u1[l][t'] = Y_l[t'][2t + 1]
#pragma unroll
    for (int l = 0; l < 2; l++)
#pragma unroll
        for (int j = 0; j < 8; j++)
            *reinterpret_cast<float4 *>(scratch[l] + t * 16 + ((2 * j + 2 * t) & 15)) =
                make_float4(x[l][2 * j].x, x[l][2 * j].y, x[l][2 * j + 1].x, x[l][2 * j + 1].y);
    __syncwarp();
#pragma unroll
    for (int l = 0; l < 2; l++)
#pragma unroll
        for (int s = 0; s < 8; s++) {
            const float4 v = *reinterpret_cast<const float4 *>(scratch[l] + s * 16 + ((2 * t + 2 * s) & 15));
            u0[l][s] = make_float2(v.x, v.y);
            u1[l][s] = make_float2(v.z, v.w);
        }
    __syncwarp();
#pragma unroll
    for (int l = 0; l < 2; l++) { dft8<false>(u0[l]); dft8<false>(u1[l]); }
}

// Inverse of lines_forward (unnormalised): from u0/u1 as lines_forward leaves them, x[l][m] = line[t + 8m].
__device__ __forceinline__ void lines_inverse(float2 (&u0)[2][8], float2 (&u1)[2][8], int t, const float2 *tw,
                                              float2 *const (&scratch)[2], float2 (&x)[2][16]) {
#pragma unroll
    for (int l = 0; l < 2; l++) { dft8<true>(u0[l]); dft8<true>(u1[l]); }
    // u0[t'] = G[t'][2t], u1[t'] = G[t'][2t+1]; twiddle by conj(W128^{t' q})
#pragma unroll
    for (int s = 1; s < 8; s++) {
        const float2 w0 = tw[(s * 2 * t) & 127], w1 = tw[(s * (2 * t + 1)) & 127];
#pragma unroll
        for (int l = 0; l < 2; l++) { u0[l][s] = fmc(u0[l][s], w0); u1[l][s] = fmc(u1[l][s], w1); }
    }
#pragma unroll
    for (int l = 0; l < 2; l++)
#pragma unroll
        for (int s = 0; s < 8; s++)
            *reinterpret_cast<float4 *>(scratch[l] + s * 16 + ((2 * t + 2 * s) & 15)) =
                make_float4(u0[l][s].x, u0[l][s].y, u1[l][s].x, u1[l][s].y);
    __syncwarp();
#pragma unroll
    for (int l = 0; l < 2; l++)
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const float4 v = *reinterpret_cast<const float4 *>(scratch[l] + t * 16 + ((2 * j + 2 * t) & 15));
            x[l][2 * j] = make_float2(v.x, v.y);
            x[l][2 * j + 1] = make_float2(v.z, v.w);
        }
    __syncwarp();
    dft16<true>(x[0]);
    dft16<true>(x[1]);
}

__device__ __forceinline__ int wrap_once(int v, int size) { return v < 0 ? v + size : (v >= size ? v - size : v); }

// Tensor-memory columns of this thread's probe-gradient accumulators: 32 detector pixels (two lines x 16), real,
// imaginary and weight planes of 32 columns each; the four warps that share a lane quadrant take 96 columns each.
__device__ __forceinline__ uint32_t acc_base(uint32_t tmem, int warp) {
    return umma::tmem_addr(tmem, 32 * (warp & 3), 96 * (warp >> 2));
}

__global__ void __launch_bounds__(kThreads, 1) fast128_kernel(Fast128Args a) {
    extern __shared__ __align__(16) float2 sm[];
    float2 *tw = sm + kN * kPitch;
    float *amp_smem = reinterpret_cast<float *>(tw + kN);  // the current position's amplitudes, 64 KB
    __shared__ uint64_t amp_bar;
    __shared__ uint32_t tmem_base;
    __shared__ int amp_fault;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = warp * 4 + (lane >> 3);  // this 8-thread group owns lines g and g + 64
    const int t = lane & 7;
    for (int i = tid; i < kN; i += kThreads) tw[i] = a.tw128[i];
    if (warp == 0) {
        umma::tmem_alloc(&tmem_base, 512);
        umma::tmem_relinquish();
    }
    const int first = a.first + blockIdx.x;
    if (tid == 0) {
        umma::mbar_init(&amp_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        amp_fault = 0;
        if (first < a.first + a.count)
            umma::bulk_load(amp_smem, a.amplitudes + (size_t)first * (kN * kN), kN * kN * sizeof(float), &amp_bar);
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t acc = acc_base(tmem_base, warp);
    if (a.accumulate) {  // an earlier band's partial of this CTA: its sums continue in the same position order
#pragma unroll
        for (int l = 0; l < 2; l++)
#pragma unroll
            for (int m0 = 0; m0 < 16; m0 += 8) {
                float gr[8], gi[8], gw[8];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int k = (g + l * kLines) * kN + t + 8 * (m0 + i);
                    const float2 v = a.partial_grad[(size_t)blockIdx.x * (kN * kN) + k];
                    gr[i] = v.x;
                    gi[i] = v.y;
                    gw[i] = a.partial_weight[(size_t)blockIdx.x * (kN * kN) + k];
                }
                const uint32_t col = acc + l * 16 + m0;
                umma::tmem_st8(col, gr);
                umma::tmem_st8(col + 32, gi);
                umma::tmem_st8(col + 64, gw);
            }
        umma::tmem_wait_st();
    } else {
        const float zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int c = 0; c < 96; c += 8) umma::tmem_st8(acc + c, zero);
        umma::tmem_wait_st();
    }
    float2 *line[2] = {sm + g * kPitch, sm + (g + kLines) * kPitch};  // the group's own rows (scratch)
    const float inv_n = 1.0f / (float)(kN * kN);
    uint32_t amp_phase = 0;
    for (int p = first; p < a.first + a.count; p += gridDim.x) {
        const int rr = a.scan.rr[p], cc = a.scan.cc[p], cls = a.scan.cls[p];
        float2 x[2][16], u0[2][8], u1[2][8];
        // exit wave, rows g and g + 64, columns t + 8m (Ptychography.swift:321-336).  Column t + 8m lies left of the
        // centre for m >= 8 (corner offset t + 8m - 128); when the whole window is inside the object no wrap is needed.
        const bool interior = cc >= kN / 2 && cc + kN / 2 <= a.object_columns;
        const float2 *orows[2];
#pragma unroll
        for (int l = 0; l < 2; l++) {
            const int row = g + l * kLines;
            const float2 *S = a.shifted + (size_t)cls * (kN * kN) + row * kN;
            orows[l] = a.object + (size_t)wrap_once(rr + (l == 0 ? row : row - kN), a.object_rows) * a.object_columns;
            if (interior) {
                const float2 *centre = orows[l] + cc + t;
#pragma unroll
                for (int m = 0; m < 16; m++) x[l][m] = fm(S[t + 8 * m], centre[m < 8 ? 8 * m : 8 * m - kN]);
            } else {
#pragma unroll
                for (int m = 0; m < 16; m++) {
                    const int xc = wrap_once(cc + t + (m < 8 ? 8 * m : 8 * m - kN), a.object_columns);
                    x[l][m] = fm(S[t + 8 * m], orows[l][xc]);
                }
            }
        }
        // row pass
        lines_forward(x, t, tw, line, u0, u1);
#pragma unroll
        for (int l = 0; l < 2; l++)
#pragma unroll
            for (int s = 0; s < 8; s++)
                *reinterpret_cast<float4 *>(line[l] + 2 * t + 16 * s) = make_float4(u0[l][s].x, u0[l][s].y, u1[l][s].x, u1[l][s].y);
        __syncthreads();
        // column pass: columns g and g + 64, rows t + 8m
#pragma unroll
        for (int l = 0; l < 2; l++)
#pragma unroll
            for (int m = 0; m < 16; m++) x[l][m] = sm[(t + 8 * m) * kPitch + g + l * kLines];
        __syncthreads();
        lines_forward(x, t, tw, line, u0, u1);
        // projection (Ptychography.swift:338-349); line l holds F[2t + parity + 16s][g + 64 l].  This position's
        // amplitudes were prefetched into shared memory ([column][h][t][4]: float4 h of the 8 threads of a group is
        // one 128-byte row, free of bank conflicts).
        if (!umma::mbar_wait(&amp_bar, amp_phase, 2000000000ull)) amp_fault = 1;
        amp_phase ^= 1u;
        double err = 0;
#pragma unroll
        for (int l = 0; l < 2; l++) {
            const float4 *A = reinterpret_cast<const float4 *>(amp_smem + (size_t)(g + l * kLines) * kN) + t;
#pragma unroll
            for (int h = 0; h < 4; h++) {
                const float4 av = A[h * 8];
                const float am[4] = {av.x, av.y, av.z, av.w};
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int j = h * 4 + e;  // j = parity * 8 + s
                    float2 &f = (j < 8) ? u0[l][j] : u1[l][j - 8];
                    const float mag = sqrtf(f.x * f.x + f.y * f.y);
                    const float miss = am[e] - mag;
                    err += (double)(miss * miss);
                    if (mag > 0.f) {
                        const float sc = (am[e] / mag - 1.0f) * inv_n;
                        f = make_float2(f.x * sc, f.y * sc);
                    } else {
                        f = make_float2(am[e] * inv_n, 0.f);
                    }
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) err += __shfl_down_sync(0xffffffffu, err, o);
        if (lane == 0) a.error[(size_t)p * kWarps + warp] = err;
        // inverse column pass
        lines_inverse(u0, u1, t, tw, line, x);
        __syncthreads();  // every group is done with its scratch rows (and the amplitude buffer) before reuse
        if (tid == 0 && p + (int)gridDim.x < a.first + a.count)
            umma::bulk_load(amp_smem, a.amplitudes + (size_t)(p + gridDim.x) * (kN * kN), kN * kN * sizeof(float),
                            &amp_bar);
#pragma unroll
        for (int l = 0; l < 2; l++)
#pragma unroll
            for (int m = 0; m < 16; m++) sm[(t + 8 * m) * kPitch + g + l * kLines] = x[l][m];
        __syncthreads();
        // inverse row pass from the row-pass layout
#pragma unroll
        for (int l = 0; l < 2; l++)
#pragma unroll
            for (int s = 0; s < 8; s++) {
                const float4 v = *reinterpret_cast<const float4 *>(line[l] + 2 * t + 16 * s);
                u0[l][s] = make_float2(v.x, v.y);
                u1[l][s] = make_float2(v.z, v.w);
            }
        __syncwarp();
        lines_inverse(u0, u1, t, tw, line, x);
#pragma unroll
        for (int l = 0; l < 2; l++) {
            float2 *out = a.dpsi + (size_t)(p - a.dpsi_first) * (kN * kN) + (g + l * kLines) * kN;
#pragma unroll
            for (int m = 0; m < 16; m++) out[t + 8 * m] = x[l][m];
        }
        // probe gradient (Ptychography.swift:356-357): conj(O[patch]) dpsi and |O|^2 added to this thread's 32 pixels,
        // in tensor memory, in this CTA's position order
#pragma unroll
        for (int l = 0; l < 2; l++)
#pragma unroll
            for (int m0 = 0; m0 < 16; m0 += 8) {
                float gr[8], gi[8], gw[8];
                const uint32_t col = acc + l * 16 + m0;
                umma::tmem_ld8(col, gr);
                umma::tmem_ld8(col + 32, gi);
                umma::tmem_ld8(col + 64, gw);
                umma::tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int m = m0 + i;
                    const int xc = interior ? cc + t + (m < 8 ? 8 * m : 8 * m - kN)
                                            : wrap_once(cc + t + (m < 8 ? 8 * m : 8 * m - kN), a.object_columns);
                    const float2 o = orows[l][xc], d = x[l][m];
                    gr[i] += o.x * d.x + o.y * d.y;
                    gi[i] += o.x * d.y - o.y * d.x;
                    gw[i] += o.x * o.x + o.y * o.y;
                }
                umma::tmem_st8(col, gr);
                umma::tmem_st8(col + 32, gi);
                umma::tmem_st8(col + 64, gw);
            }
        umma::tmem_wait_st();
    }
    // this CTA's probe-gradient partial, natural pixel order
#pragma unroll
    for (int l = 0; l < 2; l++)
#pragma unroll
        for (int m0 = 0; m0 < 16; m0 += 8) {
            float gr[8], gi[8], gw[8];
            const uint32_t col = acc + l * 16 + m0;
            umma::tmem_ld8(col, gr);
            umma::tmem_ld8(col + 32, gi);
            umma::tmem_ld8(col + 64, gw);
            umma::tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int k = (g + l * kLines) * kN + t + 8 * (m0 + i);
                a.partial_grad[(size_t)blockIdx.x * (kN * kN) + k] = make_float2(gr[i], gi[i]);
                a.partial_weight[(size_t)blockIdx.x * (kN * kN) + k] = gw[i];
            }
        }
    if (amp_fault && tid == 0) *a.fault = 1;
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (warp == 0) umma::tmem_dealloc(tmem_base, 512);
}

// [position][row][column] -> [position][column][h][t][e]: element j = 4h + e (j = parity * 8 + s) of thread t of the
// column's group, row = 2t + parity + 16s.
__global__ void permute_amplitudes_kernel(const float *in, float *out, long long positions) {
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i >= positions * kN * kN) return;
    const long long p = i / (kN * kN);
    const int rem = (int)(i - p * kN * kN);
    const int column = rem >> 7, h = (rem >> 5) & 3, t = (rem >> 2) & 7, e = rem & 3;
    const int j = 4 * h + e;
    const int row = 2 * t + (j >> 3) + 16 * (j & 7);
    out[i] = in[p * kN * kN + row * kN + column];
}

}  // namespace

bool fast128_applicable(int rows, int columns) { return rows == kN && columns == kN; }

int fast128_partials_per_position() { return kWarps; }

size_t fast128_smem() { return (size_t)(kN * kPitch + kN) * sizeof(float2) + (size_t)kN * kN * sizeof(float); }

int fast128_ctas() { return 148; }  // fixed, so the probe-gradient summation order does not depend on the device

cudaError_t configure_fast128() {
    int device = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    if ((size_t)optin < fast128_smem()) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(fast128_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fast128_smem());
}

cudaError_t launch_fast128(const Fast128Args &a, int ctas, cudaStream_t s) {
    if (a.count <= 0) return cudaSuccess;
    (void)ctas;
    const int grid = a.count < fast128_ctas() ? a.count : fast128_ctas();
    fast128_kernel<<<grid, kThreads, fast128_smem(), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_permute_amplitudes(const float *in, float *out, long long positions, cudaStream_t s) {
    const long long total = positions * kN * kN;
    permute_amplitudes_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(in, out, positions);
    return cudaGetLastError();
}

}  // namespace cubo
