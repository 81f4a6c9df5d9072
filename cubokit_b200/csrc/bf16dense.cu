// The split-BF16 position pass for a 128 x 128 detector: the 2-D DFT pair as DFT-matrix products on the tensor cores.
//
// Arithmetic (Ptychography.swift:321-350): exit wave X = S * O[patch], F = W X W (W the symmetric 128-point DFT matrix,
// unnormalised), the Fourier-modulus projection with the 1/n of ifft2 folded in, then dpsi = conj(W) F' conj(W).
// Every product is a left multiplication D = W * B with the DFT matrix as the A operand, kept in tensor memory for the
// whole kernel (re hi, re lo, im hi, im lo: 4 x 64 columns), and the data as the B operand in shared memory:
//
//   stage 1  D = W X^T      = Y^T    (Y = X W, the row transform)      B = X     K-major, row r of X per lane r
//   stage 2  D = W Y        = F                                        B = Y     K-major, row k of Y^T per lane k
//   stage 3  D = conj(W) F' = Y'                                       B = F'    MN-major, row k of F' per lane k
//   stage 4  D = conj(W) Y'^T = dpsi^T                                 B = Y'^T  K-major, row r of Y' per lane r
//
// so no stage needs a transpose: each TMEM lane's row of one stage's result is written, split into bf16 hi and lo, as
// one contiguous row of the next stage's B operand.  Each real product P Q is P_hi Q_hi + P_hi Q_lo + P_lo Q_hi (the
// lo * lo term is below FP32 resolution of the sum), accumulated in FP32 in tensor memory: 12 streams x 8 K-steps = 96
// tcgen05.mma (M = N = 128, K = 16) per stage, issued by one thread and completed through an mbarrier.  Signs of conj(W)
// and of the - Wi Bi term come from the instruction descriptor's negate bit.
//
// One persistent CTA of 256 threads per SM: thread (warp w, lane i) owns TMEM lane 32 (w mod 4) + i and column half
// w / 4.  The residual is written transposed ([position][column][row]); the amplitudes are read in 16-float chunks
// ([position][column / 16][row][column mod 16]) so a warp reads 2 KB contiguously.  Waits are bounded: a wait that runs
// out sets *fault and the CTA stops after freeing its tensor memory.
#include "engine.h"
#include "umma.cuh"

namespace cubo {

namespace {

using namespace umma;

constexpr int kN = 128;
constexpr int kThreads = 256;
constexpr uint32_t kSBO = 2048, kLBO = 128;     // canonical no-swizzle layout of a 128 x 128 bf16 plane
constexpr int kPlaneBytes = kN * kN * 2;        // 32 KB
constexpr uint64_t kWaitLimit = 2000000000ull;  // ns of wall time an mbarrier wait may take before giving up

__device__ __forceinline__ uint32_t kmajor_offset(int row, int k) {
    return (row >> 3) * kSBO + (k >> 3) * kLBO + (row & 7) * 16 + (k & 7) * 2;
}
__device__ __forceinline__ uint32_t mnmajor_offset(int k, int col) {
    return (col >> 3) * kSBO + (k >> 3) * kLBO + (k & 7) * 16 + (col & 7) * 2;
}

__device__ __forceinline__ int wrap_once(int v, int size) { return v < 0 ? v + size : (v >= size ? v - size : v); }

// Writes 8 consecutive K (or MN) values, split into hi and lo, of one row of the four B planes (16 bytes per plane).
// re/im hold 8 values; `off` is the byte offset of the chunk inside a plane.
__device__ __forceinline__ void store_chunk(uint8_t *planes, uint32_t off, const float (&re)[8], const float (&im)[8]) {
    uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        split_bf16x2(re[2 * i], re[2 * i + 1], rh[i], rl[i]);
        split_bf16x2(im[2 * i], im[2 * i + 1], ih[i], il[i]);
    }
    *reinterpret_cast<uint4 *>(planes + 0 * kPlaneBytes + off) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
    *reinterpret_cast<uint4 *>(planes + 1 * kPlaneBytes + off) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
    *reinterpret_cast<uint4 *>(planes + 2 * kPlaneBytes + off) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
    *reinterpret_cast<uint4 *>(planes + 3 * kPlaneBytes + off) = make_uint4(il[0], il[1], il[2], il[3]);
}

// The 96 MMAs of one stage, D (re at d, im at d + 128) = (conj?)W * B.
__device__ __forceinline__ void issue_stage(uint32_t tmem, uint32_t planes_smem, bool conj, bool b_mn_major) {
    // (destination 0 re / 1 im, W plane, B plane, negative)
    constexpr int prod[12][4] = {{0, 0, 0, 0}, {0, 0, 1, 0}, {0, 1, 0, 0},   // + Wr Br
                                 {0, 2, 2, 1}, {0, 2, 3, 1}, {0, 3, 2, 1},   // - Wi Bi
                                 {1, 0, 2, 0}, {1, 0, 3, 0}, {1, 1, 2, 0},   // + Wr Bi
                                 {1, 2, 0, 0}, {1, 2, 1, 0}, {1, 3, 0, 0}};  // + Wi Br
#pragma unroll 1
    for (int s = 0; s < kN / 16; s++) {
#pragma unroll
        for (int i = 0; i < 12; i++) {
            const bool neg = (prod[i][3] != 0) != (conj && prod[i][1] >= 2);
            const uint32_t idesc = idesc_bf16(128, 128, false, b_mn_major, false, neg);
            const uint64_t bdesc = smem_desc(planes_smem + prod[i][2] * kPlaneBytes + s * 2 * kLBO, kLBO, kSBO);
            mma_ts(tmem + 256 + prod[i][0] * 128, tmem + prod[i][1] * 64 + s * 8, bdesc, idesc,
                   (s > 0 || (i % 6) != 0) ? 1u : 0u);
        }
    }
}

__global__ void __launch_bounds__(kThreads, 1) bf16_position_kernel(Bf16Args a) {
    extern __shared__ __align__(1024) uint8_t planes[];  // 4 x 32 KB: the B operand
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    __shared__ int stop;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int row = 32 * (warp & 3) + lane;  // this thread's TMEM lane
    const int half = warp >> 2;              // its half of the columns
    if (warp == 0) {
        tmem_alloc(&tmem_base, 512);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        stop = 0;
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = tmem_base;
    const uint32_t lane_addr = tmem_addr(tmem, 32 * (warp & 3), 0);
    const uint32_t planes_smem = smem_u32(planes);
    // W planes into tensor memory: plane q at columns 64 q, lane m = row m, column j = W[m][2j] | W[m][2j+1] << 16
    for (int q = 0; q < 4; q++)
        for (int c0 = 0; c0 < 32; c0 += 16) {
            uint32_t r[16];
            const uint32_t *src = reinterpret_cast<const uint32_t *>(a.w_planes + ((size_t)q * kN + row) * kN) + 32 * half + c0;
#pragma unroll
            for (int j = 0; j < 16; j++) r[j] = src[j];
            tmem_st16(lane_addr + q * 64 + 32 * half + c0, r);
        }
    tmem_wait_st();
    uint32_t phase = 0;
    const float inv_n = 1.0f / (float)(kN * kN);
    // one stage's MMAs after the B operand is in shared memory; false when the wait ran out
    auto run_stage = [&](bool conj, bool mn_major) -> bool {
        fence_proxy_async();
        fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            fence_after_sync();
            issue_stage(tmem, planes_smem, conj, mn_major);
            mma_commit(&mbar);
        }
        const bool ok = mbar_wait(&mbar, phase, kWaitLimit);
        if (ok) phase ^= 1u;  // on a timeout `phase` keeps the parity still outstanding, for the drain below
        else {
            stop = 1;
            *a.fault = 1;
        }
        fence_after_sync();
        return ok;
    };
    for (int p = a.first + blockIdx.x; p < a.first + a.count; p += gridDim.x) {
        // ---- stage 1: B = X (row `row` of the exit wave, columns of this half), K-major
        {
            const int rr = a.scan.rr[p], cc = a.scan.cc[p], cls = a.scan.cls[p];
            const float2 *S = a.shifted + (size_t)cls * (kN * kN) + row * kN;
            const float2 *orow = a.object + (size_t)wrap_once(rr + (row < kN / 2 ? row : row - kN), a.object_rows) * a.object_columns;
#pragma unroll 1
            for (int c8 = 64 * half; c8 < 64 * half + 64; c8 += 8) {
                float re[8], im[8];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int c = c8 + i;
                    const int x = wrap_once(cc + (c < kN / 2 ? c : c - kN), a.object_columns);
                    const float2 s = S[c], o = orow[x];
                    re[i] = s.x * o.x - s.y * o.y;
                    im[i] = s.x * o.y + s.y * o.x;
                }
                store_chunk(planes, kmajor_offset(row, c8), re, im);
            }
        }
        run_stage(false, false);
        __syncthreads();
        if (stop) break;
        // ---- stage 2: B = Y, K-major [k][r]: lane k's row of Y^T
#pragma unroll 1
        for (int c16 = 64 * half; c16 < 64 * half + 64; c16 += 16) {
            float re[16], im[16];
            tmem_ld16(lane_addr + 256 + c16, re);
            tmem_ld16(lane_addr + 384 + c16, im);
            tmem_wait_ld();
            float r0[8], i0[8], r1[8], i1[8];
#pragma unroll
            for (int i = 0; i < 8; i++) { r0[i] = re[i]; i0[i] = im[i]; r1[i] = re[8 + i]; i1[i] = im[8 + i]; }
            store_chunk(planes, kmajor_offset(row, c16), r0, i0);
            store_chunk(planes, kmajor_offset(row, c16 + 8), r1, i1);
        }
        run_stage(false, false);
        __syncthreads();
        if (stop) break;
        // ---- projection on F (lane k_r, columns k_c of this half); stage 3: B = F', MN-major [k_r][k_c]
        {
            double err = 0;
            const float *A = a.amplitudes + (size_t)p * (kN * kN);
#pragma unroll 1
            for (int c16 = 64 * half; c16 < 64 * half + 64; c16 += 16) {
                float re[16], im[16];
                tmem_ld16(lane_addr + 256 + c16, re);
                tmem_ld16(lane_addr + 384 + c16, im);
                tmem_wait_ld();
                const float4 *am4 = reinterpret_cast<const float4 *>(A + ((size_t)(c16 >> 4) * kN + row) * 16);
#pragma unroll
                for (int h4 = 0; h4 < 4; h4++) {
                    const float4 av = am4[h4];
                    const float am[4] = {av.x, av.y, av.z, av.w};
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const int i = 4 * h4 + e;
                        const float mag = sqrtf(re[i] * re[i] + im[i] * im[i]);
                        const float miss = am[e] - mag;
                        err += (double)(miss * miss);
                        if (mag > 0.f) {
                            const float sc = (am[e] / mag - 1.0f) * inv_n;
                            re[i] *= sc;
                            im[i] *= sc;
                        } else {
                            re[i] = am[e] * inv_n;
                            im[i] = 0.f;
                        }
                    }
                }
                float r0[8], i0[8], r1[8], i1[8];
#pragma unroll
                for (int i = 0; i < 8; i++) { r0[i] = re[i]; i0[i] = im[i]; r1[i] = re[8 + i]; i1[i] = im[8 + i]; }
                store_chunk(planes, mnmajor_offset(row, c16), r0, i0);
                store_chunk(planes, mnmajor_offset(row, c16 + 8), r1, i1);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) err += __shfl_down_sync(0xffffffffu, err, o);
            if (lane == 0) a.error[(size_t)p * (kThreads / 32) + warp] = err;
        }
        run_stage(true, true);
        __syncthreads();
        if (stop) break;
        // ---- stage 4: B = Y'^T, K-major [r][k]: lane r's row of Y'
#pragma unroll 1
        for (int c16 = 64 * half; c16 < 64 * half + 64; c16 += 16) {
            float re[16], im[16];
            tmem_ld16(lane_addr + 256 + c16, re);
            tmem_ld16(lane_addr + 384 + c16, im);
            tmem_wait_ld();
            float r0[8], i0[8], r1[8], i1[8];
#pragma unroll
            for (int i = 0; i < 8; i++) { r0[i] = re[i]; i0[i] = im[i]; r1[i] = re[8 + i]; i1[i] = im[8 + i]; }
            store_chunk(planes, kmajor_offset(row, c16), r0, i0);
            store_chunk(planes, kmajor_offset(row, c16 + 8), r1, i1);
        }
        run_stage(true, false);
        __syncthreads();
        if (stop) break;
        // ---- dpsi^T: lane c, columns r of this half -> [position][c][r]
        {
            float2 *out = a.dpsi + (size_t)p * (kN * kN) + (size_t)row * kN;
#pragma unroll 1
            for (int c16 = 64 * half; c16 < 64 * half + 64; c16 += 16) {
                float re[16], im[16];
                tmem_ld16(lane_addr + 256 + c16, re);
                tmem_ld16(lane_addr + 384 + c16, im);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; i += 2)
                    *reinterpret_cast<float4 *>(out + c16 + i) = make_float4(re[i], im[i], re[i + 1], im[i + 1]);
            }
        }
        fence_before_sync();
        __syncthreads();  // every lane has read D before the next stage's MMAs overwrite it
        fence_after_sync();
    }
    fence_before_sync();
    __syncthreads();
    if (stop) {
        // a wait ran out: give the tensor core a bounded chance to drain before the columns are freed
        mbar_wait(&mbar, phase, kWaitLimit);
    }
    fence_after_sync();
    if (warp == 0) tmem_dealloc(tmem, 512);
}

// [position][row][column] -> [position][column / 16][row][column mod 16]
__global__ void permute_bf16_amplitudes_kernel(const float *in, float *out, long long positions) {
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i >= positions * kN * kN) return;
    const long long p = i / (kN * kN);
    const int rem = (int)(i - p * kN * kN);
    const int chunk = rem >> 11, row = (rem >> 4) & 127, c = rem & 15;
    out[i] = in[p * kN * kN + row * kN + chunk * 16 + c];
}

size_t bf16_smem() { return 4 * (size_t)kPlaneBytes; }

}  // namespace

bool bf16_applicable(int rows, int columns) { return rows == kN && columns == kN; }
int bf16_partials_per_position() { return kThreads / 32; }

cudaError_t configure_bf16() {
    int device = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (e != cudaSuccess) return e;
    if ((size_t)optin < bf16_smem() + 1024) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(bf16_position_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bf16_smem());
}

cudaError_t launch_bf16(const Bf16Args &a, int ctas, cudaStream_t s) {
    if (a.count <= 0) return cudaSuccess;
    const int grid = a.count < ctas ? a.count : ctas;
    bf16_position_kernel<<<grid, kThreads, bf16_smem(), s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_permute_bf16_amplitudes(const float *in, float *out, long long positions, cudaStream_t s) {
    const long long total = positions * kN * kN;
    permute_bf16_amplitudes_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(in, out, positions);
    return cudaGetLastError();
}

}  // namespace cubo
