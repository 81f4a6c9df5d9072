// Test harness for the tcgen05 helpers of cubokit_b200/csrc/umma.cuh (built and run only by tests/test_gpu_umma.py).
//
// One CTA of 256 threads computes the complex product D = W * B (128 x 128 x 128) the way the split-BF16 DFT kernel does:
// the four bf16 planes of W (re hi, re lo, im hi, im lo; [m][k]) in tensor memory as the A operand, the four planes of B
// (logical [k][n]) in shared memory as the B operand, K-major ([n][k]) or MN-major ([k][n]) canonical layout, and the
// three split products hi*hi + hi*lo + lo*hi of each real product accumulated in FP32 tensor memory.
#include <cuda_runtime.h>
#include <stdint.h>

#include "umma.cuh"

using namespace cubo::umma;

namespace {

constexpr int N = 128;

// Canonical no-swizzle layouts with core matrices adjacent in K `lbo` bytes apart and 8-row groups `sbo` bytes apart
// (lbo = 128, sbo = 2048 packs them; lbo = 144 pads 16 bytes between K chunks).
__device__ __forceinline__ uint32_t kmajor_offset(int row, int k, uint32_t lbo, uint32_t sbo) {  // row = M/N, k = K
    return (row >> 3) * sbo + (k >> 3) * lbo + (row & 7) * 16 + (k & 7) * 2;
}
__device__ __forceinline__ uint32_t mnmajor_offset(int k, int col, uint32_t lbo, uint32_t sbo) {  // col = M/N
    return (col >> 3) * sbo + (k >> 3) * lbo + (k & 7) * 16 + (col & 7) * 2;
}

// withhold_commit: issue nothing and never commit, so the completion wait must run out (the bounded-wait path).
__global__ void __launch_bounds__(256, 1) probe_kernel(const uint16_t *w, const uint16_t *b, int b_mn_major, int conj_w,
                                                       int withhold_commit, uint32_t lbo, uint32_t sbo, float *out,
                                                       int *status) {
    const uint32_t plane = 16 * sbo;  // bytes of one B plane
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        tmem_alloc(&tmem_base, 512);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(&mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t base = tmem_base;
    // W planes into tensor memory: plane q at columns q*64 .. q*64+63, lane m = row, column j = (k 2j, k 2j+1)
    const int m = 32 * (warp & 3) + lane, half = warp >> 2;
    for (int q = 0; q < 4; q++)
        for (int c0 = 0; c0 < 32; c0 += 16) {
            uint32_t r[16];
#pragma unroll
            for (int jj = 0; jj < 16; jj++) {
                const int j = 32 * half + c0 + jj;
                r[jj] = (uint32_t)w[(q * N + m) * N + 2 * j] | ((uint32_t)w[(q * N + m) * N + 2 * j + 1] << 16);
            }
            tmem_st16(tmem_addr(base, 32 * (warp & 3), q * 64 + 32 * half + c0), r);
        }
    tmem_wait_st();
    // B planes into shared memory
    for (int q = 0; q < 4; q++)
        for (int e = tid; e < N * N; e += 256) {
            const int k = e / N, n = e % N;  // logical B[k][n]
            const uint32_t off = b_mn_major ? mnmajor_offset(k, n, lbo, sbo) : kmajor_offset(n, k, lbo, sbo);
            *reinterpret_cast<uint16_t *>(smem + q * plane + off) = b[(q * N + k) * N + n];
        }
    fence_proxy_async();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (tid == 0 && !withhold_commit) {
        // (d: 0 re / 1 im, A plane, B plane, negate)
        const int prod[12][4] = {{0, 0, 0, 0}, {0, 0, 1, 0}, {0, 1, 0, 0},   // + Wr Br
                                 {0, 2, 2, 1}, {0, 2, 3, 1}, {0, 3, 2, 1},   // - Wi Bi
                                 {1, 0, 2, 0}, {1, 0, 3, 0}, {1, 1, 2, 0},   // + Wr Bi
                                 {1, 2, 0, 0}, {1, 2, 1, 0}, {1, 3, 0, 0}};  // + Wi Br
        const uint32_t smem_base = smem_u32(smem);
        for (int s = 0; s < N / 16; s++)
            for (int i = 0; i < 12; i++) {
                bool neg = prod[i][3] != 0;
                if (conj_w && prod[i][1] >= 2) neg = !neg;  // conj(W): every Wi term changes sign
                const uint32_t idesc = idesc_bf16(128, 128, false, b_mn_major != 0, false, neg);
                const uint64_t bdesc = smem_desc(smem_base + prod[i][2] * plane + s * 2 * lbo, lbo, sbo);
                const uint32_t d = base + 256 + prod[i][0] * 128;
                const uint32_t a = base + prod[i][1] * 64 + s * 8;
                const uint32_t acc = (s > 0 || (i % 6) != 0) ? 1u : 0u;
                mma_ts(d, a, bdesc, idesc, acc);
            }
        mma_commit(&mbar);
    }
    const bool done = mbar_wait(&mbar, 0, withhold_commit ? 200000000ull : 2000000000ull);
    if (!done && tid == 0) *status = 1;
    fence_after_sync();
    if (done) {
        for (int part = 0; part < 2; part++)
            for (int c0 = 0; c0 < 64; c0 += 16) {
                float v[16];
                tmem_ld16(tmem_addr(base, 32 * (warp & 3), 256 + part * 128 + 64 * half + c0), v);
                tmem_wait_ld();
#pragma unroll
                for (int jj = 0; jj < 16; jj++) out[(part * N + m) * N + 64 * half + c0 + jj] = v[jj];
            }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(base, 512);
}

}  // namespace

extern "C" int umma_probe_complex_strided(const uint16_t *w_host, const uint16_t *b_host, int b_mn_major, int conj_w,
                                          int withhold_commit, uint32_t lbo, uint32_t sbo, float *out_host) {
    if (lbo < 128 || lbo % 16 || sbo < 16 * lbo || sbo % 16) return -3;  // layouts that keep core matrices apart
    uint16_t *w = nullptr, *b = nullptr;
    float *out = nullptr;
    int *status = nullptr, st = 0;
    const size_t planes = 4 * N * N * sizeof(uint16_t);
    if (cudaMalloc(&w, planes) || cudaMalloc(&b, planes) || cudaMalloc(&out, 2 * N * N * sizeof(float)) ||
        cudaMalloc(&status, sizeof(int)))
        return -1;
    cudaMemcpy(w, w_host, planes, cudaMemcpyHostToDevice);
    cudaMemcpy(b, b_host, planes, cudaMemcpyHostToDevice);
    cudaMemset(status, 0, sizeof(int));
    cudaMemset(out, 0, 2 * N * N * sizeof(float));
    const int smem = 4 * 16 * (int)sbo;
    cudaFuncSetAttribute(probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    probe_kernel<<<1, 256, smem>>>(w, b, b_mn_major, conj_w, withhold_commit, lbo, sbo, out, status);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return -2;
    cudaMemcpy(out_host, out, 2 * N * N * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(w);
    cudaFree(b);
    cudaFree(out);
    cudaFree(status);
    return st;
}

extern "C" int umma_probe_complex(const uint16_t *w_host, const uint16_t *b_host, int b_mn_major, int conj_w,
                                  int withhold_commit, float *out_host) {
    return umma_probe_complex_strided(w_host, b_host, b_mn_major, conj_w, withhold_commit, 128, 2048, out_host);
}
