// Allocation-free forward loss: cubo_ptycho_loss_fp32_noalloc (include/cubo_ptycho.h).
//
// Who needs it: callers that cannot call cudaMalloc.  A host application whose device memory is owned by its own pool
// allocator (one that hands plugins only the buffers it manages), or a latency-critical loop that must not allocate once
// it runs (cudaMalloc can synchronise the device and stall every stream), can still evaluate the ptychographic loss
// with this entry point: it passes its own device buffers for the inputs and the output, and the one scratch buffer the
// computation needs is a fixed array compiled into this library.
//
// The computation is the forward half of the generic FP32 position pass (exit wave S * O[patch], forward 2-D FFT in
// shared memory, squared amplitude residual summed in FP64; Ptychography.swift:321-349) for integer scan centres, then a
// fixed-order FP64 sum over positions.  The per-position residuals go to `g_loss_partials`, a file-scope device array of
// kNoallocMaxPositions doubles (8 MiB) that every GPU which loads this library holds until the process exits.  Every
// slot that a call reads is written by that same call first, so nothing has to be cleared; the array keeps the last
// call's values.  All calls on a device share the one array: calls whose kernels overlap on the GPU (different streams,
// different host threads) race on it, so a caller must order them (one stream, or events).
#include <cstdint>
#include <mutex>

#include "../../include/cubo_ptycho.h"
#include "fft_smem.cuh"

namespace cubo {
namespace {

constexpr int kNoallocMaxPositions = CUBO_PTYCHO_NOALLOC_MAX_POSITIONS;
constexpr int kNoallocThreads = 512;
constexpr int kNoallocMaxN = 16384;  // detector pixels: 128 x 128 complex64 in shared memory
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_loss_partials[kNoallocMaxPositions];

// Host-side set-up state, per device: the device address of g_loss_partials (the symbol itself is only a host-side
// stand-in and must never be passed to a kernel).  It is resolved once per device and kept for the process's life; a
// cudaDeviceReset of that device would invalidate it, which the header rules out.
std::mutex g_setup_mutex;
double *g_partials_address[kMaxDevices] = {};

__device__ __forceinline__ int wrap_any(int v, int size) {
    const int m = v % size;
    return m < 0 ? m + size : m;
}

__global__ void __launch_bounds__(kNoallocThreads, 1)
noalloc_forward_kernel(int rows, int columns, int object_rows, int object_columns, const float *amplitudes,
                       const int *centre_rows, const int *centre_columns, const float2 *object, const float2 *probe,
                       Radices rad_rows, Radices rad_columns, double *partials) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = rows * columns;
    float2 *D = reinterpret_cast<float2 *>(smem_raw);
    float2 *twr = D + n;
    float2 *twc = twr + rows;
    double *scratch = reinterpret_cast<double *>(twc + columns);
    const int tid = threadIdx.x;
    const int p = blockIdx.x;
    // W_L^t = e^{-2 pi i t / L}, evaluated in FP64 and rounded once
    for (int i = tid; i < rows; i += kNoallocThreads) {
        double s, c;
        sincospi(-2.0 * (double)i / (double)rows, &s, &c);
        twr[i] = make_float2((float)c, (float)s);
    }
    for (int i = tid; i < columns; i += kNoallocThreads) {
        double s, c;
        sincospi(-2.0 * (double)i / (double)columns, &s, &c);
        twc[i] = make_float2((float)c, (float)s);
    }
    const int rr = wrap_any(centre_rows[p], object_rows), cc = wrap_any(centre_columns[p], object_columns);
    for (int k = tid; k < n; k += kNoallocThreads) {
        const int kr = k / columns, kc = k - kr * columns;
        const int y = wrap_any(rr + corner_offset(kr, rows), object_rows);
        const int x = wrap_any(cc + corner_offset(kc, columns), object_columns);
        D[k] = cmul(probe[k], object[(size_t)y * object_columns + x]);
    }
    __syncthreads();
    fft2_smem<float, kNoallocThreads, kNoallocMaxN>(D, rows, columns, rad_rows, rad_columns, twr, twc, false);
    const float *A = amplitudes + (size_t)p * n;
    double err = 0;
    for (int k = tid; k < n; k += kNoallocThreads) {
        const float2 f = D[k];
        const float miss = A[k] - sqrtf(f.x * f.x + f.y * f.y);
        err += (double)(miss * miss);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) err += __shfl_down_sync(0xffffffffu, err, o);
    if ((tid & 31) == 0) scratch[tid >> 5] = err;
    __syncthreads();
    if (tid == 0) {
        double total = 0;
        for (int w = 0; w < kNoallocThreads / 32; w++) total += scratch[w];
        partials[p] = total;
    }
}

// Fixed-order FP64 sum of partials[0, count) into *loss (one CTA).
__global__ void __launch_bounds__(1024) noalloc_sum_kernel(const double *partials, int count, double *loss) {
    __shared__ double scratch[32];
    const long long b = (long long)count * threadIdx.x / 1024, e = (long long)count * (threadIdx.x + 1) / 1024;
    double s = 0;
    for (long long i = b; i < e; i++) s += partials[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < 32; w++) t += scratch[w];
        *loss = t;
    }
}

size_t forward_smem(int rows, int columns) {
    return (size_t)(rows * columns + rows + columns) * sizeof(float2) + 32 * sizeof(double);
}

// Once per device, with that device current: resolve the scratch array's device address and raise the kernel's
// shared-memory limit.
int setup_device(int device, double **partials) {
    if (device < 0 || device >= kMaxDevices) return CUBO_PTYCHO_CUDA_ERROR;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_address[device]) {
        void *ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_loss_partials) != cudaSuccess || !ptr) {
            cudaGetLastError();
            return CUBO_PTYCHO_CUDA_ERROR;
        }
        int optin = 0;
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess ||
            cudaFuncSetAttribute(noalloc_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin) != cudaSuccess) {
            cudaGetLastError();
            return CUBO_PTYCHO_CUDA_ERROR;
        }
        g_partials_address[device] = static_cast<double *>(ptr);
    }
    *partials = g_partials_address[device];
    return CUBO_PTYCHO_OK;
}

}  // namespace
}  // namespace cubo

extern "C" CUBO_PTYCHO_API int cubo_ptycho_loss_fp32_noalloc(int rows, int columns, int object_rows, int object_columns,
                                                             int count, const float *amplitudes, const int *centre_rows,
                                                             const int *centre_columns, const float *object,
                                                             const float *probe, double *loss, void *stream) {
    using namespace cubo;
    if (!(rows > 1 && columns > 1 && object_rows >= rows && object_columns >= columns)) return CUBO_PTYCHO_INVALID_INPUT;
    if (count < 1 || count > kNoallocMaxPositions) return CUBO_PTYCHO_INVALID_INPUT;  // beyond the scratch array
    if (!amplitudes || !centre_rows || !centre_columns || !object || !probe || !loss) return CUBO_PTYCHO_INVALID_INPUT;
    // the kernels read complex samples as float2 and write the loss as one double: a pointer off that alignment would
    // fault on the device instead of returning a status
    if ((((uintptr_t)object | (uintptr_t)probe | (uintptr_t)loss) & 7) != 0 ||
        (((uintptr_t)amplitudes | (uintptr_t)centre_rows | (uintptr_t)centre_columns) & 3) != 0)
        return CUBO_PTYCHO_INVALID_INPUT;
    if ((long long)rows * columns > kNoallocMaxN) return CUBO_PTYCHO_UNSUPPORTED;
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        cudaGetLastError();
        return CUBO_PTYCHO_NO_DEVICE;
    }
    double *partials = nullptr;
    const int st = setup_device(device, &partials);
    if (st != CUBO_PTYCHO_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    noalloc_forward_kernel<<<count, kNoallocThreads, forward_smem(rows, columns), s>>>(
        rows, columns, object_rows, object_columns, amplitudes, centre_rows, centre_columns,
        reinterpret_cast<const float2 *>(object), reinterpret_cast<const float2 *>(probe), factor_length(rows),
        factor_length(columns), partials);
    if (cudaGetLastError() != cudaSuccess) return CUBO_PTYCHO_CUDA_ERROR;
    noalloc_sum_kernel<<<1, 1024, 0, s>>>(partials, count, loss);
    if (cudaGetLastError() != cudaSuccess) return CUBO_PTYCHO_CUDA_ERROR;
    return CUBO_PTYCHO_OK;
}
