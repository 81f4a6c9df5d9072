// Shared device helpers of the single-slice ptychography engine (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cubo {

template <typename T> struct Complex;
template <> struct Complex<float> { using type = float2; };
template <> struct Complex<double> { using type = double2; };
template <typename T> using C2 = typename Complex<T>::type;

template <typename T> __host__ __device__ __forceinline__ C2<T> mk(T x, T y) { C2<T> r; r.x = x; r.y = y; return r; }
template <typename V> __host__ __device__ __forceinline__ V cadd(V a, V b) { a.x += b.x; a.y += b.y; return a; }
template <typename V> __host__ __device__ __forceinline__ V csub(V a, V b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename V> __host__ __device__ __forceinline__ V cmul(V a, V b) {
    V r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
// conj(a) * b
template <typename V> __host__ __device__ __forceinline__ V cmulc(V a, V b) {
    V r; r.x = a.x * b.x + a.y * b.y; r.y = a.x * b.y - a.y * b.x; return r;
}
template <typename V> __host__ __device__ __forceinline__ V cconj(V a) { a.y = -a.y; return a; }
template <typename V, typename S> __host__ __device__ __forceinline__ V cscale(V a, S s) { a.x *= s; a.y *= s; return a; }
// multiply by -i (forward) or +i (inverse)
template <typename V> __host__ __device__ __forceinline__ V cmul_mi(V a, bool inv) {
    V r; if (inv) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; } return r;
}

// Corner-centred offset of detector index k of n: k for k < ceil(n/2), k - n otherwise (Ptychography.swift:322,326).
__host__ __device__ __forceinline__ int corner_offset(int k, int n) { return k < (n + 1) / 2 ? k : k - n; }

// fftfreq sample (Ptychography.swift:474).
__host__ __device__ __forceinline__ double frequency(int k, int n) { return (double)corner_offset(k, n) / (double)n; }

// Detector index covering object coordinate `delta = (y - centre) mod size`, or -1 when outside the window.
__device__ __forceinline__ int window_index(int delta, int n, int size) {
    const int high = (n + 1) / 2, low = n / 2;
    return delta < high ? delta : (delta >= size - low ? delta - size + n : -1);
}

}  // namespace cubo
