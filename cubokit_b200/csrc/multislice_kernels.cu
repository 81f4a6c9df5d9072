// The multislice engine's own kernels (MultislicePtychography, PtychographyEngines.swift:458-588), FP64: the object is a
// stack of slices with a Fresnel propagation between neighbours.  The engine's batched FFT and its projection, gathers
// and updates do the rest:
//
//   forward    wave_0 = the shifted probe; exit_s = wave_s x O_s[patch]; wave_{s+1} = IFFT(FFT(exit_s) x prop_s)
//   detector   chi = IFFT(projection of FFT(exit_{L-1}))
//   backward   slice s's gradient sums conj(wave_s) chi (the object gather, wave_s in place of the shifted probe);
//              chi <- chi x conj(O_s[patch]), then IFFT(FFT(chi) x conj(prop_{s-1})) for s > 0; at slice 0 the probe
//              gradient sums conj(O_0[patch]) chi (the probe gather)
//   slices     identicalSlices: every slice replaced by their mean (:566-572)
#include "engine.h"

namespace cubo {

namespace {

__device__ __forceinline__ int wrap_once(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

// out[p][k] = in[class(p)][k] x O[patch(p)][k] (conj(O) when conj_object; O = 1 when object is null), positions
// first .. first + m - 1; class(p) = scan.cls[p] when by_class, else p.  in and out may be the same buffer.
__global__ void __launch_bounds__(256) patch_multiply_kernel(const double2 *in, int by_class, const double2 *object,
                                                             int conj_object, ScanTables scan, int first, int m,
                                                             int rows, int columns, int object_rows,
                                                             int object_columns, double2 *out) {
    const int n = rows * columns;
    const long long t = (long long)blockIdx.x * 256 + threadIdx.x;
    if (t >= (long long)m * n) return;
    const int i = (int)(t / n), k = (int)(t - (long long)i * n);
    const int p = first + i;
    double2 v = in[(size_t)(by_class ? scan.cls[p] : p) * n + k];
    if (object) {
        const int kr = k / columns, kc = k - kr * columns;
        const int y = wrap_once(scan.rr[p] + corner_offset(kr, rows), object_rows);
        const int x = wrap_once(scan.cc[p] + corner_offset(kc, columns), object_columns);
        double2 o = object[(size_t)y * object_columns + x];
        if (conj_object) o.y = -o.y;
        v = cmul(v, o);
    }
    out[(size_t)p * n + k] = v;
}

// data[p][k] *= scale x prop[k] (conj(prop[k]) when conj_prop), every plane of `planes`.
__global__ void __launch_bounds__(256) spectrum_multiply_kernel(double2 *data, long long planes, int n,
                                                                const double2 *prop, int conj_prop, double scale) {
    const long long t = (long long)blockIdx.x * 256 + threadIdx.x;
    if (t >= planes * n) return;
    const int k = (int)(t % n);
    double2 w = prop[k];
    if (conj_prop) w.y = -w.y;
    const double2 v = cmul(data[t], w);
    data[t] = make_double2(v.x * scale, v.y * scale);
}

// Every slice replaced by the mean of all slices, summed slice by slice in order.
__global__ void __launch_bounds__(256) average_slices_kernel(double2 *object, int slices, long long plane) {
    const long long j = (long long)blockIdx.x * 256 + threadIdx.x;
    if (j >= plane) return;
    double sr = 0.0, si = 0.0;
    for (int s = 0; s < slices; s++) {
        const double2 v = object[(size_t)s * plane + j];
        sr += v.x;
        si += v.y;
    }
    const double2 mean = make_double2(sr / slices, si / slices);
    for (int s = 0; s < slices; s++) object[(size_t)s * plane + j] = mean;
}

unsigned blocks_for(long long total) { return (unsigned)((total + 255) / 256); }

}  // namespace

cudaError_t launch_patch_multiply(const double2 *in, bool by_class, const double2 *object, bool conj_object,
                                  ScanTables scan, int first, int m, int rows, int columns, int object_rows,
                                  int object_columns, double2 *out, cudaStream_t s) {
    if (m <= 0) return cudaSuccess;
    patch_multiply_kernel<<<blocks_for((long long)m * rows * columns), 256, 0, s>>>(
        in, by_class ? 1 : 0, object, conj_object ? 1 : 0, scan, first, m, rows, columns, object_rows, object_columns,
        out);
    return cudaGetLastError();
}

cudaError_t launch_spectrum_multiply(double2 *data, long long planes, int n, const double2 *prop, bool conj_prop,
                                     double scale, cudaStream_t s) {
    if (planes <= 0) return cudaSuccess;
    spectrum_multiply_kernel<<<blocks_for(planes * n), 256, 0, s>>>(data, planes, n, prop, conj_prop ? 1 : 0, scale);
    return cudaGetLastError();
}

cudaError_t launch_average_slices(double2 *object, int slices, long long plane, cudaStream_t s) {
    average_slices_kernel<<<blocks_for(plane), 256, 0, s>>>(object, slices, plane);
    return cudaGetLastError();
}

}  // namespace cubo
