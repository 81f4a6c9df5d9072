// FP64 probe-sized kernels: 2-D FFTs of probe fields in global memory, the probe update, the probe constraints
// (Sources/CuboPtycho/PtychographyConstraints.swift:9-83, called at Ptychography.swift:383-395), the shifted-probe table
// for fractional positions (Ptychography.swift:303-320) and the probe builder's spectrum (Ptychography.swift:155-167).
// All of this is O(n) or O(n log n) once per iteration; it runs in FP64 in every form, as the reference's Float path
// also keeps the probe spectrum and the constraints in Double (PtychographySingle.swift:109-115,202-211).
#include <cfloat>

#include "engine.h"

namespace cubo {

namespace {

constexpr int kLineThreads = 256;
constexpr int kLineMaxN = 4096;  // elements of the lines one CTA holds (64 KB of complex128)

// Rows (columns == false) or columns of `batch` rows x columns fields, lines_per_block lines per CTA.
// R0 = 0: the plan `rad` at run time; else the compile-time plan R0 x R1 x R2 (it must equal `rad`).
template <int R0, int R1, int R2>
__global__ void __launch_bounds__(kLineThreads) fft_lines_kernel(double2 *data, int rows, int columns, int batch,
                                                                 bool columns_pass, int lines_per_block, Radices rad,
                                                                 const double2 *tw_global, bool inv) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int L = columns_pass ? rows : columns;
    const int lines_total = batch * (columns_pass ? columns : rows);
    double2 *D = reinterpret_cast<double2 *>(smem_raw);
    double2 *tw = D + (size_t)lines_per_block * L;
    for (int i = threadIdx.x; i < L; i += kLineThreads) tw[i] = tw_global[i];
    const int first = blockIdx.x * lines_per_block;
    const int nl = min(lines_per_block, lines_total - first);
    const long long n = (long long)rows * columns;
    // line l: rows pass -> field l / rows, row l % rows, stride 1, one line after the other in shared memory;
    // columns pass -> field l / columns, column l % columns, stride C, staged as rows of the nl columns (element e of
    // line j at e * nl + j) so that consecutive threads read consecutive columns of one row
    // the tile comes in with 16-byte asynchronous copies (all of a thread's copies in flight at once)
    const uint32_t d0 = (uint32_t)__cvta_generic_to_shared(D);
    auto copy_in = [&](int i, long long src) {
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d0 + 16u * (uint32_t)i), "l"(data + src)
                     : "memory");
    };
    if (columns_pass) {
        if (columns % nl == 0 && kLineThreads % nl == 0) {
            // the block's nl columns lie in one field: each thread keeps its column and walks down the rows
            const long long base = (long long)(first / columns) * n + first % columns;
            const int j = threadIdx.x % nl, rows_step = kLineThreads / nl;
            for (int e = threadIdx.x / nl; e < L; e += rows_step) copy_in(e * nl + j, base + (long long)e * columns + j);
        } else {
            for (int i = threadIdx.x; i < nl * L; i += kLineThreads) {
                const int j = i % nl, e = i / nl, l = first + j;
                copy_in(i, (long long)(l / columns) * n + (long long)e * columns + (l % columns));
            }
        }
    } else {
        const long long base = (long long)first * columns;  // consecutive lines are consecutive rows
        for (int i = threadIdx.x; i < nl * L; i += kLineThreads) copy_in(i, base + i);
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    const LineGeom geom = columns_pass ? LineGeom{L, nl, nl, 1} : LineGeom{L, nl, 1, L};
    if constexpr (R0 == 0) line_fft<double, kLineThreads, kLineMaxN>(D, geom, rad, tw, inv);
    else line_fft_fixed<double, kLineThreads, kLineMaxN, R0, R1, R2>(D, geom, tw, inv);
    if (columns_pass) {
        if (columns % nl == 0 && kLineThreads % nl == 0) {
            const long long base = (long long)(first / columns) * n + first % columns;
            const int j = threadIdx.x % nl, rows_step = kLineThreads / nl;
            for (int e = threadIdx.x / nl; e < L; e += rows_step) data[base + (long long)e * columns + j] = D[e * nl + j];
        } else {
            for (int i = threadIdx.x; i < nl * L; i += kLineThreads) {
                const int j = i % nl, e = i / nl, l = first + j;
                data[(long long)(l / columns) * n + (long long)e * columns + (l % columns)] = D[i];
            }
        }
    } else {
        const long long base = (long long)first * columns;
        for (int i = threadIdx.x; i < nl * L; i += kLineThreads) data[base + i] = D[i];
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Fixed-order sum over one CTA of 1024 threads; thread 0 gets the result.
__device__ double block_sum1024(double v, double *scratch) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) scratch[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < 32; w++) t += scratch[w];
    __syncthreads();
    return t;
}

__global__ void scale_kernel(double2 *d, int count, double s) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i < count) { d[i].x *= s; d[i].y *= s; }
}

// Ptychography.swift:383-386
__global__ void probe_update_kernel(double2 *probe, const double2 *grad, const double *weight, int n,
                                    const double *max_weight, double step, double minimum) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= n) return;
    const double l = (1 - minimum) * weight[k], x = minimum * *max_weight;
    const double s = step * (1 / sqrt(1e-16 + l * l + x * x));
    probe[k].x += s * grad[k].x;
    probe[k].y += s * grad[k].y;
}

// PtychographyConstraints.swift:9-18: total intensity and its corner-centred first moments.
__global__ void __launch_bounds__(1024) moments_kernel(const double2 *p, int rows, int columns, double *sums) {
    __shared__ double scratch[32];
    double t = 0, mr = 0, mc = 0;
    const int n = rows * columns;
    for (int k = threadIdx.x; k < n; k += 1024) {
        const int r = k / columns, c = k - r * columns;
        const double w = p[k].x * p[k].x + p[k].y * p[k].y;
        t += w;
        mr += frequency(r, rows) * (double)rows * w;
        mc += frequency(c, columns) * (double)columns * w;
    }
    t = block_sum1024(t, scratch);
    mr = block_sum1024(mr, scratch);
    mc = block_sum1024(mc, scratch);
    if (threadIdx.x == 0) { sums[0] = t; sums[1] = mr; sums[2] = mc; }
}

__global__ void __launch_bounds__(1024) energy_kernel(const double2 *p, int n, double *sum) {
    __shared__ double scratch[32];
    double t = 0;
    for (int k = threadIdx.x; k < n; k += 1024) t += p[k].x * p[k].x + p[k].y * p[k].y;
    t = block_sum1024(t, scratch);
    if (threadIdx.x == 0) *sum = t;
}

__device__ __forceinline__ bool com_valid(const double *sums) { return sums[0] > 0 && isfinite(sums[0]); }

// PtychographyConstraints.swift:21-31 with (row, column) = -(centre of mass): spectrum *= e^{-2 pi i (fr row + fc col)}
__global__ void com_ramp_kernel(double2 *spec, int rows, int columns, const double *sums) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= rows * columns || !com_valid(sums)) return;
    const double row = -sums[1] / sums[0], column = -sums[2] / sums[0];
    const int r = k / columns, c = k - r * columns;
    const double phase = -2 * 3.14159265358979323846 * (frequency(r, rows) * row + frequency(c, columns) * column);
    double sn, cs;
    sincos(phase, &sn, &cs);
    const double a = spec[k].x, b = spec[k].y;
    spec[k] = make_double2(a * cs - b * sn, a * sn + b * cs);
}

__global__ void commit_kernel(double2 *probe, const double2 *candidate, int n, const double *sums) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k < n && com_valid(sums)) probe[k] = candidate[k];
}

// PtychographyConstraints.swift:62-65: keep the phase, take the initial Fourier amplitude.
__global__ void aperture_phase_kernel(double2 *spec, const double *aperture, int n) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= n) return;
    const double ph = atan2(spec[k].y, spec[k].x);
    double sn, cs;
    sincos(ph, &sn, &cs);
    spec[k] = make_double2(aperture[k] * cs, aperture[k] * sn);
}

// PtychographyConstraints.swift:43-51: the erf top-hat in cycles per pixel.
__global__ void amplitude_mask_kernel(double2 *p, int rows, int columns, double radius, double width) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= rows * columns) return;
    const int r = k / columns, c = k - r * columns;
    const double sigma = sqrt(3.14159265358979323846) / width;
    const double d = hypot(frequency(r, rows), frequency(c, columns)) - radius;
    const double mask = 0.5 * (1 - erf(sigma * d / (1 - d * d)));
    p[k].x *= mask;
    p[k].y *= mask;
}

// dst = src * sqrt(before / after) when both are positive, else dst = src (PtychographyConstraints.swift:52-54,68-70).
__global__ void renormalise_kernel(double2 *dst, const double2 *src, int n, const double *before, const double *after) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= n) return;
    const double b = *before, a = *after;
    const double s = (b > 0 && a > 0) ? sqrt(b / a) : 1.0;
    dst[k] = make_double2(src[k].x * s, src[k].y * s);
}

// PtychographyConstraints.swift:74-76
__global__ void support_kernel(double2 *p, const unsigned char *mask, int n) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k < n && !mask[k]) p[k] = make_double2(0, 0);
}

__global__ void magnitude_kernel(const double2 *d, double *out, int n) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k < n) out[k] = hypot(d[k].x, d[k].y);
}

// Ptychography.swift:304-319: spectrum times the product of a row ramp and a column ramp, one field per shift class.
__global__ void shift_ramps_kernel(const double2 *spec, const double2 *rr, const double2 *rc, int rows, int columns,
                                   int classes, double2 *out) {
    const long long n = (long long)rows * columns;
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i >= n * classes) return;
    const int cls = (int)(i / n);
    const int k = (int)(i - cls * n);
    const int r = k / columns, c = k - r * columns;
    const double2 a = rr[(size_t)cls * rows + r], b = rc[(size_t)cls * columns + c];
    const double cs = a.x * b.x - a.y * b.y, sn = a.y * b.x + a.x * b.y;
    const double2 s = spec[k];
    out[i] = make_double2(s.x * cs - s.y * sn, s.x * sn + s.y * cs);
}

template <typename T>
__global__ void convert_kernel(const double2 *in, C2<T> *out, long long count) {
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    if (i < count) out[i] = mk<T>((T)in[i].x, (T)in[i].y);
}

// Ptychography.swift:155-166: aperture with cosine rolloff times e^{-i chi}.
__global__ void probe_spectrum_kernel(double2 *out, int rows, int columns, double row_sampling, double column_sampling,
                                      double wavelength, double cutoff, double rolloff, double defocus,
                                      double astigmatism, double astigmatism_angle, double spherical, int term_count,
                                      const double *terms) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= rows * columns) return;
    const int r = k / columns, c = k - r * columns;
    const double pi = 3.14159265358979323846;
    const double qr = frequency(r, rows) / row_sampling, qc = frequency(c, columns) / column_sampling;
    const double alpha = hypot(qr, qc) * wavelength, angle = atan2(qc, qr);
    double aperture;
    if (rolloff > 0 && alpha > cutoff - rolloff) aperture = alpha > cutoff ? 0 : 0.5 * (1 + cos(pi * (alpha - cutoff + rolloff) / rolloff));
    else aperture = alpha < cutoff ? 1 : 0;
    const double a2 = alpha * alpha;
    double phase = a2 / 2 * (-defocus + astigmatism * cos(2 * (angle - astigmatism_angle))) + a2 * a2 / 4 * spherical;
    for (int t = 0; t < term_count; t++) {  // Ptychography.swift:127-132
        const int nr = (int)terms[4 * t], mr = (int)terms[4 * t + 1];
        const double radial = pow(alpha, (double)(nr + 1)) / (double)(nr + 1);
        if (mr == 0) phase += terms[4 * t + 3] * radial;
        else {
            const double an = (double)mr * angle;
            phase += terms[4 * t + 3] * radial * (terms[4 * t + 2] != 0 ? sin(an) : cos(an));
        }
    }
    const double chi = 2 * pi / wavelength * phase;
    out[k] = make_double2(aperture * cos(chi), -aperture * sin(chi));
}

inline int blocks(long long count) { return (int)((count + 255) / 256); }

}  // namespace

cudaError_t launch_fft2_f64(const Fft2Plan64 &p, double2 *data, int batch, bool inverse, cudaStream_t s) {
    static_assert(kLineMaxN * sizeof(double2) + 1024 * sizeof(double2) <= 232448, "line FFT shared memory");
    for (int pass = 0; pass < 2; pass++) {
        const bool cols = pass == 1;
        const int L = cols ? p.rows : p.columns;
        if (L > kLineMaxN) return cudaErrorInvalidValue;
        const int lines = batch * (cols ? p.columns : p.rows);
        const int lpb = kLineMaxN / L;
        const size_t smem = ((size_t)lpb * L + L) * sizeof(double2);
        const Radices &rad = cols ? p.rad_rows : p.rad_columns;
        auto plan_is = [&](int a, int b, int c) {
            const int want[3] = {a, b, c};
            const int count = c ? 3 : (b ? 2 : 1);
            if (rad.count != count) return false;
            for (int i = 0; i < count; i++)
                if (rad.r[i] != want[i]) return false;
            return true;
        };
        // compile-time plans of the usual line lengths (128 = 8 x 8 x 2, 64 = 8 x 8, 256 = 8 x 8 x 4, 32 = 8 x 4)
        auto kernel = plan_is(8, 8, 2) ? fft_lines_kernel<8, 8, 2>
                      : plan_is(8, 8, 0) ? fft_lines_kernel<8, 8, 0>
                      : plan_is(8, 8, 4) ? fft_lines_kernel<8, 8, 4>
                      : plan_is(8, 4, 0) ? fft_lines_kernel<8, 4, 0>
                                         : fft_lines_kernel<0, 0, 0>;
        kernel<<<(lines + lpb - 1) / lpb, kLineThreads, smem, s>>>(data, p.rows, p.columns, batch, cols, lpb, rad,
                                                                   cols ? p.tw_rows : p.tw_columns, inverse);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

bool line_fft_supported(int rows, int columns) { return rows <= kLineMaxN && columns <= kLineMaxN; }

// The line-FFT kernel's shared-memory limit, once per device (outside any stream capture).
cudaError_t configure_fft_lines() {
    const int bytes = (int)((kLineMaxN + kLineMaxN) * sizeof(double2));
    for (auto f : {fft_lines_kernel<0, 0, 0>, fft_lines_kernel<8, 8, 2>, fft_lines_kernel<8, 8, 0>,
                   fft_lines_kernel<8, 8, 4>, fft_lines_kernel<8, 4, 0>}) {
        const cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_scale_f64(double2 *data, int count, double scale, cudaStream_t s) {
    scale_kernel<<<blocks(count), 256, 0, s>>>(data, count, scale);
    return cudaGetLastError();
}

cudaError_t launch_probe_update(double2 *probe, const double2 *grad, const double *weight, int n,
                                const double *max_weight, double step, double minimum, cudaStream_t s) {
    probe_update_kernel<<<blocks(n), 256, 0, s>>>(probe, grad, weight, n, max_weight, step, minimum);
    return cudaGetLastError();
}

cudaError_t launch_probe_moments(const double2 *probe, int rows, int columns, double *sums, cudaStream_t s) {
    moments_kernel<<<1, 1024, 0, s>>>(probe, rows, columns, sums);
    return cudaGetLastError();
}

cudaError_t launch_energy(const double2 *data, int n, double *sum, cudaStream_t s) {
    energy_kernel<<<1, 1024, 0, s>>>(data, n, sum);
    return cudaGetLastError();
}

cudaError_t launch_com_ramp(double2 *spectrum, int rows, int columns, const double *sums, cudaStream_t s) {
    com_ramp_kernel<<<blocks(rows * columns), 256, 0, s>>>(spectrum, rows, columns, sums);
    return cudaGetLastError();
}

cudaError_t launch_commit_if_valid(double2 *probe, const double2 *candidate, int n, const double *sums,
                                   cudaStream_t s) {
    commit_kernel<<<blocks(n), 256, 0, s>>>(probe, candidate, n, sums);
    return cudaGetLastError();
}

cudaError_t launch_aperture_phase(double2 *spectrum, const double *aperture, int n, cudaStream_t s) {
    aperture_phase_kernel<<<blocks(n), 256, 0, s>>>(spectrum, aperture, n);
    return cudaGetLastError();
}

cudaError_t launch_amplitude_mask(double2 *probe, int rows, int columns, double radius, double width,
                                  cudaStream_t s) {
    amplitude_mask_kernel<<<blocks(rows * columns), 256, 0, s>>>(probe, rows, columns, radius, width);
    return cudaGetLastError();
}

cudaError_t launch_renormalise(double2 *dst, const double2 *src, int n, const double *before, const double *after,
                               cudaStream_t s) {
    renormalise_kernel<<<blocks(n), 256, 0, s>>>(dst, src, n, before, after);
    return cudaGetLastError();
}

cudaError_t launch_support_mask(double2 *probe, const unsigned char *mask, int n, cudaStream_t s) {
    support_kernel<<<blocks(n), 256, 0, s>>>(probe, mask, n);
    return cudaGetLastError();
}

cudaError_t launch_magnitude(const double2 *data, double *out, int n, cudaStream_t s) {
    magnitude_kernel<<<blocks(n), 256, 0, s>>>(data, out, n);
    return cudaGetLastError();
}

cudaError_t launch_shift_ramps(const double2 *spectrum, const double2 *ramps_rows, const double2 *ramps_columns,
                               int rows, int columns, int classes, double2 *out, cudaStream_t s) {
    shift_ramps_kernel<<<blocks((long long)rows * columns * classes), 256, 0, s>>>(spectrum, ramps_rows,
                                                                                   ramps_columns, rows, columns,
                                                                                   classes, out);
    return cudaGetLastError();
}

// The phase ramps of the shift classes (Ptychography.swift:304-311): rows[f][r] = exp(-2 pi i frequency(r) dr_f),
// columns[f][c] likewise with dc_f; fractions[f] = (dr_f, dc_f).
__global__ void ramp_table_kernel(const double2 *fractions, int classes, int rows, int columns, double2 *ramps_rows,
                                  double2 *ramps_columns) {
    const long long i = (long long)blockIdx.x * 256 + threadIdx.x;
    const int per = rows + columns;
    if (i >= (long long)classes * per) return;
    const int f = (int)(i / per), j = (int)(i - (long long)f * per);
    double sn, cs;
    if (j < rows) {
        sincospi(-2.0 * frequency(j, rows) * fractions[f].x, &sn, &cs);
        ramps_rows[(size_t)f * rows + j] = make_double2(cs, sn);
    } else {
        const int c = j - rows;
        sincospi(-2.0 * frequency(c, columns) * fractions[f].y, &sn, &cs);
        ramps_columns[(size_t)f * columns + c] = make_double2(cs, sn);
    }
}

cudaError_t launch_ramp_table(const double2 *fractions, int classes, int rows, int columns, double2 *ramps_rows,
                              double2 *ramps_columns, cudaStream_t s) {
    if (classes <= 0) return cudaSuccess;
    ramp_table_kernel<<<blocks((long long)classes * (rows + columns)), 256, 0, s>>>(fractions, classes, rows, columns,
                                                                                    ramps_rows, ramps_columns);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_convert(const double2 *in, C2<T> *out, long long count, cudaStream_t s) {
    convert_kernel<T><<<blocks(count), 256, 0, s>>>(in, out, count);
    return cudaGetLastError();
}
template cudaError_t launch_convert<float>(const double2 *, float2 *, long long, cudaStream_t);
template cudaError_t launch_convert<double>(const double2 *, double2 *, long long, cudaStream_t);

cudaError_t launch_probe_spectrum(double2 *out, int rows, int columns, double row_sampling, double column_sampling,
                                  double wavelength, double cutoff, double rolloff, double defocus, double astigmatism,
                                  double astigmatism_angle, double spherical, int term_count, const double *terms,
                                  cudaStream_t s) {
    probe_spectrum_kernel<<<blocks(rows * columns), 256, 0, s>>>(out, rows, columns, row_sampling, column_sampling,
                                                                 wavelength, cutoff, rolloff, defocus, astigmatism,
                                                                 astigmatism_angle, spherical, term_count, terms);
    return cudaGetLastError();
}

}  // namespace cubo
