// Shared-memory complex FFTs of any length for one CTA (sm_100a).
//
// A line of length L = r_1 r_2 ... r_k (radices 2, 3, 4, 5, 7, 8) is transformed by Stockham autosort stages: stage s
// reads R = r_s values at stride L/R, twiddles them by W_L^{(j mod Ns) r L/(Ns R)}, runs an R-point DFT and writes them
// at stride Ns (Ns = r_1 ... r_{s-1}), which leaves the result in natural order.  A length with any other prime factor
// is transformed by a direct O(L^2) DFT.  Every stage of every line of a 2-D pass runs at once: each thread reads its
// butterflies' inputs into registers, the CTA synchronises, and the outputs are written back in place, so no second
// buffer is needed.  Twiddles W_L^t are a table evaluated in FP64 on the host (e^{-2 pi i t / L}) and rounded once.
// The convention is NumPy's: forward e^{-2 pi i}, unnormalised; the inverse uses conjugate twiddles and no 1/L (callers
// fold the 1/n of ifft2 into the data).
#pragma once

#include "common.cuh"

namespace cubo {

constexpr int kMaxStages = 24;

// Radix schedule of one line length; r[0] == 0 means "direct DFT".
struct Radices {
    int count;
    int r[kMaxStages];
};

struct LineGeom {
    int L;       // line length
    int nlines;  // number of lines
    int elem;    // element stride
    int line;    // line stride
};

inline Radices factor_length(int L) {
    Radices out{};
    int rest = L;
    const int order[6] = {8, 4, 2, 3, 5, 7};
    for (int i = 0; i < 6; i++)
        while (rest % order[i] == 0 && out.count < kMaxStages) { out.r[out.count++] = order[i]; rest /= order[i]; }
    if (rest != 1 || L < 2) { out.count = 1; out.r[0] = 0; }
    return out;
}

template <typename T, int R>
__device__ __forceinline__ void small_dft(C2<T> (&v)[R], const C2<T> *tw, int L, bool inv) {
    // R-point DFT from the line's twiddle table: W_R^m = W_L^{m L / R}.
    C2<T> out[R];
#pragma unroll
    for (int q = 0; q < R; q++) {
        C2<T> acc = v[0];
#pragma unroll
        for (int r = 1; r < R; r++) {
            C2<T> w = tw[((r * q) % R) * (L / R)];
            if (inv) w.y = -w.y;
            acc = cadd(acc, cmul(v[r], w));
        }
        out[q] = acc;
    }
#pragma unroll
    for (int q = 0; q < R; q++) v[q] = out[q];
}

template <>
__device__ __forceinline__ void small_dft<float, 2>(float2 (&v)[2], const float2 *, int, bool) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b); v[1] = csub(a, b);
}
template <>
__device__ __forceinline__ void small_dft<double, 2>(double2 (&v)[2], const double2 *, int, bool) {
    const double2 a = v[0], b = v[1];
    v[0] = cadd(a, b); v[1] = csub(a, b);
}

template <typename V>
__device__ __forceinline__ void dft4(V &x0, V &x1, V &x2, V &x3, bool inv) {
    const V t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), t3 = cmul_mi(csub(x1, x3), inv);
    x0 = cadd(t0, t2); x2 = csub(t0, t2); x1 = cadd(t1, t3); x3 = csub(t1, t3);
}

template <>
__device__ __forceinline__ void small_dft<float, 4>(float2 (&v)[4], const float2 *, int, bool inv) {
    dft4(v[0], v[1], v[2], v[3], inv);
}
template <>
__device__ __forceinline__ void small_dft<double, 4>(double2 (&v)[4], const double2 *, int, bool inv) {
    dft4(v[0], v[1], v[2], v[3], inv);
}

template <typename T>
__device__ __forceinline__ void dft8(C2<T> (&v)[8], bool inv) {
    // Two 4-point DFTs of the even and odd samples, joined by W_8^k.
    C2<T> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6], o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4(e0, e1, e2, e3, inv);
    dft4(o0, o1, o2, o3, inv);
    const T h = (T)0.70710678118654752440;  // cos(pi/4)
    // W_8^1 = h(1 - i) forward, h(1 + i) inverse; W_8^2 = -i / +i; W_8^3 = h(-1 - i) / h(-1 + i)
    const T s = inv ? (T)1 : (T)-1;
    C2<T> w1o1 = mk<T>(h * (o1.x - s * o1.y), h * (o1.y + s * o1.x));
    C2<T> w2o2 = cmul_mi(o2, inv);
    C2<T> w3o3 = mk<T>(h * (-o3.x - s * o3.y), h * (-o3.y + s * o3.x));
    v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
    v[1] = cadd(e1, w1o1); v[5] = csub(e1, w1o1);
    v[2] = cadd(e2, w2o2); v[6] = csub(e2, w2o2);
    v[3] = cadd(e3, w3o3); v[7] = csub(e3, w3o3);
}
template <>
__device__ __forceinline__ void small_dft<float, 8>(float2 (&v)[8], const float2 *, int, bool inv) { dft8<float>(v, inv); }
template <>
__device__ __forceinline__ void small_dft<double, 8>(double2 (&v)[8], const double2 *, int, bool inv) { dft8<double>(v, inv); }

// Which (line, butterfly) work item b is: consecutive items take consecutive lines when the lines are interleaved
// (line stride 1: the same element of neighbouring lines is contiguous, so a warp's accesses are too), else
// consecutive butterflies of one line.  Only the assignment of work to threads changes, not the arithmetic.
__device__ __forceinline__ void line_item(const LineGeom &g, int per, int b, int &ln, int &j) {
    if (g.line == 1) {
        j = b / g.nlines;
        ln = b - j * g.nlines;
    } else {
        ln = b / per;
        j = b - ln * per;
    }
}

// One Stockham stage of radix R over every line of `g`, in place through registers.  All NT threads must call it.
template <typename T, int R, int NT, int ITER>
__device__ __forceinline__ void stockham_stage(C2<T> *D, const LineGeom &g, int Ns, const C2<T> *tw, bool inv) {
    const int per = g.L / R;
    const int total = g.nlines * per;
    const int tstride = g.L / (Ns * R);
    C2<T> v[ITER][R];
#pragma unroll
    for (int i = 0; i < ITER; i++) {
        const int b = threadIdx.x + i * NT;
        if (b < total) {
            int ln, j;
            line_item(g, per, b, ln, j);
            const C2<T> *x = D + ln * g.line;
#pragma unroll
            for (int r = 0; r < R; r++) v[i][r] = x[(j + r * per) * g.elem];
            const int t = (j % Ns) * tstride;
            if (t != 0) {
#pragma unroll
                for (int r = 1; r < R; r++) {
                    C2<T> w = tw[(r * t) % g.L];
                    if (inv) w.y = -w.y;
                    v[i][r] = cmul(v[i][r], w);
                }
            }
            small_dft<T, R>(v[i], tw, g.L, inv);
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ITER; i++) {
        const int b = threadIdx.x + i * NT;
        if (b < total) {
            int ln, j;
            line_item(g, per, b, ln, j);
            C2<T> *y = D + ln * g.line;
            const int base = (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
            for (int r = 0; r < R; r++) y[(base + r * Ns) * g.elem] = v[i][r];
        }
    }
    __syncthreads();
}

// Direct DFT of every line (any length), in place through registers.
template <typename T, int NT, int ITER>
__device__ __forceinline__ void direct_lines(C2<T> *D, const LineGeom &g, const C2<T> *tw, bool inv) {
    const int total = g.nlines * g.L;
    C2<T> v[ITER];
#pragma unroll
    for (int i = 0; i < ITER; i++) {
        const int b = threadIdx.x + i * NT;
        if (b < total) {
            int ln, k;
            line_item(g, g.L, b, ln, k);
            const C2<T> *x = D + ln * g.line;
            C2<T> acc = mk<T>(0, 0);
            int idx = 0;  // (m k) mod L
            for (int m = 0; m < g.L; m++) {
                C2<T> w = tw[idx];
                if (inv) w.y = -w.y;
                acc = cadd(acc, cmul(x[m * g.elem], w));
                idx += k;
                if (idx >= g.L) idx -= g.L;
            }
            v[i] = acc;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < ITER; i++) {
        const int b = threadIdx.x + i * NT;
        if (b < total) {
            int ln, k;
            line_item(g, g.L, b, ln, k);
            D[ln * g.line + k * g.elem] = v[i];
        }
    }
    __syncthreads();
}

// Transforms every line of `g` (MAXN >= nlines * L).
template <typename T, int NT, int MAXN>
__device__ __noinline__ void line_fft(C2<T> *D, const LineGeom &g, const Radices &rad, const C2<T> *tw, bool inv) {
    if (rad.r[0] == 0) {
        direct_lines<T, NT, (MAXN + NT - 1) / NT>(D, g, tw, inv);
        return;
    }
    int Ns = 1;
    for (int s = 0; s < rad.count; s++) {
        const int R = rad.r[s];
        switch (R) {
            case 2: stockham_stage<T, 2, NT, (MAXN + 2 * NT - 1) / (2 * NT)>(D, g, Ns, tw, inv); break;
            case 3: stockham_stage<T, 3, NT, (MAXN + 3 * NT - 1) / (3 * NT)>(D, g, Ns, tw, inv); break;
            case 4: stockham_stage<T, 4, NT, (MAXN + 4 * NT - 1) / (4 * NT)>(D, g, Ns, tw, inv); break;
            case 5: stockham_stage<T, 5, NT, (MAXN + 5 * NT - 1) / (5 * NT)>(D, g, Ns, tw, inv); break;
            case 7: stockham_stage<T, 7, NT, (MAXN + 7 * NT - 1) / (7 * NT)>(D, g, Ns, tw, inv); break;
            default: stockham_stage<T, 8, NT, (MAXN + 8 * NT - 1) / (8 * NT)>(D, g, Ns, tw, inv); break;
        }
        Ns *= R;
    }
}

// The same transform with the radix plan fixed at compile time (R1, R2 = 0: no stage): no run-time dispatch, so the
// compiler keeps each stage's values in registers.  The stages and their arithmetic are line_fft's for that plan.
template <typename T, int NT, int MAXN, int R0, int R1, int R2>
__device__ __forceinline__ void line_fft_fixed(C2<T> *D, const LineGeom &g, const C2<T> *tw, bool inv) {
    int Ns = 1;
    stockham_stage<T, R0, NT, (MAXN + R0 * NT - 1) / (R0 * NT)>(D, g, Ns, tw, inv);
    Ns *= R0;
    if constexpr (R1 > 0) {
        stockham_stage<T, R1, NT, (MAXN + R1 * NT - 1) / (R1 * NT)>(D, g, Ns, tw, inv);
        Ns *= R1;
    }
    if constexpr (R2 > 0) stockham_stage<T, R2, NT, (MAXN + R2 * NT - 1) / (R2 * NT)>(D, g, Ns, tw, inv);
}

// 2-D transform of a rows x columns field held row-major in shared memory: rows, then columns.
template <typename T, int NT, int MAXN>
__device__ void fft2_smem(C2<T> *D, int rows, int columns, const Radices &rad_rows, const Radices &rad_columns,
                          const C2<T> *tw_rows, const C2<T> *tw_columns, bool inv) {
    line_fft<T, NT, MAXN>(D, LineGeom{columns, rows, 1, columns}, rad_columns, tw_columns, inv);
    line_fft<T, NT, MAXN>(D, LineGeom{rows, columns, columns, 1}, rad_rows, tw_rows, inv);
}

}  // namespace cubo
