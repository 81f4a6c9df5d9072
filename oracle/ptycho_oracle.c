/*
 * FP64 C restatement of CuboPtycho's single-slice gradient descent — TEST INFRASTRUCTURE ONLY (the oracle and the
 * timed CPU baseline).  See ptycho_oracle.h for what it restates and who may load it.
 */
#include "ptycho_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* fftfreq sample k of n (Ptychography.swift:474). */
static double frequency(int k, int n) { return (double)(k < (n + 1) / 2 ? k : k - n) / (double)n; }
static int wrapped(long v, long n) { long m = v % n; return (int)(m < 0 ? m + n : m); }

/* ------------------------------------------------------------------------------------------------------------------
 * One-dimensional transform of any length, in REAL = double and REAL = float instantiations.
 * Powers of two: iterative radix-2 Cooley-Tukey (bit reversal, then log2 n butterfly passes).  Other lengths: Bluestein's
 * chirp-z, x_k w_k convolved with conj(w) through a radix-2 transform of length m >= 2n - 1, w_k = e^{-i pi k^2 / n}.
 * Twiddles and chirps are evaluated in double from their definition and rounded once.
 * ------------------------------------------------------------------------------------------------------------------ */
#define DEFINE_FFT(REAL, SUF)                                                                                          \
    typedef struct {                                                                                                   \
        int n, m, pow2;                                                                                                \
        int *rev;                   /* bit reversal, length m */                                                       \
        REAL *twr, *twi;            /* e^{-2 pi i k / m}, k < m/2 */                                                   \
        REAL *chr, *chi;            /* Bluestein chirp, length n */                                                    \
        REAL *kr, *ki;              /* transform of the wrapped conjugate chirp, length m */                           \
    } fft1##SUF;                                                                                                       \
                                                                                                                       \
    static void radix2##SUF(const fft1##SUF *p, REAL *re, REAL *im, int inverse) {                                     \
        const int m = p->m;                                                                                            \
        for (int i = 0; i < m; i++) {                                                                                  \
            int j = p->rev[i];                                                                                         \
            if (j > i) { REAL t = re[i]; re[i] = re[j]; re[j] = t; t = im[i]; im[i] = im[j]; im[j] = t; }              \
        }                                                                                                              \
        const REAL sign = inverse ? (REAL)-1 : (REAL)1;                                                                \
        for (int len = 2; len <= m; len <<= 1) {                                                                       \
            const int half = len >> 1, step = m / len;                                                                 \
            for (int i = 0; i < m; i += len) {                                                                         \
                for (int j = 0; j < half; j++) {                                                                       \
                    const REAL wr = p->twr[j * step], wi = sign * p->twi[j * step];                                    \
                    const int a = i + j, b = a + half;                                                                 \
                    const REAL xr = re[b] * wr - im[b] * wi, xi = re[b] * wi + im[b] * wr;                             \
                    re[b] = re[a] - xr; im[b] = im[a] - xi;                                                            \
                    re[a] += xr; im[a] += xi;                                                                          \
                }                                                                                                      \
            }                                                                                                          \
        }                                                                                                              \
    }                                                                                                                  \
                                                                                                                       \
    static fft1##SUF *fft1_make##SUF(int n) {                                                                          \
        fft1##SUF *p = (fft1##SUF *)calloc(1, sizeof(fft1##SUF));                                                      \
        p->n = n;                                                                                                      \
        p->pow2 = (n & (n - 1)) == 0;                                                                                  \
        int m = 1;                                                                                                     \
        while (m < (p->pow2 ? n : 2 * n - 1)) m <<= 1;                                                                 \
        p->m = m;                                                                                                      \
        int bits = 0;                                                                                                  \
        while ((1 << bits) < m) bits++;                                                                                \
        p->rev = (int *)malloc(sizeof(int) * m);                                                                       \
        for (int i = 0; i < m; i++) {                                                                                  \
            int r = 0;                                                                                                 \
            for (int b = 0; b < bits; b++) r |= ((i >> b) & 1) << (bits - 1 - b);                                      \
            p->rev[i] = r;                                                                                             \
        }                                                                                                              \
        p->twr = (REAL *)malloc(sizeof(REAL) * (m / 2 + 1));                                                           \
        p->twi = (REAL *)malloc(sizeof(REAL) * (m / 2 + 1));                                                           \
        for (int k = 0; k <= m / 2; k++) {                                                                             \
            double a = -2.0 * M_PI * (double)k / (double)m;                                                            \
            p->twr[k] = (REAL)cos(a); p->twi[k] = (REAL)sin(a);                                                        \
        }                                                                                                              \
        if (!p->pow2) {                                                                                                \
            p->chr = (REAL *)malloc(sizeof(REAL) * n); p->chi = (REAL *)malloc(sizeof(REAL) * n);                      \
            p->kr = (REAL *)calloc(m, sizeof(REAL)); p->ki = (REAL *)calloc(m, sizeof(REAL));                          \
            for (int k = 0; k < n; k++) {                                                                              \
                long long q = ((long long)k * k) % (2LL * n);                                                          \
                double a = -M_PI * (double)q / (double)n;                                                              \
                p->chr[k] = (REAL)cos(a); p->chi[k] = (REAL)sin(a);                                                    \
            }                                                                                                          \
            for (int k = 0; k < n; k++) {                                                                              \
                p->kr[k] = p->chr[k]; p->ki[k] = -p->chi[k];                                                           \
                if (k) { p->kr[m - k] = p->chr[k]; p->ki[m - k] = -p->chi[k]; }                                        \
            }                                                                                                          \
            radix2##SUF(p, p->kr, p->ki, 0);                                                                           \
        }                                                                                                              \
        return p;                                                                                                      \
    }                                                                                                                  \
                                                                                                                       \
    static void fft1_free##SUF(fft1##SUF *p) {                                                                         \
        if (!p) return;                                                                                                \
        free(p->rev); free(p->twr); free(p->twi); free(p->chr); free(p->chi); free(p->kr); free(p->ki); free(p);       \
    }                                                                                                                  \
                                                                                                                       \
    /* Unnormalised transform of one line; work holds 2 m samples (Bluestein only). */                                \
    static void fft1_run##SUF(const fft1##SUF *p, REAL *re, REAL *im, int inverse, REAL *work) {                       \
        if (p->pow2) { radix2##SUF(p, re, im, inverse); return; }                                                      \
        const int n = p->n, m = p->m;                                                                                  \
        REAL *ar = work, *ai = work + m;                                                                               \
        const REAL s = inverse ? (REAL)-1 : (REAL)1; /* the inverse is conj(fft(conj(x))) */                          \
        for (int k = 0; k < n; k++) {                                                                                  \
            const REAL xr = re[k], xi = s * im[k];                                                                     \
            ar[k] = xr * p->chr[k] - xi * p->chi[k]; ai[k] = xr * p->chi[k] + xi * p->chr[k];                          \
        }                                                                                                              \
        for (int k = n; k < m; k++) { ar[k] = 0; ai[k] = 0; }                                                          \
        radix2##SUF(p, ar, ai, 0);                                                                                     \
        for (int k = 0; k < m; k++) {                                                                                  \
            const REAL xr = ar[k] * p->kr[k] - ai[k] * p->ki[k], xi = ar[k] * p->ki[k] + ai[k] * p->kr[k];             \
            ar[k] = xr; ai[k] = xi;                                                                                    \
        }                                                                                                              \
        radix2##SUF(p, ar, ai, 1);                                                                                     \
        const REAL inv = (REAL)1 / (REAL)m;                                                                            \
        for (int k = 0; k < n; k++) {                                                                                  \
            const REAL cr = ar[k] * inv, ci = ai[k] * inv;                                                             \
            re[k] = cr * p->chr[k] - ci * p->chi[k];                                                                   \
            im[k] = s * (cr * p->chi[k] + ci * p->chr[k]);                                                             \
        }                                                                                                              \
    }                                                                                                                  \
                                                                                                                       \
    typedef struct {                                                                                                   \
        int rows, columns;                                                                                             \
        fft1##SUF *r, *c;                                                                                              \
    } fft2##SUF;                                                                                                       \
                                                                                                                       \
    static fft2##SUF fft2_make##SUF(int rows, int columns) {                                                           \
        fft2##SUF f; f.rows = rows; f.columns = columns; f.c = fft1_make##SUF(columns);                                \
        f.r = rows == columns ? f.c : fft1_make##SUF(rows);                                                            \
        return f;                                                                                                      \
    }                                                                                                                  \
    static void fft2_free##SUF(fft2##SUF *f) { if (f->r != f->c) fft1_free##SUF(f->r); fft1_free##SUF(f->c); }         \
    static size_t fft2_work##SUF(const fft2##SUF *f) {                                                                 \
        int m = f->r->m > f->c->m ? f->r->m : f->c->m;                                                                 \
        return (size_t)2 * f->rows * f->columns + 2 * (size_t)m;                                                       \
    }                                                                                                                  \
    /* NumPy fft2 / ifft2 (the inverse divides by rows*columns): rows, transpose, rows, transpose. */                 \
    static void fft2_run##SUF(const fft2##SUF *f, REAL *re, REAL *im, int inverse, REAL *work) {                       \
        const int R = f->rows, C = f->columns;                                                                         \
        REAL *tr = work, *ti = work + (size_t)R * C, *line = work + (size_t)2 * R * C;                                 \
        for (int r = 0; r < R; r++) fft1_run##SUF(f->c, re + (size_t)r * C, im + (size_t)r * C, inverse, line);       \
        for (int r = 0; r < R; r++)                                                                                    \
            for (int c = 0; c < C; c++) { tr[(size_t)c * R + r] = re[(size_t)r * C + c]; ti[(size_t)c * R + r] = im[(size_t)r * C + c]; } \
        for (int c = 0; c < C; c++) fft1_run##SUF(f->r, tr + (size_t)c * R, ti + (size_t)c * R, inverse, line);       \
        const REAL scale = inverse ? (REAL)1 / (REAL)(R * C) : (REAL)1;                                                \
        for (int r = 0; r < R; r++)                                                                                    \
            for (int c = 0; c < C; c++) {                                                                              \
                re[(size_t)r * C + c] = tr[(size_t)c * R + r] * scale; im[(size_t)r * C + c] = ti[(size_t)c * R + r] * scale; \
            }                                                                                                          \
    }

DEFINE_FFT(double, _d)
DEFINE_FFT(float, _f)

void oracle_fft2(int rows, int columns, double *re, double *im, int inverse) {
    fft2_d f = fft2_make_d(rows, columns);
    double *work = (double *)malloc(sizeof(double) * fft2_work_d(&f));
    fft2_run_d(&f, re, im, inverse, work);
    free(work);
    fft2_free_d(&f);
}

/* ------------------------------------------------------------------------------------------------ probe build */

int oracle_probe_build(int rows, int columns, double row_sampling, double column_sampling, double wavelength,
                       double cutoff, double rolloff, double defocus, double astigmatism, double astigmatism_angle,
                       double spherical_aberration, int term_count, const double *terms, double *re, double *im) {
    /* Ptychography.swift:147-153 */
    if (!(rows > 1 && columns > 1)) return 1;
    const double pos[4] = {row_sampling, column_sampling, wavelength, cutoff};
    for (int i = 0; i < 4; i++) if (!(isfinite(pos[i]) && pos[i] > 0)) return 1;
    if (!(isfinite(rolloff) && rolloff >= 0)) return 1;
    if (!(isfinite(defocus) && isfinite(astigmatism) && isfinite(astigmatism_angle) && isfinite(spherical_aberration))) return 1;
    for (int t = 0; t < term_count; t++) {
        const double nr = terms[4 * t], mr = terms[4 * t + 1], sine = terms[4 * t + 2], c = terms[4 * t + 3];
        if (!(isfinite(c) && nr >= 1 && nr <= 64 && mr >= 0 && (sine == 0 || mr > 0))) return 1;
    }
    /* Ptychography.swift:155-167 */
    for (int r = 0; r < rows; r++)
        for (int c = 0; c < columns; c++) {
            const double qr = frequency(r, rows) / row_sampling, qc = frequency(c, columns) / column_sampling;
            const double alpha = hypot(qr, qc) * wavelength, angle = atan2(qc, qr);
            double aperture;
            if (rolloff > 0 && alpha > cutoff - rolloff)
                aperture = alpha > cutoff ? 0 : 0.5 * (1 + cos(M_PI * (alpha - cutoff + rolloff) / rolloff));
            else
                aperture = alpha < cutoff ? 1 : 0;
            const double a2 = alpha * alpha;
            double phase = a2 / 2 * (-defocus + astigmatism * cos(2 * (angle - astigmatism_angle))) +
                           a2 * a2 / 4 * spherical_aberration;
            for (int t = 0; t < term_count; t++) { /* Ptychography.swift:127-132 */
                const int nr = (int)terms[4 * t], mr = (int)terms[4 * t + 1];
                const double radial = pow(alpha, (double)(nr + 1)) / (double)(nr + 1);
                if (mr == 0) phase += terms[4 * t + 3] * radial;
                else {
                    const double a = (double)mr * angle;
                    phase += terms[4 * t + 3] * radial * (terms[4 * t + 2] != 0 ? sin(a) : cos(a));
                }
            }
            const double chi = 2 * M_PI / wavelength * phase;
            re[r * columns + c] = aperture * cos(chi);
            im[r * columns + c] = -aperture * sin(chi);
        }
    oracle_fft2(rows, columns, re, im, 1);
    double norm = 0;
    for (int k = 0; k < rows * columns; k++) norm += re[k] * re[k] + im[k] * im[k];
    norm = sqrt(norm);
    if (!(norm > 0 && isfinite(norm))) return 1;
    for (int k = 0; k < rows * columns; k++) { re[k] /= norm; im[k] /= norm; }
    return 0;
}

/* ----------------------------------------------------------------------------------- probe constraints, Double */

/* PtychographyConstraints.swift:21-31: out[x] = in[x - shift]. */
static void fourier_shift(const fft2_d *f, double *re, double *im, double row, double column, double *work) {
    const int R = f->rows, C = f->columns;
    fft2_run_d(f, re, im, 0, work);
    for (int r = 0; r < R; r++)
        for (int c = 0; c < C; c++) {
            const int k = r * C + c;
            const double phase = -2 * M_PI * (frequency(r, R) * row + frequency(c, C) * column);
            const double cs = cos(phase), sn = sin(phase), a = re[k], b = im[k];
            re[k] = a * cs - b * sn; im[k] = a * sn + b * cs;
        }
    fft2_run_d(f, re, im, 1, work);
}

/* PtychographyConstraints.swift:9-18, 34-37. */
static void center_of_mass_constraint(const fft2_d *f, double *re, double *im, double *work) {
    const int R = f->rows, C = f->columns;
    double total = 0, cr = 0, cc = 0;
    for (int r = 0; r < R; r++)
        for (int c = 0; c < C; c++) {
            const int k = r * C + c;
            const double w = re[k] * re[k] + im[k] * im[k];
            total += w;
            cr += frequency(r, R) * (double)R * w;
            cc += frequency(c, C) * (double)C * w;
        }
    if (!(total > 0 && isfinite(total))) return;
    fourier_shift(f, re, im, -cr / total, -cc / total, work);
}

/* PtychographyConstraints.swift:40-55. */
static void amplitude_constraint(int R, int C, double *re, double *im, double radius, double width) {
    double before = 0, after = 0;
    for (int k = 0; k < R * C; k++) before += re[k] * re[k] + im[k] * im[k];
    const double sigma = sqrt(M_PI) / width;
    for (int r = 0; r < R; r++)
        for (int c = 0; c < C; c++) {
            const int k = r * C + c;
            const double d = hypot(frequency(r, R), frequency(c, C)) - radius;
            const double mask = 0.5 * (1 - erf(sigma * d / (1 - d * d)));
            re[k] *= mask; im[k] *= mask;
            after += re[k] * re[k] + im[k] * im[k];
        }
    if (!(before > 0 && after > 0)) return;
    const double s = sqrt(before / after);
    for (int k = 0; k < R * C; k++) { re[k] *= s; im[k] *= s; }
}

/* PtychographyConstraints.swift:59-71. */
static void aperture_constraint(const fft2_d *f, double *re, double *im, const double *aperture, double *work) {
    const int n = f->rows * f->columns;
    double before = 0, after = 0;
    for (int k = 0; k < n; k++) before += re[k] * re[k] + im[k] * im[k];
    fft2_run_d(f, re, im, 0, work);
    for (int k = 0; k < n; k++) {
        const double ph = atan2(im[k], re[k]);
        re[k] = aperture[k] * cos(ph); im[k] = aperture[k] * sin(ph);
    }
    fft2_run_d(f, re, im, 1, work);
    for (int k = 0; k < n; k++) after += re[k] * re[k] + im[k] * im[k];
    if (!(before > 0 && after > 0)) return;
    const double s = sqrt(before / after);
    for (int k = 0; k < n; k++) { re[k] *= s; im[k] *= s; }
}

static void probe_constraints(const oracle_params *pp, const fft2_d *f, double *re, double *im,
                              const double *aperture, double *work) {
    /* Ptychography.swift:387-392, py4DSTEM's order: centre of mass, aperture, amplitude. */
    if (pp->fix_probe_center_of_mass) center_of_mass_constraint(f, re, im, work);
    if (pp->fix_probe_aperture) aperture_constraint(f, re, im, aperture, work);
    if (pp->constrain_probe_amplitude)
        amplitude_constraint(f->rows, f->columns, re, im, pp->probe_amplitude_relative_radius,
                             pp->probe_amplitude_relative_width);
}

/* ------------------------------------------------------------------------------------------------- validation */

/* Ptychography.swift:247-259 (and PtychographySingle.swift:53-67).  Returns the error divisor, or -1 when invalid. */
static double validate(const oracle_params *p, int rows, int columns, int object_rows, int object_columns, int count,
                       const double *amplitudes, const float *amplitudes_f, const double *pr, const double *pc) {
    if (!(rows > 1 && columns > 1 && object_rows > 1 && object_columns > 1)) return -1;
    const long n = (long)rows * columns;
    if (!(count > 0 && p->iterations >= 0 && isfinite(p->step_size) && p->step_size > 0)) return -1;
    if (!(isfinite(p->normalization_minimum) && p->normalization_minimum >= 0 && p->normalization_minimum <= 1)) return -1;
    const double limit = (double)(INT64_MAX / 4);
    for (int i = 0; i < count; i++)
        if (!(isfinite(pr[i]) && isfinite(pc[i]) && fabs(pr[i]) < limit && fabs(pc[i]) < limit)) return -1;
    const double rad = p->probe_amplitude_relative_radius, wid = p->probe_amplitude_relative_width;
    if (!(isfinite(rad) && rad >= 0 && rad <= 0.5 && isfinite(wid) && wid > 0 && wid <= 0.5)) return -1;
    if (!(object_rows >= rows && object_columns >= columns)) return -1;
    double energy = 0;
    for (long i = 0; i < (long)count * n; i++) {
        const double a = amplitudes ? amplitudes[i] : (double)amplitudes_f[i];
        if (!(isfinite(a) && a >= 0)) return -1;
        energy += a * a;
    }
    const double d = p->error_normalization == 1 ? p->mean_intensity * (double)count : energy;
    if (!(isfinite(d) && d > 0)) return -1;
    return d;
}

/* ------------------------------------------------------------------------------------- the Double engine */

typedef struct {
    double *onr, *oni, *pn;   /* object-sized accumulators */
    double *pnr, *pni, *on;   /* probe-sized accumulators */
    double *sr, *si, *fr, *fi, *work;
    int *indices;
    unsigned char *rows_touched; /* object rows any window of this thread's positions covers */
    double error;
} thread_state;

static void thread_state_init(thread_state *t, size_t objects, size_t n, size_t work, int object_rows) {
    t->onr = (double *)calloc(objects, sizeof(double)); t->oni = (double *)calloc(objects, sizeof(double));
    t->pn = (double *)calloc(objects, sizeof(double));
    t->pnr = (double *)calloc(n, sizeof(double)); t->pni = (double *)calloc(n, sizeof(double));
    t->on = (double *)calloc(n, sizeof(double));
    t->sr = (double *)malloc(n * sizeof(double)); t->si = (double *)malloc(n * sizeof(double));
    t->fr = (double *)malloc(n * sizeof(double)); t->fi = (double *)malloc(n * sizeof(double));
    t->work = (double *)malloc(work * sizeof(double));
    t->indices = (int *)malloc(n * sizeof(int));
    t->rows_touched = (unsigned char *)calloc((size_t)object_rows, 1);
}

static void thread_state_free(thread_state *t) {
    free(t->onr); free(t->oni); free(t->pn); free(t->pnr); free(t->pni); free(t->on);
    free(t->sr); free(t->si); free(t->fr); free(t->fi); free(t->work); free(t->indices); free(t->rows_touched);
}

/* The object rows the windows of positions [begin, end) cover (the row indices of Ptychography.swift:321-336).  A thread
 * of the multi-threaded pass zeroes and hands over only these rows of its object-sized accumulators: every other row
 * holds no contribution, so the fixed-order sum over threads is unchanged while its cost no longer grows with the whole
 * object per thread. */
static void mark_rows(unsigned char *touched, int rows, int object_rows, const double *prow, int begin, int end) {
    memset(touched, 0, (size_t)object_rows);
    for (int pattern = begin; pattern < end; pattern++) {
        const long rr = (long)nearbyint(prow[pattern]);
        for (int r = 0; r < rows; r++) touched[wrapped(rr + (r < (rows + 1) / 2 ? r : r - rows), object_rows)] = 1;
    }
}

/* The per-position body of Ptychography.swift:300-358 for positions [begin, end). */
static void positions_pass(const fft2_d *f, int object_rows, int object_columns, const double *amplitudes,
                           const double *prow, const double *pcol, int begin, int end, const double *psr,
                           const double *psi, const double *prr, const double *pii, const double *orr, const double *oii,
                           int always_shift, thread_state *t) {
    const int R = f->rows, C = f->columns, n = R * C;
    double *rowCos = (double *)malloc(sizeof(double) * (R + C) * 2);
    double *rowSin = rowCos + R, *colCos = rowSin + R, *colSin = colCos + C;
    int *rowBase = (int *)malloc(sizeof(int) * (R + C)), *colIndex = rowBase + R;
    for (int pattern = begin; pattern < end; pattern++) {
        const double rr = nearbyint(prow[pattern]), cc = nearbyint(pcol[pattern]);
        const double dr = prow[pattern] - rr, dc = pcol[pattern] - cc;
        if (always_shift || dr != 0 || dc != 0) {
            for (int r = 0; r < R; r++) { const double a = -2 * M_PI * frequency(r, R) * dr; rowCos[r] = cos(a); rowSin[r] = sin(a); }
            for (int c = 0; c < C; c++) { const double a = -2 * M_PI * frequency(c, C) * dc; colCos[c] = cos(a); colSin[c] = sin(a); }
            for (int r = 0; r < R; r++) {
                const double rc = rowCos[r], rs = rowSin[r];
                for (int c = 0; c < C; c++) {
                    const int k = r * C + c;
                    const double cs = rc * colCos[c] - rs * colSin[c], sn = rs * colCos[c] + rc * colSin[c];
                    t->sr[k] = psr[k] * cs - psi[k] * sn; t->si[k] = psr[k] * sn + psi[k] * cs;
                }
            }
            fft2_run_d(f, t->sr, t->si, 1, t->work);
        } else {
            /* a shift by zero: the probe itself, without the transform pair's roundoff */
            memcpy(t->sr, prr, sizeof(double) * n); memcpy(t->si, pii, sizeof(double) * n);
        }
        for (int r = 0; r < R; r++) rowBase[r] = wrapped((long)rr + (r < (R + 1) / 2 ? r : r - R), object_rows) * object_columns;
        for (int c = 0; c < C; c++) colIndex[c] = wrapped((long)cc + (c < (C + 1) / 2 ? c : c - C), object_columns);
        for (int r = 0; r < R; r++)
            for (int c = 0; c < C; c++) {
                const int k = r * C + c, j = rowBase[r] + colIndex[c];
                t->indices[k] = j;
                t->fr[k] = t->sr[k] * orr[j] - t->si[k] * oii[j];
                t->fi[k] = t->sr[k] * oii[j] + t->si[k] * orr[j];
            }
        fft2_run_d(f, t->fr, t->fi, 0, t->work);
        const double *amp = amplitudes + (size_t)pattern * n;
        for (int k = 0; k < n; k++) {
            const double a = t->fr[k], b = t->fi[k];
            const double mag = sqrt(a * a + b * b), measured = amp[k];
            t->error += (measured - mag) * (measured - mag);
            if (mag > 0) {
                const double s = measured / mag;
                t->fr[k] = s * a - a; t->fi[k] = s * b - b;
            } else {
                t->fr[k] = measured; t->fi[k] = 0;
            }
        }
        fft2_run_d(f, t->fr, t->fi, 1, t->work);
        for (int k = 0; k < n; k++) {
            const int j = t->indices[k];
            const double sk = t->sr[k], ik = t->si[k], fk = t->fr[k], gk = t->fi[k];
            t->onr[j] += sk * fk + ik * gk; t->oni[j] += sk * gk - ik * fk;
            t->pn[j] += sk * sk + ik * ik;
            t->pnr[k] += orr[j] * fk + oii[j] * gk; t->pni[k] += orr[j] * gk - oii[j] * fk;
            t->on[k] += orr[j] * orr[j] + oii[j] * oii[j];
        }
    }
    free(rowCos); free(rowBase);
}

int oracle_reconstruct(const oracle_params *pp, int rows, int columns, int object_rows, int object_columns, int count,
                       const double *amplitudes, const double *position_rows, const double *position_columns,
                       double *object_re, double *object_im, double *probe_re, double *probe_im, double *errors) {
    const double divisor = validate(pp, rows, columns, object_rows, object_columns, count, amplitudes, NULL,
                                    position_rows, position_columns);
    if (divisor < 0) return 1;
    const int n = rows * columns;
    const size_t objects = (size_t)object_rows * object_columns;
    fft2_d f = fft2_make_d(rows, columns);
    const size_t work = fft2_work_d(&f);
    double *w = (double *)malloc(sizeof(double) * (work + 6 * (size_t)n));
    double *psr = w + work, *psi = psr + n, *aperture = psi + n, *tr = aperture + n, *ti = tr + n;
    if (pp->fix_probe_aperture) { /* PtychographyConstraints.swift:79-83 */
        memcpy(tr, probe_re, sizeof(double) * n); memcpy(ti, probe_im, sizeof(double) * n);
        fft2_run_d(&f, tr, ti, 0, w);
        for (int k = 0; k < n; k++) aperture[k] = hypot(tr[k], ti[k]);
    }
    int threads = pp->threads > 1 ? pp->threads : 1;
    if (threads > count) threads = count;
    thread_state *ts = (thread_state *)calloc(threads, sizeof(thread_state));
    for (int t = 0; t < threads; t++) {
        thread_state_init(&ts[t], objects, n, work, object_rows);
        mark_rows(ts[t].rows_touched, rows, object_rows, position_rows, (int)((long)count * t / threads),
                  (int)((long)count * (t + 1) / threads));
    }
    const double m = pp->normalization_minimum;
    const size_t row_bytes = sizeof(double) * (size_t)object_columns;
    for (int it = 0; it < pp->iterations; it++) {
        memcpy(psr, probe_re, sizeof(double) * n); memcpy(psi, probe_im, sizeof(double) * n);
        fft2_run_d(&f, psr, psi, 0, w);
        for (int t = 0; t < threads; t++) {
            thread_state *s = &ts[t];
            if (t == 0) {  /* thread 0's accumulators end up holding the sum: all of them start at zero */
                memset(s->onr, 0, sizeof(double) * objects); memset(s->oni, 0, sizeof(double) * objects);
                memset(s->pn, 0, sizeof(double) * objects);
            } else {
                for (int y = 0; y < object_rows; y++)
                    if (s->rows_touched[y]) {
                        const size_t o = (size_t)y * object_columns;
                        memset(s->onr + o, 0, row_bytes); memset(s->oni + o, 0, row_bytes); memset(s->pn + o, 0, row_bytes);
                    }
            }
            memset(s->pnr, 0, sizeof(double) * n); memset(s->pni, 0, sizeof(double) * n); memset(s->on, 0, sizeof(double) * n);
            s->error = 0;
        }
        if (threads == 1) {
            positions_pass(&f, object_rows, object_columns, amplitudes, position_rows, position_columns, 0, count, psr,
                           psi, probe_re, probe_im, object_re, object_im, pp->single_shift_fft, &ts[0]);
        } else {
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(static, 1)
#endif
            for (int t = 0; t < threads; t++) {
                const int begin = (int)((long)count * t / threads), end = (int)((long)count * (t + 1) / threads);
                positions_pass(&f, object_rows, object_columns, amplitudes, position_rows, position_columns, begin, end,
                               psr, psi, probe_re, probe_im, object_re, object_im, pp->single_shift_fft, &ts[t]);
            }
            /* fixed-order sum of the per-thread accumulators (thread 0 first) */
            for (int t = 1; t < threads; t++) {
                thread_state *a = &ts[0], *b = &ts[t];
                for (int y = 0; y < object_rows; y++) {
                    if (!b->rows_touched[y]) continue;  /* an untouched row of thread t adds nothing */
                    for (size_t j = (size_t)y * object_columns, e = j + object_columns; j < e; j++) {
                        a->onr[j] += b->onr[j]; a->oni[j] += b->oni[j]; a->pn[j] += b->pn[j];
                    }
                }
                for (int k = 0; k < n; k++) { a->pnr[k] += b->pnr[k]; a->pni[k] += b->pni[k]; a->on[k] += b->on[k]; }
                a->error += b->error;
            }
        }
        const thread_state *acc = &ts[0];
        /* Ptychography.swift:362-370 */
        double maxPN = acc->pn[0], maxON = acc->on[0];
        for (size_t j = 1; j < objects; j++) if (acc->pn[j] > maxPN) maxPN = acc->pn[j];
        for (int k = 1; k < n; k++) if (acc->on[k] > maxON) maxON = acc->on[k];
        for (size_t j = 0; j < objects; j++) {
            const double l = (1 - m) * acc->pn[j], x = m * maxPN;
            const double s = pp->step_size * (1 / sqrt(1e-16 + l * l + x * x));
            object_re[j] += s * acc->onr[j]; object_im[j] += s * acc->oni[j];
        }
        /* Ptychography.swift:378-382 */
        if (pp->constrain_object_amplitude || pp->pure_phase_object)
            for (size_t j = 0; j < objects; j++) {
                const double amp = sqrt(object_re[j] * object_re[j] + object_im[j] * object_im[j]);
                const double a = pp->pure_phase_object ? 1 : (amp < 1 ? amp : 1);
                if (amp > 0) { const double s = a / amp; object_re[j] *= s; object_im[j] *= s; }
                else { object_re[j] = a; object_im[j] = 0; }
            }
        /* Ptychography.swift:383-395 */
        if (!pp->fix_probe) {
            for (int k = 0; k < n; k++) {
                const double l = (1 - m) * acc->on[k], x = m * maxON;
                const double s = pp->step_size * (1 / sqrt(1e-16 + l * l + x * x));
                probe_re[k] += s * acc->pnr[k]; probe_im[k] += s * acc->pni[k];
            }
            probe_constraints(pp, &f, probe_re, probe_im, aperture, w);
        }
        if (pp->probe_support_mask)
            for (int k = 0; k < n; k++) if (!pp->probe_support_mask[k]) { probe_re[k] = 0; probe_im[k] = 0; }
        errors[it] = acc->error / divisor;
    }
    for (int t = 0; t < threads; t++) thread_state_free(&ts[t]);
    free(ts);
    free(w);
    fft2_free_d(&f);
    return 0;
}

/* ------------------------------------------------------------------------------------- the Float32 engine */

/* PtychographySingle.swift:40-220, in natural (untransposed) layout: the transforms, shifted probe, projection and
 * accumulations in Float32 with the inverse's 1/n folded into the column ramp and the projection; the probe spectrum and
 * the probe constraints in Double once per iteration.  Single-threaded. */
int oracle_reconstruct_single(const oracle_params *pp, int rows, int columns, int object_rows, int object_columns,
                              int count, const float *amplitudes, const double *position_rows,
                              const double *position_columns, double *object_re, double *object_im, double *probe_re,
                              double *probe_im, double *errors) {
    const double divisor = validate(pp, rows, columns, object_rows, object_columns, count, NULL, amplitudes,
                                    position_rows, position_columns);
    if (divisor < 0) return 1;
    const int R = rows, C = columns, n = R * C;
    const size_t objects = (size_t)object_rows * object_columns;
    fft2_d fd = fft2_make_d(R, C);
    fft2_f ff = fft2_make_f(R, C);
    const size_t workd = fft2_work_d(&fd), workf = fft2_work_f(&ff);
    double *wd = (double *)malloc(sizeof(double) * workd);
    double *dbl = (double *)malloc(sizeof(double) * 5 * (size_t)n);
    double *sre = dbl, *sim = sre + n, *aperture = sim + n, *dre = aperture + n, *dim = dre + n;
    float *wf = (float *)malloc(sizeof(float) * workf);
    float *nbuf = (float *)malloc(sizeof(float) * 11 * (size_t)n);
    float *psr = nbuf, *psi = psr + n, *sr = psi + n, *si = sr + n, *fr = si + n, *fi = fr + n;
    float *pnr = fi + n, *pni = pnr + n, *on = pni + n, *prb = on + n, *pib = prb + n;
    float *obuf = (float *)malloc(sizeof(float) * 5 * objects);
    float *obr = obuf, *obi = obr + objects, *onr = obi + objects, *oni = onr + objects, *pn = oni + objects;
    float *lines = (float *)malloc(sizeof(float) * 2 * (size_t)(R + C));
    float *rowCos = lines, *rowSin = rowCos + R, *colCos = rowSin + R, *colSin = colCos + C;
    int *indices = (int *)malloc(sizeof(int) * (n + R + C)), *rowBase = indices + n, *colIndex = rowBase + R;
    if (pp->fix_probe_aperture) {
        memcpy(dre, probe_re, sizeof(double) * n); memcpy(dim, probe_im, sizeof(double) * n);
        fft2_run_d(&fd, dre, dim, 0, wd);
        for (int k = 0; k < n; k++) aperture[k] = hypot(dre[k], dim[k]);
    }
    for (size_t j = 0; j < objects; j++) { obr[j] = (float)object_re[j]; obi[j] = (float)object_im[j]; }
    for (int k = 0; k < n; k++) { prb[k] = (float)probe_re[k]; pib[k] = (float)probe_im[k]; }
    const float inverseCount = 1.0f / (float)n;
    const double m = pp->normalization_minimum;
    for (int it = 0; it < pp->iterations; it++) {
        memset(onr, 0, sizeof(float) * objects); memset(oni, 0, sizeof(float) * objects); memset(pn, 0, sizeof(float) * objects);
        memset(pnr, 0, sizeof(float) * n); memset(pni, 0, sizeof(float) * n); memset(on, 0, sizeof(float) * n);
        for (int k = 0; k < n; k++) { sre[k] = prb[k]; sim[k] = pib[k]; }
        fft2_run_d(&fd, sre, sim, 0, wd);
        for (int k = 0; k < n; k++) { psr[k] = (float)sre[k]; psi[k] = (float)sim[k]; }
        double error = 0;
        for (int pattern = 0; pattern < count; pattern++) {
            const double rr = nearbyint(position_rows[pattern]), cc = nearbyint(position_columns[pattern]);
            const double dr = position_rows[pattern] - rr, dc = position_columns[pattern] - cc;
            for (int r = 0; r < R; r++) { const double a = -2 * M_PI * frequency(r, R) * dr; rowCos[r] = (float)cos(a); rowSin[r] = (float)sin(a); }
            for (int c = 0; c < C; c++) {
                const double a = -2 * M_PI * frequency(c, C) * dc;
                colCos[c] = (float)cos(a) * inverseCount; colSin[c] = (float)sin(a) * inverseCount;
            }
            for (int r = 0; r < R; r++)
                for (int c = 0; c < C; c++) {
                    const int k = r * C + c;
                    const float cs = rowCos[r] * colCos[c] - rowSin[r] * colSin[c];
                    const float sn = rowSin[r] * colCos[c] + rowCos[r] * colSin[c];
                    sr[k] = psr[k] * cs - psi[k] * sn; si[k] = psr[k] * sn + psi[k] * cs;
                }
            /* unnormalised inverse: the 1/n rides on the ramp */
            {
                float *tr = wf, *ti = wf + (size_t)n, *line = wf + 2 * (size_t)n;
                for (int r = 0; r < R; r++) fft1_run_f(ff.c, sr + (size_t)r * C, si + (size_t)r * C, 1, line);
                for (int r = 0; r < R; r++) for (int c = 0; c < C; c++) { tr[c * R + r] = sr[r * C + c]; ti[c * R + r] = si[r * C + c]; }
                for (int c = 0; c < C; c++) fft1_run_f(ff.r, tr + (size_t)c * R, ti + (size_t)c * R, 1, line);
                for (int r = 0; r < R; r++) for (int c = 0; c < C; c++) { sr[r * C + c] = tr[c * R + r]; si[r * C + c] = ti[c * R + r]; }
            }
            for (int r = 0; r < R; r++) rowBase[r] = wrapped((long)rr + (r < (R + 1) / 2 ? r : r - R), object_rows) * object_columns;
            for (int c = 0; c < C; c++) colIndex[c] = wrapped((long)cc + (c < (C + 1) / 2 ? c : c - C), object_columns);
            for (int r = 0; r < R; r++)
                for (int c = 0; c < C; c++) {
                    const int k = r * C + c, j = rowBase[r] + colIndex[c];
                    indices[k] = j;
                    fr[k] = sr[k] * obr[j] - si[k] * obi[j];
                    fi[k] = sr[k] * obi[j] + si[k] * obr[j];
                }
            fft2_run_f(&ff, fr, fi, 0, wf);
            const float *target = amplitudes + (size_t)pattern * n;
            float patternError = 0;
            for (int k = 0; k < n; k++) {
                const float a = fr[k], b = fi[k], wanted = target[k];
                const float mag = sqrtf(a * a + b * b), miss = wanted - mag;
                patternError += miss * miss;
                if (mag > 0) { const float s = wanted / mag; fr[k] = (s * a - a) * inverseCount; fi[k] = (s * b - b) * inverseCount; }
                else { fr[k] = wanted * inverseCount; fi[k] = 0; }
            }
            error += (double)patternError;
            {
                float *tr = wf, *ti = wf + (size_t)n, *line = wf + 2 * (size_t)n;
                for (int r = 0; r < R; r++) fft1_run_f(ff.c, fr + (size_t)r * C, fi + (size_t)r * C, 1, line);
                for (int r = 0; r < R; r++) for (int c = 0; c < C; c++) { tr[c * R + r] = fr[r * C + c]; ti[c * R + r] = fi[r * C + c]; }
                for (int c = 0; c < C; c++) fft1_run_f(ff.r, tr + (size_t)c * R, ti + (size_t)c * R, 1, line);
                for (int r = 0; r < R; r++) for (int c = 0; c < C; c++) { fr[r * C + c] = tr[c * R + r]; fi[r * C + c] = ti[c * R + r]; }
            }
            for (int k = 0; k < n; k++) {
                const int j = indices[k];
                const float s0 = sr[k], s1 = si[k], f0 = fr[k], f1 = fi[k], o0 = obr[j], o1 = obi[j];
                onr[j] += s0 * f0 + s1 * f1; oni[j] += s0 * f1 - s1 * f0;
                pn[j] += s0 * s0 + s1 * s1;
                pnr[k] += o0 * f0 + o1 * f1; pni[k] += o0 * f1 - o1 * f0;
                on[k] += o0 * o0 + o1 * o1;
            }
        }
        float maxPN = pn[0], maxON = on[0];
        for (size_t j = 1; j < objects; j++) if (pn[j] > maxPN) maxPN = pn[j];
        for (int k = 1; k < n; k++) if (on[k] > maxON) maxON = on[k];
        for (size_t j = 0; j < objects; j++) {
            const double l = (1 - m) * (double)pn[j], x = m * (double)maxPN;
            const float s = (float)pp->step_size * (float)(1 / sqrt(1e-16 + l * l + x * x));
            obr[j] += s * onr[j]; obi[j] += s * oni[j];
        }
        if (pp->constrain_object_amplitude || pp->pure_phase_object)
            for (size_t j = 0; j < objects; j++) {
                const float a0 = obr[j], a1 = obi[j], amp = sqrtf(a0 * a0 + a1 * a1);
                const float want = pp->pure_phase_object ? 1.0f : (amp < 1.0f ? amp : 1.0f);
                if (amp > 0) { const float s = want / amp; obr[j] = a0 * s; obi[j] = a1 * s; }
                else { obr[j] = want; obi[j] = 0; }
            }
        if (!pp->fix_probe) {
            for (int k = 0; k < n; k++) {
                const double l = (1 - m) * (double)on[k], x = m * (double)maxON;
                const float s = (float)pp->step_size * (float)(1 / sqrt(1e-16 + l * l + x * x));
                prb[k] += s * pnr[k]; pib[k] += s * pni[k];
            }
            if (pp->fix_probe_center_of_mass || pp->fix_probe_aperture || pp->constrain_probe_amplitude) {
                for (int k = 0; k < n; k++) { dre[k] = prb[k]; dim[k] = pib[k]; }
                probe_constraints(pp, &fd, dre, dim, aperture, wd);
                for (int k = 0; k < n; k++) { prb[k] = (float)dre[k]; pib[k] = (float)dim[k]; }
            }
        }
        if (pp->probe_support_mask)
            for (int k = 0; k < n; k++) if (!pp->probe_support_mask[k]) { prb[k] = 0; pib[k] = 0; }
        errors[it] = error / divisor;
    }
    for (size_t j = 0; j < objects; j++) { object_re[j] = obr[j]; object_im[j] = obi[j]; }
    for (int k = 0; k < n; k++) { probe_re[k] = prb[k]; probe_im[k] = pib[k]; }
    free(indices); free(lines); free(obuf); free(nbuf); free(wf); free(dbl); free(wd);
    fft2_free_d(&fd); fft2_free_f(&ff);
    return 0;
}
