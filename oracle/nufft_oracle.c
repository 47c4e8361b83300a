/*
 * CPU oracle for the laminography NUFFT path.  TEST INFRASTRUCTURE ONLY:
 * nothing in the product links this file; tests, smoke() and the bench's
 * CPU-baseline leg call it as the checker.
 *
 * The reference delegates every non-uniform transform to FINUFFT (third-party,
 * version unpinned; call sites include/nufft.h:37-64, include/finufft_plan.h:93-129).
 * FINUFFT is absent from the reference tree, so this file restates the
 * published transform definitions and the published exponential-of-semicircle
 * (ES) spreading method of Barnett, Magland and af Klinteberg, "A parallel
 * non-uniform fast Fourier transform library based on an exponential of
 * semicircle kernel", SIAM J. Sci. Comput. 41(5), 2019.
 *
 * Conventions (as the reference calls FINUFFT, nufft.h:37-64):
 *   3-D type 1 (points -> modes):  f[k] = sum_j c_j exp(+i k.x_j)   (iflag +1)
 *   3-D type 2 (modes -> points):  c_j  = sum_k f[k] exp(-i k.x_j)  (iflag -1)
 *   n_modes = {N1, N2, N3} = {ncols, nrows, nslices} of the volume; x pairs with
 *   N1 (fastest), y with N2, z with N3 (slowest).  Modes are centred
 *   (FINUFFT modeord 0): k = idx - floor(N/2).
 *   Complex arrays are interleaved (re, im) doubles / floats.
 *
 * Two families:
 *   oracle_nudft3d{1,2}   exact O(M N) sums in FP64 (the definitional oracle);
 *   oracle_es_{spread,interp}[_f]  ES-kernel gridding on an oversampled
 *       periodic fine grid (FP64, and FP32 for the CPU baseline timing); the
 *       FFT and deconvolution steps live in oracle.py (numpy / scipy.fft).
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* exact NUDFT                                                          */
/* ------------------------------------------------------------------ */

static void phase_row(double xj, int64_t N, int iflag, double *er, double *ei) {
    int64_t k0 = -(N / 2);
    for (int64_t i = 0; i < N; ++i) {
        double ph = (double)iflag * (double)(k0 + i) * xj;
        er[i] = cos(ph);
        ei[i] = sin(ph);
    }
}

/* type 2: c[j] = sum_k f[k] e^{iflag i k.x_j} */
void oracle_nudft3d2(int64_t M, const double *x, const double *y, const double *z,
                     int iflag, int64_t N1, int64_t N2, int64_t N3, const double *f,
                     double *c) {
#pragma omp parallel
    {
        double *e1r = malloc(sizeof(double) * N1), *e1i = malloc(sizeof(double) * N1);
        double *e2r = malloc(sizeof(double) * N2), *e2i = malloc(sizeof(double) * N2);
        double *e3r = malloc(sizeof(double) * N3), *e3i = malloc(sizeof(double) * N3);
#pragma omp for schedule(static)
        for (int64_t j = 0; j < M; ++j) {
            phase_row(x[j], N1, iflag, e1r, e1i);
            phase_row(y[j], N2, iflag, e2r, e2i);
            phase_row(z[j], N3, iflag, e3r, e3i);
            double sr = 0.0, si = 0.0;
            for (int64_t i3 = 0; i3 < N3; ++i3) {
                for (int64_t i2 = 0; i2 < N2; ++i2) {
                    double pr = e3r[i3] * e2r[i2] - e3i[i3] * e2i[i2];
                    double pi = e3r[i3] * e2i[i2] + e3i[i3] * e2r[i2];
                    const double *row = f + 2 * ((i3 * N2 + i2) * N1);
                    double rr = 0.0, ri = 0.0;
                    for (int64_t i1 = 0; i1 < N1; ++i1) {
                        double fr = row[2 * i1], fi = row[2 * i1 + 1];
                        rr += fr * e1r[i1] - fi * e1i[i1];
                        ri += fr * e1i[i1] + fi * e1r[i1];
                    }
                    sr += rr * pr - ri * pi;
                    si += rr * pi + ri * pr;
                }
            }
            c[2 * j] = sr;
            c[2 * j + 1] = si;
        }
        free(e1r); free(e1i); free(e2r); free(e2i); free(e3r); free(e3i);
    }
}

/* type 1: f[k] = sum_j c_j e^{iflag i k.x_j}  (f overwritten) */
void oracle_nudft3d1(int64_t M, const double *x, const double *y, const double *z,
                     const double *c, int iflag, int64_t N1, int64_t N2, int64_t N3,
                     double *f) {
    memset(f, 0, sizeof(double) * 2 * N1 * N2 * N3);
#pragma omp parallel
    {
        double *e1r = malloc(sizeof(double) * N1), *e1i = malloc(sizeof(double) * N1);
        double *e2r = malloc(sizeof(double) * N2), *e2i = malloc(sizeof(double) * N2);
#pragma omp for schedule(static)
        for (int64_t i3 = 0; i3 < N3; ++i3) {
            double k3 = (double)(i3 - N3 / 2);
            for (int64_t j = 0; j < M; ++j) {
                phase_row(x[j], N1, iflag, e1r, e1i);
                phase_row(y[j], N2, iflag, e2r, e2i);
                double ph = (double)iflag * k3 * z[j];
                double e3r = cos(ph), e3i = sin(ph);
                double cr = c[2 * j] * e3r - c[2 * j + 1] * e3i;
                double ci = c[2 * j] * e3i + c[2 * j + 1] * e3r;
                for (int64_t i2 = 0; i2 < N2; ++i2) {
                    double pr = cr * e2r[i2] - ci * e2i[i2];
                    double pi = cr * e2i[i2] + ci * e2r[i2];
                    double *row = f + 2 * ((i3 * N2 + i2) * N1);
                    for (int64_t i1 = 0; i1 < N1; ++i1) {
                        row[2 * i1] += pr * e1r[i1] - pi * e1i[i1];
                        row[2 * i1 + 1] += pr * e1i[i1] + pi * e1r[i1];
                    }
                }
            }
        }
        free(e1r); free(e1i); free(e2r); free(e2i);
    }
}

/* ------------------------------------------------------------------ */
/* ES-kernel gridding                                                   */
/* ------------------------------------------------------------------ */
/* Kernel: phi(t) = exp(beta (sqrt(1 - t^2) - 1)) on |t| < 1, t = 2 (l - u) / w,
 * with u = x nf / (2 pi) the point's fine-grid coordinate and l the integer
 * tap positions ceil(u - w/2) ... ceil(u - w/2) + w - 1 (taken modulo nf). */

#define ORACLE_MAXW 32

#define DEFINE_ES(REAL, SUFFIX)                                                       \
    static inline int64_t es_taps##SUFFIX(REAL xj, int64_t nf, int w, REAL beta,      \
                                          REAL *wt) {                                 \
        REAL u = xj * (REAL)nf / (REAL)(2.0 * M_PI);                                  \
        REAL l0 = ceil(u - (REAL)w / 2);                                              \
        for (int t = 0; t < w; ++t) {                                                 \
            REAL a = (REAL)2 * (l0 + (REAL)t - u) / (REAL)w;                          \
            REAL s = (REAL)1 - a * a;                                                 \
            wt[t] = s > 0 ? (REAL)exp(beta * (sqrt(s) - (REAL)1)) : (REAL)0;          \
        }                                                                             \
        int64_t l = (int64_t)l0 % nf;                                                 \
        if (l < 0) l += nf;                                                           \
        return l;                                                                     \
    }                                                                                 \
                                                                                      \
    void oracle_es_interp##SUFFIX(int64_t M, const REAL *x, const REAL *y,            \
                                  const REAL *z, int64_t nf1, int64_t nf2,            \
                                  int64_t nf3, const REAL *G, int w, REAL beta,       \
                                  REAL *c) {                                          \
        _Pragma("omp parallel for schedule(static)")                                  \
        for (int64_t j = 0; j < M; ++j) {                                             \
            REAL w1[ORACLE_MAXW], w2[ORACLE_MAXW], w3[ORACLE_MAXW];                   \
            int64_t l1 = es_taps##SUFFIX(x[j], nf1, w, beta, w1);                     \
            int64_t l2 = es_taps##SUFFIX(y[j], nf2, w, beta, w2);                     \
            int64_t l3 = es_taps##SUFFIX(z[j], nf3, w, beta, w3);                     \
            int64_t i1s[ORACLE_MAXW];                                                 \
            for (int t = 0; t < w; ++t) i1s[t] = (l1 + t) % nf1;                      \
            REAL sr = 0, si = 0;                                                      \
            for (int t3 = 0; t3 < w; ++t3) {                                          \
                int64_t i3 = (l3 + t3) % nf3;                                         \
                for (int t2 = 0; t2 < w; ++t2) {                                      \
                    int64_t i2 = (l2 + t2) % nf2;                                     \
                    const REAL *row = G + 2 * ((i3 * nf2 + i2) * nf1);                \
                    REAL rr = 0, ri = 0;                                              \
                    for (int t1 = 0; t1 < w; ++t1) {                                  \
                        rr += w1[t1] * row[2 * i1s[t1]];                              \
                        ri += w1[t1] * row[2 * i1s[t1] + 1];                          \
                    }                                                                 \
                    REAL k23 = w3[t3] * w2[t2];                                       \
                    sr += k23 * rr;                                                   \
                    si += k23 * ri;                                                   \
                }                                                                     \
            }                                                                         \
            c[2 * j] = sr;                                                            \
            c[2 * j + 1] = si;                                                        \
        }                                                                             \
    }                                                                                 \
                                                                                      \
    void oracle_es_spread##SUFFIX(int64_t M, const REAL *x, const REAL *y,            \
                                  const REAL *z, const REAL *c, int64_t nf1,          \
                                  int64_t nf2, int64_t nf3, REAL *G, int w,           \
                                  REAL beta) {                                        \
        _Pragma("omp parallel for schedule(static)")                                  \
        for (int64_t j = 0; j < M; ++j) {                                             \
            REAL w1[ORACLE_MAXW], w2[ORACLE_MAXW], w3[ORACLE_MAXW];                   \
            int64_t l1 = es_taps##SUFFIX(x[j], nf1, w, beta, w1);                     \
            int64_t l2 = es_taps##SUFFIX(y[j], nf2, w, beta, w2);                     \
            int64_t l3 = es_taps##SUFFIX(z[j], nf3, w, beta, w3);                     \
            REAL cr = c[2 * j], ci = c[2 * j + 1];                                    \
            for (int t3 = 0; t3 < w; ++t3) {                                          \
                int64_t i3 = (l3 + t3) % nf3;                                         \
                for (int t2 = 0; t2 < w; ++t2) {                                      \
                    int64_t i2 = (l2 + t2) % nf2;                                     \
                    REAL k23 = w3[t3] * w2[t2];                                       \
                    REAL *row = G + 2 * ((i3 * nf2 + i2) * nf1);                      \
                    for (int t1 = 0; t1 < w; ++t1) {                                  \
                        int64_t i1 = (l1 + t1) % nf1;                                 \
                        REAL k = k23 * w1[t1];                                        \
                        _Pragma("omp atomic")                                         \
                        row[2 * i1] += k * cr;                                        \
                        _Pragma("omp atomic")                                         \
                        row[2 * i1 + 1] += k * ci;                                    \
                    }                                                                 \
                }                                                                     \
            }                                                                         \
        }                                                                             \
    }

DEFINE_ES(double, )
DEFINE_ES(float, _f)

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
