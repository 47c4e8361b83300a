/*
 * The subset of the FINUFFT C API that the reference calls
 * (include/finufft_plan.h:35-129), declared for the checker build only (TEST
 * INFRASTRUCTURE; implemented in oracle/finufft_shim.cpp over this project's
 * ES-kernel gridding and CPU FFT).  FINUFFT itself is third-party, unpinned by
 * the reference (cmake/Findfinufft.cmake has no version) and absent here; these
 * declarations restate its published interface (FINUFFT 2.x guru interface):
 *   type 1: f[k] = sum_j c_j exp(iflag i k.x_j);  type 2: c_j = sum_k f[k] exp(iflag i k.x_j)
 *   modes centred, k = idx - floor(N/2) (modeord 0), x pairs with n_modes[0] (fastest).
 */
#ifndef ORACLE_SHIM_FINUFFT_H
#define ORACLE_SHIM_FINUFFT_H

#include <stdint.h>

#ifdef __cplusplus
#include <complex>
typedef std::complex<double> finufft_cpx;
typedef std::complex<float> finufftf_cpx;
extern "C" {
#else
typedef double _Complex finufft_cpx;
typedef float _Complex finufftf_cpx;
#endif

typedef struct finufft_opts {
    int modeord;      /* 0: centred modes (the only ordering supported) */
    int debug;
    int nthreads;     /* 0: all OpenMP threads */
    double upsampfac; /* 2.0 (the only value supported) */
} finufft_opts;

typedef struct oracle_nufft_plan_s *finufft_plan;
typedef struct oracle_nufftf_plan_s *finufftf_plan;

void finufft_default_opts(finufft_opts *o);
int finufft_makeplan(int type, int dim, int64_t *n_modes, int iflag, int ntrans, double eps, finufft_plan *plan,
                     finufft_opts *o);
int finufftf_makeplan(int type, int dim, int64_t *n_modes, int iflag, int ntrans, float eps,
                      finufftf_plan *plan, finufft_opts *o);
int finufft_setpts(finufft_plan plan, int64_t M, double *x, double *y, double *z, int64_t N, double *s,
                   double *t, double *u);
int finufftf_setpts(finufftf_plan plan, int64_t M, float *x, float *y, float *z, int64_t N, float *s, float *t,
                    float *u);
int finufft_execute(finufft_plan plan, finufft_cpx *c, finufft_cpx *f);
int finufftf_execute(finufftf_plan plan, finufftf_cpx *c, finufftf_cpx *f);
int finufft_destroy(finufft_plan plan);
int finufftf_destroy(finufftf_plan plan);

#ifdef __cplusplus
}
#endif
#endif
