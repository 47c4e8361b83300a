/*
 * The subset of the FFTW3 C API that the reference calls (include/fft.h:35-263),
 * declared for the checker build only (TEST INFRASTRUCTURE; implemented over
 * this project's CPU FFT in oracle/fftw_shim.cpp).  FFTW3 itself is absent.
 * Semantics follow FFTW's documentation: unnormalised transforms,
 * FFTW_FORWARD = exponent sign -1, r2c keeps n_last/2 + 1 outputs, c2r treats its
 * input as the half spectrum of a Hermitian array.  Only dense layouts
 * (inembed/onembed null, unit strides) are supported, as the reference uses.
 */
#ifndef ORACLE_SHIM_FFTW3_H
#define ORACLE_SHIM_FFTW3_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct oracle_fft_plan_s *fftw_plan;
typedef struct oracle_fft_plan_s *fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed,
                             int istride, int idist, fftw_complex *out, const int *onembed, int ostride,
                             int odist, int sign, unsigned flags);
fftwf_plan fftwf_plan_many_dft(int rank, const int *n, int howmany, fftwf_complex *in, const int *inembed,
                               int istride, int idist, fftwf_complex *out, const int *onembed, int ostride,
                               int odist, int sign, unsigned flags);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in, const int *inembed,
                                 int istride, int idist, fftw_complex *out, const int *onembed, int ostride,
                                 int odist, unsigned flags);
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int *n, int howmany, float *in, const int *inembed,
                                   int istride, int idist, fftwf_complex *out, const int *onembed, int ostride,
                                   int odist, unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed,
                                 int istride, int idist, double *out, const int *onembed, int ostride,
                                 int odist, unsigned flags);
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int *n, int howmany, fftwf_complex *in, const int *inembed,
                                   int istride, int idist, float *out, const int *onembed, int ostride,
                                   int odist, unsigned flags);
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float *in, fftwf_complex *out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex *in, float *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftwf_execute(const fftwf_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftwf_destroy_plan(fftwf_plan p);

#ifdef __cplusplus
}
#endif
#endif
