// Demagnetizing field of a magnetization volume (include/demag.h:13-79):
// H = F^-1[ -k (k . m^) / |k|^2 ] / N, the k = 0 term set to 0, with the
// reference's frequency grids (fftfreq along n1 and n2, rfftfreq along n3, each
// times 2 pi / n in float) and its float arithmetic order.  The three real
// 3-D transforms run as one batched cuFFT R2C / C2R pair; the spectral step is
// one kernel, in place on the three half-spectra, with the 1/N folded in.
#include "demag.cuh"

namespace lamino {

__device__ __forceinline__ float fftfreq_dev(int i, int n, float dk) {
    const int half = (n % 2 == 0) ? n / 2 : n / 2 + 1;
    return (float)(i < half ? i : i - n) * dk;
}

__global__ void k_demag_spectrum(float2 *__restrict__ S, int n1, int n2, int nk, float dk1, float dk2, float dk3,
                                 float norm) {
    const int64_t plane = (int64_t)n1 * n2 * nk;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < plane;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(idx % nk);
        const int64_t r = idx / nk;
        const int j = (int)(r % n2);
        const int i = (int)(r / n2);
        const float kx = fftfreq_dev(i, n1, dk1), ky = fftfreq_dev(j, n2, dk2), kz = (float)k * dk3;
        float kk = __fadd_rn(__fadd_rn(__fmul_rn(kx, kx), __fmul_rn(ky, ky)), __fmul_rn(kz, kz));
        const bool dc = (i == 0 && j == 0 && k == 0);
        if (dc) kk = 1.0f;
        const float kinv = (float)(1.0 / (double)kk);
        const float2 m0 = S[idx], m1 = S[plane + idx], m2 = S[2 * plane + idx];
        const float2 kdm = make_float2(__fadd_rn(__fadd_rn(__fmul_rn(kx, m0.x), __fmul_rn(ky, m1.x)), __fmul_rn(kz, m2.x)),
                                       __fadd_rn(__fadd_rn(__fmul_rn(kx, m0.y), __fmul_rn(ky, m1.y)), __fmul_rn(kz, m2.y)));
        const float kc[3] = {kx, ky, kz};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float2 h = make_float2(__fmul_rn(__fmul_rn(-kdm.x, kc[c]), kinv), __fmul_rn(__fmul_rn(-kdm.y, kc[c]), kinv));
            if (dc) h = make_float2(0.f, 0.f);
            S[c * plane + idx] = make_float2(h.x * norm, h.y * norm);
        }
    }
}

void demag(const float *m3, Dims3 d, float *h3, cudaStream_t s) {
    if (d.n1 <= 0 || d.n2 <= 0 || d.n3 <= 0) throw Error(ERR_ARG, "volume dims must be positive");
    if (d.size() > (int64_t)INT32_MAX) throw Error(ERR_ARG, "volume too large for one transform");
    const int64_t nk = d.n3 / 2 + 1;
    const int64_t plane = d.n1 * d.n2 * nk;
    DevBuf<float2> spec((size_t)(3 * plane));
    int n[3] = {(int)d.n1, (int)d.n2, (int)d.n3};
    FftPlan r2c, c2r;
    r2c.make(3, n, CUFFT_R2C, 3);
    c2r.make(3, n, CUFFT_C2R, 3);
    LAMINO_CUFFT(cufftSetStream(r2c.h, s));
    LAMINO_CUFFT(cufftSetStream(c2r.h, s));
    // cuFFT's R2C does not modify its input; the cast drops const for its signature
    LAMINO_CUFFT(cufftExecR2C(r2c.h, const_cast<float *>(m3), (cufftComplex *)spec.p));
    const float dk1 = (float)(2 * M_PI / (double)(float)d.n1);
    const float dk2 = (float)(2 * M_PI / (double)(float)d.n2);
    const float dk3 = (float)(2 * M_PI / (double)(float)d.n3);
    const float norm = (float)(1.0 / (double)(d.n1 * d.n2 * d.n3));
    k_demag_spectrum<<<grid_for(plane, 256), 256, 0, s>>>(spec.p, (int)d.n1, (int)d.n2, (int)nk, dk1, dk2, dk3,
                                                          norm);
    LAMINO_LAUNCH("k_demag_spectrum");
    LAMINO_CUFFT(cufftExecC2R(c2r.h, (cufftComplex *)spec.p, h3));
    LAMINO_CUDA(cudaStreamSynchronize(s));  // the plans and the spectrum are released on return
}

}  // namespace lamino
