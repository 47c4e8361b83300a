// Toeplitz form of the normal operator sum_gamma sysmat (src/gradient.cpp:34-89
// summed by the MBIR closures, e.g. src/mbir_sb.cpp:89-97).
#pragma once

#include <cuda_fp16.h>

#include <vector>

#include "common.cuh"
#include "fft_engine.cuh"
#include "geometry.cuh"

namespace lamino {

// FP32 spectra, FP16 spectra, or both (mixed: FP32 for refinement residuals,
// FP16 for the correction solves).
enum Precision : int { PREC_FP32 = 0, PREC_FP16 = 1, PREC_MIXED = 2 };

struct Toeplitz {
    Dims3 vol;
    int64_t L1, L2, L3, L3h;     // embedding grid (even, 2,3,5-smooth, >= 2n); L3h = L3/2 + 1
    int64_t M3;                  // L3 / 2 (packed-complex length of the real transform)
    int precision = PREC_FP32;
    // spectra in apply order: [(p2 * L3h + k3) * 6 + q][p1], p = DIF position of k
    DevBuf<float> K;             // fp32 storage
    DevBuf<__half> Kh;           // fp16 storage variant
    DevBuf<float> Kscale;        // power-of-two scale per (p2, k3) pencil of Kh
    // FFT schedules and twiddles: dim 1 (length L1), dim 2 (L2), dim 3 (packed, M3)
    FftLen f1, f2, f3;
    DevBuf<float2> tw1, tw2, tw3, twh3;  // twh3: exp(-2 pi i k / L3), k <= M3
    DevBuf<int> pos3;                    // natural k -> DIF position, length M3
    // intermediates
    DevBuf<float2> z1;           // [3][n1][n2][L3h]   after the R2C along n3 (and before C2R)
    DevBuf<float2> xa;           // [3][L2][L3h][n1p]  spectra after dim 2, pencil-major
    int64_t n1p = 0;             // pencil stride: n1 rounded up to a multiple of 8
    int kb2 = 8;                 // k3 values per CTA in the dim-2 kernels (x 8 i1 values)
    int rows1 = 8;               // rows per CTA in the dim-3 kernels
    int ct1 = 0, ct2 = 0, ct3 = 0;  // compile-time FFT lengths in use (0 = runtime schedule)

    // optional per-stage timing with CUDA events on the launching stream
    static constexpr int NSTAGE = 5;  // r2c rows, dim2 fwd, pencil (fwd x K inv), dim2 inv, c2r rows
    bool profiling = false;
    std::vector<cudaEvent_t> ev;      // NSTAGE+1 events per profiled apply
    int nprof = 0;

  private:
    std::vector<int> r1_, r2_;  // radix schedules of L1 and L2
    void init_tables(Dims3 d, int precision);
    void finish(cudaStream_t s);  // FP16 spectra, intermediates, launch shapes

  public:

    Toeplitz(const std::vector<const Geom *> &gs, Dims3 d, int precision, cudaStream_t s);
    // the operator of the union of the parts' geometries, from their FP32 spectra
    Toeplitz(const std::vector<const Toeplitz *> &parts, int precision, cudaStream_t s);
    ~Toeplitz();
    int64_t Lsize() const { return L1 * L2 * L3; }
    int64_t Ssize() const { return L1 * L2 * L3h; }
    // low = true applies with the FP16 spectra (PREC_FP16 always does; PREC_MIXED on request)
    void apply(const float *x3, float *y3, cudaStream_t s, bool low = false);
    // acc[3 g + i] += x_i . (S_g x)_i for the operators S_g of `parts` (FP32
    // spectra, this volume size): one forward half-spectrum of x with this
    // operator's buffers, no inverse transform.  acc: device doubles.
    void quadforms(const float *x3, const std::vector<const Toeplitz *> &parts, double *acc, cudaStream_t s);
    // free the work buffers of an operator kept only for its spectra
    void drop_work();
    // launch shape: rows per CTA of the n3 kernels, k3 values per CTA of the n2 kernels
    void set_shape(int rows, int kb);
    // time the valid launch shapes on this operator and keep the fastest; the
    // choice is cached per (L1, L2, L3, precision) for the process.  Returns the
    // best apply time in ms (0 when taken from the cache).
    double autotune(cudaStream_t s);
    bool has_fp32() const { return K.p != nullptr; }
    bool has_fp16() const { return Kh.p != nullptr; }
    void set_profiling(bool on, int max_applies);
    // accumulated stage milliseconds over profiled applies; returns count
    int stage_times(double *ms);
    // algorithmic bytes moved by each stage of one apply
    void stage_bytes(int64_t *b) const;
    static const char *stage_name(int i);
    // number of this library's kernels launched per apply
    static int kernels_per_apply() { return NSTAGE; }
    size_t device_bytes() const;
};

}  // namespace lamino
