// Toeplitz form of the normal operator sum_gamma sysmat (src/gradient.cpp:34-89
// summed by the MBIR closures, e.g. src/mbir_sb.cpp:89-97).
#pragma once

#include <cuda_fp16.h>

#include <vector>

#include "common.cuh"
#include "geometry.cuh"

namespace lamino {

enum Precision : int { PREC_FP32 = 0, PREC_FP16 = 1 };

struct Toeplitz {
    Dims3 vol;
    int64_t L1, L2, L3, L3h;     // embedding grid (even, 2,3,5-smooth, >= 2n) and L3/2+1
    int precision = PREC_FP32;
    DevBuf<float> K;             // 6 real half-spectra (fp32), pair order 00,11,22,01,02,12
    DevBuf<__half> Kh;           // fp16 storage variant
    DevBuf<float> Kscale;        // per-k1-plane power-of-two scales of Kh
    DevBuf<float> xpad;          // 3 zero-padded real grids (zero outside the data box)
    DevBuf<float2> xhat;         // 3 half-spectra
    DevBuf<float> ypad;          // 3 real grids (C2R outputs)
    FftPlan r2c, c2r;

    // optional per-stage timing with CUDA events on the launching stream
    static constexpr int NSTAGE = 5;  // pad, r2c, multiply, c2r, crop
    bool profiling = false;
    std::vector<cudaEvent_t> ev;      // NSTAGE+1 events per profiled apply
    int nprof = 0;

    Toeplitz(const std::vector<const Geom *> &gs, Dims3 d, int precision, cudaStream_t s);
    ~Toeplitz();
    int64_t Lsize() const { return L1 * L2 * L3; }
    int64_t Ssize() const { return L1 * L2 * L3h; }
    void apply(const float *x3, float *y3, cudaStream_t s);
    void set_profiling(bool on, int max_applies);
    // accumulated stage milliseconds over profiled applies; returns count
    int stage_times(double *ms);
    // algorithmic bytes moved by each stage of one apply
    void stage_bytes(int64_t *b) const;
    static const char *stage_name(int i);
    // number of this library's kernels launched per apply
    static int kernels_per_apply() { return 3; }
};

}  // namespace lamino
