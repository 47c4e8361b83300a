// Laminography geometry: the non-uniform frequency points of one gamma dataset.
//
// Restates include/polar_grid.h:44-75 of the reference, but stores only the
// separable factors (qX per column, qY per row, sin/cos per projection); each
// kernel regenerates a point's (x, y, z) in registers with the same float
// operations, in the same order, as the reference:
//   qX = T(k*dX - pi + dX/2), qY likewise (middle terms in double)
//   z = (-qX) sin(g) + (qY cos(th)) cos(g);  y = (-qY) sin(th);
//   x = qX cos(g) + (qY cos(th)) sin(g)
// (round-to-nearest products and sums, no contraction into FMA).  Storing
// nothing per point removes the 3 x 4 B x M coordinate arrays (26 GB at the
// 51x511x511 / 4-gamma size) and every setpts sort of the reference path.
#pragma once

#include <atomic>
#include <cmath>
#include <vector>

#include "common.cuh"

namespace lamino {

// beam_dir_vector (include/projection.h:37-41) in float.
inline void beam_dir_vector_f(float gamma, float alpha, float out[3]) {
    out[0] = std::sin(gamma) * std::sin(alpha);
    out[1] = std::cos(alpha);
    out[2] = std::cos(gamma) * std::sin(alpha);
}

struct GeomView {  // passed by value to kernels
    const float *qX, *qY, *st, *ct, *coeff;  // coeff: [3][nproj]
    int nproj, nrows, ncols;
    float sg, cg;
};

// Process-unique id of a geometry (keys caches of per-geometry point orders).
inline uint64_t next_geom_uid() {
    static std::atomic<uint64_t> n{0};
    return ++n;
}

struct Geom {
    uint64_t uid = next_geom_uid();
    int64_t nproj = 0, nrows = 0, ncols = 0;
    float gamma = 0.f, sg = 0.f, cg = 0.f;
    std::vector<float> theta;
    std::vector<float> h_coeff;  // [3][nproj]
    DevBuf<float> qX, qY, st, ct, coeff;

    Geom(const float *angles, int64_t np, int64_t nr, int64_t nc, float g)
        : nproj(np), nrows(nr), ncols(nc), gamma(g), theta(angles, angles + np) {
        if (np <= 0 || nr <= 0 || nc <= 0) throw Error(ERR_ARG, "geometry sizes must be positive");
        std::vector<float> hx(nc), hy(nr), hs(np), hc(np);
        h_coeff.resize(3 * np);
        float dX = (float)((2 * M_PI) / (double)(float)nc);
        float dY = (float)((2 * M_PI) / (double)(float)nr);
        for (int64_t k = 0; k < nc; ++k)
            hx[k] = (float)((double)((float)k * dX) - M_PI + (double)(dX / 2));
        for (int64_t j = 0; j < nr; ++j)
            hy[j] = (float)((double)((float)j * dY) - M_PI + (double)(dY / 2));
        for (int64_t i = 0; i < np; ++i) {
            hs[i] = std::sin(theta[i]);
            hc[i] = std::cos(theta[i]);
            float c[3];
            beam_dir_vector_f(g, theta[i], c);
            for (int q = 0; q < 3; ++q) h_coeff[q * np + i] = c[q];
        }
        sg = std::sin(g);
        cg = std::cos(g);
        qX.alloc(nc); qY.alloc(nr); st.alloc(np); ct.alloc(np); coeff.alloc(3 * np);
        upload(qX.p, hx.data(), (size_t)nc);
        upload(qY.p, hy.data(), (size_t)nr);
        upload(st.p, hs.data(), (size_t)np);
        upload(ct.p, hc.data(), (size_t)np);
        upload(coeff.p, h_coeff.data(), (size_t)(3 * np));
    }
    GeomView view() const {
        return GeomView{qX.p, qY.p, st.p, ct.p, coeff.p, (int)nproj, (int)nrows, (int)ncols, sg, cg};
    }
    int64_t npts() const { return nproj * nrows * ncols; }
};

// Point (p, j, k) of a geometry, in the reference's float arithmetic.
__device__ __forceinline__ void point_xyz(const GeomView &g, int p, int j, int k, float &x,
                                          float &y, float &z) {
    float qx = __ldg(g.qX + k), qy = __ldg(g.qY + j);
    float ct = __ldg(g.ct + p), st = __ldg(g.st + p);
    float qyc = __fmul_rn(qy, ct);
    x = __fadd_rn(__fmul_rn(qx, g.cg), __fmul_rn(qyc, g.sg));
    y = __fmul_rn(-qy, st);
    z = __fadd_rn(__fmul_rn(-qx, g.sg), __fmul_rn(qyc, g.cg));
}

}  // namespace lamino
