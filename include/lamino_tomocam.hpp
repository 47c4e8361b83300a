/* C++ operator surface of the reference (tomocam-lamino) over the C ABI of
 * liblamino_b200.so: the header a maintainer of the reference adds to switch
 * its FINUFFT/OpenMP path to the GPU without touching the solver or driver code.
 *
 * Include it after the reference's "polar_grid.h" (which brings "array.h" and
 * "dtypes.h"); link with -llamino_b200.  Same names, argument meaning and
 * exception types as the reference:
 *
 *   tomocam::forward   include/projection.h:52-54   -> tomocam::gpu::forward
 *   tomocam::adjoint   include/projection.h:64-66   -> tomocam::gpu::adjoint
 *   tomocam::sysmat    include/tomocam.h:50-52      -> tomocam::gpu::sysmat
 *   tomocam::gradient  include/tomocam.h:64-67      -> tomocam::gpu::gradient
 *   tomocam::residual  include/tomocam.h:79-82      -> tomocam::gpu::residual
 *   MBIR `A` closures  src/mbir_sb.cpp:89-97        -> tomocam::gpu::Normal
 *   tomocam::MBIR1/2/3 include/tomocam.h:101-154    -> tomocam::gpu::MBIR1/2/3
 *
 * Volumes are std::array<Array<float>, 3> of (n1, n2, n3) = (W, T, H) each, as
 * in the reference; projections are Array<float> (nproj, nrows, ncols).  Host
 * buffers are staged through device memory by the library.  Status codes come
 * back as std::invalid_argument (bad arguments), std::bad_alloc (out of
 * memory) or std::runtime_error (anything else), with lamino_last_error() as
 * the message.  NUFFT plans are kept per volume size for the process (the
 * reference keeps one plan per precision, sized by its first call).
 */
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "lamino.h"

namespace tomocam::gpu {

inline void check(int rc) {
    if (rc == LAMINO_OK) return;
    const char *msg = lamino_last_error();
    const std::string m = msg ? msg : "lamino error";
    if (rc == LAMINO_ERR_ARG) throw std::invalid_argument(m);
    if (rc == LAMINO_ERR_OOM) throw std::bad_alloc();
    throw std::runtime_error(m);
}

// One geometry handle per (PolarGrid, gamma): the library regenerates the points
// from the angles, so the x / y / z arrays of the grid are not read.
class Geom {
  public:
    Geom(const PolarGrid<float> &pg, float gamma) {
        const dims_t d = pg.dims();
        check(lamino_geom_create(pg.theta.data(), (int64_t)pg.nprojs(), (int64_t)d.n2, (int64_t)d.n3, gamma, &h_));
    }
    ~Geom() { lamino_geom_destroy(h_); }
    Geom(const Geom &) = delete;
    Geom &operator=(const Geom &) = delete;
    lamino_geom_t get() const { return h_; }

  private:
    lamino_geom_t h_ = nullptr;
};

// The NUFFT plan of a volume size, created on first use and kept for the process.
inline lamino_plan_t plan_for(const dims_t &d) {
    struct Del {
        void operator()(lamino_plan_s *p) const { lamino_plan_destroy(p); }
    };
    static std::mutex mu;
    static std::map<std::array<size_t, 3>, std::unique_ptr<lamino_plan_s, Del>> plans;
    std::lock_guard<std::mutex> lk(mu);
    auto &slot = plans[{d.n1, d.n2, d.n3}];
    if (!slot) {
        lamino_plan_t p = nullptr;
        check(lamino_plan_create((int64_t)d.n1, (int64_t)d.n2, (int64_t)d.n3, 1.2e-6, &p));
        slot.reset(p);
    }
    return slot.get();
}

namespace detail {
inline std::vector<float> pack3(const std::array<Array<float>, 3> &x) {
    const size_t V = x[0].size();
    if (x[1].size() != V || x[2].size() != V) throw std::invalid_argument("volume components differ in size");
    std::vector<float> v(3 * V);
    for (int i = 0; i < 3; ++i) std::copy(x[i].begin(), x[i].begin() + V, v.begin() + i * V);
    return v;
}
inline std::array<Array<float>, 3> unpack3(const std::vector<float> &v, const dims_t &d) {
    std::array<Array<float>, 3> y;
    const size_t V = d.size();
    for (int i = 0; i < 3; ++i) {
        y[i] = Array<float>(d);
        std::copy(v.begin() + i * V, v.begin() + (i + 1) * V, y[i].begin());
    }
    return y;
}
}  // namespace detail

// tomocam::forward (src/projection.cpp:42-77)
inline Array<float> forward(const std::array<Array<float>, 3> &m, const PolarGrid<float> &pg, const float &gamma) {
    const Geom g(pg, gamma);
    const std::vector<float> in = detail::pack3(m);
    Array<float> out(pg.dims());
    check(lamino_forward(plan_for(m[0].dims()), g.get(), in.data(), out.begin(), nullptr));
    return out;
}

// tomocam::adjoint (src/projection.cpp:90-126)
inline std::array<Array<float>, 3> adjoint(const Array<float> &proj, const PolarGrid<float> &pg,
                                           const dims_t &recon_dims, float gamma) {
    const Geom g(pg, gamma);
    std::vector<float> out(3 * recon_dims.size());
    check(lamino_adjoint(plan_for(recon_dims), g.get(), proj.begin(), out.data(), nullptr));
    return detail::unpack3(out, recon_dims);
}

// tomocam::sysmat (src/gradient.cpp:34-89), NUFFT form
inline std::array<Array<float>, 3> sysmat(const std::array<Array<float>, 3> &x, const PolarGrid<float> &pg,
                                          float gamma) {
    const Geom g(pg, gamma);
    const lamino_geom_t gh = g.get();
    const std::vector<float> in = detail::pack3(x);
    std::vector<float> out(in.size());
    check(lamino_sysmat(plan_for(x[0].dims()), &gh, 1, in.data(), out.data(), nullptr));
    return detail::unpack3(out, x[0].dims());
}

// tomocam::gradient (src/gradient.cpp:98-105): sysmat(m) - pT
inline std::array<Array<float>, 3> gradient(const std::array<Array<float>, 3> &m,
                                            const std::array<Array<float>, 3> &pT, const PolarGrid<float> &pg,
                                            float gamma) {
    const Geom g(pg, gamma);
    const std::vector<float> a = detail::pack3(m), b = detail::pack3(pT);
    std::vector<float> out(a.size());
    check(lamino_gradient(plan_for(m[0].dims()), g.get(), a.data(), b.data(), out.data(), nullptr));
    return detail::unpack3(out, m[0].dims());
}

// tomocam::residual (src/gradient.cpp:117-127)
inline float residual(const std::array<Array<float>, 3> &m, const std::array<Array<float>, 3> &pT,
                      const PolarGrid<float> &pg, float pTp, float gamma) {
    const Geom g(pg, gamma);
    const std::vector<float> a = detail::pack3(m), b = detail::pack3(pT);
    double r = 0.0;
    check(lamino_residual(plan_for(m[0].dims()), g.get(), a.data(), b.data(), pTp, &r, nullptr));
    return (float)r;
}

// The summed normal operator sum_gamma sysmat of the MBIR `A` closures
// (src/mbir_cg.cpp:97-105, src/mbir_sb.cpp:89-97) in Toeplitz form:
//     tomocam::gpu::Normal A(grids, out_dims);
//     opt::Function<float> f = [&](const std::array<Array<float>, 3> &x) { return A(x); };
class Normal {
  public:
    // grids: (PolarGrid, gamma) per dataset; precision LAMINO_PREC_FP32 or LAMINO_PREC_FP16
    Normal(const std::vector<std::pair<const PolarGrid<float> *, float>> &grids, const dims_t &dims,
           int precision = LAMINO_PREC_FP32)
        : dims_(dims) {
        std::vector<std::unique_ptr<Geom>> gs;
        std::vector<lamino_geom_t> hs;
        for (const auto &[pg, gamma] : grids) {
            gs.push_back(std::make_unique<Geom>(*pg, gamma));
            hs.push_back(gs.back()->get());
        }
        check(lamino_normal_create(hs.data(), (int)hs.size(), (int64_t)dims.n1, (int64_t)dims.n2, (int64_t)dims.n3,
                                   precision, &h_, nullptr));
    }
    ~Normal() { lamino_normal_destroy(h_); }
    Normal(const Normal &) = delete;
    Normal &operator=(const Normal &) = delete;

    std::array<Array<float>, 3> operator()(const std::array<Array<float>, 3> &x) const {
        const std::vector<float> in = detail::pack3(x);
        std::vector<float> out(in.size());
        check(lamino_normal_apply(h_, in.data(), out.data(), nullptr));
        return detail::unpack3(out, dims_);
    }
    lamino_normal_t get() const { return h_; }

  private:
    dims_t dims_;
    lamino_normal_t h_ = nullptr;
};

// tomocam::MBIR1 / MBIR2 / MBIR3 (include/tomocam.h:101-154).  Params: the
// reference's tomocam::ReconParams (include/config.h:146-158) or any type with
// its fields maxIters, innerIters, sigma, p, lambda, mu, tol, xtol, PAD_FACTOR.
template <class Params>
std::array<Array<float>, 3> MBIR(int method,
                                 const std::vector<std::tuple<Array<float>, std::vector<float>, float>> &datasets,
                                 const dims_t &recon_dims, const Params &params) {
    lamino_recon_params p;
    lamino_recon_params_default(&p);
    p.max_iters = (int)params.maxIters;
    p.inner_iters = (int)params.innerIters;
    p.sigma = params.sigma;
    p.p = params.p;
    p.lambda = params.lambda;
    p.mu = params.mu;
    p.tol = params.tol;
    p.xtol = params.xtol;
    p.pad_factor = params.PAD_FACTOR;
    std::vector<const float *> projs, angles;
    std::vector<int64_t> pdims;
    std::vector<float> gammas;
    for (const auto &[proj, ang, gamma] : datasets) {
        const dims_t d = proj.dims();
        if (ang.size() != d.n1) throw std::invalid_argument("one angle per projection is needed");
        projs.push_back(proj.begin());
        angles.push_back(ang.data());
        pdims.insert(pdims.end(), {(int64_t)d.n1, (int64_t)d.n2, (int64_t)d.n3});
        gammas.push_back(gamma);
    }
    std::vector<float> out(3 * recon_dims.size());
    check(lamino_mbir(method, (int)datasets.size(), projs.data(), pdims.data(), angles.data(), gammas.data(),
                      (int64_t)recon_dims.n1, (int64_t)recon_dims.n2, (int64_t)recon_dims.n3, &p, out.data(),
                      nullptr));
    return detail::unpack3(out, recon_dims);
}

template <class Params>
std::array<Array<float>, 3> MBIR1(const std::vector<std::tuple<Array<float>, std::vector<float>, float>> &datasets,
                                  const dims_t &recon_dims, const Params &params) {
    return MBIR(1, datasets, recon_dims, params);
}
template <class Params>
std::array<Array<float>, 3> MBIR2(const std::vector<std::tuple<Array<float>, std::vector<float>, float>> &datasets,
                                  const dims_t &recon_dims, const Params &params) {
    return MBIR(2, datasets, recon_dims, params);
}
template <class Params>
std::array<Array<float>, 3> MBIR3(const std::vector<std::tuple<Array<float>, std::vector<float>, float>> &datasets,
                                  const dims_t &recon_dims, const Params &params) {
    return MBIR(3, datasets, recon_dims, params);
}

}  // namespace tomocam::gpu
