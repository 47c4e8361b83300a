/*
 * C-ABI shim over the reference's own operator and solver path, compiled where
 * the sources lie (src/projection.cpp, src/gradient.cpp, src/conjgrad.cpp,
 * src/bregman.cpp, src/finitediff.cpp, src/nagopt.cpp, src/qggmrf.cpp,
 * src/mbir_cg.cpp, src/mbir_sb.cpp, src/mbir3.cpp, and the headers they
 * include), against this project's FINUFFT-API and FFTW-API shims
 * (finufft_shim.cpp, fftw_shim.cpp) and the toml++ / libtiff stubs under shim/.
 * TEST INFRASTRUCTURE ONLY: it produces the golden outputs the oracle and the
 * GPU path are pinned to, and the timed CPU path of the bench's reference arm.
 *
 * Every arithmetic step outside the NUFFT and the uniform FFTs is the
 * reference's own code.  Entry points (T = float: suffix _f, double: _d):
 *   ref_forward      tomocam::forward      src/projection.cpp:42-77
 *   ref_adjoint      tomocam::adjoint      src/projection.cpp:90-126
 *   ref_sysmat       tomocam::sysmat       src/gradient.cpp:34-89
 *   ref_normal       sum over datasets of sysmat, the MBIR closures (src/mbir_cg.cpp:97-105)
 *   ref_gradient     tomocam::gradient     src/gradient.cpp:98-105
 *   ref_residual     tomocam::residual     src/gradient.cpp:117-127
 *   ref_ramp         opt::RampPreconditioner::apply  include/precond.h:72-86
 *   ref_cgsolver     opt::cgsolver on the normal operator   src/conjgrad.cpp:37-117
 *   ref_split_bregman opt::split_bregman on the normal operator src/bregman.cpp:39-134
 *   ref_mbir         tomocam::MBIR1 / MBIR2 / MBIR3 src/mbir_cg.cpp:48, src/mbir_sb.cpp:47, src/mbir3.cpp:47
 * The reference keeps one FINUFFT plan per precision and transform type for the
 * whole process, sized by the first call (include/finufft_plan_cache.h:50-66):
 * a process must use a single volume size per precision.  Volumes are three
 * contiguous components [3][n1][n2][n3]; projections [nproj][nrows][ncols].
 * quiet != 0 silences the solvers' per-iteration prints on std::cout.
 */
#include <array>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <iostream>
#include <sstream>
#include <tuple>
#include <vector>

#include "array.h"
#include "array_ops.h"
#include "optimize.h"
#include "polar_grid.h"
#include "precond.h"
#include "projection.h"
#include "tomocam.h"

using tomocam::Array;
using tomocam::dims_t;
using tomocam::PolarGrid;

namespace {

struct Quiet {
    std::streambuf *old = nullptr;
    std::ostringstream sink;
    explicit Quiet(int on) {
        if (on) old = std::cout.rdbuf(sink.rdbuf());
    }
    ~Quiet() {
        if (old) std::cout.rdbuf(old);
    }
};

template <typename T>
Array<T> arr(const T *p, int64_t n1, int64_t n2, int64_t n3) {
    Array<T> a(dims_t(n1, n2, n3));
    std::memcpy(a.begin(), p, sizeof(T) * a.size());
    return a;
}
template <typename T>
std::array<Array<T>, 3> vec3(const T *p, int64_t n1, int64_t n2, int64_t n3) {
    const int64_t v = n1 * n2 * n3;
    return {arr(p, n1, n2, n3), arr(p + v, n1, n2, n3), arr(p + 2 * v, n1, n2, n3)};
}
template <typename T>
void put3(const std::array<Array<T>, 3> &a, T *p) {
    const size_t v = a[0].size();
    for (int i = 0; i < 3; ++i) std::memcpy(p + i * v, a[i].begin(), sizeof(T) * v);
}

template <typename T>
struct Geoms {
    std::vector<PolarGrid<T>> grids;
    std::vector<T> gammas;
    Geoms(int ng, const int64_t *nproj, const int64_t *nrows, const int64_t *ncols, const T *angles,
          const T *gammas_) {
        size_t off = 0;
        for (int g = 0; g < ng; ++g) {
            std::vector<T> th(angles + off, angles + off + nproj[g]);
            off += nproj[g];
            grids.emplace_back(th, (size_t)nrows[g], (size_t)ncols[g], gammas_[g]);
            gammas.push_back(gammas_[g]);
        }
    }
    std::array<Array<T>, 3> normal(const std::array<Array<T>, 3> &x) const {
        auto Ax = tomocam::sysmat(x, grids[0], gammas[0]);
        for (size_t j = 1; j < grids.size(); ++j) {
            auto t = tomocam::sysmat(x, grids[j], gammas[j]);
            for (int i = 0; i < 3; ++i) Ax[i] += t[i];
        }
        return Ax;
    }
};

template <typename T>
int guard(const std::function<void()> &f) {
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        std::cerr << "reference path: " << e.what() << "\n";
        return 1;
    }
}

template <typename T>
int forward_impl(const T *m3, int64_t n1, int64_t n2, int64_t n3, const T *angles, int64_t nproj, int64_t nrows,
                 int64_t ncols, T gamma, T *out) {
    return guard<T>([&] {
        std::vector<T> th(angles, angles + nproj);
        PolarGrid<T> pg(th, nrows, ncols, gamma);
        auto p = tomocam::forward(vec3(m3, n1, n2, n3), pg, gamma);
        std::memcpy(out, p.begin(), sizeof(T) * p.size());
    });
}

template <typename T>
int adjoint_impl(const T *proj, int64_t nproj, int64_t nrows, int64_t ncols, const T *angles, T gamma, int64_t n1,
                 int64_t n2, int64_t n3, T *out3) {
    return guard<T>([&] {
        std::vector<T> th(angles, angles + nproj);
        PolarGrid<T> pg(th, nrows, ncols, gamma);
        auto r = tomocam::adjoint(arr(proj, nproj, nrows, ncols), pg, dims_t(n1, n2, n3), gamma);
        put3(r, out3);
    });
}

template <typename T>
int sysmat_impl(const T *x3, int64_t n1, int64_t n2, int64_t n3, const T *angles, int64_t nproj, int64_t nrows,
                int64_t ncols, T gamma, T *out3) {
    return guard<T>([&] {
        std::vector<T> th(angles, angles + nproj);
        PolarGrid<T> pg(th, nrows, ncols, gamma);
        put3(tomocam::sysmat(vec3(x3, n1, n2, n3), pg, gamma), out3);
    });
}

template <typename T>
int normal_impl(const T *x3, int64_t n1, int64_t n2, int64_t n3, int ng, const int64_t *nproj, const int64_t *nrows,
                const int64_t *ncols, const T *angles, const T *gammas, T *out3) {
    return guard<T>([&] {
        Geoms<T> G(ng, nproj, nrows, ncols, angles, gammas);
        put3(G.normal(vec3(x3, n1, n2, n3)), out3);
    });
}

template <typename T>
int gradient_impl(const T *x3, const T *yT3, int64_t n1, int64_t n2, int64_t n3, const T *angles, int64_t nproj,
                  int64_t nrows, int64_t ncols, T gamma, T *out3) {
    return guard<T>([&] {
        std::vector<T> th(angles, angles + nproj);
        PolarGrid<T> pg(th, nrows, ncols, gamma);
        put3(tomocam::gradient(vec3(x3, n1, n2, n3), vec3(yT3, n1, n2, n3), pg, gamma), out3);
    });
}

template <typename T>
int residual_impl(const T *x3, const T *yT3, int64_t n1, int64_t n2, int64_t n3, const T *angles, int64_t nproj,
                  int64_t nrows, int64_t ncols, T yTy, T gamma, T *out) {
    return guard<T>([&] {
        std::vector<T> th(angles, angles + nproj);
        PolarGrid<T> pg(th, nrows, ncols, gamma);
        *out = tomocam::residual(vec3(x3, n1, n2, n3), vec3(yT3, n1, n2, n3), pg, yTy, gamma);
    });
}

template <typename T>
int ramp_impl(const T *in, int64_t n1, int64_t n2, int64_t n3, T *out) {
    return guard<T>([&] {
        tomocam::opt::RampPreconditioner<T> P(dims_t(n1, n2, n3));
        auto r = P.apply(arr(in, n1, n2, n3));
        std::memcpy(out, r.begin(), sizeof(T) * r.size());
    });
}

template <typename T>
int cg_impl(const T *b3, const T *x03, int64_t n1, int64_t n2, int64_t n3, int ng, const int64_t *nproj,
            const int64_t *nrows, const int64_t *ncols, const T *angles, const T *gammas, int64_t max_iter, T tol,
            int quiet, T *out3) {
    return guard<T>([&] {
        Geoms<T> G(ng, nproj, nrows, ncols, angles, gammas);
        tomocam::opt::Function<T> A = [&G](const std::array<Array<T>, 3> &x) { return G.normal(x); };
        Quiet q(quiet);
        auto x = tomocam::opt::cgsolver<T>(A, vec3(b3, n1, n2, n3), vec3(x03, n1, n2, n3), (size_t)max_iter, tol,
                                           T(0));
        put3(x, out3);
    });
}

template <typename T>
int sb_impl(const T *yT3, const T *x03, int64_t n1, int64_t n2, int64_t n3, int ng, const int64_t *nproj,
            const int64_t *nrows, const int64_t *ncols, const T *angles, const T *gammas, T lambda, T mu,
            int64_t outer, int64_t inner, T tol, T xtol, int quiet, T *out3) {
    return guard<T>([&] {
        Geoms<T> G(ng, nproj, nrows, ncols, angles, gammas);
        tomocam::opt::Function<T> A = [&G](const std::array<Array<T>, 3> &x) { return G.normal(x); };
        Quiet q(quiet);
        auto x = tomocam::opt::split_bregman<T>(A, vec3(yT3, n1, n2, n3), vec3(x03, n1, n2, n3), lambda, mu,
                                                (size_t)outer, (size_t)inner, tol, xtol);
        put3(x, out3);
    });
}

template <typename T>
int mbir_impl(int which, int ng, const T *proj, const int64_t *nproj, const int64_t *nrows, const int64_t *ncols,
              const T *angles, const T *gammas, int64_t r1, int64_t r2, int64_t r3, int64_t max_iters,
              int64_t inner_iters, double sigma, double p, double lambda, double mu, double tol, double xtol,
              int quiet, T *out3) {
    return guard<T>([&] {
        std::vector<std::tuple<Array<T>, std::vector<T>, T>> ds;
        size_t poff = 0, aoff = 0;
        for (int g = 0; g < ng; ++g) {
            Array<T> pa = arr(proj + poff, nproj[g], nrows[g], ncols[g]);
            poff += (size_t)(nproj[g] * nrows[g] * ncols[g]);
            std::vector<T> th(angles + aoff, angles + aoff + nproj[g]);
            aoff += nproj[g];
            ds.emplace_back(std::move(pa), std::move(th), gammas[g]);
        }
        tomocam::ReconParams rp;
        rp.maxIters = (size_t)max_iters;
        rp.innerIters = (size_t)inner_iters;
        rp.sigma = (float)sigma;
        rp.p = (float)p;
        rp.lambda = (float)lambda;
        rp.mu = (float)mu;
        rp.tol = (float)tol;
        rp.xtol = (float)xtol;
        Quiet q(quiet);
        const dims_t rd(r1, r2, r3);
        std::array<Array<T>, 3> r;
        if (which == 1) r = tomocam::MBIR1<T>(ds, rd, rp);
        else if (which == 2) r = tomocam::MBIR2<T>(ds, rd, rp);
        else r = tomocam::MBIR3<T>(ds, rd, rp);
        put3(r, out3);
    });
}

}  // namespace

#define REF_DEFINE(T, S)                                                                                          \
    int ref_forward##S(const T *m3, int64_t n1, int64_t n2, int64_t n3, const T *angles, int64_t nproj,          \
                       int64_t nrows, int64_t ncols, T gamma, T *out) {                                          \
        return forward_impl<T>(m3, n1, n2, n3, angles, nproj, nrows, ncols, gamma, out);                         \
    }                                                                                                             \
    int ref_adjoint##S(const T *proj, int64_t nproj, int64_t nrows, int64_t ncols, const T *angles, T gamma,      \
                       int64_t n1, int64_t n2, int64_t n3, T *out3) {                                            \
        return adjoint_impl<T>(proj, nproj, nrows, ncols, angles, gamma, n1, n2, n3, out3);                      \
    }                                                                                                             \
    int ref_sysmat##S(const T *x3, int64_t n1, int64_t n2, int64_t n3, const T *angles, int64_t nproj,           \
                      int64_t nrows, int64_t ncols, T gamma, T *out3) {                                          \
        return sysmat_impl<T>(x3, n1, n2, n3, angles, nproj, nrows, ncols, gamma, out3);                         \
    }                                                                                                             \
    int ref_normal##S(const T *x3, int64_t n1, int64_t n2, int64_t n3, int ng, const int64_t *nproj,             \
                      const int64_t *nrows, const int64_t *ncols, const T *angles, const T *gammas, T *out3) {  \
        return normal_impl<T>(x3, n1, n2, n3, ng, nproj, nrows, ncols, angles, gammas, out3);                    \
    }                                                                                                             \
    int ref_gradient##S(const T *x3, const T *yT3, int64_t n1, int64_t n2, int64_t n3, const T *angles,          \
                        int64_t nproj, int64_t nrows, int64_t ncols, T gamma, T *out3) {                         \
        return gradient_impl<T>(x3, yT3, n1, n2, n3, angles, nproj, nrows, ncols, gamma, out3);                  \
    }                                                                                                             \
    int ref_residual##S(const T *x3, const T *yT3, int64_t n1, int64_t n2, int64_t n3, const T *angles,          \
                        int64_t nproj, int64_t nrows, int64_t ncols, T yTy, T gamma, T *out) {                   \
        return residual_impl<T>(x3, yT3, n1, n2, n3, angles, nproj, nrows, ncols, yTy, gamma, out);              \
    }                                                                                                             \
    int ref_ramp##S(const T *in, int64_t n1, int64_t n2, int64_t n3, T *out) {                                   \
        return ramp_impl<T>(in, n1, n2, n3, out);                                                                \
    }                                                                                                             \
    int ref_cgsolver##S(const T *b3, const T *x03, int64_t n1, int64_t n2, int64_t n3, int ng,                   \
                        const int64_t *nproj, const int64_t *nrows, const int64_t *ncols, const T *angles,       \
                        const T *gammas, int64_t max_iter, T tol, int quiet, T *out3) {                          \
        return cg_impl<T>(b3, x03, n1, n2, n3, ng, nproj, nrows, ncols, angles, gammas, max_iter, tol, quiet,    \
                          out3);                                                                                 \
    }                                                                                                             \
    int ref_split_bregman##S(const T *yT3, const T *x03, int64_t n1, int64_t n2, int64_t n3, int ng,             \
                             const int64_t *nproj, const int64_t *nrows, const int64_t *ncols, const T *angles,  \
                             const T *gammas, T lambda, T mu, int64_t outer, int64_t inner, T tol, T xtol,       \
                             int quiet, T *out3) {                                                               \
        return sb_impl<T>(yT3, x03, n1, n2, n3, ng, nproj, nrows, ncols, angles, gammas, lambda, mu, outer,      \
                          inner, tol, xtol, quiet, out3);                                                        \
    }                                                                                                             \
    int ref_mbir##S(int which, int ng, const T *proj, const int64_t *nproj, const int64_t *nrows,                 \
                    const int64_t *ncols, const T *angles, const T *gammas, int64_t r1, int64_t r2, int64_t r3,  \
                    int64_t max_iters, int64_t inner_iters, double sigma, double p, double lambda, double mu,    \
                    double tol, double xtol, int quiet, T *out3) {                                               \
        return mbir_impl<T>(which, ng, proj, nproj, nrows, ncols, angles, gammas, r1, r2, r3, max_iters,         \
                            inner_iters, sigma, p, lambda, mu, tol, xtol, quiet, out3);                          \
    }

extern "C" {
REF_DEFINE(float, _f)
REF_DEFINE(double, _d)
}
