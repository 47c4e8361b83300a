/*
 * C-ABI shim over the reference's own dependency-free sources, compiled where
 * they lie (reference include/ and src/qggmrf.cpp, src/finitediff.cpp,
 * src/nagopt.cpp) into oracle/_ref/libtomocam_ref.so by oracle/Makefile.
 * TEST INFRASTRUCTURE ONLY: it pins the oracle's restatement of the parts of
 * the path that the reference can build without FINUFFT, FFTW, TBB, libtiff
 * or toml++:
 *   PolarGrid coordinates          include/polar_grid.h:44-75
 *   beam_dir_vector                include/projection.h:37-41
 *   pad2d / crop2d / pad3d / crop3d include/padding.h:94-232
 *   fftshift2 / ifftshift2         include/fftutils.h:85-168
 *   dot / norm2 (float accumulation) include/array_ops.h:74-92
 *   transpose                      include/array_ops.h:117-137
 *   grad_u / divergence / laplacian src/finitediff.cpp:8-71, include/bregman.h:34-36
 *   qggmrf                         src/qggmrf.cpp:60-95
 *   nagopt (vector form)           src/nagopt.cpp:116-209
 *   mask_infs_nans / mask_support  include/mask.h:29-91
 * Nothing here is part of the product.
 */
#include <array>
#include <complex>
#include <cstdint>
#include <cstring>
#include <functional>
#include <vector>

#include "array.h"
#include "array_ops.h"
#include "bregman.h"
#include "fftutils.h"
#include "logger.h"
#include "mask.h"
#include "optimize.h"
#include "padding.h"
#include "polar_grid.h"
#include "projection.h"

using tomocam::Array;
using tomocam::dims_t;

namespace {
template <typename T>
Array<T> from_ptr(const T *p, int64_t n1, int64_t n2, int64_t n3) {
    Array<T> a(dims_t(n1, n2, n3));
    std::memcpy(a.begin(), p, sizeof(T) * a.size());
    return a;
}
template <typename T>
void to_ptr(const Array<T> &a, T *p) {
    std::memcpy(p, a.begin(), sizeof(T) * a.size());
}
template <typename T>
void grid_impl(const T *angles, int64_t nproj, int64_t nrows, int64_t ncols, T gamma,
               T *x, T *y, T *z) {
    std::vector<T> th(angles, angles + nproj);
    tomocam::PolarGrid<T> pg(th, nrows, ncols, gamma);
    to_ptr(pg.x, x);
    to_ptr(pg.y, y);
    to_ptr(pg.z, z);
}
}  // namespace

extern "C" {

void ref_polar_grid_f(const float *angles, int64_t nproj, int64_t nrows, int64_t ncols,
                      float gamma, float *x, float *y, float *z) {
    grid_impl<float>(angles, nproj, nrows, ncols, gamma, x, y, z);
}
void ref_polar_grid_d(const double *angles, int64_t nproj, int64_t nrows, int64_t ncols,
                      double gamma, double *x, double *y, double *z) {
    grid_impl<double>(angles, nproj, nrows, ncols, gamma, x, y, z);
}

void ref_beam_dir_f(float gamma, float alpha, float *out) {
    auto v = tomocam::beam_dir_vector<float>(gamma, alpha);
    out[0] = v[0]; out[1] = v[1]; out[2] = v[2];
}

/* pad2d / pad3d output dims: out_dims[3] is written, out may be null (query). */
void ref_pad2d_f(const float *in, int64_t n1, int64_t n2, int64_t n3, float factor,
                 float *out, int64_t *out_dims) {
    auto a = from_ptr(in, n1, n2, n3);
    auto b = tomocam::pad2d(a, factor, tomocam::PadType::SYMMETRIC);
    out_dims[0] = b.dims().n1; out_dims[1] = b.dims().n2; out_dims[2] = b.dims().n3;
    if (out) to_ptr(b, out);
}
void ref_pad3d_f(const float *in, int64_t n1, int64_t n2, int64_t n3, float factor,
                 float *out, int64_t *out_dims) {
    auto a = from_ptr(in, n1, n2, n3);
    auto b = tomocam::pad3d(a, factor, tomocam::PadType::SYMMETRIC);
    out_dims[0] = b.dims().n1; out_dims[1] = b.dims().n2; out_dims[2] = b.dims().n3;
    if (out) to_ptr(b, out);
}
void ref_crop2d_f(const float *in, int64_t n1, int64_t n2, int64_t n3, int64_t m1,
                  int64_t m2, int64_t m3, float *out) {
    auto a = from_ptr(in, n1, n2, n3);
    to_ptr(tomocam::crop2d(a, dims_t(m1, m2, m3), tomocam::PadType::SYMMETRIC), out);
}
void ref_crop3d_f(const float *in, int64_t n1, int64_t n2, int64_t n3, int64_t m1,
                  int64_t m2, int64_t m3, float *out) {
    auto a = from_ptr(in, n1, n2, n3);
    to_ptr(tomocam::crop3d(a, dims_t(m1, m2, m3), tomocam::PadType::SYMMETRIC), out);
}

void ref_fftshift2_c(const float *in, int64_t n1, int64_t n2, int64_t n3, float *out) {
    auto a = from_ptr(reinterpret_cast<const std::complex<float> *>(in), n1, n2, n3);
    to_ptr(tomocam::fft::fftshift2(a), reinterpret_cast<std::complex<float> *>(out));
}
void ref_ifftshift2_c(const float *in, int64_t n1, int64_t n2, int64_t n3, float *out) {
    auto a = from_ptr(reinterpret_cast<const std::complex<float> *>(in), n1, n2, n3);
    to_ptr(tomocam::fft::ifftshift2(a), reinterpret_cast<std::complex<float> *>(out));
}

float ref_dot_f(const float *a, const float *b, int64_t n) {
    auto A = from_ptr(a, 1, 1, n), B = from_ptr(b, 1, 1, n);
    return tomocam::array::dot(A, B);
}
float ref_norm2_f(const float *a, int64_t n) {
    return tomocam::array::norm2(from_ptr(a, 1, 1, n));
}
void ref_transpose_f(const float *in, int64_t n1, int64_t n2, int64_t n3, int64_t a0,
                     int64_t a1, int64_t a2, float *out) {
    auto a = from_ptr(in, n1, n2, n3);
    to_ptr(tomocam::array::transpose(a, {(size_t)a0, (size_t)a1, (size_t)a2}), out);
}

void ref_grad_u_f(const float *u, int64_t n1, int64_t n2, int64_t n3, float *out3) {
    auto g = tomocam::opt::grad_u(from_ptr(u, n1, n2, n3));
    int64_t V = n1 * n2 * n3;
    for (int i = 0; i < 3; ++i) to_ptr(g[i], out3 + i * V);
}
void ref_divergence_f(const float *du3, int64_t n1, int64_t n2, int64_t n3, float *out) {
    int64_t V = n1 * n2 * n3;
    std::array<Array<float>, 3> d = {from_ptr(du3, n1, n2, n3),
                                     from_ptr(du3 + V, n1, n2, n3),
                                     from_ptr(du3 + 2 * V, n1, n2, n3)};
    to_ptr(tomocam::opt::divergence(d), out);
}
void ref_laplacian_f(const float *u, int64_t n1, int64_t n2, int64_t n3, float *out) {
    to_ptr(tomocam::opt::laplacian(from_ptr(u, n1, n2, n3)), out);
}

void ref_qggmrf_f(float *g, const float *x, int64_t n1, int64_t n2, int64_t n3,
                  float sigma, float p) {
    auto G = from_ptr(g, n1, n2, n3);
    tomocam::opt::qggmrf<float>(G, from_ptr(x, n1, n2, n3), sigma, p);
    to_ptr(G, g);
}
void ref_qggmrf_d(double *g, const double *x, int64_t n1, int64_t n2, int64_t n3,
                  double sigma, double p) {
    auto G = from_ptr(g, n1, n2, n3);
    tomocam::opt::qggmrf<double>(G, from_ptr(x, n1, n2, n3), sigma, p);
    to_ptr(G, g);
}

/* nagopt (vector form) driven through C callbacks on packed 3-component arrays. */
typedef void (*ref_grad_cb)(const float *x3, float *g3, void *ctx);
typedef float (*ref_loss_cb)(const float *x3, void *ctx);

void ref_nagopt_f(ref_grad_cb gcb, ref_loss_cb lcb, void *ctx, float *x3, int64_t n1,
                  int64_t n2, int64_t n3, int64_t max_iters, float lipschitz, float tol,
                  float xtol, int64_t max_inner) {
    int64_t V = n1 * n2 * n3;
    using Vec = std::array<Array<float>, 3>;
    auto pack = [V](const Vec &v, std::vector<float> &buf) {
        buf.resize(3 * V);
        for (int i = 0; i < 3; ++i) std::memcpy(buf.data() + i * V, v[i].begin(), sizeof(float) * V);
    };
    std::function<Vec(const Vec &)> grad = [&](const Vec &x) {
        std::vector<float> xb, gb(3 * V);
        pack(x, xb);
        gcb(xb.data(), gb.data(), ctx);
        Vec g = {from_ptr(gb.data(), n1, n2, n3), from_ptr(gb.data() + V, n1, n2, n3),
                 from_ptr(gb.data() + 2 * V, n1, n2, n3)};
        return g;
    };
    std::function<float(const Vec &)> loss = [&](const Vec &x) {
        std::vector<float> xb;
        pack(x, xb);
        return lcb(xb.data(), ctx);
    };
    Vec x = {from_ptr(x3, n1, n2, n3), from_ptr(x3 + V, n1, n2, n3),
             from_ptr(x3 + 2 * V, n1, n2, n3)};
    tomocam::Logger quiet(tomocam::LogMode::SILENT);
    Vec r = tomocam::opt::nagopt<float>(grad, loss, x, (size_t)max_iters, lipschitz, tol,
                                        xtol, (size_t)max_inner, &quiet);
    for (int i = 0; i < 3; ++i) to_ptr(r[i], x3 + i * V);
}


void ref_mask_infs_nans_f(const float *in, int64_t n1, int64_t n2, int64_t n3, float *out) {
    to_ptr(tomocam::mask_infs_nans(from_ptr(in, n1, n2, n3)), out);
}
void ref_mask_support_f(const float *in, int64_t n1, int64_t n2, int64_t n3, int64_t d1, int64_t d2, int64_t d3,
                        const float *theta, float gamma, float *out) {
    std::vector<float> th(theta, theta + n1);
    to_ptr(tomocam::mask_support(from_ptr(in, n1, n2, n3), dims_t(d1, d2, d3), th, gamma), out);
}
}  // extern "C"
