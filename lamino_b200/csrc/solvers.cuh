// Solver kernels and host-side solver loops (CG, split-Bregman, NAG, power
// iteration) over packed 3-component volumes [3][n1][n2][n3].
#pragma once

#include <functional>

#include "common.cuh"
#include "fft_engine.cuh"

namespace lamino {

using OpFn = std::function<void(const float *x3, float *y3, cudaStream_t)>;

// Device scalar scratch for FP64 reductions (pinned host mirror).
struct Reducer {
    double *d = nullptr;   // device accumulators
    double *h = nullptr;   // pinned host copy (from a per-thread cache: cudaFreeHost waits for the device)
    int cap = 0;
    DevBuf<double> dbuf;
    explicit Reducer(int n = 16);
    ~Reducer();
    Reducer(const Reducer &) = delete;
    Reducer &operator=(const Reducer &) = delete;
    void zero(int n, cudaStream_t s);
    void fetch(int n, cudaStream_t s);  // copies and synchronises
};

// ---- vector kernels (n = element count) ----
void vec_lin2(float *out, float a, const float *x, float b, const float *y, int64_t n, cudaStream_t s);
void vec_scale(float *out, float a, const float *x, int64_t n, cudaStream_t s);
// out[slot] += sum (double) x*y
void vec_dot(const float *x, const float *y, int64_t n, double *out, cudaStream_t s);
// out[slot+c] += sum_c (x_c - y_c)^2 per component c of 3 (y may be null)
void vec_sqdist3(const float *x, const float *y, int64_t V, double *out3, cudaStream_t s);
// max element (as double, via ordered-int trick on floats)
void vec_max(const float *x, int64_t n, double *out, cudaStream_t s);

// ---- regularisers / finite differences (one component of dims d) ----
void qggmrf_add(float *g, const float *x, Dims3 d, float sigma, float p, cudaStream_t s);
void grad_u(const float *u, Dims3 d, float *out3, cudaStream_t s);
void divergence(const float *du3, Dims3 d, float *out, cudaStream_t s);
void laplacian_axpy(float *y, float mu, const float *u, Dims3 d, cudaStream_t s);  // y += mu*lap(u)
// rhs_i = yT_i + mu * divergence(d_i - b_i), i = 0..2 (d, b: [3][3][V])
void sb_rhs(const float *yT3, const float *d9, const float *b9, float mu, Dims3 dims, float *rhs3, cudaStream_t s);
// isotropic shrink + Bregman update from grad_u(x_i) computed on the fly
void sb_shrink(const float *x3, float *d9, float *b9, float lam, float mu, Dims3 dims, cudaStream_t s);

// ---- ramp preconditioner (include/precond.h:33-87) ----
struct RampPrecond {
    Dims3 d;
    FftPlan r2c, c2r;
    DevBuf<float2> spec;
    DevBuf<float> filt;  // the filter (2-D path) or the n2 convolution kernels (column path)
    bool cols = false;   // 1-D transforms along n3 and a circulant convolution along n2
    bool blue = false;        // (with cols) the n3 transforms as Bluestein convolutions
    bool blue_fixed = false;  // of length 1458 on the compile-time pipeline (else runtime M)
    DevBuf<float2> chirp, vfwd, vinv, tw;  // Bluestein tables: chirp, kernel spectra, twiddles
    FftLen blue_f{};                       // schedule of the Bluestein length M
    explicit RampPrecond(Dims3 d);
    void apply3(const float *r3, float *z3, cudaStream_t s);  // all 3 components
};

// ---- solver loops (host control flow mirrors the reference) ----
struct CgStats { int iters = 0; double last_res = 0; };

// Buffers, ramp preconditioner (cuFFT plans) and reduction slots of one PCG,
// allocated once per solve so repeated calls (split-Bregman inner solves,
// refinement cycles) allocate and free nothing.
struct CgWork {
    Dims3 d;
    DevBuf<float> r, p, z, Ap, e1, e2;  // e1, e2: refinement residual / correction
    RampPrecond M;
    Reducer red;
    explicit CgWork(Dims3 dd)
        : d(dd), r(3 * dd.size()), p(3 * dd.size()), z(3 * dd.size()), Ap(3 * dd.size()), M(dd), red(4) {}
};

// src/conjgrad.cpp:37-117.  x3 holds x0 on entry and the solution on exit.
CgStats cgsolver(const OpFn &A, const float *y3, float *x3, Dims3 d, int max_iter, float tol, cudaStream_t s);
CgStats cgsolver(const OpFn &A, const float *y3, float *x3, CgWork &w, int max_iter, float tol, cudaStream_t s);

// Mixed-precision PCG: `refinements` cycles of  r = y - A_hi x  (FP32 operator,
// FP64 reductions), then `inner` PCG iterations on A_lo d = r from d = 0, x += d.
CgStats cgsolver_refined(const OpFn &A_hi, const OpFn &A_lo, const float *y3, float *x3, Dims3 d, int inner,
                         int refinements, float tol, cudaStream_t s);
CgStats cgsolver_refined(const OpFn &A_hi, const OpFn &A_lo, const float *y3, float *x3, CgWork &w, int inner,
                         int refinements, float tol, cudaStream_t s);

// src/bregman.cpp:39-134.  x3 in/out.  With A_lo set, each outer iteration solves
// its linear subproblem as x_old + d, d from PCG on A_lo against the residual of
// A (refinement cycles as cgsolver_refined).
int split_bregman_refined(const OpFn &A, const OpFn &A_lo, int refinements, const float *yT3, float *x3, Dims3 d,
                          float lam, float mu, int outer_max, int inner_max, float tol, float xtol, cudaStream_t s);
int split_bregman(const OpFn &A, const float *yT3, float *x3, Dims3 d, float lam, float mu, int outer_max,
                  int inner_max, float tol, float xtol, cudaStream_t s);

// src/nagopt.cpp:116-209 (vector form); grad and loss are closures.
using GradFn = std::function<void(const float *x3, float *g3, cudaStream_t)>;
// A loss split so that several evaluations share one host read: enqueue(x, acc)
// adds the loss's nterms partial sums of x into device doubles acc[0..nterms)
// (zeroed by the caller) without reading them; value(terms) forms the loss from
// the fetched sums on the host.
struct LossTerms {
    int nterms = 0;
    std::function<void(const float *x3, double *acc, cudaStream_t)> enqueue;
    std::function<double(const double *terms)> value;
};
int nagopt(const GradFn &grad, const LossTerms &loss, float *x3, Dims3 d, int max_iters, float lipschitz, float tol,
           float xtol, int max_inner, cudaStream_t s);

// The same solve advanced one line-search step at a time, so that several
// solves on their own streams can share host synchronisation: enqueue() queues
// a step's work and the asynchronous copy of its reductions; once the stream
// has reached that point (the caller synchronises it), finish() reads them,
// takes the step's decisions and returns whether the solve has ended.
class NagSolve {
  public:
    NagSolve(GradFn grad, LossTerms loss, float *x3, Dims3 d, int max_iters, float lipschitz, float tol, float xtol,
             int max_inner, cudaStream_t s);
    void enqueue();
    bool finish();
    bool done() const { return done_; }
    int iterations() const { return it_; }
    cudaStream_t stream() const { return s_; }

  private:
    GradFn grad_;
    LossTerms loss_;
    float *x_;
    Dims3 d_;
    int max_iters_, max_inner_;
    float tol_, xtol_;
    cudaStream_t s_;
    DevBuf<float> xold_, y_, g_;
    Reducer red_;
    double t_ = 1, tnew_ = 1, xerr_ = 1e300;
    float step_, step_prev_;
    int it_ = 0, inner_ = 0;
    bool done_ = false;
};

// power iteration for ||A|| (src/lipschitz.cpp:31-53, made to work: seeded start, FP64 norms)
double lipschitz(const OpFn &A, Dims3 d, int max_iters, double tol, unsigned long long seed, cudaStream_t s);

}  // namespace lamino
