// MBIR drivers on the GPU path: src/mbir_cg.cpp:48-128 (MBIR1, CG),
// src/mbir_sb.cpp:47-114 (MBIR2, split Bregman), src/mbir3.cpp:47-135 (MBIR3,
// NAG + qGGMRF).  Setup, solver and crop keep the reference's order of
// operations and its quirks (different projection padding for MBIR1 vs 2/3,
// yT subtracted once per gamma in the MBIR3 gradient, `mu` passed as the
// Lipschitz constant, per-component square roots in the MBIR3 loss).
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "graph.cuh"
#include <chrono>

#include "mbir.cuh"

namespace lamino {

int64_t pad_dim(int64_t n, float f) {
    int64_t npad = 2 * ((int64_t)((float)n * f) / 2);
    return n + npad;
}

__global__ void k_norm_pad2d(const float *__restrict__ in, int64_t np, int nr, int nc, float mx, int onr, int onc,
                             int d1, int d2, float *__restrict__ out) {
    const int64_t M = np * nr * nc;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x) {
        int k = (int)(i % nc);
        int64_t r = i / nc;
        int j = (int)(r % nr);
        int64_t p = r / nr;
        out[(p * onr + j + d1) * onc + k + d2] = in[i] / mx;
    }
}

void normalize_pad2d(const float *proj, int64_t np, int64_t nr, int64_t nc, float mx, float factor,
                     DevBuf<float> &out, int64_t &onr, int64_t &onc, cudaStream_t s) {
    int64_t p2 = 0, p3 = 0;
    if (!(factor < 1.e-06f)) {
        p2 = 2 * ((int64_t)((float)nr * factor) / 2);
        p3 = 2 * ((int64_t)((float)nc * factor) / 2);
    }
    onr = nr + p2;
    onc = nc + p3;
    const int64_t need = np * onr * onc;
    if ((int64_t)out.n < need) out.alloc(need);  // a buffer from an earlier dataset is reused
    LAMINO_CUDA(cudaMemsetAsync(out.p, 0, need * sizeof(float), s));
    k_norm_pad2d<<<grid_for(np * nr * nc, 256), 256, 0, s>>>(proj, np, (int)nr, (int)nc, mx, (int)onr, (int)onc,
                                                            (int)(p2 / 2), (int)(p3 / 2), out.p);
    LAMINO_LAUNCH("k_norm_pad2d");
}

__global__ void k_crop3d3(const float *__restrict__ in, int f1, int f2, int f3, int t1, int t2, int t3, int o1,
                          int o2, int o3, float *__restrict__ out) {
    const int64_t V = (int64_t)t1 * t2 * t3, VF = (int64_t)f1 * f2 * f3;
    const int c = blockIdx.y;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
        int k = (int)(i % t3);
        int64_t r = i / t3;
        int j = (int)(r % t2);
        int a = (int)(r / t2);
        out[c * V + i] = in[c * VF + ((int64_t)(a + o1) * f2 + j + o2) * f3 + k + o3];
    }
}

void crop3d3(const float *in, Dims3 from, Dims3 to, float *out, cudaStream_t s) {
    dim3 g(grid_for(to.size(), 256), 3);
    k_crop3d3<<<g, 256, 0, s>>>(in, (int)from.n1, (int)from.n2, (int)from.n3, (int)to.n1, (int)to.n2, (int)to.n3,
                                (int)((from.n1 - to.n1) / 2), (int)((from.n2 - to.n2) / 2),
                                (int)((from.n3 - to.n3) / 2), out);
    LAMINO_LAUNCH("k_crop3d3");
}

__global__ void k_axpy_scalar(float *__restrict__ y, float a, const float *__restrict__ x, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] += a * x[i];
}

static Dims3 padded_dims(int method, Dims3 recon, const ReconParams &prm) {
    // volume padding: MBIR1 uses T(PAD-1.0); MBIR2/3 use (T(PAD) - 1) in float
    float vfac = method == 1 ? (float)((double)prm.pad_factor - 1.0) : prm.pad_factor - 1.0f;
    return Dims3{pad_dim(recon.n1, vfac), pad_dim(recon.n2, vfac), pad_dim(recon.n3, vfac)};
}

static float proj_pad_factor(int method, const ReconParams &prm) {
    // projection padding: MBIR1 pads by PAD-1, MBIR2/3 by PAD itself
    return method == 1 ? (float)((double)prm.pad_factor - 1.0) : prm.pad_factor;
}

static int64_t pad2d_len(int64_t n, float factor) {
    return factor < 1.e-06f ? n : n + 2 * ((int64_t)((float)n * factor) / 2);
}

int64_t mbir_footprint(int method, const std::vector<std::array<int64_t, 3>> &proj_dims, Dims3 recon,
                       const ReconParams &prm) {
    const Dims3 od = padded_dims(method, recon, prm);
    const float pf = proj_pad_factor(method, prm);
    const int64_t V = od.size();
    int64_t raw = 0, maxpts = 0;
    for (auto &d : proj_dims) {
        raw += d[0] * d[1] * d[2] * 4;
        maxpts = std::max<int64_t>(maxpts, d[0] * pad2d_len(d[1], pf) * pad2d_len(d[2], pf));
    }
    const int w = es_width(prm.eps);
    const int64_t nf = next_smooth_even(std::max<int64_t>(2 * od.n1, 2 * w)) *
                       next_smooth_even(std::max<int64_t>(2 * od.n2, 2 * w)) *
                       next_smooth_even(std::max<int64_t>(2 * od.n3, 2 * w));
    // setup: raw + padded projections, projection spectra + 2-D FFT work, fine grids + 3-D FFT work
    const int64_t setup = raw + maxpts * 4 + 2 * maxpts * 8 + (6 + 1) * nf * 8 + 3 * V * 4;
    const int64_t L1 = next_smooth_even(2 * od.n1), L2 = next_smooth_even(2 * od.n2), L3 = next_smooth_even(2 * od.n3);
    const int64_t S = L1 * L2 * (L3 / 2 + 1), L = L1 * L2 * L3;
    const int64_t n1p = (od.n1 + 7) / 8 * 8;
    const int64_t kb = prm.op_kind == OP_TOEPLITZ_FP32 ? 4 : (prm.op_kind == OP_TOEPLITZ_FP16 ? 2 : 6);
    const int64_t inter = 3 * od.n1 * od.n2 * (L3 / 2 + 1) * 8 + 3 * L2 * (L3 / 2 + 1) * n1p * 8;
    int64_t op = 6 * S * kb + inter;
    const int64_t build = 6 * L * 4 + 2 * S * 8;  // transient kernel grids + R2C output and work
    if (method == 3) op += (int64_t)proj_dims.size() * (6 * S * 4 + inter);  // per-gamma operators for the loss
    if (prm.op_kind == OP_NUFFT) op = (6 + 1) * nf * 8 + 2 * maxpts * 8;
    const int64_t state = (method == 2 ? 40 : 12) * V * 4 + 3 * V * 4;
    const int64_t solve = op + state + (prm.op_kind == OP_NUFFT ? 0 : build);
    const int64_t peak = std::max(setup, solve + 3 * V * 4 + raw);
    return peak + peak / 4 + (64LL << 20);  // cuFFT work areas and allocator slack
}

static double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

MbirPhases &last_mbir_phases() {
    static thread_local MbirPhases p;
    return p;
}

MbirJob::MbirJob(int method, const std::vector<Dataset> &data, Dims3 recon, const ReconParams &prm, float *out3,
                 cudaStream_t s, cudaStream_t solve_stream)
    : method_(method), data_(data), recon_(recon), prm_(prm), out3_(out3), s_(s), ss_(solve_stream ? solve_stream : s) {
    if (method < 1 || method > 3) throw Error(ERR_ARG, "method must be 1 (CG), 2 (split Bregman) or 3 (NAG)");
    if (data.empty()) throw Error(ERR_ARG, "no datasets");
    od_ = padded_dims(method, recon, prm);
    V_ = od_.size();
    n_ = 3 * V_;
}
MbirJob::~MbirJob() = default;

void MbirJob::prepare() {
    const int method = method_;
    const ReconParams &prm = prm_;
    const std::vector<Dataset> &data = data_;
    cudaStream_t s = s_;
    const Dims3 od = od_;
    const int64_t V = V_, n = n_;
    const float pfac = proj_pad_factor(method, prm);
    const bool graphs = prm.use_graphs != 0;
    t0_ = now_s();

    plan_.reset(new NufftPlan(od, prm.eps));
    t_plan_ = now_s();
    yT_.alloc(n);
    LAMINO_CUDA(cudaMemsetAsync(yT_.p, 0, yT_.bytes(), s));
    Reducer red(8);
    DevBuf<float> y;  // normalised, padded projections of the dataset in hand
    for (const Dataset &ds : data) {
        red.zero(1, s);
        vec_max(ds.proj, ds.nproj * ds.nrows * ds.ncols, red.d, s);
        red.fetch(1, s);
        float mx = (float)red.h[0];
        int64_t nr, nc;
        normalize_pad2d(ds.proj, ds.nproj, ds.nrows, ds.ncols, mx, pfac, y, nr, nc, s);
        geoms_.emplace_back(new Geom(ds.angles, ds.nproj, nr, nc, ds.gamma));
        const double ta = now_s();
        plan_->adjoint(*geoms_.back(), y.p, yT_.p, true, s);
        LAMINO_CUDA(cudaStreamSynchronize(s));
        t_adj_ += now_s() - ta;
    }
    for (auto &g : geoms_) gptr_.push_back(g.get());

    t_setup_ = now_s();

    // normal operator sum_gamma sysmat; MBIR3 also needs one operator per gamma
    // for its loss, and then the sum is formed from their spectra
    const bool mixed = prm.op_kind == OP_TOEPLITZ_MIXED;
    if (prm.op_kind == OP_NUFFT) {
        NufftPlan *pl = plan_.get();
        if (prm.autotune) {
            const double tt = now_s();
            pl->autotune_bins(gptr_, 1, s);
            t_tune_ += now_s() - tt;
        }
        A_raw_ = [pl, this](const float *x, float *y, cudaStream_t st) { pl->normal(gptr_, x, y, st); };
        if (method == 3)
            for (const Geom *g : gptr_)
                Ag_.push_back([pl, g](const float *xx, float *yy, cudaStream_t st) { pl->normal({g}, xx, yy, st); });
    } else {
        plan_.reset();  // the fine grids are only needed for the setup adjoints
        int prec = prm.op_kind == OP_TOEPLITZ_FP16 ? PREC_FP16 : (mixed ? PREC_MIXED : PREC_FP32);
        if (method == 3) {
            for (const Geom *g : gptr_) {
                Tg_.emplace_back(new Toeplitz({g}, od, PREC_FP32, s));
                Tg_.back()->drop_work();  // kept for its spectra (loss quadratic forms, the sum)
                parts_.push_back(Tg_.back().get());
            }
            T_.reset(new Toeplitz(parts_, prec, s));
        } else {
            T_.reset(new Toeplitz(gptr_, od, prec, s));
        }
        Toeplitz *tp = T_.get();
        if (prm.autotune) {
            const double tt = now_s();
            tp->autotune(s);
            t_tune_ += now_s() - tt;
        }
        A_raw_ = [tp](const float *x, float *y, cudaStream_t st) { tp->apply(x, y, st, false); };
        if (mixed) A_lo_raw_ = [tp](const float *x, float *y, cudaStream_t st) { tp->apply(x, y, st, true); };
    }
    gA_.reset(new GraphedOp(A_raw_, graphs));
    gA_lo_.reset(new GraphedOp(A_lo_raw_ ? A_lo_raw_ : A_raw_, graphs));

    x_.alloc(n);
    LAMINO_CUDA(cudaMemsetAsync(x_.p, 0, x_.bytes(), s));
    LAMINO_CUDA(cudaStreamSynchronize(s));
    t_build_ = now_s();
    if (method != 3) return;  // s has drained: the solve stream needs no wait

    red.zero(1, s);
    vec_dot(yT_.p, yT_.p, n, red.d, s);
    red.fetch(1, s);
    const double yTy = red.h[0];
    const float ng = (float)gptr_.size();
    // gradient: sum_gamma (sysmat x - yT) + qGGMRF (src/mbir3.cpp:91-103), one graph per input
    gGrad_.reset(new GraphedOp(
        [this, ng, n, V](const float *xx, float *g, cudaStream_t st) {
            A_raw_(xx, g, st);
            k_axpy_scalar<<<grid_for(n, 256), 256, 0, st>>>(g, -ng, yT_.p, n);
            LAMINO_LAUNCH("k_axpy_scalar");
            for (int i = 0; i < 3; ++i) qggmrf_add(g + i * V, xx + i * V, od_, prm_.sigma, prm_.p, st);
        },
        graphs));
    GradFn grad = [this](const float *xx, float *g, cudaStream_t st) {
        (*gGrad_)(xx, g, st);
        ++extra_applies_;
    };
    // loss (src/mbir3.cpp:108-116): sum over gamma and component of
    // sqrt(x_i . S_g x_i - 2 x_i . yT_i + yTy).  Toeplitz forms get every
    // x_i . S_g x_i from one forward half-spectrum of x (Parseval); the NUFFT
    // form applies each S_g.  The terms land in the caller's (zeroed) device
    // slots; the graph is keyed by (input, slot) pointers.
    const int ngi = (int)gptr_.size();
    if (!T_) Sx_.alloc(n);
    gLoss_.reset(new GraphedOp(
        [this, ngi, V](const float *xx, float *slot, cudaStream_t st) {
            double *acc = reinterpret_cast<double *>(slot);
            if (T_) {
                T_->quadforms(xx, parts_, acc, st);
            } else {
                for (int q = 0; q < ngi; ++q) {
                    Ag_[q](xx, Sx_.p, st);
                    for (int i = 0; i < 3; ++i) vec_dot(xx + i * V, Sx_.p + i * V, V, acc + 3 * q + i, st);
                }
            }
            for (int i = 0; i < 3; ++i) vec_dot(xx + i * V, yT_.p + i * V, V, acc + 3 * ngi + i, st);
        },
        graphs));
    LossTerms loss;
    loss.nterms = 3 * ngi + 3;
    loss.enqueue = [this, ngi](const float *xx, double *acc, cudaStream_t st) {
        (*gLoss_)(xx, reinterpret_cast<float *>(acc), st);
        extra_applies_ += T_ ? 0 : ngi;
    };
    loss.value = [ngi, yTy](const double *h) {
        double e = 0.0;
        for (int q = 0; q < ngi; ++q)
            for (int i = 0; i < 3; ++i) e += std::sqrt(h[3 * q + i] - 2.0 * h[3 * ngi + i] + yTy);
        return e;
    };
    float lip = prm.mu;
    if (!(lip > 0.f)) {  // estimate: 30 power iterations of sum_gamma sysmat (qGGMRF curvature neglected)
        lip = (float)lipschitz(gA_->as_fn(), od, 30, 0.0, 12345ULL, s);
        if (!(lip > 0.f)) lip = 1.f;
    }
    if (ss_ != s) {  // the solve stream starts after the work queued on s
        cudaEvent_t ev;
        LAMINO_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        LAMINO_CUDA(cudaEventRecord(ev, s));
        LAMINO_CUDA(cudaStreamWaitEvent(ss_, ev, 0));
        LAMINO_CUDA(cudaEventDestroy(ev));
    }
    nag_.reset(new NagSolve(grad, loss, x_.p, od, prm.max_iters, lip, prm.tol, prm.xtol, prm.inner_iters, ss_));
}

void MbirJob::solve() {
    const ReconParams &prm = prm_;
    cudaStream_t s = ss_;
    const bool mixed = prm.op_kind == OP_TOEPLITZ_MIXED;
    OpFn A = gA_->as_fn();
    OpFn A_lo = mixed ? gA_lo_->as_fn() : OpFn();
    if (method_ == 1) {
        if (mixed) {
            int R = std::max(1, prm.refinements);
            cgsolver_refined(A, A_lo, yT_.p, x_.p, od_, std::max(1, prm.max_iters / R), R, prm.tol, s);
        } else {
            cgsolver(A, yT_.p, x_.p, od_, prm.max_iters, prm.tol, s);
        }
    } else if (method_ == 2) {
        split_bregman_refined(A, A_lo, mixed ? std::max(1, prm.refinements) : 0, yT_.p, x_.p, od_, prm.lambda, prm.mu,
                              prm.max_iters, prm.inner_iters, prm.tol, prm.xtol, s);
    } else {
        while (!nag_->done()) {
            nag_->enqueue();
            LAMINO_CUDA(cudaStreamSynchronize(s));
            nag_->finish();
        }
    }
}

void MbirJob::finish() {
    crop3d3(x_.p, od_, recon_, out3_, ss_);
    LAMINO_CUDA(cudaStreamSynchronize(ss_));
    MbirPhases &ph = last_mbir_phases();
    ph.setup_s = t_setup_ - t0_;
    ph.build_s = t_build_ - t_setup_;
    ph.solve_s = now_s() - t_build_;
    ph.applies = gA_->calls() + gA_lo_->calls() + extra_applies_;
    ph.plan_s = t_plan_ - t0_;
    ph.adjoint_s = t_adj_;
    ph.tune_s = t_tune_;
}

void mbir(int method, const std::vector<Dataset> &data, Dims3 recon, const ReconParams &prm, float *out3,
          cudaStream_t s) {
    MbirJob job(method, data, recon, prm, out3, s);
    job.prepare();
    job.solve();
    job.finish();
}

}  // namespace lamino
