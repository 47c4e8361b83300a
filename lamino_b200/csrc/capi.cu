// C ABI of lamino_b200 (declared in include/lamino.h).  Every entry point
// converts C++ exceptions into status codes plus a thread-local message, and
// stages host buffers through device memory when it is given host pointers.
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lamino.h"
#include "batch.cuh"
#include "demag.cuh"
#include "server.cuh"

using namespace lamino;

struct lamino_geom_s {
    std::unique_ptr<Geom> g;
};
struct lamino_plan_s {
    std::unique_ptr<NufftPlan> p;
};
struct lamino_normal_s {
    std::unique_ptr<Toeplitz> t;
    DevBuf<float> sx, sy;  // staging for host-pointer calls, kept across calls
    // lamino_normal_apply_many: two input and two output stagings, a copy-in and a
    // copy-out stream, and the events that order them (created on first use)
    DevBuf<float> px[2], py[2];
    cudaStream_t h2d = nullptr, d2h = nullptr;
    cudaEvent_t ev_in[2] = {nullptr, nullptr}, ev_done[2] = {nullptr, nullptr}, ev_out[2] = {nullptr, nullptr};
    cudaEvent_t ev_start = nullptr;
    ~lamino_normal_s() {
        for (int i = 0; i < 2; ++i) {
            if (ev_in[i]) cudaEventDestroy(ev_in[i]);
            if (ev_done[i]) cudaEventDestroy(ev_done[i]);
            if (ev_out[i]) cudaEventDestroy(ev_out[i]);
        }
        if (ev_start) cudaEventDestroy(ev_start);
        if (h2d) cudaStreamDestroy(h2d);
        if (d2h) cudaStreamDestroy(d2h);
    }
};
struct lamino_op_s {
    OpFn fn;
    Dims3 d;
};
struct lamino_server_s {
    std::unique_ptr<Server> s;
};

namespace {
thread_local std::string g_err;

int fail(int code, const char *msg) {
    g_err = msg;
    return code;
}

bool is_device_ptr(const void *p) {
    if (!p) return false;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Input array: device pointer as is, host pointer copied in.
template <typename T>
struct In {
    const T *d = nullptr;
    DevBuf<T> own;
    bool host = false;
    In(const T *p, size_t n, cudaStream_t s) {
        if (!p) throw Error(ERR_ARG, "null input pointer");
        if (is_device_ptr(p)) {
            d = p;
        } else {
            host = true;
            own.alloc(n);
            LAMINO_CUDA(cudaMemcpyAsync(own.p, p, n * sizeof(T), cudaMemcpyHostToDevice, s));
            d = own.p;
        }
    }
};

// Output array: device pointer as is, host pointer filled on finish().
template <typename T>
struct Out {
    T *d = nullptr;
    T *h = nullptr;
    size_t n = 0;
    DevBuf<T> own;
    Out(T *p, size_t count, cudaStream_t s, bool preload = false) : n(count) {
        if (!p) throw Error(ERR_ARG, "null output pointer");
        if (is_device_ptr(p)) {
            d = p;
        } else {
            h = p;
            own.alloc(count);
            d = own.p;
            if (preload) LAMINO_CUDA(cudaMemcpyAsync(own.p, p, n * sizeof(T), cudaMemcpyHostToDevice, s));
        }
    }
    void finish(cudaStream_t s) {
        if (h) LAMINO_CUDA(cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, s));
        if (h) LAMINO_CUDA(cudaStreamSynchronize(s));
    }
};

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

Dims3 dims_of(int64_t n1, int64_t n2, int64_t n3) {
    if (n1 <= 0 || n2 <= 0 || n3 <= 0) throw Error(ERR_ARG, "dims must be positive");
    return Dims3{n1, n2, n3};
}

std::vector<const Geom *> geoms_of(const lamino_geom_t *gs, int n) {
    if (!gs || n <= 0) throw Error(ERR_ARG, "need at least one geometry");
    std::vector<const Geom *> v;
    for (int i = 0; i < n; ++i) {
        if (!gs[i] || !gs[i]->g) throw Error(ERR_ARG, "null geometry handle");
        v.push_back(gs[i]->g.get());
    }
    return v;
}

__global__ void k_points(GeomView g, float *x, float *y, float *z) {
    const uint32_t M = (uint32_t)g.nproj * g.nrows * g.ncols;
    for (uint32_t pid = blockIdx.x * blockDim.x + threadIdx.x; pid < M; pid += gridDim.x * blockDim.x) {
        uint32_t plane = (uint32_t)g.nrows * g.ncols;
        int p = (int)(pid / plane);
        uint32_t r = pid - p * plane;
        int j = (int)(r / g.ncols), k = (int)(r % g.ncols);
        point_xyz(g, p, j, k, x[pid], y[pid], z[pid]);
    }
}

__global__ void k_sub(float *out, const float *a, const float *b, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[i] - b[i];
}
}  // namespace

#define API_BEGIN try {
#define API_END                                                        \
    }                                                                  \
    catch (const Error &e) { return fail(e.code, e.what()); }          \
    catch (const std::bad_alloc &) { return fail(ERR_OOM, "host out of memory"); } \
    catch (const std::exception &e) { return fail(ERR_STATE, e.what()); } \
    return LAMINO_OK;

extern "C" {

const char *lamino_last_error(void) { return g_err.c_str(); }
const char *lamino_version(void) { return "lamino_b200 0.1.0 (sm_100a)"; }

int lamino_geom_create(const float *angles, int64_t nproj, int64_t nrows, int64_t ncols, float gamma,
                       lamino_geom_t *out) {
    API_BEGIN
    if (!angles || !out) throw Error(ERR_ARG, "null argument");
    auto h = std::make_unique<lamino_geom_s>();
    h->g.reset(new Geom(angles, nproj, nrows, ncols, gamma));
    *out = h.release();
    API_END
}

int lamino_geom_points(lamino_geom_t g, float *x, float *y, float *z, void *stream) {
    API_BEGIN
    if (!g) throw Error(ERR_ARG, "null geometry");
    size_t M = (size_t)g->g->npts();
    Out<float> ox(x, M, S(stream)), oy(y, M, S(stream)), oz(z, M, S(stream));
    k_points<<<grid_for(M, 256), 256, 0, S(stream)>>>(g->g->view(), ox.d, oy.d, oz.d);
    LAMINO_LAUNCH("k_points");
    ox.finish(S(stream)); oy.finish(S(stream)); oz.finish(S(stream));
    API_END
}

int lamino_geom_destroy(lamino_geom_t g) {
    API_BEGIN
    delete g;
    API_END
}

int lamino_plan_create(int64_t n1, int64_t n2, int64_t n3, double eps, lamino_plan_t *out) {
    API_BEGIN
    if (!out) throw Error(ERR_ARG, "null argument");
    if (!(eps > 0)) throw Error(ERR_ARG, "eps must be positive");
    auto h = std::make_unique<lamino_plan_s>();
    h->p.reset(new NufftPlan(dims_of(n1, n2, n3), eps));
    *out = h.release();
    API_END
}

int lamino_plan_destroy(lamino_plan_t p) {
    API_BEGIN
    delete p;
    API_END
}

int lamino_plan_set_bins(lamino_plan_t p, int b1, int b2, int b3) {
    API_BEGIN
    if (!p) throw Error(ERR_ARG, "null plan");
    p->p->set_bins(b1, b2, b3);
    API_END
}

int lamino_plan_autotune(lamino_plan_t p, const lamino_geom_t *geoms, int ngeom, int objective, int *bins,
                         double *best_ms, void *stream) {
    API_BEGIN
    if (!p) throw Error(ERR_ARG, "null plan");
    auto gs = geoms_of(geoms, ngeom);
    double ms = p->p->autotune_bins(gs, objective, S(stream));
    if (bins) {
        bins[0] = p->p->bins.b1;
        bins[1] = p->p->bins.b2;
        bins[2] = p->p->bins.b3;
    }
    if (best_ms) *best_ms = ms;
    API_END
}

int lamino_nufft3d2(lamino_plan_t p, lamino_geom_t g, const float *modes, float *c, void *stream) {
    API_BEGIN
    if (!p || !g) throw Error(ERR_ARG, "null handle");
    size_t V = (size_t)p->p->vol.size(), M = (size_t)g->g->npts();
    In<float2> in(reinterpret_cast<const float2 *>(modes), V, S(stream));
    Out<float2> out(reinterpret_cast<float2 *>(c), M, S(stream));
    p->p->type2(*g->g, in.d, out.d, S(stream));
    out.finish(S(stream));
    API_END
}

int lamino_nufft3d1(lamino_plan_t p, lamino_geom_t g, const float *c, float *modes, void *stream) {
    API_BEGIN
    if (!p || !g) throw Error(ERR_ARG, "null handle");
    size_t V = (size_t)p->p->vol.size(), M = (size_t)g->g->npts();
    In<float2> in(reinterpret_cast<const float2 *>(c), M, S(stream));
    Out<float2> out(reinterpret_cast<float2 *>(modes), V, S(stream));
    p->p->type1(*g->g, in.d, out.d, S(stream));
    out.finish(S(stream));
    API_END
}

int lamino_forward(lamino_plan_t p, lamino_geom_t g, const float *m3, float *proj, void *stream) {
    API_BEGIN
    if (!p || !g) throw Error(ERR_ARG, "null handle");
    size_t V = (size_t)p->p->vol.size(), M = (size_t)g->g->npts();
    In<float> in(m3, 3 * V, S(stream));
    Out<float> out(proj, M, S(stream));
    p->p->forward(*g->g, in.d, out.d, S(stream));
    out.finish(S(stream));
    API_END
}

int lamino_adjoint(lamino_plan_t p, lamino_geom_t g, const float *proj, float *m3, void *stream) {
    API_BEGIN
    if (!p || !g) throw Error(ERR_ARG, "null handle");
    size_t V = (size_t)p->p->vol.size(), M = (size_t)g->g->npts();
    In<float> in(proj, M, S(stream));
    Out<float> out(m3, 3 * V, S(stream));
    p->p->adjoint(*g->g, in.d, out.d, false, S(stream));
    out.finish(S(stream));
    API_END
}

int lamino_sysmat(lamino_plan_t p, const lamino_geom_t *geoms, int ngeom, const float *x3, float *y3,
                  void *stream) {
    API_BEGIN
    if (!p) throw Error(ERR_ARG, "null plan");
    auto gs = geoms_of(geoms, ngeom);
    size_t V = (size_t)p->p->vol.size();
    In<float> in(x3, 3 * V, S(stream));
    Out<float> out(y3, 3 * V, S(stream));
    p->p->normal(gs, in.d, out.d, S(stream));
    out.finish(S(stream));
    API_END
}

int lamino_gradient(lamino_plan_t p, lamino_geom_t g, const float *f3, const float *yT3, float *out3,
                    void *stream) {
    API_BEGIN
    if (!p || !g) throw Error(ERR_ARG, "null handle");
    size_t V = (size_t)p->p->vol.size();
    In<float> in(f3, 3 * V, S(stream)), yt(yT3, 3 * V, S(stream));
    Out<float> out(out3, 3 * V, S(stream));
    p->p->normal({g->g.get()}, in.d, out.d, S(stream));
    k_sub<<<grid_for(3 * V, 256), 256, 0, S(stream)>>>(out.d, out.d, yt.d, (int64_t)(3 * V));
    LAMINO_LAUNCH("k_sub");
    out.finish(S(stream));
    API_END
}

int lamino_residual(lamino_plan_t p, lamino_geom_t g, const float *f3, const float *yT3, float yTy, double *res,
                    void *stream) {
    API_BEGIN
    if (!p || !g || !res) throw Error(ERR_ARG, "null argument");
    int64_t V = p->p->vol.size();
    In<float> in(f3, 3 * V, S(stream)), yt(yT3, 3 * V, S(stream));
    DevBuf<float> Ax(3 * V);
    p->p->normal({g->g.get()}, in.d, Ax.p, S(stream));
    Reducer red(6);
    red.zero(6, S(stream));
    for (int i = 0; i < 3; ++i) {
        vec_dot(in.d + i * V, Ax.p + i * V, V, red.d + i, S(stream));
        vec_dot(in.d + i * V, yt.d + i * V, V, red.d + 3 + i, S(stream));
    }
    red.fetch(6, S(stream));
    double e = 0;
    for (int i = 0; i < 3; ++i) e += std::sqrt(red.h[i] - 2.0 * red.h[3 + i] + (double)yTy);
    *res = e;
    API_END
}

int lamino_normal_create(const lamino_geom_t *geoms, int ngeom, int64_t n1, int64_t n2, int64_t n3, int precision,
                         lamino_normal_t *out, void *stream) {
    API_BEGIN
    if (!out) throw Error(ERR_ARG, "null argument");
    auto gs = geoms_of(geoms, ngeom);
    auto h = std::make_unique<lamino_normal_s>();
    h->t.reset(new Toeplitz(gs, dims_of(n1, n2, n3), precision, S(stream)));
    *out = h.release();
    API_END
}

int lamino_normal_apply(lamino_normal_t op, const float *x3, float *y3, void *stream) {
    API_BEGIN
    if (!op) throw Error(ERR_ARG, "null operator");
    if (!x3 || !y3) throw Error(ERR_ARG, "null array");
    const size_t n = 3 * (size_t)op->t->vol.size();
    cudaStream_t s = S(stream);
    const float *xd = x3;
    float *yd = y3;
    const bool xh = !is_device_ptr(x3), yh = !is_device_ptr(y3);
    if (xh) {
        if (op->sx.n != n) op->sx.alloc(n);
        LAMINO_CUDA(cudaMemcpyAsync(op->sx.p, x3, n * 4, cudaMemcpyHostToDevice, s));
        xd = op->sx.p;
    }
    if (yh) {
        if (op->sy.n != n) op->sy.alloc(n);
        yd = op->sy.p;
    }
    op->t->apply(xd, yd, s);
    if (yh) LAMINO_CUDA(cudaMemcpyAsync(y3, yd, n * 4, cudaMemcpyDeviceToHost, s));
    if (xh || yh) LAMINO_CUDA(cudaStreamSynchronize(s));
    API_END
}

int lamino_normal_apply_many(lamino_normal_t op, int count, const float *const *x3s, float *const *y3s,
                             void *stream) {
    API_BEGIN
    if (!op || !x3s || !y3s) throw Error(ERR_ARG, "null argument");
    if (count < 0) throw Error(ERR_ARG, "count must be non-negative");
    const size_t n = 3 * (size_t)op->t->vol.size();
    for (int i = 0; i < count; ++i) {
        if (!x3s[i] || !y3s[i]) throw Error(ERR_ARG, "null array in the batch");
        if (is_device_ptr(x3s[i]) || is_device_ptr(y3s[i]))
            throw Error(ERR_ARG, "lamino_normal_apply_many takes host buffers (use lamino_normal_apply on device data)");
    }
    if (count == 0) return 0;
    cudaStream_t s = S(stream);
    if (!op->h2d) {
        LAMINO_CUDA(cudaStreamCreateWithFlags(&op->h2d, cudaStreamNonBlocking));
        LAMINO_CUDA(cudaStreamCreateWithFlags(&op->d2h, cudaStreamNonBlocking));
        for (int i = 0; i < 2; ++i) {
            LAMINO_CUDA(cudaEventCreateWithFlags(&op->ev_in[i], cudaEventDisableTiming));
            LAMINO_CUDA(cudaEventCreateWithFlags(&op->ev_done[i], cudaEventDisableTiming));
            LAMINO_CUDA(cudaEventCreateWithFlags(&op->ev_out[i], cudaEventDisableTiming));
        }
        LAMINO_CUDA(cudaEventCreateWithFlags(&op->ev_start, cudaEventDisableTiming));
    }
    const int nb = count > 1 ? 2 : 1;
    for (int b = 0; b < nb; ++b) {
        if (op->px[b].n != n) op->px[b].alloc(n);
        if (op->py[b].n != n) op->py[b].alloc(n);
    }
    // the copy streams start after the work already queued on the caller's stream
    LAMINO_CUDA(cudaEventRecord(op->ev_start, s));
    LAMINO_CUDA(cudaStreamWaitEvent(op->h2d, op->ev_start, 0));
    LAMINO_CUDA(cudaStreamWaitEvent(op->d2h, op->ev_start, 0));
    for (int i = 0; i < count; ++i) {
        const int b = i % nb;
        // input b is free once apply i - 2 finished reading it
        if (i >= nb) LAMINO_CUDA(cudaStreamWaitEvent(op->h2d, op->ev_done[b], 0));
        LAMINO_CUDA(cudaMemcpyAsync(op->px[b].p, x3s[i], n * 4, cudaMemcpyHostToDevice, op->h2d));
        LAMINO_CUDA(cudaEventRecord(op->ev_in[b], op->h2d));
        LAMINO_CUDA(cudaStreamWaitEvent(s, op->ev_in[b], 0));
        // output b is free once the copy-out of result i - 2 finished
        if (i >= nb) LAMINO_CUDA(cudaStreamWaitEvent(s, op->ev_out[b], 0));
        op->t->apply(op->px[b].p, op->py[b].p, s);
        LAMINO_CUDA(cudaEventRecord(op->ev_done[b], s));
        LAMINO_CUDA(cudaStreamWaitEvent(op->d2h, op->ev_done[b], 0));
        LAMINO_CUDA(cudaMemcpyAsync(y3s[i], op->py[b].p, n * 4, cudaMemcpyDeviceToHost, op->d2h));
        LAMINO_CUDA(cudaEventRecord(op->ev_out[b], op->d2h));
    }
    // join both copy streams into the caller's stream, then wait for all of it
    LAMINO_CUDA(cudaStreamWaitEvent(s, op->ev_out[(count - 1) % nb], 0));
    LAMINO_CUDA(cudaStreamWaitEvent(s, op->ev_in[(count - 1) % nb], 0));
    LAMINO_CUDA(cudaStreamSynchronize(s));
    API_END
}

int lamino_normal_profile(lamino_normal_t op, int enable, int max_applies) {
    API_BEGIN
    if (!op) throw Error(ERR_ARG, "null operator");
    if (enable && max_applies <= 0) throw Error(ERR_ARG, "max_applies must be positive");
    op->t->set_profiling(enable != 0, max_applies);
    API_END
}

int lamino_normal_stage_times(lamino_normal_t op, int *nstages, double *ms, int64_t *bytes, int *napplies,
                              int *kernels_per_apply) {
    API_BEGIN
    if (!op || !nstages) throw Error(ERR_ARG, "null argument");
    *nstages = Toeplitz::NSTAGE;
    double t[Toeplitz::NSTAGE];
    int64_t b[Toeplitz::NSTAGE];
    int na = op->t->stage_times(t);
    op->t->stage_bytes(b);
    for (int k = 0; k < Toeplitz::NSTAGE; ++k) {
        if (ms) ms[k] = t[k];
        if (bytes) bytes[k] = b[k];
    }
    if (napplies) *napplies = na;
    if (kernels_per_apply) *kernels_per_apply = Toeplitz::kernels_per_apply();
    API_END
}

int lamino_normal_info(lamino_normal_t op, int64_t *L, int64_t *bytes) {
    API_BEGIN
    if (!op) throw Error(ERR_ARG, "null operator");
    const Toeplitz &t = *op->t;
    if (L) { L[0] = t.L1; L[1] = t.L2; L[2] = t.L3; }
    if (bytes) *bytes = (int64_t)t.device_bytes();
    API_END
}

int lamino_normal_quadforms(lamino_normal_t op, const lamino_normal_t *parts, int nparts, const float *x3,
                            double *out, void *stream) {
    API_BEGIN
    if (!op || !parts || nparts <= 0 || !out) throw Error(ERR_ARG, "null argument");
    std::vector<const Toeplitz *> ps;
    for (int i = 0; i < nparts; ++i) {
        if (!parts[i]) throw Error(ERR_ARG, "null operator");
        ps.push_back(parts[i]->t.get());
    }
    cudaStream_t s = S(stream);
    In<float> in(x3, (size_t)(3 * op->t->vol.size()), s);
    DevBuf<double> acc((size_t)(3 * nparts));
    LAMINO_CUDA(cudaMemsetAsync(acc.p, 0, acc.bytes(), s));
    op->t->quadforms(in.d, ps, acc.p, s);
    LAMINO_CUDA(cudaMemcpyAsync(out, acc.p, acc.bytes(), cudaMemcpyDeviceToHost, s));
    LAMINO_CUDA(cudaStreamSynchronize(s));
    API_END
}

int lamino_normal_autotune(lamino_normal_t op, int *rows, int *kb, double *best_ms, void *stream) {
    API_BEGIN
    if (!op) throw Error(ERR_ARG, "null operator");
    double ms = op->t->autotune(S(stream));
    if (rows) *rows = op->t->rows1;
    if (kb) *kb = op->t->kb2;
    if (best_ms) *best_ms = ms;
    API_END
}

int lamino_normal_destroy(lamino_normal_t op) {
    API_BEGIN
    delete op;
    API_END
}

int lamino_qggmrf(float *g, const float *x, int64_t n1, int64_t n2, int64_t n3, float sigma, float p,
                  void *stream) {
    API_BEGIN
    Dims3 d = dims_of(n1, n2, n3);
    In<float> xi(x, d.size(), S(stream));
    Out<float> go(g, d.size(), S(stream), true);
    qggmrf_add(go.d, xi.d, d, sigma, p, S(stream));
    go.finish(S(stream));
    API_END
}

int lamino_grad_u(const float *u, int64_t n1, int64_t n2, int64_t n3, float *out3, void *stream) {
    API_BEGIN
    Dims3 d = dims_of(n1, n2, n3);
    In<float> ui(u, d.size(), S(stream));
    Out<float> o(out3, 3 * d.size(), S(stream));
    grad_u(ui.d, d, o.d, S(stream));
    o.finish(S(stream));
    API_END
}

int lamino_divergence(const float *du3, int64_t n1, int64_t n2, int64_t n3, float *out, void *stream) {
    API_BEGIN
    Dims3 d = dims_of(n1, n2, n3);
    In<float> di(du3, 3 * d.size(), S(stream));
    Out<float> o(out, d.size(), S(stream));
    divergence(di.d, d, o.d, S(stream));
    o.finish(S(stream));
    API_END
}

int lamino_demag(const float *m3, int64_t n1, int64_t n2, int64_t n3, float *h3, void *stream) {
    API_BEGIN
    Dims3 d = dims_of(n1, n2, n3);
    In<float> mi(m3, (size_t)(3 * d.size()), S(stream));
    Out<float> o(h3, (size_t)(3 * d.size()), S(stream));
    demag(mi.d, d, o.d, S(stream));
    o.finish(S(stream));
    API_END
}

int lamino_laplacian(const float *u, int64_t n1, int64_t n2, int64_t n3, float *out, void *stream) {
    API_BEGIN
    Dims3 d = dims_of(n1, n2, n3);
    In<float> ui(u, d.size(), S(stream));
    Out<float> o(out, d.size(), S(stream));
    // laplacian_axpy works on 3 components; run it on a 3-slot scratch
    DevBuf<float> u3(3 * d.size()), y3(3 * d.size());
    LAMINO_CUDA(cudaMemsetAsync(u3.p, 0, u3.bytes(), S(stream)));
    LAMINO_CUDA(cudaMemcpyAsync(u3.p, ui.d, d.size() * 4, cudaMemcpyDeviceToDevice, S(stream)));
    LAMINO_CUDA(cudaMemsetAsync(y3.p, 0, y3.bytes(), S(stream)));
    laplacian_axpy(y3.p, 1.0f, u3.p, d, S(stream));
    LAMINO_CUDA(cudaMemcpyAsync(o.d, y3.p, d.size() * 4, cudaMemcpyDeviceToDevice, S(stream)));
    o.finish(S(stream));
    LAMINO_CUDA(cudaStreamSynchronize(S(stream)));
    API_END
}

int lamino_ramp_precond(const float *r3, int64_t n1, int64_t n2, int64_t n3, float *z3, void *stream) {
    API_BEGIN
    Dims3 d = dims_of(n1, n2, n3);
    In<float> ri(r3, 3 * d.size(), S(stream));
    Out<float> o(z3, 3 * d.size(), S(stream));
    RampPrecond M(d);
    M.apply3(ri.d, o.d, S(stream));
    o.finish(S(stream));
    LAMINO_CUDA(cudaStreamSynchronize(S(stream)));
    API_END
}

int lamino_op_from_normal(lamino_normal_t n, lamino_op_t *out) {
    API_BEGIN
    if (!n || !out) throw Error(ERR_ARG, "null argument");
    auto h = std::make_unique<lamino_op_s>();
    Toeplitz *t = n->t.get();
    h->fn = [t](const float *x, float *y, cudaStream_t s) { t->apply(x, y, s); };
    h->d = t->vol;
    *out = h.release();
    API_END
}

int lamino_op_from_plan(lamino_plan_t p, const lamino_geom_t *geoms, int ngeom, lamino_op_t *out) {
    API_BEGIN
    if (!p || !out) throw Error(ERR_ARG, "null argument");
    auto gs = geoms_of(geoms, ngeom);
    auto h = std::make_unique<lamino_op_s>();
    NufftPlan *pl = p->p.get();
    h->fn = [pl, gs](const float *x, float *y, cudaStream_t s) { pl->normal(gs, x, y, s); };
    h->d = pl->vol;
    *out = h.release();
    API_END
}

int lamino_op_apply(lamino_op_t op, const float *x3, float *y3, void *stream) {
    API_BEGIN
    if (!op) throw Error(ERR_ARG, "null operator");
    size_t V = (size_t)op->d.size();
    In<float> in(x3, 3 * V, S(stream));
    Out<float> out(y3, 3 * V, S(stream));
    op->fn(in.d, out.d, S(stream));
    out.finish(S(stream));
    API_END
}

int lamino_op_destroy(lamino_op_t op) {
    API_BEGIN
    delete op;
    API_END
}

int lamino_cgsolver(lamino_op_t A, const float *y3, float *x3, int64_t n1, int64_t n2, int64_t n3, int max_iter,
                    float tol, int *iters, void *stream) {
    API_BEGIN
    if (!A) throw Error(ERR_ARG, "null operator");
    Dims3 d = dims_of(n1, n2, n3);
    In<float> yi(y3, 3 * d.size(), S(stream));
    Out<float> xo(x3, 3 * d.size(), S(stream), true);
    CgStats st = cgsolver(A->fn, yi.d, xo.d, d, max_iter, tol, S(stream));
    if (iters) *iters = st.iters;
    xo.finish(S(stream));
    LAMINO_CUDA(cudaStreamSynchronize(S(stream)));
    API_END
}

int lamino_split_bregman(lamino_op_t A, const float *yT3, float *x3, int64_t n1, int64_t n2, int64_t n3,
                         float lambda, float mu, int outer_max, int inner_max, float tol, float xtol, int *iters,
                         void *stream) {
    API_BEGIN
    if (!A) throw Error(ERR_ARG, "null operator");
    Dims3 d = dims_of(n1, n2, n3);
    In<float> yi(yT3, 3 * d.size(), S(stream));
    Out<float> xo(x3, 3 * d.size(), S(stream), true);
    int it = split_bregman(A->fn, yi.d, xo.d, d, lambda, mu, outer_max, inner_max, tol, xtol, S(stream));
    if (iters) *iters = it;
    xo.finish(S(stream));
    API_END
}

int lamino_lipschitz(lamino_op_t A, int64_t n1, int64_t n2, int64_t n3, int max_iters, double tol, uint64_t seed,
                     double *L, void *stream) {
    API_BEGIN
    if (!A || !L) throw Error(ERR_ARG, "null argument");
    *L = lipschitz(A->fn, dims_of(n1, n2, n3), max_iters, tol, seed, S(stream));
    API_END
}

void lamino_recon_params_default(lamino_recon_params *p) {
    if (!p) return;
    ReconParams d;
    p->max_iters = d.max_iters;
    p->inner_iters = d.inner_iters;
    p->sigma = d.sigma;
    p->p = d.p;
    p->lambda = d.lambda;
    p->mu = d.mu;
    p->tol = d.tol;
    p->xtol = d.xtol;
    p->pad_factor = d.pad_factor;
    p->op_kind = d.op_kind;
    p->eps = d.eps;
    p->refinements = d.refinements;
    p->use_graphs = d.use_graphs;
    p->autotune = d.autotune;
}

static ReconParams params_of(const lamino_recon_params *params) {
    ReconParams prm;
    prm.max_iters = params->max_iters;
    prm.inner_iters = params->inner_iters;
    prm.sigma = params->sigma;
    prm.p = params->p;
    prm.lambda = params->lambda;
    prm.mu = params->mu;
    prm.tol = params->tol;
    prm.xtol = params->xtol;
    prm.pad_factor = params->pad_factor;
    prm.op_kind = params->op_kind;
    prm.eps = params->eps;
    prm.refinements = params->refinements;
    prm.use_graphs = params->use_graphs;
    prm.autotune = params->autotune;
    if (prm.max_iters < 0 || prm.inner_iters < 0) throw Error(ERR_ARG, "iteration counts must be >= 0");
    if (prm.op_kind < 0 || prm.op_kind > 3) throw Error(ERR_ARG, "op_kind must be 0..3");
    return prm;
}

// A caller on the legacy default stream gets a private non-blocking stream for
// the whole reconstruction (ordered after the caller's earlier default-stream
// work), so the solver iterations can be graph-captured; the call still returns
// only when the result is complete.
struct CallStream {
    cudaStream_t s = nullptr;
    bool owned = false;
    explicit CallStream(void *user) {
        s = S(user);
        if (s) return;
        LAMINO_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        owned = true;
        cudaEvent_t e;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess) {
            cudaEventRecord(e, nullptr);
            cudaStreamWaitEvent(s, e, 0);
            cudaEventDestroy(e);
        }
    }
    ~CallStream() {
        if (owned) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }
};

int lamino_mbir(int method, int nds, const float *const *projs, const int64_t *pdims, const float *const *angles,
                const float *gammas, int64_t r1, int64_t r2, int64_t r3, const lamino_recon_params *params,
                float *out3, void *stream) {
    API_BEGIN
    if (nds <= 0 || !projs || !pdims || !angles || !gammas || !params) throw Error(ERR_ARG, "null argument");
    Dims3 rd = dims_of(r1, r2, r3);
    ReconParams prm = params_of(params);
    CallStream cs(stream);
    std::vector<std::unique_ptr<In<float>>> ins;
    std::vector<Dataset> data;
    for (int i = 0; i < nds; ++i) {
        int64_t np = pdims[3 * i], nr = pdims[3 * i + 1], nc = pdims[3 * i + 2];
        if (np <= 0 || nr <= 0 || nc <= 0) throw Error(ERR_ARG, "projection dims must be positive");
        ins.emplace_back(new In<float>(projs[i], (size_t)(np * nr * nc), cs.s));
        data.push_back(Dataset{ins.back()->d, np, nr, nc, angles[i], gammas[i]});
    }
    Out<float> o(out3, 3 * rd.size(), cs.s);
    mbir(method, data, rd, prm, o.d, cs.s);
    o.finish(cs.s);
    API_END
}

int lamino_mbir_phases(double *setup_s, double *build_s, double *solve_s, int64_t *applies, double *parts) {
    API_BEGIN
    const MbirPhases &p = last_mbir_phases();
    if (setup_s) *setup_s = p.setup_s;
    if (build_s) *build_s = p.build_s;
    if (solve_s) *solve_s = p.solve_s;
    if (applies) *applies = p.applies;
    if (parts) {
        parts[0] = p.plan_s;
        parts[1] = p.adjoint_s;
        parts[2] = p.tune_s;
    }
    API_END
}

int lamino_mbir_footprint(int method, int nds, const int64_t *pdims, int64_t r1, int64_t r2, int64_t r3,
                          const lamino_recon_params *params, int64_t *bytes) {
    API_BEGIN
    if (nds <= 0 || !pdims || !params || !bytes) throw Error(ERR_ARG, "null argument");
    if (method < 1 || method > 3) throw Error(ERR_ARG, "method must be 1, 2 or 3");
    std::vector<std::array<int64_t, 3>> pd;
    for (int i = 0; i < nds; ++i) pd.push_back({pdims[3 * i], pdims[3 * i + 1], pdims[3 * i + 2]});
    *bytes = mbir_footprint(method, pd, dims_of(r1, r2, r3), params_of(params));
    API_END
}

int lamino_mbir3_batch(int nreq, const int *nds, const float *const *projs, const int64_t *pdims,
                       const float *const *angles, const float *gammas, const int64_t *rdims,
                       const lamino_recon_params *params, float *const *out3, int64_t budget, int threads,
                       double *times, int64_t *counts, int64_t *stats) {
    API_BEGIN
    if (nreq < 0) throw Error(ERR_ARG, "negative request count");
    if (nreq > 0 && (!nds || !projs || !pdims || !angles || !gammas || !rdims || !params || !out3))
        throw Error(ERR_ARG, "null argument");
    std::vector<BatchRequest> reqs((size_t)nreq);
    int64_t k = 0;  // running dataset index
    for (int r = 0; r < nreq; ++r) {
        if (nds[r] <= 0) throw Error(ERR_ARG, "every request needs at least one dataset");
        BatchRequest &q = reqs[(size_t)r];
        for (int i = 0; i < nds[r]; ++i, ++k) {
            const int64_t np = pdims[3 * k], nr = pdims[3 * k + 1], nc = pdims[3 * k + 2];
            if (np <= 0 || nr <= 0 || nc <= 0) throw Error(ERR_ARG, "projection dims must be positive");
            if (!projs[k] || !angles[k]) throw Error(ERR_ARG, "null dataset pointer");
            q.projs.push_back(projs[k]);
            q.pdims.push_back({np, nr, nc});
            q.angles.push_back(angles[k]);
            q.gammas.push_back(gammas[k]);
        }
        q.recon = dims_of(rdims[3 * r], rdims[3 * r + 1], rdims[3 * r + 2]);
        q.prm = params_of(&params[r]);
        q.out = out3[r];
    }
    BatchStats st;
    mbir3_batch(reqs, budget, threads, &st);
    for (int r = 0; r < nreq; ++r) {
        if (times) {
            times[2 * r] = reqs[(size_t)r].t_ready;
            times[2 * r + 1] = reqs[(size_t)r].t_done;
        }
        if (counts) {
            counts[2 * r] = reqs[(size_t)r].iterations;
            counts[2 * r + 1] = reqs[(size_t)r].phases.applies;
        }
    }
    if (stats) {
        stats[0] = st.peak_in_use;
        stats[1] = st.peak_live;
        stats[2] = st.steps;
        stats[3] = (int64_t)(st.wall_s * 1e6);
    }
    API_END
}

int lamino_server_create(int64_t budget, int slots, int flags, double dry_run_ms, lamino_server_t *out) {
    API_BEGIN
    if (!out) throw Error(ERR_ARG, "null argument");
    auto h = std::make_unique<lamino_server_s>();
    h->s.reset(new Server(budget, slots, (flags & 1) != 0, dry_run_ms));
    *out = h.release();
    API_END
}

int lamino_server_submit(lamino_server_t srv, int method, int nds, const float *const *projs, const int64_t *pdims,
                         const float *const *angles, const float *gammas, int64_t r1, int64_t r2, int64_t r3,
                         const lamino_recon_params *params, int64_t *id) {
    API_BEGIN
    if (!srv || nds <= 0 || !projs || !pdims || !angles || !gammas || !params || !id)
        throw Error(ERR_ARG, "null argument");
    if (method < 1 || method > 3) throw Error(ERR_ARG, "method must be 1, 2 or 3");
    auto r = std::make_unique<ServeRequest>();
    r->t_submit = Server::now();  // latency counts the input copy below
    r->method = method;
    r->recon = dims_of(r1, r2, r3);
    r->prm = params_of(params);
    for (int i = 0; i < nds; ++i) {
        int64_t np = pdims[3 * i], nr = pdims[3 * i + 1], nc = pdims[3 * i + 2];
        if (np <= 0 || nr <= 0 || nc <= 0) throw Error(ERR_ARG, "projection dims must be positive");
        if (!projs[i] || !angles[i]) throw Error(ERR_ARG, "null dataset pointer");
        size_t m = (size_t)(np * nr * nc);
        r->projs.emplace_back(m);
        if (is_device_ptr(projs[i]))
            LAMINO_CUDA(cudaMemcpy(r->projs.back().data(), projs[i], m * 4, cudaMemcpyDeviceToHost));
        else
            std::memcpy(r->projs.back().data(), projs[i], m * 4);
        r->pdims.push_back({np, nr, nc});
        r->angles.emplace_back(angles[i], angles[i] + np);
        r->gammas.push_back(gammas[i]);
    }
    r->footprint = mbir_footprint(method, r->pdims, r->recon, r->prm);
    Server::Use use(*srv->s);
    *id = srv->s->submit(std::move(r));
    API_END
}

int lamino_server_wait(lamino_server_t srv, int64_t id, double timeout_s, float *out3, double *queue_s,
                       double *run_s, double *latency_s, double *phases) {
    API_BEGIN
    if (!srv) throw Error(ERR_ARG, "null server");
    Server::Use use(*srv->s);
    ServeRequest *r = nullptr;
    if (!srv->s->wait(id, timeout_s, &r)) throw Error(ERR_TIMEOUT, "request not finished within the timeout");
    if (r->status != OK) {
        int code = r->status;
        std::string msg = r->err;
        srv->s->release(id);
        throw Error(code, msg);
    }
    if (out3) std::memcpy(out3, r->result.data(), r->result.size() * 4);
    if (queue_s) *queue_s = r->t_start - r->t_submit;
    if (run_s) *run_s = r->t_done - r->t_start;
    if (latency_s) *latency_s = r->t_done - r->t_submit;
    if (phases) {
        phases[0] = r->phases.setup_s;
        phases[1] = r->phases.build_s;
        phases[2] = r->phases.solve_s;
        phases[3] = (double)r->phases.applies;
        phases[4] = r->phases.plan_s;
        phases[5] = r->phases.adjoint_s;
        phases[6] = r->phases.tune_s;
    }
    srv->s->release(id);
    API_END
}

int lamino_server_stats(lamino_server_t srv, int64_t *st) {
    API_BEGIN
    if (!srv || !st) throw Error(ERR_ARG, "null argument");
    Server::Use use(*srv->s);
    ServerStats x = srv->s->stats();
    int64_t v[10] = {x.submitted, x.completed, x.failed, x.in_use, x.peak_in_use,
                     x.budget, x.active, x.peak_active, x.queued, x.slots};
    std::memcpy(st, v, sizeof(v));
    API_END
}

int lamino_server_destroy(lamino_server_t srv) {
    API_BEGIN
    delete srv;
    API_END
}

// ---------------------------------------------------------------------------
// Allocation-free residual.
//
// Callers that cannot allocate device memory use lamino_residual_noalloc: a
// reconstruction service that overlaps several requests on one GPU evaluates
// this residual (the MBIR3 loss) inside its Nesterov line search, and a
// cudaMalloc/cudaFree there would stall every other request (cudaFree waits
// for the whole device); a caller whose device memory is owned by another
// allocator (a framework's caching allocator that has reserved most of HBM)
// may not be able to obtain fresh device memory at all.  Its scratch -- A f
// (3 volumes) and the six FP64 reduction slots -- lives in the static array
// below, of fixed size on every GPU that loads this library until exit.
// ---------------------------------------------------------------------------

namespace {
constexpr size_t kNoAllocScratchBytes = (size_t)96 << 20;  // 96 MiB
constexpr size_t kNoAllocHeader = 256;                      // 6 doubles, padded to 256 B
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
void *g_noalloc_ptr[kMaxDevices] = {nullptr};
std::mutex g_noalloc_mu;

// Device address of the static scratch for the current device, resolved once
// per device with that device current.
void *noalloc_scratch() {
    int dev = 0;
    LAMINO_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error(ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            throw Error(ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch failed: ") +
                                      cudaGetErrorString(e));
        }
        g_noalloc_ptr[dev] = p;
    }
    return g_noalloc_ptr[dev];
}
}  // namespace

extern "C" int lamino_residual_noalloc(lamino_plan_t p, lamino_geom_t g, const float *f3, const float *yT3,
                                       float yTy, double *res, void *stream) {
    API_BEGIN
    if (!p || !g || !res) throw Error(ERR_ARG, "null argument");
    const int64_t V = p->p->vol.size();
    const size_t need = kNoAllocHeader + (size_t)3 * V * sizeof(float);
    if (need > kNoAllocScratchBytes)
        throw Error(ERR_ARG, "lamino_residual_noalloc: volume of " + std::to_string(V) +
                                 " voxels exceeds the static scratch (at most " +
                                 std::to_string((kNoAllocScratchBytes - kNoAllocHeader) / 12) + " voxels)");
    if (!is_device_ptr(f3) || !is_device_ptr(yT3))
        throw Error(ERR_ARG, "lamino_residual_noalloc needs device pointers for f and yT");
    cudaStream_t s = S(stream);
    unsigned char *base = static_cast<unsigned char *>(noalloc_scratch());
    double *acc = reinterpret_cast<double *>(base);
    float *Ax = reinterpret_cast<float *>(base + kNoAllocHeader);
    LAMINO_CUDA(cudaMemsetAsync(acc, 0, 6 * sizeof(double), s));  // slots keep the last call's sums
    const Geom *gp = g->g.get();
    p->p->normal_ptrs(&gp, 1, f3, Ax, s);
    for (int i = 0; i < 3; ++i) {
        vec_dot(f3 + i * V, Ax + i * V, V, acc + i, s);
        vec_dot(f3 + i * V, yT3 + i * V, V, acc + 3 + i, s);
    }
    double h[6];
    LAMINO_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, s));
    LAMINO_CUDA(cudaStreamSynchronize(s));
    double e = 0;
    for (int i = 0; i < 3; ++i) e += std::sqrt(h[i] - 2.0 * h[3 + i] + (double)yTy);
    *res = e;
    API_END
}

}  // extern "C"
