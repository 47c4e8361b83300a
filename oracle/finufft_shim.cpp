// FINUFFT C-API subset (3-D types 1 and 2) for the checker build of the
// reference's own sources (TEST INFRASTRUCTURE ONLY).  It serves the call sites
// of include/finufft_plan.h:35-129 (makeplan with upsampfac 2, setpts on the
// PolarGrid coordinates, execute, destroy) so that src/projection.cpp and
// src/gradient.cpp run unmodified.
//
// FINUFFT is third-party and absent (version unpinned by the reference).  This
// restates its published method (Barnett, Magland & af Klinteberg, SIAM J. Sci.
// Comput. 41(5), 2019): exponential-of-semicircle kernel
// phi(t) = exp(beta (sqrt(1 - t^2) - 1)), width w = ceil(log10(10 / eps)) (2..16),
// beta = 2.30 w (2.20, 2.26, 2.38 for w = 2, 3, 4), fine grid nf = the smallest
// even 2,3,5-smooth size >= max(2 N, 2 w), deconvolution by the kernel's Fourier
// transform from Gauss-Legendre quadrature.  Arithmetic runs in the plan's
// precision (float plans in float), like FINUFFT's.
//
// Spreading is deterministic: points are bucketed by the first fine-grid plane
// they touch along z (setpts, like FINUFFT's per-call sort), and each OpenMP
// thread owns a slab of planes and applies only the taps that fall in it.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "cpu_fft.hpp"
#include "shim/finufft.h"

namespace {

int64_t next_smooth_even(int64_t n) {
    if (n < 2) n = 2;
    if (n & 1) ++n;
    while (!cfft::smooth235(n)) n += 2;
    return n;
}

// Gauss-Legendre nodes / weights on [-1, 1] (Newton on P_n)
void gauss_legendre(int n, std::vector<double> &t, std::vector<double> &wq) {
    t.resize(n);
    wq.resize(n);
    for (int i = 0; i < n; ++i) {
        double x = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = x;
            for (int k = 2; k <= n; ++k) {
                const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            const double dp = n * (x * p1 - p0) / (x * x - 1.0);
            const double dx = p1 / dp;
            x -= dx;
            if (std::fabs(dx) < 1e-16) break;
        }
        double p0 = 1.0, p1 = x;
        for (int k = 2; k <= n; ++k) {
            const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
            p0 = p1;
            p1 = p2;
        }
        const double dp = n * (x * p1 - p0) / (x * x - 1.0);
        t[i] = x;
        wq[i] = 2.0 / ((1.0 - x * x) * dp * dp);
    }
}

template <class R>
struct Nufft {
    int type = 0, iflag = 0;
    int64_t N[3] = {1, 1, 1};   // modes: x (fastest), y, z
    int64_t nf[3] = {2, 2, 2};
    int w = 7;
    R beta = 16.1;
    std::vector<R> corr[3];     // 1 / phihat(k), centred order
    int64_t M = 0;
    const R *pt[3] = {nullptr, nullptr, nullptr};
    std::vector<uint32_t> order;  // points by first z plane
    std::vector<int64_t> bstart;  // bucket offsets, nf[2] + 1

    int make(int type_, int64_t *n_modes, int iflag_, double eps, double upsampfac) {
        if (type_ != 1 && type_ != 2) return 1;
        if (upsampfac != 2.0) return 1;
        type = type_;
        iflag = iflag_ >= 0 ? 1 : -1;
        w = (int)std::ceil(std::log10(10.0 / eps));
        w = std::max(2, std::min(w, 16));
        double bo = 2.30;
        if (w == 2) bo = 2.20;
        if (w == 3) bo = 2.26;
        if (w == 4) bo = 2.38;
        beta = (R)(bo * w);
        std::vector<double> t, wq;
        gauss_legendre(200, t, wq);
        for (int d = 0; d < 3; ++d) {
            N[d] = n_modes[d];
            nf[d] = next_smooth_even(std::max<int64_t>(2 * N[d], 2 * w));
            corr[d].resize(N[d]);
            for (int64_t i = 0; i < N[d]; ++i) {
                const double k = (double)(i - N[d] / 2);
                double s = 0.0;
                for (size_t q = 0; q < t.size(); ++q) {
                    const double phi = std::exp((double)beta * (std::sqrt(1.0 - t[q] * t[q]) - 1.0));
                    s += wq[q] * phi * std::cos(k * M_PI * w * t[q] / (double)nf[d]);
                }
                corr[d][i] = (R)(1.0 / (0.5 * w * s));
            }
        }
        return 0;
    }

    // start tap l (mod nf) and the w weights for coordinate x on a grid of nf
    inline int64_t taps(R x, int64_t n, R *wt) const {
        const R u = x * (R)n / (R)(2.0 * M_PI);
        const R l0 = std::ceil(u - (R)w / 2);
        for (int t = 0; t < w; ++t) {
            const R a = (R)2 * (l0 + (R)t - u) / (R)w;
            const R s = (R)1 - a * a;
            wt[t] = s > 0 ? (R)std::exp(beta * (std::sqrt(s) - (R)1)) : (R)0;
        }
        int64_t l = (int64_t)l0 % n;
        if (l < 0) l += n;
        return l;
    }

    int setpts(int64_t M_, const R *x, const R *y, const R *z) {
        if (M_ < 0 || M_ > (int64_t)UINT32_MAX) return 1;
        M = M_;
        pt[0] = x;
        pt[1] = y;
        pt[2] = z;
        const int64_t n3 = nf[2];
        std::vector<uint16_t> l3(M);
        bstart.assign(n3 + 1, 0);
        const int nt = cfft::threads();
        std::vector<std::vector<int64_t>> cnt(nt, std::vector<int64_t>(n3, 0));
#pragma omp parallel num_threads(nt)
        {
#ifdef _OPENMP
            const int tid = omp_get_thread_num();
#else
            const int tid = 0;
#endif
            R wt[16];
#pragma omp for schedule(static)
            for (int64_t j = 0; j < M; ++j) {
                const int64_t l = taps(z[j], n3, wt);
                l3[j] = (uint16_t)l;
                ++cnt[tid][l];
            }
        }
        // exclusive offsets per (bucket, thread) so the scatter keeps point order
        std::vector<std::vector<int64_t>> off(nt, std::vector<int64_t>(n3, 0));
        int64_t acc = 0;
        for (int64_t b = 0; b < n3; ++b) {
            bstart[b] = acc;
            for (int t = 0; t < nt; ++t) {
                off[t][b] = acc;
                acc += cnt[t][b];
            }
        }
        bstart[n3] = acc;
        order.resize(M);
#pragma omp parallel num_threads(nt)
        {
#ifdef _OPENMP
            const int tid = omp_get_thread_num();
#else
            const int tid = 0;
#endif
#pragma omp for schedule(static)
            for (int64_t j = 0; j < M; ++j) order[off[tid][l3[j]]++] = (uint32_t)j;
        }
        return 0;
    }

    void spread(const std::complex<R> *c, R *G) const {
        const int64_t n1 = nf[0], n2 = nf[1], n3 = nf[2];
        const int nt = cfft::threads();
        const int64_t nslab = std::max<int64_t>(1, std::min<int64_t>(nt, n3 / w));
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
        for (int64_t s = 0; s < nslab; ++s) {
            const int64_t Z0 = s * n3 / nslab, Z1 = (s + 1) * n3 / nslab;
            const int64_t nstart = std::min<int64_t>(n3, Z1 - Z0 + w - 1);
            R w1[16], w2[16], w3[16];
            int64_t i1s[16];
            for (int64_t q = 0; q < nstart; ++q) {
                const int64_t p = ((Z0 - (w - 1) + q) % n3 + n3) % n3;
                for (int64_t b = bstart[p]; b < bstart[p + 1]; ++b) {
                    const int64_t j = order[b];
                    const int64_t l1 = taps(pt[0][j], n1, w1);
                    const int64_t l2 = taps(pt[1][j], n2, w2);
                    taps(pt[2][j], n3, w3);
                    for (int t = 0; t < w; ++t) i1s[t] = (l1 + t) % n1;
                    const R cr = c[j].real(), ci = c[j].imag();
                    for (int t3 = 0; t3 < w; ++t3) {
                        const int64_t i3 = (p + t3) % n3;
                        if (i3 < Z0 || i3 >= Z1) continue;
                        for (int t2 = 0; t2 < w; ++t2) {
                            const int64_t i2 = (l2 + t2) % n2;
                            const R k23 = w3[t3] * w2[t2];
                            R *row = G + 2 * ((i3 * n2 + i2) * n1);
                            if (l1 + w <= n1) {
                                R *r = row + 2 * l1;
                                for (int t1 = 0; t1 < w; ++t1) {
                                    const R k = k23 * w1[t1];
                                    r[2 * t1] += k * cr;
                                    r[2 * t1 + 1] += k * ci;
                                }
                            } else {
                                for (int t1 = 0; t1 < w; ++t1) {
                                    const R k = k23 * w1[t1];
                                    row[2 * i1s[t1]] += k * cr;
                                    row[2 * i1s[t1] + 1] += k * ci;
                                }
                            }
                        }
                    }
                }
            }
        }
    }

    void interp(const R *G, std::complex<R> *c) const {
        const int64_t n1 = nf[0], n2 = nf[1], n3 = nf[2];
#pragma omp parallel for schedule(static, 4096)
        for (int64_t b = 0; b < M; ++b) {
            const int64_t j = order[b];
            R w1[16], w2[16], w3[16];
            int64_t i1s[16];
            const int64_t l1 = taps(pt[0][j], n1, w1);
            const int64_t l2 = taps(pt[1][j], n2, w2);
            const int64_t l3 = taps(pt[2][j], n3, w3);
            for (int t = 0; t < w; ++t) i1s[t] = (l1 + t) % n1;
            R sr = 0, si = 0;
            for (int t3 = 0; t3 < w; ++t3) {
                const int64_t i3 = (l3 + t3) % n3;
                for (int t2 = 0; t2 < w; ++t2) {
                    const int64_t i2 = (l2 + t2) % n2;
                    const R *row = G + 2 * ((i3 * n2 + i2) * n1);
                    R rr = 0, ri = 0;
                    if (l1 + w <= n1) {
                        const R *r = row + 2 * l1;
                        for (int t1 = 0; t1 < w; ++t1) {
                            rr += w1[t1] * r[2 * t1];
                            ri += w1[t1] * r[2 * t1 + 1];
                        }
                    } else {
                        for (int t1 = 0; t1 < w; ++t1) {
                            rr += w1[t1] * row[2 * i1s[t1]];
                            ri += w1[t1] * row[2 * i1s[t1] + 1];
                        }
                    }
                    const R k23 = w3[t3] * w2[t2];
                    sr += k23 * rr;
                    si += k23 * ri;
                }
            }
            c[j] = std::complex<R>(sr, si);
        }
    }

    int execute(std::complex<R> *c, std::complex<R> *f) const {
        const int64_t n1 = nf[0], n2 = nf[1], n3 = nf[2];
        const int64_t total = n1 * n2 * n3;
        // the fine grid, zeroed by all threads (a serial fill of GBs would dominate small calls)
        std::unique_ptr<std::complex<R>[]> Gbuf(new std::complex<R>[total]);
        std::complex<R> *Gd = Gbuf.get();
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < total; ++i) Gd[i] = std::complex<R>(0, 0);
        struct {
            std::complex<R> *p;
            std::complex<R> *data() const { return p; }
            std::complex<R> &operator[](int64_t i) const { return p[i]; }
        } G{Gd};
        R *Gr = reinterpret_cast<R *>(G.data());
        if (type == 1) {
            spread(c, Gr);
            cfft::fftn(G.data(), {n3, n2, n1}, iflag);
#pragma omp parallel for schedule(static)
            for (int64_t i3 = 0; i3 < N[2]; ++i3) {
                const int64_t g3 = ((i3 - N[2] / 2) % n3 + n3) % n3;
                for (int64_t i2 = 0; i2 < N[1]; ++i2) {
                    const int64_t g2 = ((i2 - N[1] / 2) % n2 + n2) % n2;
                    const R c23 = corr[2][i3] * corr[1][i2];
                    for (int64_t i1 = 0; i1 < N[0]; ++i1) {
                        const int64_t g1 = ((i1 - N[0] / 2) % n1 + n1) % n1;
                        f[(i3 * N[1] + i2) * N[0] + i1] = G[(g3 * n2 + g2) * n1 + g1] * (c23 * corr[0][i1]);
                    }
                }
            }
        } else {
#pragma omp parallel for schedule(static)
            for (int64_t i3 = 0; i3 < N[2]; ++i3) {
                const int64_t g3 = ((i3 - N[2] / 2) % n3 + n3) % n3;
                for (int64_t i2 = 0; i2 < N[1]; ++i2) {
                    const int64_t g2 = ((i2 - N[1] / 2) % n2 + n2) % n2;
                    const R c23 = corr[2][i3] * corr[1][i2];
                    for (int64_t i1 = 0; i1 < N[0]; ++i1) {
                        const int64_t g1 = ((i1 - N[0] / 2) % n1 + n1) % n1;
                        G[(g3 * n2 + g2) * n1 + g1] = f[(i3 * N[1] + i2) * N[0] + i1] * (c23 * corr[0][i1]);
                    }
                }
            }
            cfft::fftn(G.data(), {n3, n2, n1}, iflag);
            interp(Gr, c);
        }
        return 0;
    }
};

}  // namespace

struct oracle_nufft_plan_s {
    Nufft<double> p;
};
struct oracle_nufftf_plan_s {
    Nufft<float> p;
};

extern "C" {

void finufft_default_opts(finufft_opts *o) {
    o->modeord = 0;
    o->debug = 0;
    o->nthreads = 0;
    o->upsampfac = 2.0;
}

int finufft_makeplan(int type, int dim, int64_t *n_modes, int iflag, int ntrans, double eps, finufft_plan *plan,
                     finufft_opts *o) {
    if (dim != 3 || ntrans != 1 || (o && o->modeord != 0)) return 1;
    auto *p = new oracle_nufft_plan_s;
    if (p->p.make(type, n_modes, iflag, eps, o ? o->upsampfac : 2.0)) {
        delete p;
        return 1;
    }
    *plan = p;
    return 0;
}
int finufftf_makeplan(int type, int dim, int64_t *n_modes, int iflag, int ntrans, float eps,
                      finufftf_plan *plan, finufft_opts *o) {
    if (dim != 3 || ntrans != 1 || (o && o->modeord != 0)) return 1;
    auto *p = new oracle_nufftf_plan_s;
    if (p->p.make(type, n_modes, iflag, eps, o ? o->upsampfac : 2.0)) {
        delete p;
        return 1;
    }
    *plan = p;
    return 0;
}
int finufft_setpts(finufft_plan plan, int64_t M, double *x, double *y, double *z, int64_t, double *, double *,
                   double *) {
    return plan->p.setpts(M, x, y, z);
}
int finufftf_setpts(finufftf_plan plan, int64_t M, float *x, float *y, float *z, int64_t, float *, float *,
                    float *) {
    return plan->p.setpts(M, x, y, z);
}
int finufft_execute(finufft_plan plan, finufft_cpx *c, finufft_cpx *f) { return plan->p.execute(c, f); }
int finufftf_execute(finufftf_plan plan, finufftf_cpx *c, finufftf_cpx *f) { return plan->p.execute(c, f); }
int finufft_destroy(finufft_plan plan) {
    delete plan;
    return 0;
}
int finufftf_destroy(finufftf_plan plan) {
    delete plan;
    return 0;
}

}  // extern "C"
