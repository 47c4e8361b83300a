// CPU FFT for the checker libraries (TEST INFRASTRUCTURE ONLY: nothing in the
// product includes this file).  It backs the FFTW-API shim (fftw_shim.cpp) and
// the FINUFFT-API shim (finufft_shim.cpp) that let the reference's own operator
// and solver sources compile unmodified without FFTW3 or FINUFFT.
//
// Algorithm: recursive mixed-radix decimation in time (Cooley-Tukey) with
// radices 4, 2, 3, 5 and a generic odd radix; a length with a prime factor above
// 64 runs as a Bluestein chirp convolution (X_k = c_k sum_j (x_j c_j) conj(c_{k-j}),
// c_j = exp(s i pi j^2 / n)) over a 2,3,5-smooth length >= 2n - 1.  Transforms
// are unnormalised, sign -1 forward and +1 backward, like FFTW's.  Multi-dimensional
// transforms run axis by axis; strided axes are gathered in blocks of lines.
#pragma once

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace cfft {

template <class R>
using cpx = std::complex<R>;

template <class R>
inline cpx<R> cmul(cpx<R> a, cpx<R> b) {
    return cpx<R>(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}
template <class R>
inline cpx<R> cmulc(cpx<R> a, cpx<R> b) {  // a * conj(b)
    return cpx<R>(a.real() * b.real() + a.imag() * b.imag(), a.imag() * b.real() - a.real() * b.imag());
}

inline bool smooth235(int64_t n) {
    for (int p : {2, 3, 5})
        while (n % p == 0) n /= p;
    return n == 1;
}

inline int64_t next_smooth(int64_t n) {
    while (!smooth235(n)) ++n;
    return n;
}

template <class R>
class Plan1 {
  public:
    explicit Plan1(int n) : n_(n) {
        int m = n;
        int big = 0;
        for (int p = 2; (int64_t)p * p <= m; ++p)
            while (m % p == 0) {
                if (p > 64) big = 1;
                m /= p;
            }
        if (m > 64) big = 1;
        if (big) {
            m_ = (int)next_smooth(2 * (int64_t)n - 1);
            sub_.reset(new Plan1<R>(m_));
            chirp_.resize(n);
            for (int64_t j = 0; j < n; ++j) {
                // exp(-i pi j^2 / n), argument reduced exactly modulo 2n
                const int64_t r = (j * j) % (2 * (int64_t)n);
                const double a = -M_PI * (double)r / (double)n;
                chirp_[j] = cpx<R>((R)std::cos(a), (R)std::sin(a));
            }
            // spectra of the kernel conj(c_d) (forward) and c_d (backward), d in (-n, n)
            for (int s = 0; s < 2; ++s) {
                std::vector<cpx<R>> b(m_, cpx<R>(0, 0));
                for (int64_t d = 0; d < n; ++d) {
                    const cpx<R> c = s == 0 ? std::conj(chirp_[d]) : chirp_[d];
                    b[d] = c;
                    if (d) b[m_ - d] = c;
                }
                std::vector<cpx<R>> w(sub_->work_size());
                sub_->exec(b.data(), -1, w.data());
                bk_[s] = std::move(b);
            }
            return;
        }
        m = n;
        while (m % 4 == 0) { fac_.push_back(4); m /= 4; }
        while (m % 2 == 0) { fac_.push_back(2); m /= 2; }
        for (int p = 3; m > 1; p += 2)
            while (m % p == 0) { fac_.push_back(p); m /= p; }
        tw_.resize(n);
        for (int k = 0; k < n; ++k) {
            const double a = -2.0 * M_PI * (double)k / (double)n;
            tw_[k] = cpx<R>((R)std::cos(a), (R)std::sin(a));
        }
    }
    int size() const { return n_; }
    size_t work_size() const { return m_ ? (size_t)2 * m_ + sub_->work_size() : (size_t)n_; }

    // In-place transform of one contiguous line; work holds work_size() values.
    void exec(cpx<R> *x, int sign, cpx<R> *work) const {
        if (n_ == 1) return;
        if (m_) {
            cpx<R> *a = work, *sw = work + 2 * m_;
            for (int j = 0; j < n_; ++j) a[j] = sign < 0 ? cmul(x[j], chirp_[j]) : cmulc(x[j], chirp_[j]);
            for (int j = n_; j < m_; ++j) a[j] = cpx<R>(0, 0);
            sub_->exec(a, -1, sw);
            const cpx<R> *b = bk_[sign < 0 ? 0 : 1].data();
            for (int j = 0; j < m_; ++j) a[j] = cmul(a[j], b[j]);
            sub_->exec(a, +1, sw);
            const R inv = (R)1 / (R)m_;
            for (int k = 0; k < n_; ++k) {
                const cpx<R> v = a[k] * inv;
                x[k] = sign < 0 ? cmul(v, chirp_[k]) : cmulc(v, chirp_[k]);
            }
            return;
        }
        std::memcpy(work, x, sizeof(cpx<R>) * n_);
        rec(work, 1, x, n_, 0, sign);
    }

  private:
    int n_;
    std::vector<int> fac_;
    std::vector<cpx<R>> tw_;  // exp(-2 pi i k / n)
    int m_ = 0;               // Bluestein length (0: direct)
    std::vector<cpx<R>> chirp_;
    std::vector<cpx<R>> bk_[2];
    std::unique_ptr<Plan1<R>> sub_;

    cpx<R> w(int64_t e, int sign) const {  // exp(sign 2 pi i e / n)
        const cpx<R> t = tw_[e % n_];
        return sign < 0 ? t : std::conj(t);
    }

    // out[0..n) = DFT of in[0], in[stride], ..., in[(n-1) stride]
    void rec(const cpx<R> *in, int64_t stride, cpx<R> *out, int n, int fi, int sign) const {
        const int p = fac_[fi], m = n / p;
        if (m == 1) {
            for (int q = 0; q < p; ++q) out[q] = in[q * stride];
        } else {
            for (int q = 0; q < p; ++q) rec(in + q * stride, stride * p, out + q * m, m, fi + 1, sign);
        }
        const int64_t ts = n_ / n;  // W_n = W_N^ts
        const R s = sign < 0 ? (R)-1 : (R)1;
        if (p == 2) {
            for (int k = 0; k < m; ++k) {
                const cpx<R> a = out[k], b = k ? cmul(out[k + m], w(ts * k, sign)) : out[k + m];
                out[k] = a + b;
                out[k + m] = a - b;
            }
        } else if (p == 4) {
            for (int k = 0; k < m; ++k) {
                cpx<R> a0 = out[k], a1 = out[k + m], a2 = out[k + 2 * m], a3 = out[k + 3 * m];
                if (k) {
                    a1 = cmul(a1, w(ts * k, sign));
                    a2 = cmul(a2, w(2 * ts * k, sign));
                    a3 = cmul(a3, w(3 * ts * k, sign));
                }
                const cpx<R> t0 = a0 + a2, t1 = a0 - a2, t2 = a1 + a3, d = a1 - a3;
                const cpx<R> t3(-s * d.imag(), s * d.real());  // sign i (a1 - a3)
                out[k] = t0 + t2;
                out[k + 2 * m] = t0 - t2;
                out[k + m] = t1 + t3;
                out[k + 3 * m] = t1 - t3;
            }
        } else if (p == 3) {
            const R c = (R)-0.5, sn = s * (R)0.86602540378443864676;
            for (int k = 0; k < m; ++k) {
                cpx<R> a0 = out[k], a1 = out[k + m], a2 = out[k + 2 * m];
                if (k) {
                    a1 = cmul(a1, w(ts * k, sign));
                    a2 = cmul(a2, w(2 * ts * k, sign));
                }
                const cpx<R> t = a1 + a2, d = a1 - a2;
                const cpx<R> mm = a0 + t * c;
                const cpx<R> r(-sn * d.imag(), sn * d.real());
                out[k] = a0 + t;
                out[k + m] = mm + r;
                out[k + 2 * m] = mm - r;
            }
        } else {
            std::vector<cpx<R>> t(p), wp(p);
            for (int q = 0; q < p; ++q) wp[q] = w((int64_t)q * (n_ / p), sign);  // W_p^q
            for (int k = 0; k < m; ++k) {
                for (int q = 0; q < p; ++q)
                    t[q] = (k && q) ? cmul(out[k + q * m], w(ts * k * q, sign)) : out[k + q * m];
                for (int r = 0; r < p; ++r) {
                    cpx<R> acc = t[0];
                    int e = 0;
                    for (int q = 1; q < p; ++q) {
                        e += r;
                        if (e >= p) e -= p;
                        acc += cmul(t[q], wp[e]);
                    }
                    out[k + r * m] = acc;
                }
            }
        }
    }
};

// Eight lines at a time, structure of arrays (re[i][lane], im[i][lane]), by the
// Stockham autosort recursion (decimation in frequency): a stage of radix r over
// a sequence of length n with stride s maps x to y with
//   y[q + s (r p + k)] = w_n^{p k} sum_j x[q + s (p + j n / r)] w_r^{j k},
// p < n / r, q < s, then continues on length n / r with stride s r, swapping
// x and y; the result is in natural order.  Radices 4, 2, 3, 5 and any odd
// factor up to 64 (direct DFT); the innermost loop runs over the 8 lines, so
// it vectorises.  Used for lengths without a prime factor above 64.
template <class R>
class BatchPlan {
  public:
    static constexpr int LANES = 8;
    explicit BatchPlan(int n) : n_(n) {
        int m = n;
        while (m % 4 == 0) { rad_.push_back(4); m /= 4; }
        while (m % 2 == 0) { rad_.push_back(2); m /= 2; }
        for (int p = 3; m > 1; p += 2)
            while (m % p == 0) { rad_.push_back(p); m /= p; }
        // per stage twiddles w_len^{p k} (forward sign), p < len / r, k < r
        int len = n;
        for (int r : rad_) {
            const int mm = len / r;
            std::vector<cpx<R>> t((size_t)mm * r);
            for (int p = 0; p < mm; ++p)
                for (int k = 0; k < r; ++k) {
                    const double a = -2.0 * M_PI * (double)((int64_t)p * k % len) / (double)len;
                    t[(size_t)p * r + k] = cpx<R>((R)std::cos(a), (R)std::sin(a));
                }
            tw_.push_back(std::move(t));
            std::vector<cpx<R>> d((size_t)r);
            for (int k = 0; k < r; ++k) {
                const double a = -2.0 * M_PI * (double)k / (double)r;
                d[k] = cpx<R>((R)std::cos(a), (R)std::sin(a));
            }
            dft_.push_back(std::move(d));
            len = mm;
        }
    }
    static bool usable(int n) {
        int m = n;
        for (int p = 2; m > 1 && p <= 64; ++p)
            while (m % p == 0) m /= p;
        return m == 1;
    }
    // x, y: 2 n LANES values each (re block then im block); the result ends in x
    void exec(R *x, R *y, int sign) const {
        R *a = x, *b = y;
        int len = n_, s = 1;
        for (size_t st = 0; st < rad_.size(); ++st) {
            stage(rad_[st], len, s, tw_[st].data(), dft_[st].data(), a, b, sign);
            std::swap(a, b);
            len /= rad_[st];
            s *= rad_[st];
        }
        if (a != x) std::memcpy(x, a, sizeof(R) * 2 * (size_t)n_ * LANES);
    }

  private:
    int n_;
    std::vector<int> rad_;
    std::vector<std::vector<cpx<R>>> tw_, dft_;

    // radix-r butterfly on 8 lanes (b = DFT_r(a)); r in {2, 3, 4} fixed at compile time
    template <int RAD>
    static inline void bfly(R (&ar)[RAD][LANES], R (&ai)[RAD][LANES], R (&br)[RAD][LANES], R (&bi)[RAD][LANES],
                            R sg) {
        if constexpr (RAD == 2) {
            for (int l = 0; l < LANES; ++l) {
                br[0][l] = ar[0][l] + ar[1][l];
                bi[0][l] = ai[0][l] + ai[1][l];
                br[1][l] = ar[0][l] - ar[1][l];
                bi[1][l] = ai[0][l] - ai[1][l];
            }
        } else if constexpr (RAD == 3) {
            const R c = (R)-0.5, sn = sg * (R)0.86602540378443864676;
            for (int l = 0; l < LANES; ++l) {
                const R tr = ar[1][l] + ar[2][l], ti = ai[1][l] + ai[2][l];
                const R dr = ar[1][l] - ar[2][l], di = ai[1][l] - ai[2][l];
                const R mr = ar[0][l] + c * tr, mi = ai[0][l] + c * ti;
                br[0][l] = ar[0][l] + tr;
                bi[0][l] = ai[0][l] + ti;
                br[1][l] = mr + sn * di;  // m -/+ i sn d
                bi[1][l] = mi - sn * dr;
                br[2][l] = mr - sn * di;
                bi[2][l] = mi + sn * dr;
            }
        } else {
            static_assert(RAD == 4, "fixed radices 2, 3, 4");
            for (int l = 0; l < LANES; ++l) {
                const R t0r = ar[0][l] + ar[2][l], t0i = ai[0][l] + ai[2][l];
                const R t1r = ar[0][l] - ar[2][l], t1i = ai[0][l] - ai[2][l];
                const R t2r = ar[1][l] + ar[3][l], t2i = ai[1][l] + ai[3][l];
                const R dr = ar[1][l] - ar[3][l], di = ai[1][l] - ai[3][l];
                const R t3r = sg * di, t3i = -sg * dr;  // -i d (forward), +i d (backward)
                br[0][l] = t0r + t2r;
                bi[0][l] = t0i + t2i;
                br[2][l] = t0r - t2r;
                bi[2][l] = t0i - t2i;
                br[1][l] = t1r + t3r;
                bi[1][l] = t1i + t3i;
                br[3][l] = t1r - t3r;
                bi[3][l] = t1i - t3i;
            }
        }
    }

    template <int RAD>
    void stage_fixed(int len, int s, const cpx<R> *__restrict tw, const R *__restrict x, R *__restrict y,
                     int sign) const {
        const int m = len / RAD;
        const size_t N = (size_t)n_ * LANES;
        const R *__restrict xr = x;
        const R *__restrict xi = x + N;
        R *__restrict yr = y;
        R *__restrict yi = y + N;
        const R sg = sign < 0 ? (R)1 : (R)-1;
        for (int p = 0; p < m; ++p) {
            R wr[RAD], wi[RAD];
            for (int k = 0; k < RAD; ++k) {
                wr[k] = tw[(size_t)p * RAD + k].real();
                wi[k] = sg * tw[(size_t)p * RAD + k].imag();
            }
            for (int q = 0; q < s; ++q) {
                R ar[RAD][LANES], ai[RAD][LANES], br[RAD][LANES], bi[RAD][LANES];
                for (int j = 0; j < RAD; ++j) {
                    const size_t o = ((size_t)q + (size_t)s * (p + (size_t)j * m)) * LANES;
                    for (int l = 0; l < LANES; ++l) {
                        ar[j][l] = xr[o + l];
                        ai[j][l] = xi[o + l];
                    }
                }
                bfly<RAD>(ar, ai, br, bi, sg);
                for (int k = 0; k < RAD; ++k) {
                    const size_t o = ((size_t)q + (size_t)s * ((size_t)RAD * p + k)) * LANES;
                    for (int l = 0; l < LANES; ++l) {
                        yr[o + l] = wr[k] * br[k][l] - wi[k] * bi[k][l];
                        yi[o + l] = wr[k] * bi[k][l] + wi[k] * br[k][l];
                    }
                }
            }
        }
    }

    void stage(int r, int len, int s, const cpx<R> *tw, const cpx<R> *dft, const R *x, R *y, int sign) const {
        if (r == 2) return stage_fixed<2>(len, s, tw, x, y, sign);
        if (r == 3) return stage_fixed<3>(len, s, tw, x, y, sign);
        if (r == 4) return stage_fixed<4>(len, s, tw, x, y, sign);
        // any other odd factor up to 64: direct DFT
        const int m = len / r;
        const size_t N = (size_t)n_ * LANES;
        const R *xr = x, *xi = x + N;
        R *yr = y, *yi = y + N;
        const R sg = sign < 0 ? (R)1 : (R)-1;
        std::vector<R> ar((size_t)r * LANES), ai((size_t)r * LANES);
        for (int p = 0; p < m; ++p)
            for (int q = 0; q < s; ++q) {
                for (int j = 0; j < r; ++j) {
                    const size_t o = ((size_t)q + (size_t)s * (p + (size_t)j * m)) * LANES;
                    for (int l = 0; l < LANES; ++l) {
                        ar[j * LANES + l] = xr[o + l];
                        ai[j * LANES + l] = xi[o + l];
                    }
                }
                for (int k = 0; k < r; ++k) {
                    R br[LANES], bi[LANES];
                    for (int l = 0; l < LANES; ++l) {
                        br[l] = ar[l];
                        bi[l] = ai[l];
                    }
                    int e = 0;
                    for (int j = 1; j < r; ++j) {
                        e += k;
                        if (e >= r) e -= r;
                        const R wr = dft[e].real(), wi = sg * dft[e].imag();
                        for (int l = 0; l < LANES; ++l) {
                            br[l] += wr * ar[j * LANES + l] - wi * ai[j * LANES + l];
                            bi[l] += wr * ai[j * LANES + l] + wi * ar[j * LANES + l];
                        }
                    }
                    const cpx<R> w = tw[(size_t)p * r + k];
                    const R wr = w.real(), wi = sg * w.imag();
                    const size_t o = ((size_t)q + (size_t)s * ((size_t)r * p + k)) * LANES;
                    for (int l = 0; l < LANES; ++l) {
                        yr[o + l] = wr * br[l] - wi * bi[l];
                        yi[o + l] = wr * bi[l] + wi * br[l];
                    }
                }
            }
    }
};

inline int threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

// Transform along the middle axis of data viewed as [outer][n][inner].
template <class R>
void fft_axis(cpx<R> *data, int64_t outer, int64_t n, int64_t inner, int sign) {
    if (n <= 1) return;
    if (BatchPlan<R>::usable((int)n)) {
        // lines in groups of 8: gathered into structure-of-arrays buffers
        constexpr int64_t B = BatchPlan<R>::LANES;
        const BatchPlan<R> plan((int)n);
        const int64_t nblk = (inner + B - 1) / B;
        const int64_t groups = inner == 1 ? (outer + B - 1) / B : outer * nblk;
#pragma omp parallel
        {
            std::vector<R> x(2 * n * B), y(2 * n * B);
            R *xr = x.data(), *xi = x.data() + n * B;
#pragma omp for schedule(static)
            for (int64_t t = 0; t < groups; ++t) {
                // line b of the group: element i at base + b * lstride + i * istride
                cpx<R> *base;
                int64_t nb, lstride, istride;
                if (inner == 1) {
                    base = data + t * B * n;
                    nb = std::min(B, outer - t * B);
                    lstride = n;
                    istride = 1;
                } else {
                    const int64_t o = t / nblk, j0 = (t % nblk) * B;
                    base = data + o * n * inner + j0;
                    nb = std::min(B, inner - j0);
                    lstride = 1;
                    istride = inner;
                }
                for (int64_t i = 0; i < n; ++i)
                    for (int64_t b = 0; b < B; ++b) {
                        const cpx<R> v = b < nb ? base[b * lstride + i * istride] : cpx<R>(0, 0);
                        xr[i * B + b] = v.real();
                        xi[i * B + b] = v.imag();
                    }
                plan.exec(x.data(), y.data(), sign);
                for (int64_t i = 0; i < n; ++i)
                    for (int64_t b = 0; b < nb; ++b) base[b * lstride + i * istride] = cpx<R>(xr[i * B + b], xi[i * B + b]);
            }
        }
        return;
    }
    Plan1<R> plan((int)n);
    const size_t ws = plan.work_size();
    if (inner == 1) {
#pragma omp parallel
        {
            std::vector<cpx<R>> work(ws);
#pragma omp for schedule(static)
            for (int64_t o = 0; o < outer; ++o) plan.exec(data + o * n, sign, work.data());
        }
        return;
    }
    constexpr int64_t B = 16;
    const int64_t nblk = (inner + B - 1) / B;
#pragma omp parallel
    {
        std::vector<cpx<R>> work(ws), buf(B * n);
#pragma omp for schedule(static)
        for (int64_t t = 0; t < outer * nblk; ++t) {
            const int64_t o = t / nblk, j0 = (t % nblk) * B;
            const int64_t nb = std::min(B, inner - j0);
            cpx<R> *base = data + o * n * inner + j0;
            for (int64_t i = 0; i < n; ++i)
                for (int64_t b = 0; b < nb; ++b) buf[b * n + i] = base[i * inner + b];
            for (int64_t b = 0; b < nb; ++b) plan.exec(buf.data() + b * n, sign, work.data());
            for (int64_t i = 0; i < n; ++i)
                for (int64_t b = 0; b < nb; ++b) base[i * inner + b] = buf[b * n + i];
        }
    }
}

// Unnormalised multi-dimensional complex transform of a row-major array (dims[0] slowest).
template <class R>
void fftn(cpx<R> *data, const std::vector<int64_t> &dims, int sign) {
    int64_t total = 1;
    for (auto d : dims) total *= d;
    int64_t inner = total;
    int64_t outer = 1;
    for (size_t a = 0; a < dims.size(); ++a) {
        inner /= dims[a];
        fft_axis(data, outer, dims[a], inner, sign);
        outer *= dims[a];
    }
}

}  // namespace cfft
