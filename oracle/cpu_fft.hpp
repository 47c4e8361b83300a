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
