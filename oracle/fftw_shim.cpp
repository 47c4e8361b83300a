// FFTW3 API subset over this project's CPU FFT (cpu_fft.hpp), for the checker
// build of the reference's own sources (TEST INFRASTRUCTURE ONLY).  Serves the
// call sites of include/fft.h:35-263: batched 2-D c2c (fft2 / ifft2), batched
// 2-D r2c / c2r (fft2_r2c / fft2_c2r, used by include/precond.h:72-86) and 3-D
// r2c / c2r (fft3_r2c / fft3_c2r).  A plan records its arguments; execute runs
// the transform.  c2r does not modify its input.
#include <complex>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "cpu_fft.hpp"
#include "shim/fftw3.h"

namespace {

enum Kind { C2C, R2C, C2R };

struct PlanBase {
    virtual ~PlanBase() = default;
    virtual void run() = 0;
};

template <class R>
struct PlanT : PlanBase {
    Kind kind;
    std::vector<int64_t> n;  // logical transform dims (last fastest)
    int64_t howmany, idist, odist;
    void *in, *out;
    int sign;
    void run() override;
};

template <class R>
void PlanT<R>::run() {
    using C = std::complex<R>;
    int64_t total = 1;
    for (auto d : n) total *= d;
    const int64_t nl = n.back(), nh = nl / 2 + 1;
    const int64_t rows = total / nl;
    for (int64_t b = 0; b < howmany; ++b) {
        if (kind == C2C) {
            const C *src = reinterpret_cast<const C *>(in) + b * idist;
            C *dst = reinterpret_cast<C *>(out) + b * odist;
            if (src != dst) std::memmove(dst, src, sizeof(C) * total);
            cfft::fftn(dst, n, sign);
        } else if (kind == R2C) {
            const R *src = reinterpret_cast<const R *>(in) + b * idist;
            C *dst = reinterpret_cast<C *>(out) + b * odist;
            std::vector<C> full(total);
            for (int64_t i = 0; i < total; ++i) full[i] = C(src[i], 0);
            cfft::fftn(full.data(), n, -1);
            for (int64_t r = 0; r < rows; ++r)
                for (int64_t k = 0; k < nh; ++k) dst[r * nh + k] = full[r * nl + k];
        } else {  // C2R: inverse along the leading axes on the half spectrum, then Hermitian rows
            const C *src = reinterpret_cast<const C *>(in) + b * idist;
            R *dst = reinterpret_cast<R *>(out) + b * odist;
            std::vector<C> half(src, src + rows * nh);
            int64_t before = 1, after = rows;  // [before][n[a]][after * nh]
            for (size_t a = 0; a + 1 < n.size(); ++a) {
                after /= n[a];
                cfft::fft_axis(half.data(), before, n[a], after * nh, +1);
                before *= n[a];
            }
            cfft::Plan1<R> plan((int)nl);
            std::vector<C> work(plan.work_size()), line(nl);
            for (int64_t r = 0; r < rows; ++r) {
                const C *h = half.data() + r * nh;
                for (int64_t k = 0; k < nh; ++k) line[k] = h[k];
                for (int64_t k = nh; k < nl; ++k) line[k] = std::conj(h[nl - k]);
                plan.exec(line.data(), +1, work.data());
                for (int64_t j = 0; j < nl; ++j) dst[r * nl + j] = line[j].real();
            }
        }
    }
}

template <class R>
PlanBase *make(Kind kind, int rank, const int *n, int howmany, void *in, const int *inembed, int istride,
               int idist, void *out, const int *onembed, int ostride, int odist, int sign) {
    if (inembed || onembed || istride != 1 || ostride != 1 || rank < 1)
        throw std::invalid_argument("fftw shim: only dense unit-stride layouts are supported");
    auto *p = new PlanT<R>;
    p->kind = kind;
    p->n.assign(n, n + rank);
    p->howmany = howmany;
    p->idist = idist;
    p->odist = odist;
    p->in = in;
    p->out = out;
    p->sign = sign;
    return p;
}

}  // namespace

struct oracle_fft_plan_s {
    PlanBase *impl;
};

static oracle_fft_plan_s *wrap(PlanBase *p) { return new oracle_fft_plan_s{p}; }

extern "C" {

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed,
                             int istride, int idist, fftw_complex *out, const int *onembed, int ostride,
                             int odist, int sign, unsigned) {
    return wrap(make<double>(C2C, rank, n, howmany, in, inembed, istride, idist, out, onembed, ostride, odist, sign));
}
fftwf_plan fftwf_plan_many_dft(int rank, const int *n, int howmany, fftwf_complex *in, const int *inembed,
                               int istride, int idist, fftwf_complex *out, const int *onembed, int ostride,
                               int odist, int sign, unsigned) {
    return wrap(make<float>(C2C, rank, n, howmany, in, inembed, istride, idist, out, onembed, ostride, odist, sign));
}
fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany, double *in, const int *inembed,
                                 int istride, int idist, fftw_complex *out, const int *onembed, int ostride,
                                 int odist, unsigned) {
    return wrap(make<double>(R2C, rank, n, howmany, in, inembed, istride, idist, out, onembed, ostride, odist, -1));
}
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int *n, int howmany, float *in, const int *inembed,
                                   int istride, int idist, fftwf_complex *out, const int *onembed, int ostride,
                                   int odist, unsigned) {
    return wrap(make<float>(R2C, rank, n, howmany, in, inembed, istride, idist, out, onembed, ostride, odist, -1));
}
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany, fftw_complex *in, const int *inembed,
                                 int istride, int idist, double *out, const int *onembed, int ostride,
                                 int odist, unsigned) {
    return wrap(make<double>(C2R, rank, n, howmany, in, inembed, istride, idist, out, onembed, ostride, odist, +1));
}
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int *n, int howmany, fftwf_complex *in, const int *inembed,
                                   int istride, int idist, float *out, const int *onembed, int ostride,
                                   int odist, unsigned) {
    return wrap(make<float>(C2R, rank, n, howmany, in, inembed, istride, idist, out, onembed, ostride, odist, +1));
}
fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double *in, fftw_complex *out, unsigned) {
    const int n[3] = {n0, n1, n2};
    return wrap(make<double>(R2C, 3, n, 1, in, nullptr, 1, 0, out, nullptr, 1, 0, -1));
}
fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float *in, fftwf_complex *out, unsigned) {
    const int n[3] = {n0, n1, n2};
    return wrap(make<float>(R2C, 3, n, 1, in, nullptr, 1, 0, out, nullptr, 1, 0, -1));
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex *in, double *out, unsigned) {
    const int n[3] = {n0, n1, n2};
    return wrap(make<double>(C2R, 3, n, 1, in, nullptr, 1, 0, out, nullptr, 1, 0, +1));
}
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex *in, float *out, unsigned) {
    const int n[3] = {n0, n1, n2};
    return wrap(make<float>(C2R, 3, n, 1, in, nullptr, 1, 0, out, nullptr, 1, 0, +1));
}
void fftw_execute(const fftw_plan p) { p->impl->run(); }
void fftwf_execute(const fftwf_plan p) { p->impl->run(); }
void fftw_destroy_plan(fftw_plan p) {
    delete p->impl;
    delete p;
}
void fftwf_destroy_plan(fftwf_plan p) {
    delete p->impl;
    delete p;
}

}  // extern "C"
