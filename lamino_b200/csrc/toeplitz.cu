// Toeplitz normal operator for the laminography geometry (sm_100a).
//
// sum_gamma sysmat(x) (src/gradient.cpp:34-89, summed as in src/mbir_sb.cpp:89-97)
// is y_i[k] = sum_k' sum_j c_i c_j (1/(nrows ncols)) Re(sum_pts e^{i (k-k').q}) x_j[k'],
// a 3x3 block convolution whose kernel depends only on d = k - k'.  Because each
// projection's points form a centred planar lattice q = qX a(gamma) + qY b(theta, gamma),
// the lattice sum factorises into two Dirichlet kernels:
//   T_ij[d] = (1/(nr nc)) sum_gamma D_nc(d.a) sum_theta c_i c_j D_nr(d.b),
//   D_n(s) = sin(pi s) / sin(pi s / n),
// which is real and even, so its spectrum on an even embedding grid is real.
// The kernel is evaluated in closed form (FP64 phase reduction, float sinpi),
// never by spreading points, then transformed once; each apply is a zero-padded
// R2C, a 3x3 symmetric multiply with 6 real spectra and a C2R plus crop.
#include <cmath>
#include <vector>

#include "nufft.cuh"
#include "toeplitz.cuh"

namespace lamino {

struct TProj {
    double ct, st;
    double w[6];  // c_i c_j for pairs 00, 11, 22, 01, 02, 12
};
struct TGam {
    double cg, sg, inv_scale;
    int nrows, ncols, p0, np;
};

// D_n(s) = sin(pi s) / sin(pi s / n), with the 0/0 limit n (-1)^{m (n-1)} at s = m n.
__device__ __forceinline__ double dirichlet(double s, int n) {
    double m1 = rint(s);
    double f1 = s - m1;
    double q = s / (double)n;
    double m2 = rint(q);
    double f2 = q - m2;
    long long i1 = (long long)m1, i2 = (long long)m2;
    if (f2 == 0.0) return ((i2 * (long long)(n - 1)) & 1LL) ? -(double)n : (double)n;
    float num = sinpif((float)f1);
    float den = sinpif((float)f2);
    float r = num / den;
    return ((i1 + i2) & 1LL) ? -(double)r : (double)r;
}

// One thread per cell with d_z = m1 in [0, n1); writes T[d] and its mirror T[-d].
__global__ void __launch_bounds__(256) k_toeplitz_kernel(
    float *__restrict__ T, int64_t L1, int64_t L2, int64_t L3, int n1, int n2, int n3,
    const TGam *__restrict__ gams, int ngam, const TProj *__restrict__ projs) {
    const int64_t ny = 2 * n2 - 1, nx = 2 * n3 - 1;
    const int64_t total = (int64_t)n1 * ny * nx;
    const int64_t LS = L1 * L2 * L3;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int dx = (int)(idx % nx) - (n3 - 1);
        int64_t r = idx / nx;
        int dy = (int)(r % ny) - (n2 - 1);
        int dz = (int)(r / ny);
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int gi = 0; gi < ngam; ++gi) {
            const TGam G = gams[gi];
            double Da = dirichlet((double)dx * G.cg - (double)dz * G.sg, G.ncols) * G.inv_scale;
            double u = (double)dx * G.sg + (double)dz * G.cg;
            double part[6] = {0, 0, 0, 0, 0, 0};
            for (int p = 0; p < G.np; ++p) {
                const TProj P = projs[G.p0 + p];
                double Db = dirichlet(P.ct * u - (double)dy * P.st, G.nrows);
#pragma unroll
                for (int q = 0; q < 6; ++q) part[q] = fma(P.w[q], Db, part[q]);
            }
#pragma unroll
            for (int q = 0; q < 6; ++q) acc[q] = fma(Da, part[q], acc[q]);
        }
        int64_t m1 = dz, m2 = dy < 0 ? dy + L2 : dy, m3 = dx < 0 ? dx + L3 : dx;
        int64_t c0 = (m1 * L2 + m2) * L3 + m3;
        int64_t mm1 = (L1 - m1) % L1, mm2 = (L2 - m2) % L2, mm3 = (L3 - m3) % L3;
        int64_t c1 = (mm1 * L2 + mm2) * L3 + mm3;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
            T[q * LS + c0] = (float)acc[q];
            T[q * LS + c1] = (float)acc[q];
        }
    }
}

// K_q = Re(spectrum) * norm
__global__ void k_take_real(const float2 *__restrict__ S, int64_t n, float norm, float *__restrict__ K) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        K[i] = S[i].x * norm;
}

// per-k1-plane max |K| over the 6 spectra -> power-of-two scale; then fp16 store
__global__ void k_plane_scale(const float *__restrict__ K, int64_t L1, int64_t plane, float *__restrict__ scale) {
    int64_t k1 = blockIdx.x;
    float m = 0.f;
    for (int q = 0; q < 6; ++q)
        for (int64_t i = threadIdx.x; i < plane; i += blockDim.x)
            m = fmaxf(m, fabsf(K[(q * L1 + k1) * plane + i]));
    __shared__ float red[256];
    red[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // map the plane maximum to at most 2^14 (well inside fp16's 65504)
        float mx = red[0];
        float sc = 1.f;
        if (mx > 0.f) sc = exp2f(floorf(log2f(mx)) - 14.f);
        scale[k1] = sc;
    }
}

__global__ void k_to_half(const float *__restrict__ K, int64_t L1, int64_t plane, const float *__restrict__ scale,
                          __half *__restrict__ Kh) {
    int64_t n = 6 * L1 * plane;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t k1 = (i / plane) % L1;
        Kh[i] = __float2half_rn(K[i] / scale[k1]);
    }
}

__global__ void k_pad3(const float *__restrict__ x, int n1, int n2, int n3, float *__restrict__ xp, int64_t L2,
                       int64_t L3, int64_t LS) {
    const int comp = blockIdx.y;
    const int64_t V = (int64_t)n1 * n2 * n3;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < V;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i3 = (int)(idx % n3);
        int64_t r = idx / n3;
        int i2 = (int)(r % n2);
        int i1 = (int)(r / n2);
        xp[comp * LS + ((int64_t)i1 * L2 + i2) * L3 + i3] = x[comp * V + idx];
    }
}

__global__ void k_crop3(const float *__restrict__ yp, int n1, int n2, int n3, int64_t L2, int64_t L3, int64_t LS,
                        float *__restrict__ y) {
    const int comp = blockIdx.y;
    const int64_t V = (int64_t)n1 * n2 * n3;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < V;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int i3 = (int)(idx % n3);
        int64_t r = idx / n3;
        int i2 = (int)(r % n2);
        int i1 = (int)(r / n2);
        y[comp * V + idx] = yp[comp * LS + ((int64_t)i1 * L2 + i2) * L3 + i3];
    }
}

__global__ void k_mul_fp32(float2 *__restrict__ X, int64_t S, const float *__restrict__ K) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < S; i += (int64_t)gridDim.x * blockDim.x) {
        float2 a = X[i], b = X[S + i], c = X[2 * S + i];
        float k00 = K[i], k11 = K[S + i], k22 = K[2 * S + i];
        float k01 = K[3 * S + i], k02 = K[4 * S + i], k12 = K[5 * S + i];
        X[i] = make_float2(k00 * a.x + k01 * b.x + k02 * c.x, k00 * a.y + k01 * b.y + k02 * c.y);
        X[S + i] = make_float2(k01 * a.x + k11 * b.x + k12 * c.x, k01 * a.y + k11 * b.y + k12 * c.y);
        X[2 * S + i] = make_float2(k02 * a.x + k12 * b.x + k22 * c.x, k02 * a.y + k12 * b.y + k22 * c.y);
    }
}

__global__ void k_mul_fp16(float2 *__restrict__ X, int64_t S, int64_t plane, const __half *__restrict__ K,
                           const float *__restrict__ scale) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < S; i += (int64_t)gridDim.x * blockDim.x) {
        float sc = scale[i / plane];
        float2 a = X[i], b = X[S + i], c = X[2 * S + i];
        float k00 = __half2float(K[i]) * sc, k11 = __half2float(K[S + i]) * sc, k22 = __half2float(K[2 * S + i]) * sc;
        float k01 = __half2float(K[3 * S + i]) * sc, k02 = __half2float(K[4 * S + i]) * sc,
              k12 = __half2float(K[5 * S + i]) * sc;
        X[i] = make_float2(k00 * a.x + k01 * b.x + k02 * c.x, k00 * a.y + k01 * b.y + k02 * c.y);
        X[S + i] = make_float2(k01 * a.x + k11 * b.x + k12 * c.x, k01 * a.y + k11 * b.y + k12 * c.y);
        X[2 * S + i] = make_float2(k02 * a.x + k12 * b.x + k22 * c.x, k02 * a.y + k12 * b.y + k22 * c.y);
    }
}

static int64_t embed_len(int64_t n) {
    // smallest even 2,3,5-smooth L >= 2n  (L >= 2n-1 suffices for a linear convolution)
    return next_smooth_even(2 * n);
}

Toeplitz::Toeplitz(const std::vector<const Geom *> &gs, Dims3 d, int prec, cudaStream_t s) : vol(d), precision(prec) {
    if (gs.empty()) throw Error(ERR_ARG, "Toeplitz operator needs at least one geometry");
    if (d.n1 <= 0 || d.n2 <= 0 || d.n3 <= 0) throw Error(ERR_ARG, "volume dims must be positive");
    if (prec != PREC_FP32 && prec != PREC_FP16) throw Error(ERR_ARG, "precision must be 0 (fp32) or 1 (fp16)");
    L1 = embed_len(d.n1);
    L2 = embed_len(d.n2);
    L3 = embed_len(d.n3);
    L3h = L3 / 2 + 1;
    if (Lsize() > (int64_t)INT32_MAX) throw Error(ERR_ARG, "volume too large for the Toeplitz embedding");

    // geometry tables in double
    std::vector<TGam> hg;
    std::vector<TProj> hp;
    for (const Geom *g : gs) {
        TGam G;
        double gm = (double)g->gamma;
        G.cg = std::cos(gm);
        G.sg = std::sin(gm);
        G.inv_scale = 1.0 / (double)(g->nrows * g->ncols);
        G.nrows = (int)g->nrows;
        G.ncols = (int)g->ncols;
        G.p0 = (int)hp.size();
        G.np = (int)g->nproj;
        hg.push_back(G);
        for (int64_t i = 0; i < g->nproj; ++i) {
            double th = (double)g->theta[i];
            double c[3] = {std::sin(gm) * std::sin(th), std::cos(th), std::cos(gm) * std::sin(th)};
            TProj P;
            P.ct = std::cos(th);
            P.st = std::sin(th);
            P.w[0] = c[0] * c[0]; P.w[1] = c[1] * c[1]; P.w[2] = c[2] * c[2];
            P.w[3] = c[0] * c[1]; P.w[4] = c[0] * c[2]; P.w[5] = c[1] * c[2];
            hp.push_back(P);
        }
    }
    DevBuf<TGam> dg(hg.size());
    DevBuf<TProj> dp(hp.size());
    LAMINO_CUDA(cudaMemcpyAsync(dg.p, hg.data(), hg.size() * sizeof(TGam), cudaMemcpyHostToDevice, s));
    LAMINO_CUDA(cudaMemcpyAsync(dp.p, hp.data(), hp.size() * sizeof(TProj), cudaMemcpyHostToDevice, s));

    // kernel on the embedding grid, 6 pairs
    DevBuf<float> T(6 * Lsize());
    LAMINO_CUDA(cudaMemsetAsync(T.p, 0, T.bytes(), s));
    int64_t cells = d.n1 * (2 * d.n2 - 1) * (2 * d.n3 - 1);
    k_toeplitz_kernel<<<grid_for(cells, 256, 148LL * 64), 256, 0, s>>>(
        T.p, L1, L2, L3, (int)d.n1, (int)d.n2, (int)d.n3, dg.p, (int)hg.size(), dp.p);
    LAMINO_LAUNCH("k_toeplitz_kernel");

    int n[3] = {(int)L1, (int)L2, (int)L3};
    LAMINO_CUFFT(cufftPlanMany(&r2c.h, 3, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, 1));
    r2c.valid = true;
    LAMINO_CUFFT(cufftPlanMany(&c2r.h, 3, n, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, 1));
    c2r.valid = true;
    LAMINO_CUFFT(cufftSetStream(r2c.h, s));
    LAMINO_CUFFT(cufftSetStream(c2r.h, s));

    xhat.alloc(3 * Ssize());
    K.alloc(6 * Ssize());
    float norm = (float)(1.0 / ((double)L1 * L2 * L3));
    for (int q = 0; q < 6; ++q) {
        LAMINO_CUFFT(cufftExecR2C(r2c.h, T.p + q * Lsize(), (cufftComplex *)xhat.p));
        k_take_real<<<grid_for(Ssize(), 256), 256, 0, s>>>(xhat.p, Ssize(), norm, K.p + q * Ssize());
        LAMINO_LAUNCH("k_take_real");
    }
    if (precision == PREC_FP16) {
        Kh.alloc(6 * Ssize());
        Kscale.alloc(L1);
        k_plane_scale<<<(unsigned)L1, 256, 0, s>>>(K.p, L1, L2 * L3h, Kscale.p);
        LAMINO_LAUNCH("k_plane_scale");
        k_to_half<<<grid_for(6 * Ssize(), 256), 256, 0, s>>>(K.p, L1, L2 * L3h, Kscale.p, Kh.p);
        LAMINO_LAUNCH("k_to_half");
        LAMINO_CUDA(cudaStreamSynchronize(s));
        K.release();
    }
    LAMINO_CUDA(cudaStreamSynchronize(s));
    T.release();
    xpad.alloc(3 * Lsize());
    LAMINO_CUDA(cudaMemsetAsync(xpad.p, 0, xpad.bytes(), s));
    ypad.alloc(3 * Lsize());
    LAMINO_CUDA(cudaStreamSynchronize(s));
}

Toeplitz::~Toeplitz() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
}

void Toeplitz::set_profiling(bool on, int max_applies) {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    ev.clear();
    nprof = 0;
    profiling = on;
    if (on) {
        ev.resize((size_t)max_applies * (NSTAGE + 1));
        for (auto &e : ev) LAMINO_CUDA(cudaEventCreate(&e));
    }
}

int Toeplitz::stage_times(double *ms) {
    for (int k = 0; k < NSTAGE; ++k) ms[k] = 0.0;
    for (int a = 0; a < nprof; ++a) {
        for (int k = 0; k < NSTAGE; ++k) {
            float t = 0.f;
            LAMINO_CUDA(cudaEventSynchronize(ev[a * (NSTAGE + 1) + k + 1]));
            LAMINO_CUDA(cudaEventElapsedTime(&t, ev[a * (NSTAGE + 1) + k], ev[a * (NSTAGE + 1) + k + 1]));
            ms[k] += t;
        }
    }
    return nprof;
}

const char *Toeplitz::stage_name(int i) {
    static const char *names[NSTAGE] = {"pad", "r2c", "multiply", "c2r", "crop"};
    return (i >= 0 && i < NSTAGE) ? names[i] : "";
}

void Toeplitz::stage_bytes(int64_t *b) const {
    const int64_t V = vol.size(), S = Ssize(), L = Lsize();
    const int64_t bk = precision == PREC_FP16 ? 2 : 4;
    b[0] = 3 * V * 4 * 2;                    // read x, write the data box of xpad
    b[1] = 3 * (L * 4 + S * 8);              // one pass: read real grid, write half-spectrum
    b[2] = 3 * S * 8 * 2 + 6 * S * bk;       // read + write 3 spectra, read 6 kernel spectra
    b[3] = 3 * (S * 8 + L * 4);              // one pass: read half-spectrum, write real grid
    b[4] = 3 * V * 4 * 2;                    // read the data box of ypad, write y
}

void Toeplitz::apply(const float *x3, float *y3, cudaStream_t s) {
    const bool prof = profiling && (size_t)(nprof + 1) * (NSTAGE + 1) <= ev.size();
    cudaEvent_t *E = prof ? &ev[(size_t)nprof * (NSTAGE + 1)] : nullptr;
    if (prof) LAMINO_CUDA(cudaEventRecord(E[0], s));
    dim3 g3(grid_for(vol.size(), 256), 3);
    k_pad3<<<g3, 256, 0, s>>>(x3, (int)vol.n1, (int)vol.n2, (int)vol.n3, xpad.p, L2, L3, Lsize());
    LAMINO_LAUNCH("k_pad3");
    if (prof) LAMINO_CUDA(cudaEventRecord(E[1], s));
    LAMINO_CUFFT(cufftSetStream(r2c.h, s));
    LAMINO_CUFFT(cufftSetStream(c2r.h, s));
    for (int c = 0; c < 3; ++c)
        LAMINO_CUFFT(cufftExecR2C(r2c.h, xpad.p + c * Lsize(), (cufftComplex *)(xhat.p + c * Ssize())));
    if (prof) LAMINO_CUDA(cudaEventRecord(E[2], s));
    if (precision == PREC_FP16) {
        k_mul_fp16<<<grid_for(Ssize(), 256), 256, 0, s>>>(xhat.p, Ssize(), L2 * L3h, Kh.p, Kscale.p);
        LAMINO_LAUNCH("k_mul_fp16");
    } else {
        k_mul_fp32<<<grid_for(Ssize(), 256), 256, 0, s>>>(xhat.p, Ssize(), K.p);
        LAMINO_LAUNCH("k_mul_fp32");
    }
    if (prof) LAMINO_CUDA(cudaEventRecord(E[3], s));
    for (int c = 0; c < 3; ++c)
        LAMINO_CUFFT(cufftExecC2R(c2r.h, (cufftComplex *)(xhat.p + c * Ssize()), ypad.p + c * Lsize()));
    if (prof) LAMINO_CUDA(cudaEventRecord(E[4], s));
    dim3 gc(grid_for(vol.size(), 256), 3);
    k_crop3<<<gc, 256, 0, s>>>(ypad.p, (int)vol.n1, (int)vol.n2, (int)vol.n3, L2, L3, Lsize(), y3);
    LAMINO_LAUNCH("k_crop3");
    if (prof) {
        LAMINO_CUDA(cudaEventRecord(E[5], s));
        ++nprof;
    }
}

}  // namespace lamino
