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
// never by spreading points, and transformed once (cuFFT, build only).  Each
// apply is five kernels of this file over the zero-padded embedding, with the
// padding never materialised: R2C rows along n3, a pruned FFT along n2, one
// kernel per (k2, k3) pencil doing the n1 transform, the 3x3 multiply with the
// 6 real spectra and the inverse n1 transform in shared memory, then the two
// inverse passes.  Spectra and intermediates stay in digit-reversed position
// order (fft_engine.cuh), so no pass reorders data.
#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "nufft.cuh"
#include "toeplitz.cuh"

namespace lamino {

struct TProj {
    double ct, st;
    float w[6];  // c_i c_j for pairs 00, 11, 22, 01, 02, 12
};
struct TGam {
    double cg, sg, inv_scale;
    double inv_nrows, inv_ncols;
    int nrows, ncols, p0, np;
};

// sin(pi x) for |x| <= 1/2: the Taylor series of sin through the x^11 term
// (truncation error below 6e-8 on the interval), Horner in x^2 in float;
// max relative error 1.7e-7 against double sin (checked on 2e5 points).
__device__ __forceinline__ float sinpi_half(float x) {
    constexpr double P = 3.14159265358979323846;
    constexpr double P2 = P * P;
    constexpr float c1 = (float)P;
    constexpr float c3 = (float)(-P * P2 / 6.0);
    constexpr float c5 = (float)(P * P2 * P2 / 120.0);
    constexpr float c7 = (float)(-P * P2 * P2 * P2 / 5040.0);
    constexpr float c9 = (float)(P * P2 * P2 * P2 * P2 / 362880.0);
    constexpr float c11 = (float)(-P * P2 * P2 * P2 * P2 * P2 / 39916800.0);
    const float x2 = x * x;
    float p = fmaf(c11, x2, c9);
    p = fmaf(p, x2, c7);
    p = fmaf(p, x2, c5);
    p = fmaf(p, x2, c3);
    p = fmaf(p, x2, c1);
    return p * x;
}

// D_n(s) = sin(pi s) / sin(pi s / n), with the 0/0 limit n (-1)^{m (n-1)} at s = m n.
// inv_n = 1/n in double: s / n only feeds the fractional part f2 (s is an exact
// multiple of n only at s = 0, where the product is exact too).
__device__ __forceinline__ float dirichlet(double s, int n, double inv_n) {
    double m1 = rint(s);
    double f1 = s - m1;
    double q = s * inv_n;
    double m2 = rint(q);
    double f2 = q - m2;
    long long i1 = (long long)m1, i2 = (long long)m2;
    if (f2 == 0.0) return ((i2 * (long long)(n - 1)) & 1LL) ? -(float)n : (float)n;
    float num = sinpi_half((float)f1);
    float den = sinpi_half((float)f2);
    float r = __fdividef(num, den);
    return ((i1 + i2) & 1LL) ? -r : r;
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
            double Da = (double)dirichlet((double)dx * G.cg - (double)dz * G.sg, G.ncols, G.inv_ncols) * G.inv_scale;
            double u = (double)dx * G.sg + (double)dz * G.cg;
            // per-dataset sums over the projections in float (|terms| <= nrows), then FP64
            float part[6] = {0, 0, 0, 0, 0, 0};
            for (int p = 0; p < G.np; ++p) {
                const TProj P = projs[G.p0 + p];
                const float Db = dirichlet(P.ct * u - (double)dy * P.st, G.nrows, G.inv_nrows);
#pragma unroll
                for (int q = 0; q < 6; ++q) part[q] = fmaf(P.w[q], Db, part[q]);
            }
#pragma unroll
            for (int q = 0; q < 6; ++q) acc[q] = fma(Da, (double)part[q], acc[q]);
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

// ---------------------------------------------------------------------------
// spectra in apply order
// ---------------------------------------------------------------------------

// K[(pen * 6 + q) * L1 + p1] = Re(S[(nat1[p1] * L2 + nat2[p2]) * L3h + k3]) * norm, pen = p2 * L3h + k3
__global__ void k_take_real_perm(const float2 *__restrict__ S, int L1, int L2, int L3h, const int *__restrict__ nat1,
                                 const int *__restrict__ nat2, int q, float norm, float *__restrict__ K) {
    const int64_t total = (int64_t)L1 * L2 * L3h;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        int p1 = (int)(i % L1);
        int64_t pen = i / L1;
        int k3 = (int)(pen % L3h);
        int p2 = (int)(pen / L3h);
        float v = S[((int64_t)nat1[p1] * L2 + nat2[p2]) * L3h + k3].x * norm;
        K[(pen * 6 + q) * L1 + p1] = v;
    }
}

// per-pencil max |K| over its 6 x L1 values -> power-of-two scale; fp16 store
__global__ void k_pencil_scale(const float *__restrict__ K, int L1, float *__restrict__ scale) {
    const int64_t pen = blockIdx.x;
    const float *Kp = K + pen * 6 * L1;
    float m = 0.f;
    for (int i = threadIdx.x; i < 6 * L1; i += blockDim.x) m = fmaxf(m, fabsf(Kp[i]));
    __shared__ float red[256];
    red[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        float mx = red[0];
        scale[pen] = mx > 0.f ? exp2f(floorf(log2f(mx)) - 14.f) : 1.f;  // max maps below 2^15
    }
}

__global__ void k_to_half(const float *__restrict__ K, int64_t n, int L1, const float *__restrict__ scale,
                          __half *__restrict__ Kh) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        Kh[i] = __float2half_rn(K[i] / scale[i / (6 * (int64_t)L1)]);
}

// ---------------------------------------------------------------------------
// apply kernels
// ---------------------------------------------------------------------------

// independent global loads kept in flight per thread in the load phases
constexpr int LD_BATCH = 8;

// Rows of M3 = 729 (schedule 9, 9, 9): the first radix-9 stage (one block, 81
// offsets) runs in registers on the way in (k_r2c_rows) and its inverse on the
// way out (k_c2r_rows).  Item (r, n) holds the packed values n + 81 j of row r.
constexpr int R729_OFS = 81;

__device__ __forceinline__ void rows729_load(const float *__restrict__ xb, int nr, int n3,
                                             const float2 *__restrict__ tw3, float2 *__restrict__ sm, int ps,
                                             int tid, int nth) {
    for (int t = tid; t < nr * R729_OFS; t += nth) {
        const int r = t / R729_OFS, n = t - r * R729_OFS;
        const float *xr = xb + (int64_t)r * n3;
        float2 x[9];
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            const int i = 2 * (n + R729_OFS * j);
            x[j].x = i < n3 ? xr[i] : 0.f;
            x[j].y = i + 1 < n3 ? xr[i + 1] : 0.f;
        }
        dft_small<9, false>(x);
        if (n != 0) {
            float2 w[9];
            twiddle_powers<9>(tw3, n, w);
#pragma unroll
            for (int k = 1; k < 9; ++k) x[k] = c_mul(x[k], w[k]);
        }
        float2 *sp = sm + r * ps + n;
#pragma unroll
        for (int k = 0; k < 9; ++k) sp[R729_OFS * k] = x[k];
    }
}

__device__ __forceinline__ void rows729_store(const float2 *__restrict__ sm, int nr, int ps, int n3,
                                              const float2 *__restrict__ tw3, float *__restrict__ yb, int tid,
                                              int nth) {
    for (int t = tid; t < nr * R729_OFS; t += nth) {
        const int r = t / R729_OFS, n = t - r * R729_OFS;
        const float2 *sp = sm + r * ps + n;
        float2 a[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) a[k] = sp[R729_OFS * k];
        if (n != 0) {
            float2 w[9];
            twiddle_powers<9>(tw3, n, w);
#pragma unroll
            for (int k = 1; k < 9; ++k) a[k] = c_mulc(a[k], w[k]);
        }
        dft_small<9, true>(a);
        float *yr = yb + (int64_t)r * n3;
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            const int i = 2 * (n + R729_OFS * j);
            if (i < n3) yr[i] = a[j].x;
            if (i + 1 < n3) yr[i + 1] = a[j].y;
        }
    }
}

// ---- register DFTs of composite lengths (two-stage row and pencil transforms) ----
// cos / sin of 2 pi m / R for the composite register DFTs (R = 15, 18, 25)
__host__ __device__ constexpr float wr_c(int R, int m) {
    if (R == 18) {
        constexpr float t[18] = {
        1.0f, 0.9396926207859084f, 0.766044443118978f, 0.5000000000000001f, 0.17364817766693041f,
        -0.1736481776669303f, -0.4999999999999998f, -0.7660444431189779f, -0.9396926207859083f, -1.0f,
        -0.9396926207859084f, -0.7660444431189783f, -0.5000000000000004f, -0.17364817766693033f,
        0.17364817766692997f, 0.49999999999999933f, 0.7660444431189778f, 0.9396926207859084f};
        return t[m];
    }
    if (R == 15) {
        constexpr float t[15] = {
        1.0f, 0.9135454576426009f, 0.6691306063588582f, 0.30901699437494745f, -0.10452846326765333f,
        -0.4999999999999998f, -0.8090169943749473f, -0.9781476007338057f, -0.9781476007338057f,
        -0.8090169943749476f, -0.5000000000000004f, -0.10452846326765423f, 0.30901699437494723f,
        0.6691306063588585f, 0.913545457642601f};
        return t[m];
    }
    if (R == 25) {
        constexpr float t[25] = {
        1.0f, 0.9685831611286311f, 0.8763066800438636f, 0.7289686274214116f, 0.5358267949789965f,
        0.30901699437494745f, 0.06279051952931353f, -0.1873813145857246f, -0.4257792915650727f,
        -0.6374239897486897f, -0.8090169943749473f, -0.9297764858882513f, -0.9921147013144778f,
        -0.9921147013144779f, -0.9297764858882515f, -0.8090169943749478f, -0.6374239897486895f,
        -0.42577929156507216f, -0.18738131458572463f, 0.06279051952931283f, 0.30901699437494723f,
        0.5358267949789968f, 0.7289686274214112f, 0.8763066800438631f, 0.968583161128631f};
        return t[m];
    }
    return 1.f;
}
__host__ __device__ constexpr float wr_s(int R, int m) {
    if (R == 18) {
        constexpr float t[18] = {
        0.0f, 0.3420201433256687f, 0.6427876096865393f, 0.8660254037844386f, 0.984807753012208f,
        0.984807753012208f, 0.8660254037844387f, 0.6427876096865395f, 0.3420201433256689f, 0.0f,
        -0.34202014332566866f, -0.6427876096865389f, -0.8660254037844384f, -0.984807753012208f,
        -0.9848077530122081f, -0.866025403784439f, -0.6427876096865396f, -0.3420201433256686f};
        return t[m];
    }
    if (R == 15) {
        constexpr float t[15] = {
        0.0f, 0.40673664307580015f, 0.7431448254773941f, 0.9510565162951535f, 0.9945218953682734f,
        0.8660254037844387f, 0.5877852522924732f, 0.20791169081775931f, -0.20791169081775907f, -0.587785252292473f,
        -0.8660254037844384f, -0.9945218953682733f, -0.9510565162951536f, -0.743144825477394f, -0.40673664307580015f};
        return t[m];
    }
    if (R == 25) {
        constexpr float t[25] = {
        0.0f, 0.2486898871648548f, 0.4817536741017153f, 0.6845471059286886f, 0.8443279255020151f,
        0.9510565162951535f, 0.9980267284282716f, 0.9822872507286887f, 0.9048270524660195f, 0.7705132427757893f,
        0.5877852522924732f, 0.36812455268467814f, 0.12533323356430454f, -0.12533323356430429f,
        -0.3681245526846779f, -0.5877852522924727f, -0.7705132427757894f, -0.9048270524660198f,
        -0.9822872507286887f, -0.9980267284282716f, -0.9510565162951536f, -0.844327925502015f, -0.684547105928689f,
        -0.4817536741017161f, -0.24868988716485535f};
        return t[m];
    }
    return 0.f;
}

// Composite register DFT of R1 R2 points (Cooley-Tukey, input i = R2 i1 + i2,
// output k = k1 + R1 k2, twiddles W_R^(i2 k1) as constants).
template <int R1, int R2, bool INV>
__device__ __forceinline__ void dft_cs(float2 (&v)[R1 * R2]) {
    constexpr int R = R1 * R2;
    float2 a[R];
#pragma unroll
    for (int i2 = 0; i2 < R2; ++i2) {
        float2 x[R1];
#pragma unroll
        for (int i1 = 0; i1 < R1; ++i1) x[i1] = v[R2 * i1 + i2];
        dft_small<R1, INV>(x);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) {
            const int m = (i2 * k1) % R;
            a[i2 * R1 + k1] = m == 0 ? x[k1] : c_mul_k(x[k1], wr_c(R, m), INV ? wr_s(R, m) : -wr_s(R, m));
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
        float2 y[R2];
#pragma unroll
        for (int i2 = 0; i2 < R2; ++i2) y[i2] = a[i2 * R1 + k1];
        dft_small<R2, INV>(y);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = y[k2];
    }
}

// register DFT of R points
template <int R, bool INV>
__device__ __forceinline__ void dft_reg(float2 (&v)[R]) {
    if constexpr (R == 27) dft27<INV>(v);
    else if constexpr (R == 25) dft_cs<5, 5, INV>(v);
    else if constexpr (R == 15) dft_cs<3, 5, INV>(v);
    else if constexpr (R == 18) dft_cs<2, 9, INV>(v);
    else dft_small<R, INV>(v);
}

// v[k] *= (b w^(e k)) (INV: its conjugate), k < A, w = tw[1]: two table loads
// (w^e, w^5e) and at most four products per value.
template <int A, bool INV>
__device__ __forceinline__ void twiddle_lin(const float2 *__restrict__ tw, int e, int L, float2 b, float2 (&v)[A]) {
    constexpr int R0 = 5, R1 = (A + R0 - 1) / R0;
    const float2 z = __ldg(tw + e % L), z5 = __ldg(tw + (5 * e) % L);
    float2 p0[R0];
    p0[0] = b;
#pragma unroll
    for (int k0 = 1; k0 < R0; ++k0) p0[k0] = c_mul(p0[k0 - 1], z);
    float2 q = z5;
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
#pragma unroll
        for (int k0 = 0; k0 < R0; ++k0) {
            const int k = k0 + R0 * k1;
            if (k < A) {
                const float2 t = k1 == 0 ? p0[k0] : c_mul(p0[k0], q);
                v[k] = INV ? c_mulc(v[k], t) : c_mul(v[k], t);
            }
        }
        if (k1 > 0) q = c_mul(q, z5);
    }
}

// Rows of M3 = 729 as 27 x 27 (schedule 27, 27; positions
// fft_positions(729, {27, 27})): one warp per row, lanes 0..26 busy.  The first
// stage (27-point DFTs over the packed values n + 27 j, twiddles w729^{n k})
// runs between the global rows and shared memory, the second (a 27-point DFT
// per block of 27 positions) in place in shared memory; the inverses mirror
// them.  Each value makes one trip through shared memory between the stages.
__device__ __forceinline__ void rows27_load(const float *__restrict__ xb, int nr, int n3,
                                            const float2 *__restrict__ tw3, float2 *__restrict__ sm, int ps) {
    const int r = threadIdx.x >> 5, n = threadIdx.x & 31;
    if (r < nr && n < 27) {
        const float *xr = xb + (int64_t)r * n3;
        float2 v[27];
#pragma unroll
        for (int j = 0; j < 27; ++j) {
            const int i = 2 * (n + 27 * j);
            v[j].x = i < n3 ? xr[i] : 0.f;
            v[j].y = i + 1 < n3 ? xr[i + 1] : 0.f;
        }
        dft27<false>(v);
        twiddle27<false>(tw3, n, make_float2(1.f, 0.f), v);
        float2 *sp = sm + r * ps + n;
#pragma unroll
        for (int k = 0; k < 27; ++k) sp[27 * k] = v[k];
    }
    __syncthreads();
}

// the second stage in shared memory (the caller synchronises before it)
template <bool INV>
__device__ __forceinline__ void rows27_mid(float2 *__restrict__ sm, int nr, int ps) {
    const int r = threadIdx.x >> 5, b = threadIdx.x & 31;
    if (r < nr && b < 27) {
        float2 *row = sm + r * ps + 27 * b;
        float2 v[27];
#pragma unroll
        for (int j = 0; j < 27; ++j) v[j] = row[j];
        dft27<INV>(v);
#pragma unroll
        for (int k = 0; k < 27; ++k) row[k] = v[k];
    }
    __syncthreads();
}

__device__ __forceinline__ void rows27_store(const float2 *__restrict__ sm, int nr, int ps, int n3,
                                             const float2 *__restrict__ tw3, float *__restrict__ yb) {
    const int r = threadIdx.x >> 5, n = threadIdx.x & 31;
    if (r < nr && n < 27) {
        const float2 *sp = sm + r * ps + n;
        float2 v[27];
#pragma unroll
        for (int k = 0; k < 27; ++k) v[k] = sp[27 * k];
        twiddle27<true>(tw3, n, make_float2(1.f, 0.f), v);
        dft27<true>(v);
        float *yr = yb + (int64_t)r * n3;
#pragma unroll
        for (int j = 0; j < 27; ++j) {
            const int i = 2 * (n + 27 * j);
            if (i < n3) yr[i] = v[j].x;
            if (i + 1 < n3) yr[i + 1] = v[j].y;
        }
    }
}

// Rows of M3 = A B in the same two register stages (schedule A, B; positions
// fft_positions(M3, {A, B})): one warp per row; lane n < B takes the packed
// values n + B j (j < A), lane b < A the B-point block b.
template <int M3>
struct RowTwo {
    static constexpr bool on = false;
    static constexpr int A = 0, B = 0;
};
template <>
struct RowTwo<375> {
    static constexpr bool on = true;
    static constexpr int A = 15, B = 25;
};
template <>
struct RowTwo<270> {
    static constexpr bool on = true;
    static constexpr int A = 15, B = 18;
};

template <int A, int B>
__device__ __forceinline__ void rows2s_load(const float *__restrict__ xb, int nr, int n3,
                                            const float2 *__restrict__ tw3, float2 *__restrict__ sm, int ps) {
    const int r = threadIdx.x >> 5, n = threadIdx.x & 31;
    if (r < nr && n < B) {
        const float *xr = xb + (int64_t)r * n3;
        float2 v[A];
#pragma unroll
        for (int j = 0; j < A; ++j) {
            const int i = 2 * (n + B * j);
            v[j].x = i < n3 ? xr[i] : 0.f;
            v[j].y = i + 1 < n3 ? xr[i + 1] : 0.f;
        }
        dft_reg<A, false>(v);
        twiddle_lin<A, false>(tw3, n, A * B, make_float2(1.f, 0.f), v);
        float2 *sp = sm + r * ps + n;
#pragma unroll
        for (int k = 0; k < A; ++k) sp[B * k] = v[k];
    }
    __syncthreads();
}

template <int A, int B, bool INV>
__device__ __forceinline__ void rows2s_mid(float2 *__restrict__ sm, int nr, int ps) {
    const int r = threadIdx.x >> 5, b = threadIdx.x & 31;
    if (r < nr && b < A) {
        float2 *row = sm + r * ps + B * b;
        float2 v[B];
#pragma unroll
        for (int j = 0; j < B; ++j) v[j] = row[j];
        dft_reg<B, INV>(v);
#pragma unroll
        for (int k = 0; k < B; ++k) row[k] = v[k];
    }
    __syncthreads();
}

template <int A, int B>
__device__ __forceinline__ void rows2s_store(const float2 *__restrict__ sm, int nr, int ps, int n3,
                                             const float2 *__restrict__ tw3, float *__restrict__ yb) {
    const int r = threadIdx.x >> 5, n = threadIdx.x & 31;
    if (r < nr && n < B) {
        const float2 *sp = sm + r * ps + n;
        float2 v[A];
#pragma unroll
        for (int k = 0; k < A; ++k) v[k] = sp[B * k];
        twiddle_lin<A, true>(tw3, n, A * B, make_float2(1.f, 0.f), v);
        dft_reg<A, true>(v);
        float *yr = yb + (int64_t)r * n3;
#pragma unroll
        for (int j = 0; j < A; ++j) {
            const int i = 2 * (n + B * j);
            if (i < n3) yr[i] = v[j].x;
            if (i + 1 < n3) yr[i + 1] = v[j].y;
        }
    }
}

// DIF position of packed frequency k: digit reversal of k = k0 + 27 k1 for the
// 27 x 27 schedule of 729, the table otherwise
template <int N3>
__device__ __forceinline__ int row_pos(const int *__restrict__ pos3, int k) {
    if constexpr (N3 == 729) return 27 * (k % 27) + k / 27;
    else if constexpr (RowTwo<N3>::on) return RowTwo<N3>::B * (k % RowTwo<N3>::A) + k / RowTwo<N3>::A;
    else return __ldg(pos3 + k);
}

// rows with a warp per row: 729 and the two-register-stage lengths
__host__ __device__ constexpr bool warp_rows(int M3) { return M3 == 729 || M3 == 375 || M3 == 270; }
// threads of a rows CTA of R rows: one warp per row where the lengths run in registers
__host__ __device__ constexpr int rows_threads(int M3, int R) { return warp_rows(M3) && R <= 8 ? 32 * R : 256; }

// The first stage of a runtime-length row transform (radix R0 over the whole
// packed row of M3, m0 = M3 / R0 offsets) in registers on the way in and its
// inverse on the way out, as rows729_load / rows729_store for other lengths.
template <int R0>
__device__ __forceinline__ void rowslead_load(const float *__restrict__ xb, int nr, int n3, int M3,
                                              const float2 *__restrict__ tw3, float2 *__restrict__ sm, int ps,
                                              int tid, int nth) {
    const int m0 = M3 / R0;
    for (int t = tid; t < nr * m0; t += nth) {
        const int r = t / m0, n = t - r * m0;
        const float *xr = xb + (int64_t)r * n3;
        float2 x[R0];
#pragma unroll
        for (int j = 0; j < R0; ++j) {
            const int i = 2 * (n + m0 * j);
            x[j].x = i < n3 ? xr[i] : 0.f;
            x[j].y = i + 1 < n3 ? xr[i + 1] : 0.f;
        }
        dft_small<R0, false>(x);
        if (n != 0) {
            float2 w[R0];
            twiddle_powers<R0>(tw3, n, w);
#pragma unroll
            for (int k = 1; k < R0; ++k) x[k] = c_mul(x[k], w[k]);
        }
        float2 *sp = sm + r * ps + n;
#pragma unroll
        for (int k = 0; k < R0; ++k) sp[m0 * k] = x[k];
    }
}

template <int R0>
__device__ __forceinline__ void rowslead_store(const float2 *__restrict__ sm, int nr, int ps, int n3, int M3,
                                               const float2 *__restrict__ tw3, float *__restrict__ yb, int tid,
                                               int nth) {
    const int m0 = M3 / R0;
    for (int t = tid; t < nr * m0; t += nth) {
        const int r = t / m0, n = t - r * m0;
        const float2 *sp = sm + r * ps + n;
        float2 a[R0];
#pragma unroll
        for (int k = 0; k < R0; ++k) a[k] = sp[m0 * k];
        if (n != 0) {
            float2 w[R0];
            twiddle_powers<R0>(tw3, n, w);
#pragma unroll
            for (int k = 1; k < R0; ++k) a[k] = c_mulc(a[k], w[k]);
        }
        dft_small<R0, true>(a);
        float *yr = yb + (int64_t)r * n3;
#pragma unroll
        for (int j = 0; j < R0; ++j) {
            const int i = 2 * (n + m0 * j);
            if (i < n3) yr[i] = a[j].x;
            if (i + 1 < n3) yr[i + 1] = a[j].y;
        }
    }
}

template <bool STORE>
__device__ __forceinline__ void rowslead_any(const FftLen &F3, const float *xb, const float2 *smc, float2 *sm,
                                             float *yb, int nr, int n3, int ps, int tid, int nth) {
#define LAMINO_ROWS_CASE(R)                                                            \
    case R:                                                                            \
        if constexpr (STORE) rowslead_store<R>(smc, nr, ps, n3, F3.n, F3.tw, yb, tid, nth); \
        else rowslead_load<R>(xb, nr, n3, F3.n, F3.tw, sm, ps, tid, nth);               \
        break;
    switch (F3.radix[0]) {
        LAMINO_ROWS_CASE(2)
        LAMINO_ROWS_CASE(3)
        LAMINO_ROWS_CASE(4)
        LAMINO_ROWS_CASE(5)
        LAMINO_ROWS_CASE(8)
        default: LAMINO_ROWS_CASE(9)
    }
#undef LAMINO_ROWS_CASE
}

// A1: real rows along n3 (zero-padded to L3) -> half spectrum k3 in [0, M3], via the
// packed-complex M3-point DIF and the even/odd split.  N3: compile-time M3 or 0.
template <int N3>
__global__ void __launch_bounds__(256, warp_rows(N3) ? 3 : 4) k_r2c_rows(const float *__restrict__ x, int64_t nrows, int n3, FftLen F3,
                                                  const int *__restrict__ pos3, const float2 *__restrict__ twh,
                                                  int R, float2 *__restrict__ z1) {
    extern __shared__ float2 sm[];
    const int M3 = N3 ? N3 : F3.n;
    const int ps = M3 + 1;
    const int64_t row0 = (int64_t)blockIdx.x * R;
    const int nr = (int)min((int64_t)R, nrows - row0);
    if constexpr (N3 == 729) {
        rows27_load(x + row0 * n3, nr, n3, F3.tw, sm, ps);
        rows27_mid<false>(sm, nr, ps);
    } else if constexpr (RowTwo<N3>::on) {
        rows2s_load<RowTwo<N3>::A, RowTwo<N3>::B>(x + row0 * n3, nr, n3, F3.tw, sm, ps);
        rows2s_mid<RowTwo<N3>::A, RowTwo<N3>::B, false>(sm, nr, ps);
    } else if constexpr (N3 != 0) {  // compile-time schedule: the first stage in registers
        rowslead_load<CtRowSched<N3>::r[0]>(x + row0 * n3, nr, n3, N3, F3.tw, sm, ps, threadIdx.x, blockDim.x);
        __syncthreads();
        ct_forward<N3, 1, CtRowSched<N3>>(sm, nr, ps, F3.tw, threadIdx.x, blockDim.x);
    } else if (F3.ns >= 1) {  // runtime length: the first stage in registers as well
        rowslead_any<false>(F3, x + row0 * n3, nullptr, sm, nullptr, nr, n3, ps, threadIdx.x, blockDim.x);
        __syncthreads();
        fft_forward(sm, nr, ps, F3, 1, threadIdx.x, blockDim.x);
    } else {
        const int total = nr * M3;
        const float *xb = x + row0 * n3;
        for (int t0 = threadIdx.x; t0 < total; t0 += LD_BATCH * blockDim.x) {
            float2 v[LD_BATCH];
#pragma unroll
            for (int u = 0; u < LD_BATCH; ++u) {
                int t = t0 + u * blockDim.x;
                int r = t / M3, m = t - r * M3, i = 2 * m;
                v[u].x = (t < total && i < n3) ? xb[(int64_t)r * n3 + i] : 0.f;
                v[u].y = (t < total && i + 1 < n3) ? xb[(int64_t)r * n3 + i + 1] : 0.f;
            }
#pragma unroll
            for (int u = 0; u < LD_BATCH; ++u) {
                int t = t0 + u * blockDim.x;
                if (t < total) {
                    int r = t / M3;
                    sm[r * ps + (t - r * M3)] = v[u];
                }
            }
        }
        __syncthreads();
        fft_fwd_any<N3, 0>(sm, nr, ps, F3, threadIdx.x, blockDim.x);
    }
    for (int t = threadIdx.x; t < nr * (M3 + 1); t += blockDim.x) {
        int r = t / (M3 + 1), k = t - r * (M3 + 1);
        int ka = (k == M3) ? 0 : k;
        int kb = (k == 0) ? 0 : M3 - k;
        float2 Zk = sm[r * ps + row_pos<N3>(pos3, ka)];
        float2 Zm = sm[r * ps + row_pos<N3>(pos3, kb)];
        Zm.y = -Zm.y;
        float2 sum = c_add(Zk, Zm), dif = c_sub(Zk, Zm);
        float2 wd = c_mul(__ldg(twh + k), dif);
        // X = (sum - i w dif) / 2
        z1[(row0 + r) * (M3 + 1) + k] = make_float2(0.5f * (sum.x + wd.y), 0.5f * (sum.y - wd.x));
    }
}

// Tiles of the n2 passes: 8 consecutive i1 x KB (8) consecutive k3 per CTA.  Shared
// pencil p = ii * KB + kk has stride ps = L2 + pad with ps = 2 (mod 16), so the 16
// lanes of each 8-byte shared access phase (8 kk x 2 rows) hit distinct banks in the
// load, FFT and transpose phases.  xa pencils have stride n1p (a multiple of 8), so
// each thread moves its 8 i1 values as 64 aligned bytes.
constexpr int D2_IB = 8;
// shared pencil stride for KB k3 values per tile: ps = 16 / KB (mod 16)
__host__ __device__ constexpr int d2_stride(int L2, int KB) {
    return L2 + ((((16 / KB) - L2) % 16) + 16) % 16;
}
// dynamic shared memory of an n2-pass CTA (float2 values): the tile plus the
// skew of the L2 = 144 layout
__host__ __device__ constexpr int d2_smem_values(int L2, int KB) {
    return L2 == 144 ? D2_IB * KB * 145 + (D2_IB * KB / 16 + 1) * 4 : D2_IB * KB * d2_stride(L2, KB);
}


// n2 passes of L2 = 144 (schedule 2, 8, 9): the zero-padded radix-2 stage and the
// radix-8 stage (two blocks of 72, 9 offsets each) run in registers on the way in
// (k_dim2_fwd) and their inverses on the way out (k_dim2_inv); the radix-9 stage
// (blocks of 9 positions, no twiddles) runs in registers on the way out to xa
// (and in from xa), fused with the transpose.  Item (ii, n, kk), kk fastest,
// holds the values i2 = n + 9 j of tile row kk * 8 + ii; rows are 145 values
// apart (odd) plus a skew of 4 per 16 rows, so with KB = 4 the 16 lanes of each
// 8-byte access phase hit distinct banks in the lead (kk x n) and tail (ii x kk)
// phases.
constexpr int D2_144_OFS = 9;
__device__ __forceinline__ int d2_row144(int r) { return r * 145 + (r >> 4) * 4; }

// threads of an n2-pass CTA: one per item of the fused stages for L2 = 144
__host__ __device__ constexpr int d2_threads(int L2, int KB) {
    return (L2 == 144 && KB <= 4) ? D2_144_OFS * D2_IB * KB : 256;
}

__device__ __forceinline__ void dim2_144_load(const float2 *__restrict__ z1, int n1, int n2, int L3h, int c, int i1b,
                                              int k3b, int nk, int KB, int ps, const float2 *__restrict__ tw2,
                                              float2 *__restrict__ sm, int tid, int nth) {
    const int total = D2_IB * D2_144_OFS * KB;
    for (int t = tid; t < total; t += nth) {
        const int kk = t % KB, r = t / KB;
        const int n = r % D2_144_OFS, ii = r / D2_144_OFS;
        const int i1 = i1b + ii;
        const bool live = kk < nk && i1 < n1;
        float2 x[8], u[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int i2 = n + D2_144_OFS * j;
            x[j] = (live && i2 < n2) ? z1[(((int64_t)c * n1 + i1) * n2 + i2) * L3h + k3b + kk] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) u[j] = c_mul(x[j], __ldg(tw2 + n + D2_144_OFS * j));
        dft_small<8, false>(x);
        dft_small<8, false>(u);
        if (n != 0) {
            float2 w[8];
            twiddle_powers<8>(tw2, 2 * n, w);
#pragma unroll
            for (int k = 1; k < 8; ++k) {
                x[k] = c_mul(x[k], w[k]);
                u[k] = c_mul(u[k], w[k]);
            }
        }
        float2 *sp = sm + d2_row144(kk * D2_IB + ii) + n;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            sp[D2_144_OFS * k] = x[k];
            sp[72 + D2_144_OFS * k] = u[k];
        }
    }
}

__device__ __forceinline__ void dim2_144_store(const float2 *__restrict__ sm, int n1, int n2, int L3h, int c,
                                               int i1b, int k3b, int nk, int KB, int ps,
                                               const float2 *__restrict__ tw2, float2 *__restrict__ z1, int tid,
                                               int nth) {
    const int total = D2_IB * D2_144_OFS * KB;
    for (int t = tid; t < total; t += nth) {
        const int kk = t % KB, r = t / KB;
        const int n = r % D2_144_OFS, ii = r / D2_144_OFS;
        const int i1 = i1b + ii;
        if (kk >= nk || i1 >= n1) continue;
        const float2 *sp = sm + d2_row144(kk * D2_IB + ii) + n;
        float2 a[8], b[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            a[k] = sp[D2_144_OFS * k];
            b[k] = sp[72 + D2_144_OFS * k];
        }
        if (n != 0) {
            float2 w[8];
            twiddle_powers<8>(tw2, 2 * n, w);
#pragma unroll
            for (int k = 1; k < 8; ++k) {
                a[k] = c_mulc(a[k], w[k]);
                b[k] = c_mulc(b[k], w[k]);
            }
        }
        dft_small<8, true>(a);
        dft_small<8, true>(b);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int i2 = n + D2_144_OFS * j;
            if (i2 < n2)
                z1[(((int64_t)c * n1 + i1) * n2 + i2) * L3h + k3b + kk] =
                    c_add(a[j], c_mulc(b[j], __ldg(tw2 + i2)));
        }
    }
}

// The radix-9 stage of 144 and the transposing store of its outputs into
// xa[((c L2 + p2) L3h + k3) n1p + i1]: item (ii, kk, b), ii fastest, so lanes
// 0..7 write the 8 i1 values of one (p2, k3) run (64 B) for each of the 9
// outputs p2 = 9 b + k.
__device__ __forceinline__ void dim2_144_tail_store(const float2 *__restrict__ sm, int L3h, int n1p, int c,
                                                    int i1b, int k3b, int nk, int KB, float2 *__restrict__ xa,
                                                    int tid, int nth) {
    const int64_t pstride = (int64_t)L3h * n1p;
    for (int t = tid; t < D2_IB * KB * 16; t += nth) {
        const int ii = t % D2_IB, r = t / D2_IB;
        const int kk = r % KB, b = r / KB;
        if (kk >= nk) continue;
        const float2 *sp = sm + d2_row144(kk * D2_IB + ii) + 9 * b;
        float2 v[9];
#pragma unroll
        for (int j = 0; j < 9; ++j) v[j] = sp[j];
        dft_small<9, false>(v);
        float2 *dst = xa + (((int64_t)c * 144 + 9 * b) * L3h + k3b + kk) * n1p + i1b + ii;
#pragma unroll
        for (int k = 0; k < 9; ++k) dst[k * pstride] = v[k];
    }
}

// its inverse: the transposing load from xa and the inverse radix-9 stage
__device__ __forceinline__ void dim2_144_tail_load(const float2 *__restrict__ xa, int L3h, int n1p, int c, int i1b,
                                                   int k3b, int nk, int KB, float2 *__restrict__ sm, int tid,
                                                   int nth) {
    const int64_t pstride = (int64_t)L3h * n1p;
    const int total = D2_IB * KB * 16;
    // two items per pass: their 18 loads are in flight together
    for (int t0 = tid; t0 < total; t0 += 2 * nth) {
        float2 v[2][9];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int t = t0 + u * nth;
            const int ii = t % D2_IB, r = t / D2_IB;
            const int kk = r % KB, b = r / KB;
            if (t < total && kk < nk) {
                const float2 *src = xa + (((int64_t)c * 144 + 9 * b) * L3h + k3b + kk) * n1p + i1b + ii;
#pragma unroll
                for (int k = 0; k < 9; ++k) v[u][k] = src[k * pstride];
            }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int t = t0 + u * nth;
            const int ii = t % D2_IB, r = t / D2_IB;
            const int kk = r % KB, b = r / KB;
            if (t < total && kk < nk) {
                dft_small<9, true>(v[u]);
                float2 *sp = sm + d2_row144(kk * D2_IB + ii) + 9 * b;
#pragma unroll
                for (int j = 0; j < 9; ++j) sp[j] = v[u][j];
            }
        }
    }
}

// n2 passes of the other compile-time lengths L2 = 2 R1 R2 (schedule 2, R1, R2:
// 20, 48, 64, 90) with the last stage fused into the transposes, as for 144:
// item (ii, n, kk), kk fastest, holds the values i2 = n + R2 j (j < R1) of tile
// pencil ii KB + kk (rows ps apart); the zero-padded radix-2 and the radix-R1
// stage run in registers on the way in (d2f_load), the radix-R2 stage of each
// block of R2 positions on the way out to xa (d2f_tail_store: item (ii, kk, b),
// ii fastest, so 8 lanes write one 64-byte i1 run), and their inverses mirror
// them (d2f_tail_load, d2f_store).
template <int R1, int R2>
__device__ __forceinline__ void d2f_load(const float2 *__restrict__ z1, int n1, int n2, int L3h, int c, int i1b,
                                         int k3b, int nk, int KB, int ps, const float2 *__restrict__ tw2,
                                         float2 *__restrict__ sm, int tid, int nth) {
    constexpr int M = R1 * R2;
    const int total = D2_IB * R2 * KB;
    for (int t = tid; t < total; t += nth) {
        const int kk = t % KB, r = t / KB;
        const int n = r % R2, ii = r / R2;
        const int i1 = i1b + ii;
        const bool live = kk < nk && i1 < n1;
        float2 x[R1], u[R1];
#pragma unroll
        for (int j = 0; j < R1; ++j) {
            const int i2 = n + R2 * j;
            x[j] = (live && i2 < n2) ? z1[(((int64_t)c * n1 + i1) * n2 + i2) * L3h + k3b + kk] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < R1; ++j) u[j] = c_mul(x[j], __ldg(tw2 + n + R2 * j));
        dft_small<R1, false>(x);
        dft_small<R1, false>(u);
        if (n != 0) {
            float2 w[R1];
            twiddle_powers<R1>(tw2, 2 * n, w);
#pragma unroll
            for (int k = 1; k < R1; ++k) {
                x[k] = c_mul(x[k], w[k]);
                u[k] = c_mul(u[k], w[k]);
            }
        }
        float2 *sp = sm + (ii * KB + kk) * ps + n;
#pragma unroll
        for (int k = 0; k < R1; ++k) {
            sp[R2 * k] = x[k];
            sp[M + R2 * k] = u[k];
        }
    }
}

template <int R1, int R2>
__device__ __forceinline__ void d2f_tail_store(const float2 *__restrict__ sm, int L3h, int n1p, int c, int i1b,
                                               int k3b, int nk, int KB, int ps, float2 *__restrict__ xa, int tid,
                                               int nth) {
    constexpr int L = 2 * R1 * R2;
    const int64_t pstride = (int64_t)L3h * n1p;
    for (int t = tid; t < D2_IB * KB * 2 * R1; t += nth) {
        const int ii = t % D2_IB, r = t / D2_IB;
        const int kk = r % KB, b = r / KB;
        if (kk >= nk) continue;
        const float2 *sp = sm + (ii * KB + kk) * ps + R2 * b;
        float2 v[R2];
#pragma unroll
        for (int j = 0; j < R2; ++j) v[j] = sp[j];
        dft_small<R2, false>(v);
        float2 *dst = xa + (((int64_t)c * L + R2 * b) * L3h + k3b + kk) * n1p + i1b + ii;
#pragma unroll
        for (int k = 0; k < R2; ++k) dst[k * pstride] = v[k];
    }
}

template <int R1, int R2>
__device__ __forceinline__ void d2f_tail_load(const float2 *__restrict__ xa, int L3h, int n1p, int c, int i1b,
                                              int k3b, int nk, int KB, int ps, float2 *__restrict__ sm, int tid,
                                              int nth) {
    constexpr int L = 2 * R1 * R2;
    const int64_t pstride = (int64_t)L3h * n1p;
    for (int t = tid; t < D2_IB * KB * 2 * R1; t += nth) {
        const int ii = t % D2_IB, r = t / D2_IB;
        const int kk = r % KB, b = r / KB;
        if (kk >= nk) continue;
        const float2 *src = xa + (((int64_t)c * L + R2 * b) * L3h + k3b + kk) * n1p + i1b + ii;
        float2 v[R2];
#pragma unroll
        for (int k = 0; k < R2; ++k) v[k] = src[k * pstride];
        dft_small<R2, true>(v);
        float2 *sp = sm + (ii * KB + kk) * ps + R2 * b;
#pragma unroll
        for (int j = 0; j < R2; ++j) sp[j] = v[j];
    }
}

template <int R1, int R2>
__device__ __forceinline__ void d2f_store(const float2 *__restrict__ sm, int n1, int n2, int L3h, int c, int i1b,
                                          int k3b, int nk, int KB, int ps, const float2 *__restrict__ tw2,
                                          float2 *__restrict__ z1, int tid, int nth) {
    constexpr int M = R1 * R2;
    const int total = D2_IB * R2 * KB;
    for (int t = tid; t < total; t += nth) {
        const int kk = t % KB, r = t / KB;
        const int n = r % R2, ii = r / R2;
        const int i1 = i1b + ii;
        if (kk >= nk || i1 >= n1) continue;
        const float2 *sp = sm + (ii * KB + kk) * ps + n;
        float2 a[R1], b[R1];
#pragma unroll
        for (int k = 0; k < R1; ++k) {
            a[k] = sp[R2 * k];
            b[k] = sp[M + R2 * k];
        }
        if (n != 0) {
            float2 w[R1];
            twiddle_powers<R1>(tw2, 2 * n, w);
#pragma unroll
            for (int k = 1; k < R1; ++k) {
                a[k] = c_mulc(a[k], w[k]);
                b[k] = c_mulc(b[k], w[k]);
            }
        }
        dft_small<R1, true>(a);
        dft_small<R1, true>(b);
#pragma unroll
        for (int j = 0; j < R1; ++j) {
            const int i2 = n + R2 * j;
            if (i2 < n2)
                z1[(((int64_t)c * n1 + i1) * n2 + i2) * L3h + k3b + kk] = c_add(a[j], c_mulc(b[j], __ldg(tw2 + i2)));
        }
    }
}

// The same register stages for a runtime L2 (schedule 2, R1, ...): item (ii, n, kk),
// kk fastest, holds the values i2 = n + m1 j of tile pencil ii * KB + kk,
// m1 = L2 / (2 R1); the stages from 2 on run in shared memory.
template <int R1>
__device__ __forceinline__ void dim2lead_load(const float2 *__restrict__ z1, int n1, int n2, int L3h, int c, int i1b,
                                              int k3b, int nk, int KB, int ps, int L2,
                                              const float2 *__restrict__ tw2, float2 *__restrict__ sm, int tid,
                                              int nth) {
    const int half = L2 / 2, m1 = half / R1;
    const int total = D2_IB * m1 * KB;
    for (int t = tid; t < total; t += nth) {
        const int kk = t % KB, r = t / KB;
        const int ii = r / m1, n = r - ii * m1;
        const int i1 = i1b + ii;
        const bool live = kk < nk && i1 < n1;
        float2 x[R1], u[R1];
#pragma unroll
        for (int j = 0; j < R1; ++j) {
            const int i2 = n + m1 * j;
            x[j] = (live && i2 < n2) ? z1[(((int64_t)c * n1 + i1) * n2 + i2) * L3h + k3b + kk] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < R1; ++j) u[j] = c_mul(x[j], __ldg(tw2 + n + m1 * j));
        dft_small<R1, false>(x);
        dft_small<R1, false>(u);
        if (n != 0) {
            float2 w[R1];
            twiddle_powers<R1>(tw2, 2 * n, w);
#pragma unroll
            for (int k = 1; k < R1; ++k) {
                x[k] = c_mul(x[k], w[k]);
                u[k] = c_mul(u[k], w[k]);
            }
        }
        float2 *sp = sm + (ii * KB + kk) * ps + n;
#pragma unroll
        for (int k = 0; k < R1; ++k) {
            sp[m1 * k] = x[k];
            sp[half + m1 * k] = u[k];
        }
    }
}

template <int R1>
__device__ __forceinline__ void dim2lead_store(const float2 *__restrict__ sm, int n1, int n2, int L3h, int c,
                                               int i1b, int k3b, int nk, int KB, int ps, int L2,
                                               const float2 *__restrict__ tw2, float2 *__restrict__ z1, int tid,
                                               int nth) {
    const int half = L2 / 2, m1 = half / R1;
    const int total = D2_IB * m1 * KB;
    for (int t = tid; t < total; t += nth) {
        const int kk = t % KB, r = t / KB;
        const int ii = r / m1, n = r - ii * m1;
        const int i1 = i1b + ii;
        if (kk >= nk || i1 >= n1) continue;
        const float2 *sp = sm + (ii * KB + kk) * ps + n;
        float2 a[R1], b[R1];
#pragma unroll
        for (int k = 0; k < R1; ++k) {
            a[k] = sp[m1 * k];
            b[k] = sp[half + m1 * k];
        }
        if (n != 0) {
            float2 w[R1];
            twiddle_powers<R1>(tw2, 2 * n, w);
#pragma unroll
            for (int k = 1; k < R1; ++k) {
                a[k] = c_mulc(a[k], w[k]);
                b[k] = c_mulc(b[k], w[k]);
            }
        }
        dft_small<R1, true>(a);
        dft_small<R1, true>(b);
#pragma unroll
        for (int j = 0; j < R1; ++j) {
            const int i2 = n + m1 * j;
            if (i2 < n2)
                z1[(((int64_t)c * n1 + i1) * n2 + i2) * L3h + k3b + kk] = c_add(a[j], c_mulc(b[j], __ldg(tw2 + i2)));
        }
    }
}

#define LAMINO_DIM2_LEAD(FN, R1SEL, ...)                       \
    switch (R1SEL) {                                           \
        case 2: FN<2>(__VA_ARGS__); break;                     \
        case 3: FN<3>(__VA_ARGS__); break;                     \
        case 4: FN<4>(__VA_ARGS__); break;                     \
        case 5: FN<5>(__VA_ARGS__); break;                     \
        case 8: FN<8>(__VA_ARGS__); break;                     \
        default: FN<9>(__VA_ARGS__); break;                    \
    }

// A2: columns along n2 (zero-padded to L2) -> pencil-major xa[((c L2 + p2) L3h + k3) n1p + i1]
template <int N2>
__global__ void __launch_bounds__(288, 4) k_dim2_fwd(const float2 *__restrict__ z1, int n1, int n2, int L3h, int n1p,
                                                  FftLen F2, const float2 *__restrict__ tw2, int KB,
                                                  float2 *__restrict__ xa) {
    extern __shared__ float2 sm[];
    const int i1b = blockIdx.x * D2_IB, k3b = blockIdx.y * KB, c = blockIdx.z;
    const int nk = min(KB, L3h - k3b);
    const int L2 = N2 ? N2 : F2.n;
    const int ps = d2_stride(L2, KB), half = L2 / 2;
    if constexpr (N2 == 144) {
        dim2_144_load(z1, n1, n2, L3h, c, i1b, k3b, nk, KB, ps, tw2, sm, threadIdx.x, blockDim.x);
        __syncthreads();
        dim2_144_tail_store(sm, L3h, n1p, c, i1b, k3b, nk, KB, xa, threadIdx.x, blockDim.x);
    } else if constexpr (N2 != 0) {  // compile-time 2, R1, R2: lead stages in registers, the last fused with the store
        static_assert(CtSched<N2>::ns == 3, "fused n2 passes take three-stage schedules");
        d2f_load<CtSched<N2>::r[1], CtSched<N2>::r[2]>(z1, n1, n2, L3h, c, i1b, k3b, nk, KB, ps, tw2, sm,
                                                        threadIdx.x, blockDim.x);
        __syncthreads();
        d2f_tail_store<CtSched<N2>::r[1], CtSched<N2>::r[2]>(sm, L3h, n1p, c, i1b, k3b, nk, KB, ps, xa, threadIdx.x,
                                                              blockDim.x);
    } else if (F2.ns >= 2) {  // runtime length: the outer stages in registers as well
        LAMINO_DIM2_LEAD(dim2lead_load, F2.radix[1], z1, n1, n2, L3h, c, i1b, k3b, nk, KB, ps, L2, tw2, sm,
                         (int)threadIdx.x, (int)blockDim.x)
        __syncthreads();
        fft_forward(sm, D2_IB * KB, ps, F2, 2, threadIdx.x, blockDim.x);
    } else {
        // load: kk fastest (coalesced along k3); D2_BATCH independent loads in flight per thread
        constexpr int D2_BATCH = 4;
        const int total = D2_IB * half * KB;
        for (int t0 = threadIdx.x; t0 < total; t0 += D2_BATCH * blockDim.x) {
            float2 v[D2_BATCH];
#pragma unroll
            for (int u = 0; u < D2_BATCH; ++u) {
                int t = t0 + u * blockDim.x;
                int kk = t % KB;
                int r = t / KB;
                int i2 = r % half;
                int i1 = i1b + r / half;
                v[u] = make_float2(0.f, 0.f);
                if (t < total && kk < nk && i2 < n2 && i1 < n1)
                    v[u] = z1[(((int64_t)c * n1 + i1) * n2 + i2) * L3h + k3b + kk];
            }
#pragma unroll
            for (int u = 0; u < D2_BATCH; ++u) {
                int t = t0 + u * blockDim.x;
                if (t < total) {
                    int kk = t % KB;
                    int r = t / KB;
                    int i2 = r % half;
                    int ii = r / half;
                    float2 *pp = sm + (ii * KB + kk) * ps;
                    pp[i2] = v[u];
                    pp[i2 + half] = c_mul(v[u], __ldg(tw2 + i2));
                }
            }
        }
        __syncthreads();
        fft_fwd_any<N2, 1>(sm, D2_IB * KB, ps, F2, threadIdx.x, blockDim.x);
    }
    if constexpr (N2 == 0) {
        // store: four lanes per (p2, kk) run of 8 i1 values (64 B), one float4 each,
        // so a warp writes 8 runs rather than 32
        for (int t = threadIdx.x; t < L2 * nk * (D2_IB / 2); t += blockDim.x) {
            const int h = t % (D2_IB / 2), it = t / (D2_IB / 2);
            const int kk = it % nk, p2 = it / nk;
            float4 *dst = reinterpret_cast<float4 *>(xa + (((int64_t)c * L2 + p2) * L3h + k3b + kk) * n1p + i1b);
            const float2 a = sm[((2 * h) * KB + kk) * ps + p2];
            const float2 b = sm[((2 * h + 1) * KB + kk) * ps + p2];
            dst[h] = make_float4(a.x, a.y, b.x, b.y);
        }
    }
}

// Pencil rows for fft1458_load / fft1458_store: component c of the pencil at pv,
// n1 values, components cs apart.
struct PencilRows {
    float2 *pv;
    int64_t cs;
    int n1;
    __device__ __forceinline__ float2 get(int c, int i) const {
        return i < n1 ? pv[c * cs + i] : make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ bool want(int i) const { return i < n1; }
    __device__ __forceinline__ void put(int c, int i, float2 v) const { pv[c * cs + i] = v; }
};

// ---- n1 transforms of length 1458 = 2 x 27 x 27 (the 721-voxel axis) ----
// Six warps per pencil: warp (c, h) = (w / 2, w % 2), lanes 0..26 busy.  Forward
// DIF with the schedule 2, 27, 27 (positions fft_positions(1458, {2, 27, 27})):
// half h of component c holds y_h[i] = x_i w^{h i}, w = exp(-2 pi i / 1458), x_i = 0
// from n1 on.  Lane n of warp (c, h) takes y_h[n + 27 j] = w^{h n} x_{n+27j}
// W54^{h j} (W54 = w^27), forms the 27-point DFT of x_{n+27j} W54^{hj}, multiplies
// output k by w^{n (2k + h)} (the common w^{hn} and the stage twiddle
// w^{2 n k}) and stores it at position 729 h + n + 27 k; the second stage is a
// 27-point DFT per block of 27 positions, in place.  Each value makes one trip
// through shared memory between the stages (two with the 2, 9, 9, 9 schedule).
// The inverse runs the stages backwards; warp (c, 1) leaves its half times
// conj(w^i) in shared memory and warp (c, 0) adds it to its own and stores.
constexpr int P1458_THREADS = 192;
// cos / sin of 2 pi j / 54, j = 0..26 (compile-time j: folded into the instructions)
__host__ __device__ constexpr float w54c(int j) {
    constexpr float t[27] = {1.f, 0.99323835774194302317f, 0.97304487057982380627f, 0.93969262078590842791f,
                             0.89363264032341227505f, 0.83548781141293648744f, 0.76604444311897801345f,
                             0.68624163786873360049f, 0.59715859170278617896f, 0.50000000000000011102f,
                             0.39607976603915689973f, 0.28680323271109031680f, 0.17364817766693041445f,
                             0.05814482891047567659f, -0.05814482891047577373f, -0.17364817766693008139f,
                             -0.28680323271109020578f, -0.39607976603915678870f, -0.49999999999999977796f,
                             -0.59715859170278595691f, -0.68624163786873348947f, -0.76604444311897823550f,
                             -0.83548781141293626540f, -0.89363264032341216403f, -0.93969262078590831688f,
                             -0.97304487057982380627f, -0.99323835774194302317f};
    return t[j];
}
__host__ __device__ constexpr float w54s(int j) {
    constexpr float t[27] = {0.f, 0.11609291412523023435f, 0.23061587074244016549f, 0.34202014332566871291f,
                             0.44879918020046216665f, 0.54950897807080600899f, 0.64278760968653925190f,
                             0.72737364157304862378f, 0.80212319275504373461f, 0.86602540378443859659f,
                             0.91821610688027399672f, 0.95798951231548890028f, 0.98480775301220802032f,
                             0.99830815827126817563f, 0.99830815827126817563f, 0.98480775301220813134f,
                             0.95798951231548890028f, 0.91821610688027399672f, 0.86602540378443870761f,
                             0.80212319275504395666f, 0.72737364157304884582f, 0.64278760968653914087f,
                             0.54950897807080623103f, 0.44879918020046233318f, 0.34202014332566887944f,
                             0.23061587074244033202f, 0.11609291412522992903f};
    return t[j];
}

// Load (zero-padded), both forward stages; ends after a barrier with the DIF
// spectrum of the 3 components in sm[c * 1458 + p].
__device__ __forceinline__ void p1458_forward(const PencilRows &rows, const float2 *__restrict__ tw,
                                              float2 *__restrict__ sm) {
    const int w = threadIdx.x >> 5, n = threadIdx.x & 31;
    const int c = w >> 1, h = w & 1;
    float2 *half = sm + c * 1458 + h * 729;
    if (n < 27) {
        float2 v[27];
#pragma unroll
        for (int j = 0; j < 27; ++j) v[j] = rows.get(c, n + 27 * j);
        if (h) {
#pragma unroll
            for (int j = 1; j < 27; ++j) v[j] = c_mul_k(v[j], w54c(j), -w54s(j));
        }
        dft27<false>(v);
        twiddle27<false>(tw, 2 * n, h ? __ldg(tw + n) : make_float2(1.f, 0.f), v);  // w^{n (2k + h)}
#pragma unroll
        for (int k = 0; k < 27; ++k) half[n + 27 * k] = v[k];
    }
    __syncthreads();
    if (n < 27) {
        float2 *row = half + 27 * n;
        float2 v[27];
#pragma unroll
        for (int j = 0; j < 27; ++j) v[j] = row[j];
        dft27<false>(v);
#pragma unroll
        for (int k = 0; k < 27; ++k) row[k] = v[k];
    }
    __syncthreads();
}

// Both inverse stages and the pruned store of the first n1 values (the caller
// synchronises after writing the spectrum).
__device__ __forceinline__ void p1458_inverse(const PencilRows &rows, const float2 *__restrict__ tw,
                                              float2 *__restrict__ sm) {
    const int w = threadIdx.x >> 5, n = threadIdx.x & 31;
    const int c = w >> 1, h = w & 1;
    float2 *half = sm + c * 1458 + h * 729;
    if (n < 27) {
        float2 *row = half + 27 * n;
        float2 v[27];
#pragma unroll
        for (int k = 0; k < 27; ++k) v[k] = row[k];
        dft27<true>(v);
#pragma unroll
        for (int j = 0; j < 27; ++j) row[j] = v[j];
    }
    __syncthreads();
    float2 v[27];
    if (n < 27) {
#pragma unroll
        for (int k = 0; k < 27; ++k) v[k] = half[n + 27 * k];
        twiddle27<true>(tw, 2 * n, h ? __ldg(tw + n) : make_float2(1.f, 0.f), v);
        dft27<true>(v);
        if (h) {  // this half times conj(w^i) = conj(w^{n}) conj(W54^j); the first factor came with the twiddles
#pragma unroll
            for (int j = 0; j < 27; ++j) half[n + 27 * j] = j ? c_mul_k(v[j], w54c(j), w54s(j)) : v[j];
        }
    }
    __syncthreads();
    if (h == 0 && n < 27) {
        const float2 *other = half + 729;
#pragma unroll
        for (int j = 0; j < 27; ++j) {
            const int i = n + 27 * j;
            if (rows.want(i)) rows.put(c, i, c_add(v[j], other[i]));
        }
    }
}

// Forward n1 transform of L = 2 A B (the 1458 scheme of p1458_forward with A-
// and B-point stages): six warps per pencil, warp (c, h); lane n < B takes
// y_h[n + B j] = w^{h n} x_{n+B j} W_{2A}^{h j} (W_{2A} = w^B, from the table),
// forms its A-point DFT, multiplies output k by w^{n (2k + h)} and stores it at
// position A B h + n + B k; lane m < A then runs the B-point DFT of block m in
// place.  DIF positions: fft_positions(L, {2, A, B}).
template <int A, int B>
__device__ __forceinline__ void p2s_forward(const PencilRows &rows, const float2 *__restrict__ tw,
                                            float2 *__restrict__ sm) {
    constexpr int M = A * B, L = 2 * M;
    const int w = threadIdx.x >> 5, n = threadIdx.x & 31;
    const int c = w >> 1, h = w & 1;
    float2 *half = sm + c * L + h * M;
    if (n < B) {
        float2 v[A];
#pragma unroll
        for (int j = 0; j < A; ++j) v[j] = rows.get(c, n + B * j);
        if (h) {
#pragma unroll
            for (int j = 1; j < A; ++j) v[j] = c_mul(v[j], __ldg(tw + B * j));
        }
        dft_reg<A, false>(v);
        twiddle_lin<A, false>(tw, 2 * n, L, h ? __ldg(tw + n) : make_float2(1.f, 0.f), v);
#pragma unroll
        for (int k = 0; k < A; ++k) half[n + B * k] = v[k];
    }
    __syncthreads();
    if (n < A) {
        float2 *row = half + B * n;
        float2 v[B];
#pragma unroll
        for (int j = 0; j < B; ++j) v[j] = row[j];
        dft_reg<B, false>(v);
#pragma unroll
        for (int k = 0; k < B; ++k) row[k] = v[k];
    }
    __syncthreads();
}

// Its inverse and the pruned store of the first n1 values (the caller
// synchronises after writing the spectrum).
template <int A, int B>
__device__ __forceinline__ void p2s_inverse(const PencilRows &rows, const float2 *__restrict__ tw,
                                            float2 *__restrict__ sm) {
    constexpr int M = A * B, L = 2 * M;
    const int w = threadIdx.x >> 5, n = threadIdx.x & 31;
    const int c = w >> 1, h = w & 1;
    float2 *half = sm + c * L + h * M;
    if (n < A) {
        float2 *row = half + B * n;
        float2 v[B];
#pragma unroll
        for (int k = 0; k < B; ++k) v[k] = row[k];
        dft_reg<B, true>(v);
#pragma unroll
        for (int j = 0; j < B; ++j) row[j] = v[j];
    }
    __syncthreads();
    float2 v[A];
    if (n < B) {
#pragma unroll
        for (int k = 0; k < A; ++k) v[k] = half[n + B * k];
        twiddle_lin<A, true>(tw, 2 * n, L, h ? __ldg(tw + n) : make_float2(1.f, 0.f), v);
        dft_reg<A, true>(v);
        if (h) {  // this half times conj(w^i) = conj(w^n) conj(W_{2A}^j); the first factor came with the twiddles
#pragma unroll
            for (int j = 0; j < A; ++j) half[n + B * j] = j ? c_mulc(v[j], __ldg(tw + B * j)) : v[j];
        }
    }
    __syncthreads();
    if (h == 0 && n < B) {
        const float2 *other = half + M;
#pragma unroll
        for (int j = 0; j < A; ++j) {
            const int i = n + B * j;
            if (rows.want(i)) rows.put(c, i, c_add(v[j], other[i]));
        }
    }
}

// the n1 lengths run in two register stages, as (A, B); 1458 = 2 x 27 x 27 has its own
// kernels (p1458_*) with constant W_54 tables
template <int L>
struct TwoStage {
    static constexpr bool on = false;
    static constexpr int A = 0, B = 0;
};
template <>
struct TwoStage<750> {
    static constexpr bool on = true;
    static constexpr int A = 15, B = 25;
};
template <>
struct TwoStage<540> {
    static constexpr bool on = true;
    static constexpr int A = 15, B = 18;
};
// (360 as 12 x 15 and 180 as 9 x 10 were slower than their compile-time
// shared-memory schedules: too few lanes busy per warp)
// threads of a pencil CTA: six warps for the register-stage lengths, 256 otherwise
__host__ __device__ constexpr int pencil_threads(int L) {
    return (L == 1458 || L == 750 || L == 540) ? P1458_THREADS : 256;
}
// the register-stage schedule (2, A, B) of an n1 length, empty when it has none
static std::vector<int> two_stage_schedule(int L) {
    switch (L) {
        case 750: return {2, TwoStage<750>::A, TwoStage<750>::B};
        case 540: return {2, TwoStage<540>::A, TwoStage<540>::B};
        default: return {};
    }
}

// B: one (p2, k3) pencil of the 3 components along n1: DIF (zero-padded), 3x3
// symmetric multiply with the spectra (same position order), undo, first n1 kept.
// In place on xa.  N1: compile-time L1 or 0.  At L1 = 1458, five CTAs of 256
// threads per SM (48 registers, 35 KB of shared memory each); four otherwise.
template <bool HALF, int N1>
__global__ void __launch_bounds__(pencil_threads(N1), 4) k_pencil(float2 *__restrict__ xa, int n1, int n1p, int L2, int L3h, FftLen F1,
                                                const float2 *__restrict__ tw1, const float *__restrict__ K,
                                                const __half *__restrict__ Kh, const float *__restrict__ kscale) {
    extern __shared__ float2 sm[];
    const int64_t pen = blockIdx.x;
    const int L1 = N1 ? N1 : F1.n;
    const int half = L1 / 2;
    const int64_t cs = (int64_t)L2 * L3h * n1p;  // component stride in xa
    float2 *pv = xa + pen * n1p;
    // the pencil's 6 spectra (one contiguous range) start moving into L2 while
    // the forward transform runs, so the multiply does not wait on HBM
    if (threadIdx.x == 0) {
        if constexpr (HALF) prefetch_l2(Kh + pen * 6 * L1, (size_t)6 * L1 * sizeof(__half));
        else prefetch_l2(K + pen * 6 * L1, (size_t)6 * L1 * sizeof(float));
    }
    if constexpr (N1 == 1458) {
        p1458_forward(PencilRows{pv, cs, n1}, tw1, sm);
    } else if constexpr (TwoStage<N1>::on) {
        p2s_forward<TwoStage<N1>::A, TwoStage<N1>::B>(PencilRows{pv, cs, n1}, tw1, sm);
    } else if constexpr (N1 != 0) {  // compile-time schedule: lead stages in registers, the rest fixed
        fftlead_load<CtSched<N1>::r[1]>(PencilRows{pv, cs, n1}, tw1, sm, N1, N1, threadIdx.x, blockDim.x);
        __syncthreads();
        ct_forward<N1, 2>(sm, 3, N1, tw1, threadIdx.x, blockDim.x);
    } else if (F1.ns >= 2) {  // runtime length: the outer stages in registers as well
        fftlead_any<false>(PencilRows{pv, cs, n1}, F1, sm, L1, threadIdx.x, blockDim.x);
        __syncthreads();
        fft_forward(sm, 3, L1, F1, 2, threadIdx.x, blockDim.x);
    } else {
        for (int t0 = threadIdx.x; t0 < 3 * half; t0 += LD_BATCH * blockDim.x) {
            float2 v[LD_BATCH];
#pragma unroll
            for (int u = 0; u < LD_BATCH; ++u) {
                int t = t0 + u * blockDim.x;
                int c = t / half, i1 = t - c * half;
                v[u] = (t < 3 * half && i1 < n1) ? pv[c * cs + i1] : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < LD_BATCH; ++u) {
                int t = t0 + u * blockDim.x;
                if (t < 3 * half) {
                    int c = t / half, i1 = t - c * half;
                    sm[c * L1 + i1] = v[u];
                    sm[c * L1 + i1 + half] = c_mul(v[u], __ldg(tw1 + i1));
                }
            }
        }
        __syncthreads();
        fft_fwd_any<N1, 1>(sm, 3, L1, F1, threadIdx.x, blockDim.x);
    }
    const float sc = HALF ? kscale[pen] : 1.f;
    // two adjacent positions per thread (L1 is even): 8-byte spectrum loads and
    // 16-byte shared accesses; KU pairs whose 6 spectra are in flight together
    constexpr int KU = 2;
    const int L1h = L1 / 2;
    for (int q0 = threadIdx.x; q0 < L1h; q0 += KU * blockDim.x) {
        float2 kv[KU][6];
#pragma unroll
        for (int u = 0; u < KU; ++u) {
            const int pp = q0 + u * blockDim.x;
            if (pp < L1h) {
                if (HALF) {
                    const __half2 *Kp = reinterpret_cast<const __half2 *>(Kh + pen * 6 * L1) + pp;
#pragma unroll
                    for (int q = 0; q < 6; ++q) {
                        const float2 k = __half22float2(Kp[q * L1h]);
                        kv[u][q] = make_float2(k.x * sc, k.y * sc);
                    }
                } else {
                    const float2 *Kp = reinterpret_cast<const float2 *>(K + pen * 6 * L1) + pp;
#pragma unroll
                    for (int q = 0; q < 6; ++q) kv[u][q] = Kp[q * L1h];
                }
            }
        }
#pragma unroll
        for (int u = 0; u < KU; ++u) {
            const int pp = q0 + u * blockDim.x;
            if (pp < L1h) {
                float4 *s0 = reinterpret_cast<float4 *>(sm) + pp;
                float4 *s1 = reinterpret_cast<float4 *>(sm + L1) + pp;
                float4 *s2 = reinterpret_cast<float4 *>(sm + 2 * L1) + pp;
                const float4 a = *s0, b = *s1, c = *s2;
                const float2 k00 = kv[u][0], k11 = kv[u][1], k22 = kv[u][2], k01 = kv[u][3], k02 = kv[u][4],
                             k12 = kv[u][5];
                *s0 = make_float4(k00.x * a.x + k01.x * b.x + k02.x * c.x, k00.x * a.y + k01.x * b.y + k02.x * c.y,
                                  k00.y * a.z + k01.y * b.z + k02.y * c.z, k00.y * a.w + k01.y * b.w + k02.y * c.w);
                *s1 = make_float4(k01.x * a.x + k11.x * b.x + k12.x * c.x, k01.x * a.y + k11.x * b.y + k12.x * c.y,
                                  k01.y * a.z + k11.y * b.z + k12.y * c.z, k01.y * a.w + k11.y * b.w + k12.y * c.w);
                *s2 = make_float4(k02.x * a.x + k12.x * b.x + k22.x * c.x, k02.x * a.y + k12.x * b.y + k22.x * c.y,
                                  k02.y * a.z + k12.y * b.z + k22.y * c.z, k02.y * a.w + k12.y * b.w + k22.y * c.w);
            }
        }
    }
    __syncthreads();
    if constexpr (N1 == 1458) {
        p1458_inverse(PencilRows{pv, cs, n1}, tw1, sm);
    } else if constexpr (TwoStage<N1>::on) {
        p2s_inverse<TwoStage<N1>::A, TwoStage<N1>::B>(PencilRows{pv, cs, n1}, tw1, sm);
    } else if constexpr (N1 != 0) {
        ct_inverse<N1, CtSched<N1>::ns - 1, 2>(sm, 3, N1, tw1, threadIdx.x, blockDim.x);
        fftlead_store<CtSched<N1>::r[1]>(PencilRows{pv, cs, n1}, tw1, sm, N1, N1, threadIdx.x, blockDim.x);
    } else if (F1.ns >= 2) {
        fft_inverse(sm, 3, L1, F1, 2, threadIdx.x, blockDim.x);
        fftlead_any<true>(PencilRows{pv, cs, n1}, F1, sm, L1, threadIdx.x, blockDim.x);
    } else {
        fft_inv_any<N1, 1>(sm, 3, L1, F1, threadIdx.x, blockDim.x);
        for (int t = threadIdx.x; t < 3 * n1; t += blockDim.x) {
            int c = t / n1, i1 = t - c * n1;
            pv[c * cs + i1] = c_add(sm[c * L1 + i1], c_mulc(sm[c * L1 + i1 + half], __ldg(tw1 + i1)));
        }
    }
}

// Quadratic forms x_i . (S_g x)_i of up to kMaxQuadSets operators S_g sharing
// this pencil layout, by Parseval on the half spectrum: after the forward
// pencil FFT, sum_p1 w(k3) Re(conj(X_i) (K_g X)_i), w = 1 on the k3 = 0 and
// Nyquist planes and 2 elsewhere (K is real and even, X Hermitian).
constexpr int kMaxQuadSets = 8;
struct QuadSets {
    const float *K[kMaxQuadSets];
};

template <int N1>
__global__ void __launch_bounds__(pencil_threads(N1)) k_pencil_quad(const float2 *__restrict__ xa, int n1, int n1p, int L2, int L3h,
                                                     FftLen F1, const float2 *__restrict__ tw1, QuadSets ks, int ng,
                                                     double *__restrict__ acc) {
    extern __shared__ float2 sm[];
    __shared__ float red[8][3 * kMaxQuadSets];
    const int64_t pen = blockIdx.x;
    const int L1 = N1 ? N1 : F1.n;
    const int half = L1 / 2;
    const int64_t cs = (int64_t)L2 * L3h * n1p;
    const float2 *pv = xa + pen * n1p;
    if constexpr (N1 == 1458) {
        p1458_forward(PencilRows{const_cast<float2 *>(pv), cs, n1}, tw1, sm);  // reads only
    } else if constexpr (TwoStage<N1>::on) {
        p2s_forward<TwoStage<N1>::A, TwoStage<N1>::B>(PencilRows{const_cast<float2 *>(pv), cs, n1}, tw1, sm);
    } else if constexpr (N1 != 0) {
        fftlead_load<CtSched<N1>::r[1]>(PencilRows{const_cast<float2 *>(pv), cs, n1}, tw1, sm, N1, N1,
                                        threadIdx.x, blockDim.x);
        __syncthreads();
        ct_forward<N1, 2>(sm, 3, N1, tw1, threadIdx.x, blockDim.x);
    } else if (F1.ns >= 2) {
        fftlead_any<false>(PencilRows{const_cast<float2 *>(pv), cs, n1}, F1, sm, L1, threadIdx.x, blockDim.x);
        __syncthreads();
        fft_forward(sm, 3, L1, F1, 2, threadIdx.x, blockDim.x);
    } else {
        for (int t = threadIdx.x; t < 3 * half; t += blockDim.x) {
            int c = t / half, i1 = t - c * half;
            float2 v = i1 < n1 ? pv[c * cs + i1] : make_float2(0.f, 0.f);
            sm[c * L1 + i1] = v;
            sm[c * L1 + i1 + half] = c_mul(v, __ldg(tw1 + i1));
        }
        __syncthreads();
        fft_fwd_any<N1, 1>(sm, 3, L1, F1, threadIdx.x, blockDim.x);
    }
    float part[kMaxQuadSets][3];
#pragma unroll
    for (int g = 0; g < kMaxQuadSets; ++g) part[g][0] = part[g][1] = part[g][2] = 0.f;
    for (int p1 = threadIdx.x; p1 < L1; p1 += blockDim.x) {
        const float2 a = sm[p1], b = sm[L1 + p1], c = sm[2 * L1 + p1];
#pragma unroll
        for (int g = 0; g < kMaxQuadSets; ++g) {
            if (g < ng) {
                const float *Kp = ks.K[g] + pen * 6 * L1 + p1;
                const float k00 = Kp[0], k11 = Kp[L1], k22 = Kp[2 * L1], k01 = Kp[3 * L1], k02 = Kp[4 * L1],
                            k12 = Kp[5 * L1];
                const float2 y0 = make_float2(k00 * a.x + k01 * b.x + k02 * c.x, k00 * a.y + k01 * b.y + k02 * c.y);
                const float2 y1 = make_float2(k01 * a.x + k11 * b.x + k12 * c.x, k01 * a.y + k11 * b.y + k12 * c.y);
                const float2 y2 = make_float2(k02 * a.x + k12 * b.x + k22 * c.x, k02 * a.y + k12 * b.y + k22 * c.y);
                part[g][0] += a.x * y0.x + a.y * y0.y;
                part[g][1] += b.x * y1.x + b.y * y1.y;
                part[g][2] += c.x * y2.x + c.y * y2.y;
            }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int g = 0; g < kMaxQuadSets; ++g) {
        if (g < ng) {
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                float v = part[g][i];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
                if (lane == 0) red[warp][g * 3 + i] = v;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < 3 * ng) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += (double)red[w][threadIdx.x];
        const int k3 = (int)(pen % L3h);
        const double wk = (k3 == 0 || k3 == L3h - 1) ? 1.0 : 2.0;
        atomicAdd(acc + threadIdx.x, wk * t);
    }
}

// C2: undo along k2 (positions -> natural), first n2 rows kept, back into z1 rows
template <int N2>
__global__ void __launch_bounds__(288, 4) k_dim2_inv(const float2 *__restrict__ xa, int n1, int n2, int L3h, int n1p,
                                                  FftLen F2, const float2 *__restrict__ tw2, int KB,
                                                  float2 *__restrict__ z1) {
    extern __shared__ float2 sm[];
    const int i1b = blockIdx.x * D2_IB, k3b = blockIdx.y * KB, c = blockIdx.z;
    const int nk = min(KB, L3h - k3b);
    const int L2 = N2 ? N2 : F2.n;
    const int ps = d2_stride(L2, KB), half = L2 / 2;
    if constexpr (N2 == 144) {
        dim2_144_tail_load(xa, L3h, n1p, c, i1b, k3b, nk, KB, sm, threadIdx.x, blockDim.x);
        __syncthreads();
        dim2_144_store(sm, n1, n2, L3h, c, i1b, k3b, nk, KB, ps, tw2, z1, threadIdx.x, blockDim.x);
        return;
    } else if constexpr (N2 != 0) {
        d2f_tail_load<CtSched<N2>::r[1], CtSched<N2>::r[2]>(xa, L3h, n1p, c, i1b, k3b, nk, KB, ps, sm, threadIdx.x,
                                                             blockDim.x);
        __syncthreads();
        d2f_store<CtSched<N2>::r[1], CtSched<N2>::r[2]>(sm, n1, n2, L3h, c, i1b, k3b, nk, KB, ps, tw2, z1,
                                                         threadIdx.x, blockDim.x);
        return;
    }
    // load: four lanes per (p2, kk) run of 8 i1 values (64 B), one float4 each, so a
    // warp reads 8 runs rather than 32; D2_LD runs in flight per thread
    constexpr int D2_LD = 4;
    const int ltotal = L2 * KB * (D2_IB / 2);
    for (int t0 = threadIdx.x; t0 < ltotal; t0 += D2_LD * blockDim.x) {
        float4 q[D2_LD];
#pragma unroll
        for (int u = 0; u < D2_LD; ++u) {
            const int t = t0 + u * blockDim.x;
            const int h = t % (D2_IB / 2), it = t / (D2_IB / 2);
            const int kk = it % KB, p2 = it / KB;
            q[u] = (t < ltotal && kk < nk)
                       ? reinterpret_cast<const float4 *>(xa + (((int64_t)c * L2 + p2) * L3h + k3b + kk) * n1p + i1b)[h]
                       : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < D2_LD; ++u) {
            const int t = t0 + u * blockDim.x;
            if (t < ltotal) {
                const int h = t % (D2_IB / 2), it = t / (D2_IB / 2);
                const int kk = it % KB, p2 = it / KB;
                sm[((2 * h) * KB + kk) * ps + p2] = make_float2(q[u].x, q[u].y);
                sm[((2 * h + 1) * KB + kk) * ps + p2] = make_float2(q[u].z, q[u].w);
            }
        }
    }
    __syncthreads();
    if (F2.ns >= 2) {
        fft_inverse(sm, D2_IB * KB, ps, F2, 2, threadIdx.x, blockDim.x);
        LAMINO_DIM2_LEAD(dim2lead_store, F2.radix[1], sm, n1, n2, L3h, c, i1b, k3b, nk, KB, ps, L2, tw2, z1,
                         (int)threadIdx.x, (int)blockDim.x)
        return;
    }
    fft_inv_any<N2, 1>(sm, D2_IB * KB, ps, F2, threadIdx.x, blockDim.x);
    // store: kk fastest (coalesced along k3)
    for (int t = threadIdx.x; t < D2_IB * n2 * nk; t += blockDim.x) {
        int kk = t % nk;
        int r = t / nk;
        int i2 = r % n2;
        int ii = r / n2;
        int i1 = i1b + ii;
        if (i1 < n1) {
            const float2 *pp = sm + (ii * KB + kk) * ps;
            z1[(((int64_t)c * n1 + i1) * n2 + i2) * L3h + k3b + kk] =
                c_add(pp[i2], c_mulc(pp[i2 + half], __ldg(tw2 + i2)));
        }
    }
}

// C1: half spectrum k3 in [0, M3] -> real rows (first n3 kept), the inverse of A1
// returning L3 x (unnormalised; the 1/(L1 L2 L3) lives in the spectra).
template <int N3>
__global__ void __launch_bounds__(256) k_c2r_rows(const float2 *__restrict__ z1, int64_t nrows, int n3, FftLen F3,
                                                  const int *__restrict__ pos3, const float2 *__restrict__ twh, int R,
                                                  float *__restrict__ y) {
    extern __shared__ float2 sm[];
    const int M3 = N3 ? N3 : F3.n;
    const int ps = M3 + 1;
    const int64_t row0 = (int64_t)blockIdx.x * R;
    const int nr = (int)min((int64_t)R, nrows - row0);
    for (int t0 = threadIdx.x; t0 < nr * M3; t0 += LD_BATCH * blockDim.x) {
        float2 Xk[LD_BATCH], Xm[LD_BATCH];
#pragma unroll
        for (int u = 0; u < LD_BATCH; ++u) {
            int t = t0 + u * blockDim.x;
            int r = t / M3, k = t - r * M3;
            if (t < nr * M3) {
                const float2 *Xr = z1 + (row0 + r) * (M3 + 1);
                Xk[u] = Xr[k];
                Xm[u] = Xr[M3 - k];
            }
        }
#pragma unroll
        for (int u = 0; u < LD_BATCH; ++u) {
            int t = t0 + u * blockDim.x;
            if (t < nr * M3) {
                int r = t / M3, k = t - r * M3;
                float2 xm = make_float2(Xm[u].x, -Xm[u].y);
                float2 E = c_add(Xk[u], xm);
                float2 O = c_mulc(c_sub(Xk[u], xm), __ldg(twh + k));
                sm[r * ps + row_pos<N3>(pos3, k)] = make_float2(E.x - O.y, E.y + O.x);  // E + i O
            }
        }
    }
    __syncthreads();
    if constexpr (N3 == 729) {
        rows27_mid<true>(sm, nr, ps);
        rows27_store(sm, nr, ps, n3, F3.tw, y + row0 * n3);
        return;
    } else if constexpr (RowTwo<N3>::on) {
        rows2s_mid<RowTwo<N3>::A, RowTwo<N3>::B, true>(sm, nr, ps);
        rows2s_store<RowTwo<N3>::A, RowTwo<N3>::B>(sm, nr, ps, n3, F3.tw, y + row0 * n3);
        return;
    } else if constexpr (N3 != 0) {
        ct_inverse<N3, CtRowSched<N3>::ns - 1, 1, CtRowSched<N3>>(sm, nr, ps, F3.tw, threadIdx.x, blockDim.x);
        rowslead_store<CtRowSched<N3>::r[0]>(sm, nr, ps, n3, N3, F3.tw, y + row0 * n3, threadIdx.x, blockDim.x);
        return;
    }
    if (F3.ns >= 1) {
        fft_inverse(sm, nr, ps, F3, 1, threadIdx.x, blockDim.x);
        rowslead_any<true>(F3, nullptr, sm, nullptr, y + row0 * n3, nr, n3, ps, threadIdx.x, blockDim.x);
        return;
    }
    fft_inv_any<N3, 0>(sm, nr, ps, F3, threadIdx.x, blockDim.x);
    for (int t = threadIdx.x; t < nr * M3; t += blockDim.x) {
        int r = t / M3, m = t - r * M3;
        float2 z = sm[r * ps + m];
        float *yr = y + (row0 + r) * n3;
        int i = 2 * m;
        if (i < n3) yr[i] = z.x;
        if (i + 1 < n3) yr[i + 1] = z.y;
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

std::vector<int> fft_schedule(int n, bool lead2) {
    std::vector<int> r;
    int m = n;
    for (int q : {9, 8, 5, 4, 3, 2})
        while (m % q == 0 && m > 1) { r.push_back(q); m /= q; }
    if (m != 1) throw Error(ERR_ARG, "FFT length must be 2,3,5-smooth");
    if (lead2) {
        if (n % 2) throw Error(ERR_ARG, "zero-padded FFT length must be even");
        auto it = std::find(r.begin(), r.end(), 2);
        if (it != r.end()) r.erase(it);
        else if ((it = std::find(r.begin(), r.end(), 4)) != r.end()) *it = 2;
        else if ((it = std::find(r.begin(), r.end(), 8)) != r.end()) *it = 4;
    }
    // even radices first, odd ones last: the last stages read with stride = radix,
    // which is conflict-free in 8-byte shared-memory banks only when it is odd
    std::stable_sort(r.begin(), r.end(), [](int a, int b) { return (a % 2 == 0) && (b % 2 == 1); });
    if (lead2) r.insert(r.begin(), 2);
    if ((int)r.size() > FFT_MAX_STAGES) throw Error(ERR_ARG, "FFT length has too many stages");
    return r;
}

std::vector<int> fft_positions(int n, const std::vector<int> &radix) {
    std::vector<int> pos(n, 0);
    if (radix.empty()) return pos;
    int r = radix[0], m = n / r;
    std::vector<int> sub = fft_positions(m, std::vector<int>(radix.begin() + 1, radix.end()));
    for (int k = 0; k < n; ++k) pos[k] = m * (k % r) + sub[k / r];
    return pos;
}

__global__ void k_add_into(float *a, const float *b, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[i] += b[i];
}

// The dynamic shared-memory limit is a per-function attribute shared by every
// operator (and host thread) of the process on a device: it is only ever raised,
// under a lock, so an operator built concurrently for a smaller volume cannot
// lower it beneath one that is launching with more.
void raise_smem_limit(const void *f, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, int> limit;
    int dev = 0;
    LAMINO_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    int &cur = limit[{dev, f}];
    if (bytes <= cur) return;
    LAMINO_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    cur = bytes;
}

static FftLen make_len(int n, bool lead2, DevBuf<float2> &tw, std::vector<int> *radix_out) {
    std::vector<int> r = fft_schedule(n, lead2);
    FftLen F{};
    F.n = n;
    F.ns = (int)r.size();
    int b = n;
    for (int s = 0; s < F.ns; ++s) {
        F.radix[s] = r[s];
        F.bsz[s] = b;
        F.dm[s] = FastDiv::make((uint32_t)(b / r[s]));
        F.dnb[s] = FastDiv::make((uint32_t)(n / r[s]));
        F.dblk[s] = FastDiv::make((uint32_t)(n / b));
        b /= r[s];
    }
    std::vector<float2> h(n);
    for (int e = 0; e < n; ++e) {
        double a = -2.0 * M_PI * (double)e / (double)n;
        h[e] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    tw.alloc(n);
    upload(tw.p, h.data(), (size_t)n);
    F.tw = tw.p;
    if (radix_out) *radix_out = r;
    return F;
}

static int64_t embed_len(int64_t n) {
    // smallest even 2,3,5-smooth L >= 2n (L >= 2n-1 suffices for a linear convolution)
    return next_smooth_even(2 * n);
}

static void raise_rows_smem(int bytes);
static void raise_d2_smem(int bytes);

// whether the n1 length has a compile-time pencil schedule equal to the runtime
// one r (the spectra are stored in the runtime schedule's DIF positions)
template <int N>
static bool ct_equal(const std::vector<int> &r) {
    if ((int)r.size() != CtSched<N>::ns) return false;
    for (int i = 0; i < CtSched<N>::ns; ++i)
        if (r[i] != CtSched<N>::r[i]) return false;
    return true;
}
template <int N>
static bool ct_row_equal(const std::vector<int> &r) {
    if ((int)r.size() != CtRowSched<N>::ns) return false;
    for (int i = 0; i < CtRowSched<N>::ns; ++i)
        if (r[i] != CtRowSched<N>::r[i]) return false;
    return true;
}
static bool ct_row_matches(int M, const std::vector<int> &r) {
    switch (M) {
        case 180: return ct_row_equal<180>(r);
        case 90: return ct_row_equal<90>(r);
        default: return false;
    }
}
static bool ct_schedule_matches(int L, const std::vector<int> &r) {  // n1 (pencil) lengths
    switch (L) {
        case 360: return ct_equal<360>(r);
        case 180: return ct_equal<180>(r);
        default: return false;
    }
}
static bool ct_dim2_matches(int L, const std::vector<int> &r) {  // n2 lengths
    switch (L) {
        case 90: return ct_equal<90>(r);
        case 64: return ct_equal<64>(r);
        case 48: return ct_equal<48>(r);
        case 20: return ct_equal<20>(r);
        default: return false;
    }
}

void Toeplitz::init_tables(Dims3 d, int prec) {
    if (d.n1 <= 0 || d.n2 <= 0 || d.n3 <= 0) throw Error(ERR_ARG, "volume dims must be positive");
    if (prec != PREC_FP32 && prec != PREC_FP16 && prec != PREC_MIXED)
        throw Error(ERR_ARG, "precision must be 0 (fp32), 1 (fp16) or 2 (mixed)");
    L1 = embed_len(d.n1);
    L2 = embed_len(d.n2);
    L3 = embed_len(d.n3);
    L3h = L3 / 2 + 1;
    M3 = L3 / 2;
    if (Lsize() > (int64_t)INT32_MAX) throw Error(ERR_ARG, "volume too large for the Toeplitz embedding");
    if (3 * L1 * (int64_t)sizeof(float2) > 227 * 1024) throw Error(ERR_ARG, "n1 too large for the pencil kernel");

    // FFT schedules, twiddles and position maps
    std::vector<int> r1, r2, r3;
    f1 = make_len((int)L1, true, tw1, &r1);
    f2 = make_len((int)L2, true, tw2, &r2);
    f3 = make_len((int)M3, false, tw3, &r3);
    if (M3 == 729) r3 = {27, 27};  // the compile-time rows (rows27_load / rows27_mid)
    if (M3 == 375) r3 = {RowTwo<375>::A, RowTwo<375>::B};  // two register stages (rows2s_*)
    if (M3 == 270) r3 = {RowTwo<270>::A, RowTwo<270>::B};
    {
        std::vector<float2> h(M3 + 1);
        for (int64_t k = 0; k <= M3; ++k) {
            double a = -2.0 * M_PI * (double)k / (double)L3;
            h[k] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
        twh3.alloc(M3 + 1);
        upload(twh3.p, h.data(), h.size());
        std::vector<int> p3 = fft_positions((int)M3, r3);
        pos3.alloc(M3);
        upload(pos3.p, p3.data(), (size_t)M3);
    }
    // the compile-time n1 transform of 1458 runs the schedule 2, 27, 27 (p1458_forward)
    // the n1 transforms with register stages run the schedules 2, 27, 27 (1458) and
    // 2, A, B (TwoStage lengths)
    const std::vector<int> r2s = two_stage_schedule((int)L1);
    r1_ = L1 == 1458 ? std::vector<int>{2, 27, 27} : (r2s.empty() ? r1 : r2s);
    r2_ = r2;
}

Toeplitz::Toeplitz(const std::vector<const Geom *> &gs, Dims3 d, int prec, cudaStream_t s) : vol(d), precision(prec) {
    if (gs.empty()) throw Error(ERR_ARG, "Toeplitz operator needs at least one geometry");
    init_tables(d, prec);
    std::vector<int> nat1(L1), nat2(L2);
    {
        std::vector<int> p1 = fft_positions((int)L1, r1_), p2 = fft_positions((int)L2, r2_);
        for (int k = 0; k < (int)L1; ++k) nat1[p1[k]] = k;
        for (int k = 0; k < (int)L2; ++k) nat2[p2[k]] = k;
    }
    DevBuf<int> dnat1(L1), dnat2(L2);
    upload(dnat1.p, nat1.data(), (size_t)L1);
    upload(dnat2.p, nat2.data(), (size_t)L2);

    // geometry tables in double
    std::vector<TGam> hg;
    std::vector<TProj> hp;
    for (const Geom *g : gs) {
        TGam G;
        double gm = (double)g->gamma;
        G.cg = std::cos(gm);
        G.sg = std::sin(gm);
        G.inv_scale = 1.0 / (double)(g->nrows * g->ncols);
        G.inv_nrows = 1.0 / (double)g->nrows;
        G.inv_ncols = 1.0 / (double)g->ncols;
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
            P.w[0] = (float)(c[0] * c[0]); P.w[1] = (float)(c[1] * c[1]); P.w[2] = (float)(c[2] * c[2]);
            P.w[3] = (float)(c[0] * c[1]); P.w[4] = (float)(c[0] * c[2]); P.w[5] = (float)(c[1] * c[2]);
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

    // one-off uniform R2C per pair (cuFFT), real part stored in apply order
    FftPlan r2c;
    int n[3] = {(int)L1, (int)L2, (int)L3};
    r2c.make(3, n, CUFFT_R2C, 1);
    LAMINO_CUFFT(cufftSetStream(r2c.h, s));
    DevBuf<float2> spec(Ssize());
    K.alloc(6 * Ssize());
    float norm = (float)(1.0 / ((double)L1 * L2 * L3));
    for (int q = 0; q < 6; ++q) {
        LAMINO_CUFFT(cufftExecR2C(r2c.h, T.p + q * Lsize(), (cufftComplex *)spec.p));
        k_take_real_perm<<<grid_for(Ssize(), 256), 256, 0, s>>>(spec.p, (int)L1, (int)L2, (int)L3h, dnat1.p,
                                                                 dnat2.p, q, norm, K.p);
        LAMINO_LAUNCH("k_take_real_perm");
    }
    T.release();
    spec.release();
    finish(s);
}

// Sum of operators over disjoint geometry sets: the kernel is linear in the
// geometry, so its spectra add.
Toeplitz::Toeplitz(const std::vector<const Toeplitz *> &parts, int prec, cudaStream_t s)
    : vol(parts.empty() ? Dims3{0, 0, 0} : parts[0]->vol), precision(prec) {
    if (parts.empty()) throw Error(ERR_ARG, "Toeplitz sum needs at least one operator");
    for (const Toeplitz *t : parts) {
        if (!t || !t->has_fp32()) throw Error(ERR_ARG, "Toeplitz sum needs operators with FP32 spectra");
        if (t->vol.n1 != vol.n1 || t->vol.n2 != vol.n2 || t->vol.n3 != vol.n3)
            throw Error(ERR_ARG, "Toeplitz sum needs operators of one volume size");
    }
    init_tables(vol, prec);
    K.alloc(6 * Ssize());
    LAMINO_CUDA(cudaMemcpyAsync(K.p, parts[0]->K.p, K.bytes(), cudaMemcpyDeviceToDevice, s));
    for (size_t i = 1; i < parts.size(); ++i) {
        k_add_into<<<grid_for(6 * Ssize(), 256), 256, 0, s>>>(K.p, parts[i]->K.p, 6 * Ssize());
        LAMINO_LAUNCH("k_add_into");
    }
    finish(s);
}

void Toeplitz::finish(cudaStream_t s) {
    const Dims3 d = vol;
    if (precision != PREC_FP32) {
        Kh.alloc(6 * Ssize());
        Kscale.alloc(L2 * L3h);
        k_pencil_scale<<<(unsigned)(L2 * L3h), 256, 0, s>>>(K.p, (int)L1, Kscale.p);
        LAMINO_LAUNCH("k_pencil_scale");
        k_to_half<<<grid_for(6 * Ssize(), 256), 256, 0, s>>>(K.p, 6 * Ssize(), (int)L1, Kscale.p, Kh.p);
        LAMINO_LAUNCH("k_to_half");
    }
    LAMINO_CUDA(cudaStreamSynchronize(s));
    if (precision == PREC_FP16) K.release();

    // intermediates and launch shapes
    n1p = (d.n1 + D2_IB - 1) / D2_IB * D2_IB;
    z1.alloc(3 * d.n1 * d.n2 * L3h);
    xa.alloc(3 * L2 * L3h * n1p);
    rows1 = (int)std::max<int64_t>(1, std::min<int64_t>(8, (96 * 1024) / (L3h * (int64_t)sizeof(float2))));
    kb2 = 4;
    while (kb2 > 1 && d2_smem_values((int)L2, kb2) * (int64_t)sizeof(float2) > 160 * 1024) kb2 /= 2;
    if (d2_smem_values((int)L2, kb2) * (int64_t)sizeof(float2) > 200 * 1024)
        throw Error(ERR_ARG, "n2 too large for the n2-pass kernels");
    ct1 = (L1 == 1458 || !two_stage_schedule((int)L1).empty() || ct_schedule_matches((int)L1, r1_)) ? (int)L1 : 0;
    ct2 = (L2 == 144 || ct_dim2_matches((int)L2, r2_)) ? (int)L2 : 0;
    ct3 = (warp_rows((int)M3) || ct_row_matches((int)M3, fft_schedule((int)M3, false))) ? (int)M3 : 0;
    const int smem_rows = rows1 * (int)L3h * (int)sizeof(float2);
    const int smem_d2 = d2_smem_values((int)L2, kb2) * (int)sizeof(float2);
    const int smem_pen = 3 * (int)L1 * (int)sizeof(float2);
    auto attr = [](const void *f, int bytes) { raise_smem_limit(f, bytes); };
    raise_rows_smem(smem_rows);
    raise_d2_smem(smem_d2);
    attr((const void *)k_pencil<false, 0>, smem_pen);
    attr((const void *)k_pencil<true, 0>, smem_pen);
    attr((const void *)k_pencil<false, 1458>, smem_pen);
    attr((const void *)k_pencil<true, 1458>, smem_pen);
    attr((const void *)k_pencil_quad<0>, smem_pen);
    attr((const void *)k_pencil_quad<1458>, smem_pen);
    for (const void *f : {(const void *)k_pencil<false, 750>, (const void *)k_pencil<true, 750>,
                          (const void *)k_pencil_quad<750>, (const void *)k_pencil<false, 540>,
                          (const void *)k_pencil<true, 540>, (const void *)k_pencil_quad<540>,
                          (const void *)k_pencil<false, 360>, (const void *)k_pencil<true, 360>,
                          (const void *)k_pencil_quad<360>, (const void *)k_pencil<false, 180>,
                          (const void *)k_pencil<true, 180>, (const void *)k_pencil_quad<180>})
        attr(f, smem_pen);
}

Toeplitz::~Toeplitz() {
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
}

size_t Toeplitz::device_bytes() const {
    return K.bytes() + Kh.bytes() + Kscale.bytes() + z1.bytes() + xa.bytes() + tw1.bytes() + tw2.bytes() +
           tw3.bytes() + twh3.bytes() + pos3.bytes();
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
    static const char *names[NSTAGE] = {"r2c_rows", "dim2_fwd", "pencil", "dim2_inv", "c2r_rows"};
    return (i >= 0 && i < NSTAGE) ? names[i] : "";
}

void Toeplitz::stage_bytes(int64_t *b) const {
    const int64_t V = vol.size();
    const int64_t Z = 3 * vol.n1 * vol.n2 * L3h * 8;   // z1 bytes
    const int64_t X = 3 * L2 * L3h * vol.n1 * 8;        // xa bytes (the n1p padding is not counted)
    const int64_t bk = precision == PREC_FP32 ? 4 : 2;
    b[0] = 3 * V * 4 + Z;                               // read x, write z1
    b[1] = Z + X;                                       // read z1, write xa
    b[2] = 2 * X + 6 * L2 * L3h * L1 * bk;              // read + write xa, read the 6 spectra
    b[3] = X + Z;                                       // read xa, write z1
    b[4] = Z + 3 * V * 4;                               // read z1, write y
}

// the pencil kernel of the operator's n1 length: compile-time schedules for the
// lengths in CtSched (ct1), the runtime one otherwise (ct1 = 0)
template <bool HALF>
static void launch_pencil(int ct1, unsigned grid, int smem, cudaStream_t s, float2 *xa, int n1, int np1, int l2,
                          int l3h, const FftLen &f1, const float2 *tw1, const float *K, const __half *Kh,
                          const float *ksc) {
    switch (ct1) {
#define LAMINO_PENCIL(N)                                                                                       \
    case N:                                                                                                    \
        k_pencil<HALF, N><<<grid, pencil_threads(N), smem, s>>>(xa, n1, np1, l2, l3h, f1, tw1, K, \
                                                                              Kh, ksc);                        \
        break;
        LAMINO_PENCIL(1458)
        LAMINO_PENCIL(750)
        LAMINO_PENCIL(540)
        LAMINO_PENCIL(360)
        LAMINO_PENCIL(180)
        LAMINO_PENCIL(0)
#undef LAMINO_PENCIL
        default: throw Error(ERR_STATE, "no pencil kernel for this length");
    }
}

// the n2-pass kernels of the operator's n2 length (ct2: a compile-time length, 0
// = runtime schedule)
#define LAMINO_D2_LENGTHS(X) X(144) X(90) X(64) X(48) X(20) X(0)
static void launch_dim2_fwd(int ct2, dim3 grid, int kb, int smem, cudaStream_t s, const float2 *z1, int n1, int n2,
                            int l3h, int np1, const FftLen &f2, const float2 *tw2, float2 *xa) {
    switch (ct2) {
#define LAMINO_D2F(N)                                                                                           \
    case N:                                                                                                     \
        k_dim2_fwd<N><<<grid, N == 0 ? 256 : d2_threads(N, kb), smem, s>>>(z1, n1, n2, l3h, np1, f2, tw2, kb, xa); \
        break;
        LAMINO_D2_LENGTHS(LAMINO_D2F)
#undef LAMINO_D2F
        default: throw Error(ERR_STATE, "no n2-pass kernel for this length");
    }
}
static void launch_dim2_inv(int ct2, dim3 grid, int kb, int smem, cudaStream_t s, const float2 *xa, int n1, int n2,
                            int l3h, int np1, const FftLen &f2, const float2 *tw2, float2 *z1) {
    switch (ct2) {
#define LAMINO_D2I(N)                                                                                           \
    case N:                                                                                                     \
        k_dim2_inv<N><<<grid, N == 0 ? 256 : d2_threads(N, kb), smem, s>>>(xa, n1, n2, l3h, np1, f2, tw2, kb, z1); \
        break;
        LAMINO_D2_LENGTHS(LAMINO_D2I)
#undef LAMINO_D2I
        default: throw Error(ERR_STATE, "no n2-pass kernel for this length");
    }
}
static void raise_d2_smem(int bytes) {
#define LAMINO_D2_ATTR(N)                                           \
    raise_smem_limit((const void *)k_dim2_fwd<N>, bytes);           \
    raise_smem_limit((const void *)k_dim2_inv<N>, bytes);
    LAMINO_D2_LENGTHS(LAMINO_D2_ATTR)
#undef LAMINO_D2_ATTR
}

// the row kernels of the operator's packed n3 length (ct3: compile-time 729 or
// a CtRowSched length, 0 = runtime schedule)
#define LAMINO_ROW_LENGTHS(X) X(729) X(375) X(270) X(180) X(90) X(0)
static void launch_r2c(int ct3, unsigned grid, int rows, int smem, cudaStream_t s, const float *x, int64_t nrows,
                       int n3, const FftLen &f3, const int *pos3, const float2 *twh3, float2 *z1) {
    switch (ct3) {
#define LAMINO_R2C(N)                                                                                         \
    case N:                                                                                                   \
        k_r2c_rows<N><<<grid, rows_threads(N == 0 ? 1 : N, rows), smem, s>>>(x, nrows, n3, f3, pos3, twh3, rows, \
                                                                             z1);                             \
        break;
        LAMINO_ROW_LENGTHS(LAMINO_R2C)
#undef LAMINO_R2C
        default: throw Error(ERR_STATE, "no row kernel for this length");
    }
}
static void launch_c2r(int ct3, unsigned grid, int rows, int smem, cudaStream_t s, const float2 *z1, int64_t nrows,
                       int n3, const FftLen &f3, const int *pos3, const float2 *twh3, float *y) {
    switch (ct3) {
#define LAMINO_C2R(N)                                                                                         \
    case N:                                                                                                   \
        k_c2r_rows<N><<<grid, rows_threads(N == 0 ? 1 : N, rows), smem, s>>>(z1, nrows, n3, f3, pos3, twh3, rows, \
                                                                             y);                              \
        break;
        LAMINO_ROW_LENGTHS(LAMINO_C2R)
#undef LAMINO_C2R
        default: throw Error(ERR_STATE, "no row kernel for this length");
    }
}
static void raise_rows_smem(int bytes) {
#define LAMINO_ROWS_ATTR(N)                                           \
    raise_smem_limit((const void *)k_r2c_rows<N>, bytes);             \
    raise_smem_limit((const void *)k_c2r_rows<N>, bytes);
    LAMINO_ROW_LENGTHS(LAMINO_ROWS_ATTR)
#undef LAMINO_ROWS_ATTR
}

void Toeplitz::apply(const float *x3, float *y3, cudaStream_t s, bool low) {
    if (!z1.p || !xa.p) throw Error(ERR_STATE, "Toeplitz operator has no work buffers");
    const bool prof = profiling && (size_t)(nprof + 1) * (NSTAGE + 1) <= ev.size();
    cudaEvent_t *E = prof ? &ev[(size_t)nprof * (NSTAGE + 1)] : nullptr;
    const int64_t nrows = 3 * vol.n1 * vol.n2;
    const unsigned grows = (unsigned)((nrows + rows1 - 1) / rows1);
    const int smem_rows = rows1 * (int)L3h * (int)sizeof(float2);
    const int smem_d2 = d2_smem_values((int)L2, kb2) * (int)sizeof(float2);
    const int smem_pen = 3 * (int)L1 * (int)sizeof(float2);
    const dim3 gd2((unsigned)((vol.n1 + D2_IB - 1) / D2_IB), (unsigned)((L3h + kb2 - 1) / kb2), 3);
    const int n1 = (int)vol.n1, n2 = (int)vol.n2, n3 = (int)vol.n3, l2 = (int)L2, l3h = (int)L3h, np1 = (int)n1p;
    const unsigned gpen = (unsigned)(L2 * L3h);
    if (prof) LAMINO_CUDA(cudaEventRecord(E[0], s));
    launch_r2c(ct3, grows, rows1, smem_rows, s, x3, nrows, n3, f3, pos3.p, twh3.p, z1.p);
    LAMINO_LAUNCH("k_r2c_rows");
    if (prof) LAMINO_CUDA(cudaEventRecord(E[1], s));
    launch_dim2_fwd(ct2, gd2, kb2, smem_d2, s, z1.p, n1, n2, l3h, np1, f2, tw2.p, xa.p);
    LAMINO_LAUNCH("k_dim2_fwd");
    if (prof) LAMINO_CUDA(cudaEventRecord(E[2], s));
    const bool h = precision == PREC_FP16 || (precision == PREC_MIXED && low);
    if (h) launch_pencil<true>(ct1, gpen, smem_pen, s, xa.p, n1, np1, l2, l3h, f1, tw1.p, nullptr, Kh.p, Kscale.p);
    else launch_pencil<false>(ct1, gpen, smem_pen, s, xa.p, n1, np1, l2, l3h, f1, tw1.p, K.p, nullptr, nullptr);
    LAMINO_LAUNCH("k_pencil");
    if (prof) LAMINO_CUDA(cudaEventRecord(E[3], s));
    launch_dim2_inv(ct2, gd2, kb2, smem_d2, s, xa.p, n1, n2, l3h, np1, f2, tw2.p, z1.p);
    LAMINO_LAUNCH("k_dim2_inv");
    if (prof) LAMINO_CUDA(cudaEventRecord(E[4], s));
    launch_c2r(ct3, grows, rows1, smem_rows, s, z1.p, nrows, n3, f3, pos3.p, twh3.p, y3);
    LAMINO_LAUNCH("k_c2r_rows");
    if (prof) {
        LAMINO_CUDA(cudaEventRecord(E[5], s));
        ++nprof;
    }
}

void Toeplitz::quadforms(const float *x3, const std::vector<const Toeplitz *> &parts, double *acc,
                         cudaStream_t s) {
    if (!z1.p || !xa.p) throw Error(ERR_STATE, "Toeplitz operator has no work buffers");
    if (parts.empty()) return;
    for (const Toeplitz *t : parts) {
        if (!t || !t->has_fp32()) throw Error(ERR_ARG, "quadratic forms need operators with FP32 spectra");
        if (t->vol.n1 != vol.n1 || t->vol.n2 != vol.n2 || t->vol.n3 != vol.n3)
            throw Error(ERR_ARG, "quadratic forms need operators of this volume size");
    }
    const int64_t nrows = 3 * vol.n1 * vol.n2;
    const unsigned grows = (unsigned)((nrows + rows1 - 1) / rows1);
    const int smem_rows = rows1 * (int)L3h * (int)sizeof(float2);
    const int smem_d2 = d2_smem_values((int)L2, kb2) * (int)sizeof(float2);
    const int smem_pen = 3 * (int)L1 * (int)sizeof(float2);
    const dim3 gd2((unsigned)((vol.n1 + D2_IB - 1) / D2_IB), (unsigned)((L3h + kb2 - 1) / kb2), 3);
    const int n1 = (int)vol.n1, n2 = (int)vol.n2, n3 = (int)vol.n3, l2 = (int)L2, l3h = (int)L3h, np1 = (int)n1p;
    const unsigned gpen = (unsigned)(L2 * L3h);
    launch_r2c(ct3, grows, rows1, smem_rows, s, x3, nrows, n3, f3, pos3.p, twh3.p, z1.p);
    LAMINO_LAUNCH("k_r2c_rows");
    launch_dim2_fwd(ct2, gd2, kb2, smem_d2, s, z1.p, n1, n2, l3h, np1, f2, tw2.p, xa.p);
    LAMINO_LAUNCH("k_dim2_fwd");
    for (size_t g0 = 0; g0 < parts.size(); g0 += kMaxQuadSets) {
        QuadSets qs{};
        const int ng = (int)std::min<size_t>(kMaxQuadSets, parts.size() - g0);
        for (int g = 0; g < ng; ++g) qs.K[g] = parts[g0 + g]->K.p;
        switch (ct1) {
#define LAMINO_QUAD(N)                                                                                          \
    case N:                                                                                                     \
        k_pencil_quad<N><<<gpen, pencil_threads(N), smem_pen, s>>>(xa.p, n1, np1, l2, l3h, f1,    \
                                                                              tw1.p, qs, ng, acc + 3 * g0); \
        break;
            LAMINO_QUAD(1458)
            LAMINO_QUAD(750)
            LAMINO_QUAD(540)
            LAMINO_QUAD(360)
            LAMINO_QUAD(180)
            LAMINO_QUAD(0)
#undef LAMINO_QUAD
            default: throw Error(ERR_STATE, "no pencil kernel for this length");
        }
        LAMINO_LAUNCH("k_pencil_quad");
    }
}

void Toeplitz::set_shape(int rows, int kb) {
    if (rows < 1 || kb < 1) throw Error(ERR_ARG, "launch shape values must be positive");
    if (warp_rows(ct3) && rows > 8) throw Error(ERR_ARG, "rows of this length run one warp per row, at most 8 per CTA");
    const int64_t smem_rows = (int64_t)rows * L3h * (int64_t)sizeof(float2);
    const int64_t smem_d2 = (int64_t)d2_smem_values((int)L2, kb) * (int64_t)sizeof(float2);
    if (smem_rows > 200 * 1024 || smem_d2 > 200 * 1024) throw Error(ERR_ARG, "launch shape exceeds shared memory");
    rows1 = rows;
    kb2 = kb;
    raise_rows_smem((int)smem_rows);
    raise_d2_smem((int)smem_d2);
}

namespace {
std::mutex g_shape_mu;
std::map<std::array<int64_t, 4>, std::pair<int, int>> g_shape_cache;
}  // namespace

double Toeplitz::autotune(cudaStream_t s) {
    const std::array<int64_t, 4> key{L1, L2, L3, (int64_t)precision};
    {
        std::lock_guard<std::mutex> lk(g_shape_mu);
        auto it = g_shape_cache.find(key);
        if (it != g_shape_cache.end()) {
            set_shape(it->second.first, it->second.second);
            return 0.0;
        }
    }
    const int64_t n = 3 * vol.size();
    DevBuf<float> x((size_t)n), y((size_t)n);
    LAMINO_CUDA(cudaMemsetAsync(x.p, 0, x.bytes(), s));  // timing does not depend on the values
    cudaEvent_t e0, e1;
    LAMINO_CUDA(cudaEventCreate(&e0));
    LAMINO_CUDA(cudaEventCreate(&e1));
    const int r0 = rows1, k0 = kb2;
    double best = 1e300;
    int br = r0, bk = k0;
    const bool was_prof = profiling;
    profiling = false;
    for (int rows : {2, 4, 8}) {
        for (int kb : {2, 4, 8}) {
            try {
                set_shape(rows, kb);
            } catch (const Error &) {
                continue;
            }
            apply(x.p, y.p, s);  // warm-up
            LAMINO_CUDA(cudaEventRecord(e0, s));
            for (int r = 0; r < 2; ++r) apply(x.p, y.p, s);
            LAMINO_CUDA(cudaEventRecord(e1, s));
            LAMINO_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            LAMINO_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (ms / 2.0 < best) {
                best = ms / 2.0;
                br = rows;
                bk = kb;
            }
        }
    }
    profiling = was_prof;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    set_shape(br, bk);
    std::lock_guard<std::mutex> lk(g_shape_mu);
    g_shape_cache[key] = {br, bk};
    return best;
}

void Toeplitz::drop_work() {
    z1.release();
    xa.release();
}

}  // namespace lamino
