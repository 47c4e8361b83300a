// Solver kernels and loops for the laminography reconstructions (sm_100a).
//
// Arithmetic follows the reference's float expressions element by element
// (including where it promotes to double); reductions use FP64 accumulation
// with warp-shuffle trees instead of the reference's serial float sums.
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "fft_engine.cuh"
#include "solvers.cuh"

namespace lamino {

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------

namespace {
// Pinned host blocks of the calling thread, kept for reuse until it exits.
struct PinnedCache {
    std::vector<std::pair<double *, int>> free_;
    double *take(int n) {
        for (size_t i = 0; i < free_.size(); ++i)
            if (free_[i].second >= n) {
                double *p = free_[i].first;
                free_.erase(free_.begin() + (long)i);
                return p;
            }
        double *p = nullptr;
        LAMINO_CUDA(cudaMallocHost((void **)&p, sizeof(double) * std::max(n, 64)));
        return p;
    }
    void give(double *p, int n) { free_.emplace_back(p, std::max(n, 64)); }
    ~PinnedCache() {
        for (auto &b : free_) cudaFreeHost(b.first);
    }
};
PinnedCache &pinned_cache() {
    static thread_local PinnedCache c;
    return c;
}
}  // namespace

Reducer::Reducer(int n) : cap(n) {
    dbuf.alloc((size_t)n);
    d = dbuf.p;
    h = pinned_cache().take(n);
}
Reducer::~Reducer() {
    if (h) pinned_cache().give(h, cap);
}
void Reducer::zero(int n, cudaStream_t s) { LAMINO_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * n, s)); }
void Reducer::fetch(int n, cudaStream_t s) {
    LAMINO_CUDA(cudaMemcpyAsync(h, d, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    LAMINO_CUDA(cudaStreamSynchronize(s));
}

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double ws[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) ws[wid] = v;
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? ws[threadIdx.x] : 0.0;
    if (wid == 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;
}

__global__ void k_dot(const float *__restrict__ x, const float *__restrict__ y, int64_t n, double *out) {
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += (double)x[i] * (double)y[i];
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(out, s);
}

__global__ void k_sqdist3(const float *__restrict__ x, const float *__restrict__ y, int64_t V, double *out3) {
    const int c = blockIdx.y;
    double s = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
        float v = y ? (x[c * V + i] - y[c * V + i]) : x[c * V + i];
        s += (double)v * (double)v;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(out3 + c, s);
}

__device__ __forceinline__ int float_key(float f) {
    int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}

__global__ void k_max(const float *__restrict__ x, int64_t n, int *out) {
    int m = INT_MIN;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, float_key(x[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void k_key_to_double(const int *key, double *out) {
    int k = *key;
    int i = k >= 0 ? k : k ^ 0x7fffffff;
    *out = (double)__int_as_float(i);
}

void vec_dot(const float *x, const float *y, int64_t n, double *out, cudaStream_t s) {
    k_dot<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(x, y, n, out);
    LAMINO_LAUNCH("k_dot");
}
void vec_sqdist3(const float *x, const float *y, int64_t V, double *out3, cudaStream_t s) {
    dim3 g(grid_for(V, 256, 148 * 4), 3);
    k_sqdist3<<<g, 256, 0, s>>>(x, y, V, out3);
    LAMINO_LAUNCH("k_sqdist3");
}
void vec_max(const float *x, int64_t n, double *out, cudaStream_t s) {
    static_assert(sizeof(double) >= sizeof(int), "slot size");
    int *key = reinterpret_cast<int *>(out);  // use the slot's storage for the int key
    int init = INT_MIN;
    LAMINO_CUDA(cudaMemcpyAsync(key, &init, sizeof(int), cudaMemcpyHostToDevice, s));
    k_max<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(x, n, key);
    LAMINO_LAUNCH("k_max");
    k_key_to_double<<<1, 1, 0, s>>>(key, out);
    LAMINO_LAUNCH("k_key_to_double");
    LAMINO_CUDA(cudaStreamSynchronize(s));  // `init` lives on this stack frame
}

__global__ void k_lin2(float *__restrict__ out, float a, const float *__restrict__ x, float b,
                       const float *__restrict__ y, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a * x[i] + (y ? b * y[i] : 0.f);
}
void vec_lin2(float *out, float a, const float *x, float b, const float *y, int64_t n, cudaStream_t s) {
    k_lin2<<<grid_for(n, 256), 256, 0, s>>>(out, a, x, b, y, n);
    LAMINO_LAUNCH("k_lin2");
}
void vec_scale(float *out, float a, const float *x, int64_t n, cudaStream_t s) { vec_lin2(out, a, x, 0.f, nullptr, n, s); }

// One thread per (k, j) column of voxels (and component): k = blockIdx.x * kVoxX +
// threadIdx.x, j = blockIdx.y, and a contiguous run of the planes z = comp * n1 + i
// for blockIdx.z (PlaneRun), so no thread divides its index.  About 148 x 64 CTAs in all.
struct Idx3 {
    int i, j, k;
};
constexpr int kVoxX = 128;
// this CTA's contiguous run of planes [z0, z1) of nz: neighbouring planes follow
// each other in one thread, so their shared rows are still in L1
struct PlaneRun {
    int z0, z1;
    __device__ PlaneRun(int nz) {
        const int per = (nz + (int)gridDim.z - 1) / (int)gridDim.z;
        z0 = (int)blockIdx.z * per;
        z1 = min(nz, z0 + per);
    }
};
static dim3 vox_grid(Dims3 d, int ncomp) {
    if (d.n2 > 65535) throw Error(ERR_ARG, "n2 above 65535 is not supported by the voxel kernels");
    const int64_t gx = (d.n3 + kVoxX - 1) / kVoxX, gy = d.n2;
    const int64_t gz = std::max<int64_t>(1, std::min<int64_t>({d.n1 * ncomp, 65535, 148LL * 64 / (gx * gy) + 1}));
    return dim3((unsigned)gx, (unsigned)gy, (unsigned)gz);
}

// ---------------------------------------------------------------------------
// qGGMRF (src/qggmrf.cpp:25-95)
// ---------------------------------------------------------------------------

__constant__ float c_qggmrf_w[27] = {0.0302f, 0.037f, 0.0302f, 0.037f, 0.0523f, 0.037f, 0.0302f, 0.037f, 0.0302f,
                                     0.037f,  0.0523f, 0.037f, 0.0532f, 0.f,     0.0523f, 0.037f, 0.0523f, 0.037f,
                                     0.0302f, 0.037f, 0.0302f, 0.037f, 0.0523f, 0.037f, 0.0302f, 0.037f, 0.0302f};

// rho'(delta) with q = 2, C = 0.001, evaluated with the reference's float/double mix
// Derivative of the qGGMRF potential (src/qggmrf.cpp:42-57), q = 2, C = 0.001,
// in float (powf for |delta|^(q-p)); the reference evaluates parts of it in
// double, which moves the result by ~1e-7 relative.
struct QgConst {
    float qmp;         // q - p
    float inv_sqp;     // 1 / sigma^(q-p)
    float inv_sq;      // 1 / sigma^q
    float at_zero;     // q / (sigma^q C)
};
__device__ __forceinline__ float d_potential(float delta, const QgConst &k) {
    const float C = 0.001f;
    const float ad = fabsf(delta);
    if (!(ad > 0.f)) return k.at_zero;
    const float t1 = powf(ad, k.qmp) * k.inv_sqp;
    const float t3 = C + t1;
    const float r = 1.0f / t3;
    const float a = delta * r * k.inv_sq;
    return a * (2.0f - k.qmp * t1 * r);
}

// qGGMRF gradient: g[interior] += sum over the 26 neighbours of w_d rho'(x[c+d] -
// x[c]) (src/qggmrf.cpp:60-95), with each neighbour pair's derivative evaluated
// once.  rho'(-delta) = -rho'(delta) exactly in float for delta != 0 (the sign only
// flips a product), and both sides take rho'(0) = q / (sigma^q C) at delta = 0,
// so the 13 "forward" directions (dx = +1, and dx = 0 with (dy, dz) after
// (0, 0)) give every pair: the owner c keeps rho'(x[c+d] - x[c]) for its own
// sum and leaves the other side's term in shared memory.  A CTA owns a tile of
// QG_TJ x QG_TK columns (j, k) and marches through a run of planes i; its
// threads cover the tile plus a one-column halo, whose pairs reach into the
// tile.  The 26 terms of every voxel are added in the reference's order (dx,
// dy, dz from -1 to 1), as a direct 26-neighbour loop would add them.
constexpr int QG_TJ = 12, QG_TK = 32;  // 476 threads, 42 KB of shared memory
constexpr int QG_HJ = QG_TJ + 2, QG_HK = QG_TK + 2, QG_THREADS = QG_HJ * QG_HK;

__global__ void __launch_bounds__(QG_THREADS) k_qggmrf_pairs(float *__restrict__ g, const float *__restrict__ x,
                                                             int n1, int n2, int n3, QgConst kq) {
    __shared__ float q9[2][9][QG_THREADS];  // other-side terms of the dx = +1 pairs, planes i - 1 and i
    __shared__ float q4[4][QG_THREADS];     // other-side terms of the dx = 0 forward pairs, plane i
    const int t = threadIdx.x;
    const int tx = t % QG_HK, ty = t / QG_HK;
    const int k = blockIdx.x * QG_TK - 1 + tx, j = blockIdx.y * QG_TJ - 1 + ty;
    const bool col = j >= 0 && j < n2 && k >= 0 && k < n3;
    const bool fin = tx >= 1 && tx <= QG_TK && ty >= 1 && ty <= QG_TJ && j >= 1 && j <= n2 - 2 && k >= 1 &&
                     k <= n3 - 2;
    const int64_t sj = n3, si = (int64_t)n2 * n3;
    const PlaneRun pr(n1);
    float p9[9], p4[4];
    // own derivatives of plane i's forward pairs; other sides into shared memory
    auto pairs = [&](int i, int buf, bool with4) {
        if (!col || i < 0 || i >= n1) return;
        const int64_t c = i * si + j * sj + k;
        const float u = x[c];
        if (i + 1 < n1) {
#pragma unroll
            for (int dy = -1; dy < 2; ++dy)
#pragma unroll
                for (int dz = -1; dz < 2; ++dz) {
                    const int e = (dy + 1) * 3 + (dz + 1);
                    if (j + dy < 0 || j + dy >= n2 || k + dz < 0 || k + dz >= n3) continue;
                    const float delta = x[c + si + dy * sj + dz] - u;
                    const float pv = d_potential(delta, kq);
                    p9[e] = pv;
                    q9[buf][e][t] = !(fabsf(delta) > 0.f) ? kq.at_zero : -pv;
                }
        }
        if (with4) {
            const int dys[4] = {0, 1, 1, 1}, dzs[4] = {1, -1, 0, 1};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int dy = dys[e], dz = dzs[e];
                if (j + dy >= n2 || k + dz < 0 || k + dz >= n3) continue;
                const float delta = x[c + dy * sj + dz] - u;
                const float pv = d_potential(delta, kq);
                p4[e] = pv;
                q4[e][t] = !(fabsf(delta) > 0.f) ? kq.at_zero : -pv;
            }
        }
    };
    int buf = 0;
    pairs(pr.z0 - 1, buf, false);  // plane z0 - 1's dx = +1 pairs feed plane z0
    for (int i = pr.z0; i < pr.z1; ++i) {
        buf ^= 1;
        pairs(i, buf, true);
        __syncthreads();
        if (fin && i >= 1 && i <= n1 - 2) {
            const int pb = buf ^ 1;
            float sum = 0.f;
            // dx = -1: pairs owned by plane i - 1, at column (j + dy, k + dz), direction (1, -dy, -dz)
#pragma unroll
            for (int dy = -1; dy < 2; ++dy)
#pragma unroll
                for (int dz = -1; dz < 2; ++dz)
                    sum += c_qggmrf_w[(dy + 1) * 3 + (dz + 1)] *
                           q9[pb][(1 - dy) * 3 + (1 - dz)][t + dy * QG_HK + dz];
            // dx = 0, dy = -1: owned by (j - 1, k + dz), direction (0, 1, -dz)
            sum += c_qggmrf_w[9] * q4[3][t - QG_HK - 1];
            sum += c_qggmrf_w[10] * q4[2][t - QG_HK];
            sum += c_qggmrf_w[11] * q4[1][t - QG_HK + 1];
            // dx = 0, dy = 0: (0, 0, -1) owned by (j, k - 1); (0, 0, 1) own
            sum += c_qggmrf_w[12] * q4[0][t - 1];
            sum += c_qggmrf_w[14] * p4[0];
            // dx = 0, dy = 1: own
            sum += c_qggmrf_w[15] * p4[1];
            sum += c_qggmrf_w[16] * p4[2];
            sum += c_qggmrf_w[17] * p4[3];
            // dx = +1: own
#pragma unroll
            for (int e = 0; e < 9; ++e) sum += c_qggmrf_w[18 + e] * p9[e];
            g[i * si + j * sj + k] += sum;
        }
        __syncthreads();
    }
}

void qggmrf_add(float *g, const float *x, Dims3 d, float sigma, float p, cudaStream_t s) {
    if (d.n1 < 3 || d.n2 < 3 || d.n3 < 3) return;  // no interior voxels
    float sigma_q = std::pow(sigma, 2.0f);
    float sigma_qp = std::pow(sigma, 2.0f - p);
    QgConst kq;
    kq.qmp = 2.0f - p;
    kq.inv_sqp = (float)(1.0 / (double)sigma_qp);
    kq.inv_sq = (float)(1.0 / (double)sigma_q);
    kq.at_zero = (float)(2.0 / ((double)sigma_q * 0.001));
    if (d.n2 > (int64_t)65535 * QG_TJ) throw Error(ERR_ARG, "n2 too large for the qGGMRF kernel");
    const int64_t gx = (d.n3 + QG_TK - 1) / QG_TK, gy = (d.n2 + QG_TJ - 1) / QG_TJ;
    const int64_t gz = std::max<int64_t>(1, std::min<int64_t>({d.n1, 65535, 148LL * 6 / (gx * gy) + 1}));
    k_qggmrf_pairs<<<dim3((unsigned)gx, (unsigned)gy, (unsigned)gz), QG_THREADS, 0, s>>>(g, x, (int)d.n1, (int)d.n2,
                                                                                        (int)d.n3, kq);
    LAMINO_LAUNCH("k_qggmrf_pairs");
}

// ---------------------------------------------------------------------------
// finite differences (src/finitediff.cpp:8-71, include/bregman.h:34-36)
// ---------------------------------------------------------------------------

__device__ __forceinline__ bool interior(int i, int j, int k, int n1, int n2, int n3) {
    return i >= 1 && i < n1 - 1 && j >= 1 && j < n2 - 1 && k >= 1 && k < n3 - 1;
}

// grad along dim `dim` at (i,j,k): (u[+] - u[-]) / 2.0 on interior, else 0 (float result)
__device__ __forceinline__ float gdir(const float *__restrict__ u, int i, int j, int k, int n1, int n2, int n3,
                                      int dim) {
    if (!interior(i, j, k, n1, n2, n3)) return 0.f;
    int64_t c = ((int64_t)i * n2 + j) * n3 + k;
    int64_t st = dim == 0 ? (int64_t)n2 * n3 : (dim == 1 ? n3 : 1);
    return (u[c + st] - u[c - st]) * 0.5f;  // the reference's (float diff) / 2.0: halving is exact
}

__global__ void __launch_bounds__(kVoxX) k_grad_u(const float *__restrict__ u, int n1, int n2, int n3,
                                                  float *__restrict__ out3) {
    const int k = blockIdx.x * kVoxX + threadIdx.x, j = blockIdx.y;
    if (k >= n3) return;
    const int64_t V = (int64_t)n1 * n2 * n3;
    const PlaneRun pr(n1);
    for (int i = pr.z0; i < pr.z1; ++i) {
        const int64_t t = ((int64_t)i * n2 + j) * n3 + k;
        for (int dim = 0; dim < 3; ++dim) out3[dim * V + t] = gdir(u, i, j, k, n1, n2, n3, dim);
    }
}

// negative divergence of a 3-field given by an accessor
template <class F>
__device__ __forceinline__ float neg_div(const F &f, int i, int j, int k, int n1, int n2, int n3) {
    if (!interior(i, j, k, n1, n2, n3)) return 0.f;
    double a = -(double)(f(0, i + 1, j, k) - f(0, i - 1, j, k)) / 2.0;
    double b = (double)(f(1, i, j + 1, k) - f(1, i, j - 1, k)) / 2.0;
    double c = (double)(f(2, i, j, k + 1) - f(2, i, j, k - 1)) / 2.0;
    return (float)(a - b - c);
}

__global__ void __launch_bounds__(kVoxX) k_divergence(const float *__restrict__ du3, int n1, int n2, int n3,
                                                      float *__restrict__ out) {
    const int k = blockIdx.x * kVoxX + threadIdx.x, j = blockIdx.y;
    if (k >= n3) return;
    const int64_t V = (int64_t)n1 * n2 * n3;
    auto f = [&](int dim, int i, int j, int k) { return du3[dim * V + ((int64_t)i * n2 + j) * n3 + k]; };
    const PlaneRun pr(n1);
    for (int i = pr.z0; i < pr.z1; ++i) out[((int64_t)i * n2 + j) * n3 + k] = neg_div(f, i, j, k, n1, n2, n3);
}

// y += mu * divergence(grad_u(u)) for the 3 contiguous components.  The stencil
// reaches the centre and +-2 along each axis; a thread marches along i through a
// run of planes of one component (blockIdx.z = comp * runs + run) with
// u[i-2 .. i+2] of its (j, k) column in registers, so each voxel loads u[i+3]
// and the j and k neighbours only.  Same arithmetic as gdir / neg_div: float
// differences halved in float, combined in double.
__global__ void __launch_bounds__(kVoxX) k_laplacian_axpy(float *__restrict__ y, float mu, const float *__restrict__ u,
                                                          int n1, int n2, int n3) {
    const int k = blockIdx.x * kVoxX + threadIdx.x, j = blockIdx.y;
    if (k >= n3) return;
    const int runs = (int)gridDim.z / 3;
    const int comp = (int)blockIdx.z / runs, run = (int)blockIdx.z - comp * runs;
    const int per = (n1 + runs - 1) / runs;
    const int i0 = run * per, i1 = min(n1, i0 + per);
    if (i0 >= i1) return;
    const int64_t V = (int64_t)n1 * n2 * n3, s1 = (int64_t)n2 * n3;
    const bool jk_in = j >= 1 && j <= n2 - 2 && k >= 1 && k <= n3 - 2;
    const int64_t col = (int64_t)j * n3 + k;
    const float *uc = u + comp * V + col;
    float *yc = y + comp * V + col;
    auto ld = [&](int ii) { return (ii >= 0 && ii < n1) ? uc[ii * s1] : 0.f; };
    float w0 = ld(i0 - 2), w1 = ld(i0 - 1), w2 = ld(i0), w3 = ld(i0 + 1), w4 = ld(i0 + 2);
    for (int i = i0; i < i1; ++i) {
        float l = 0.f;
        if (jk_in && i >= 1 && i <= n1 - 2) {
            const float *pc = uc + (int64_t)i * s1;
            const float g0p = i + 1 <= n1 - 2 ? (w4 - w2) * 0.5f : 0.f;
            const float g0m = i - 1 >= 1 ? (w2 - w0) * 0.5f : 0.f;
            const float g1p = j + 1 <= n2 - 2 ? (pc[2 * n3] - w2) * 0.5f : 0.f;
            const float g1m = j - 1 >= 1 ? (w2 - pc[-2 * n3]) * 0.5f : 0.f;
            const float g2p = k + 1 <= n3 - 2 ? (pc[2] - w2) * 0.5f : 0.f;
            const float g2m = k - 1 >= 1 ? (w2 - pc[-2]) * 0.5f : 0.f;
            const double a = -(double)(g0p - g0m) / 2.0;
            const double b = (double)(g1p - g1m) / 2.0;
            const double c = (double)(g2p - g2m) / 2.0;
            l = (float)(a - b - c);
        }
        yc[(int64_t)i * s1] += l * mu;
        w0 = w1;
        w1 = w2;
        w2 = w3;
        w3 = w4;
        w4 = ld(i + 3);
    }
}

__global__ void __launch_bounds__(kVoxX) k_sb_rhs(const float *__restrict__ yT, const float *__restrict__ d9,
                                                  const float *__restrict__ b9, float mu, int n1, int n2, int n3,
                                                  float *__restrict__ rhs) {
    const int k = blockIdx.x * kVoxX + threadIdx.x, j = blockIdx.y;
    if (k >= n3) return;
    const int64_t V = (int64_t)n1 * n2 * n3;
    const PlaneRun pr(3 * n1);
    for (int z = pr.z0; z < pr.z1; ++z) {
        const int comp = z / n1, i = z - comp * n1;
        const float *dc = d9 + 3 * comp * V, *bc = b9 + 3 * comp * V;
        auto f = [&](int dim, int ii, int jj, int kk) {
            int64_t c = dim * V + ((int64_t)ii * n2 + jj) * n3 + kk;
            return dc[c] - bc[c];
        };
        const int64_t t = ((int64_t)i * n2 + j) * n3 + k;
        const float dv = neg_div(f, i, j, k, n1, n2, n3);
        rhs[comp * V + t] = yT[comp * V + t] + dv * mu;
    }
}

__global__ void __launch_bounds__(kVoxX) k_sb_shrink(const float *__restrict__ x3, float *__restrict__ d9,
                                                     float *__restrict__ b9, float lam, float mu, int n1, int n2,
                                                     int n3) {
    const int k = blockIdx.x * kVoxX + threadIdx.x, jj = blockIdx.y;
    if (k >= n3) return;
    const int64_t V = (int64_t)n1 * n2 * n3;
    const float eps = 1e-8f;
    const float thr = lam / mu;
    const PlaneRun prn(n1);
    for (int ii = prn.z0; ii < prn.z1; ++ii) {
        const int64_t t = ((int64_t)ii * n2 + jj) * n3 + k;
        const Idx3 p{ii, jj, k};
        float gx[9], tb[9];
        float sk = 1.0f * eps;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                gx[i * 3 + j] = gdir(x3 + i * V, p.i, p.j, p.k, n1, n2, n3, j);
                tb[i * 3 + j] = gx[i * 3 + j] + b9[(i * 3 + j) * V + t];
                sk += tb[i * 3 + j] * tb[i * 3 + j];
            }
        sk = sqrtf(sk);
        float m = fmaxf(sk - thr, 0.f);
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            float dv = m * (tb[q] / sk);
            d9[q * V + t] = dv;
            b9[q * V + t] += gx[q] - dv;
        }
    }
}

void grad_u(const float *u, Dims3 d, float *out3, cudaStream_t s) {
    k_grad_u<<<vox_grid(d, 1), kVoxX, 0, s>>>(u, (int)d.n1, (int)d.n2, (int)d.n3, out3);
    LAMINO_LAUNCH("k_grad_u");
}
void divergence(const float *du3, Dims3 d, float *out, cudaStream_t s) {
    k_divergence<<<vox_grid(d, 1), kVoxX, 0, s>>>(du3, (int)d.n1, (int)d.n2, (int)d.n3, out);
    LAMINO_LAUNCH("k_divergence");
}
void laplacian_axpy(float *y, float mu, const float *u, Dims3 d, cudaStream_t s) {
    dim3 g = vox_grid(d, 1);  // runs of planes per component, 3 components
    g.z = (unsigned)std::max<int64_t>(1, std::min<int64_t>(g.z, 65535 / 3)) * 3;
    k_laplacian_axpy<<<g, kVoxX, 0, s>>>(y, mu, u, (int)d.n1, (int)d.n2, (int)d.n3);
    LAMINO_LAUNCH("k_laplacian_axpy");
}
void sb_rhs(const float *yT3, const float *d9, const float *b9, float mu, Dims3 dims, float *rhs3, cudaStream_t s) {
    k_sb_rhs<<<vox_grid(dims, 3), kVoxX, 0, s>>>(yT3, d9, b9, mu, (int)dims.n1, (int)dims.n2, (int)dims.n3, rhs3);
    LAMINO_LAUNCH("k_sb_rhs");
}
void sb_shrink(const float *x3, float *d9, float *b9, float lam, float mu, Dims3 dims, cudaStream_t s) {
    k_sb_shrink<<<vox_grid(dims, 1), kVoxX, 0, s>>>(x3, d9, b9, lam, mu, (int)dims.n1, (int)dims.n2,
                                                    (int)dims.n3);
    LAMINO_LAUNCH("k_sb_shrink");
}

// ---------------------------------------------------------------------------
// ramp preconditioner (include/precond.h:33-87)
// ---------------------------------------------------------------------------

__global__ void k_filter_mul(float2 *__restrict__ S, const float *__restrict__ f, int64_t plane, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        float w = f[i % plane];
        S[i].x *= w;
        S[i].y *= w;
    }
}

// Along n2 the filter step (forward DFT, multiply by the ramp, inverse DFT) is a
// circulant convolution for each k3 column, z(:, k3) = G_k3 (*) x(:, k3), with
// G_k3[d] = sum_k2 f(k2, k3) cos(2 pi k2 d / n2): f is real and even in k2, so G_k3
// is real (and even).  One CTA per (n1 slice, RC_KB consecutive k3 columns): the
// column tile twice over in shared memory (so m - d + n2 needs no wrap), lanes on
// columns, warps on output rows, taps summed in order d = 0 .. n2-1.
constexpr int RC_KB = 32;
constexpr int RC_WARPS = 8;
constexpr int RC_ROWS = 9;  // output rows per thread: 8 warps x 9 rows cover n2 <= 72 in one pass
constexpr int kRampConvMaxN2 = 128;

__global__ void __launch_bounds__(RC_WARPS * 32) k_ramp_cols(float2 *__restrict__ S, const float *__restrict__ G,
                                                             int n2, int h3) {
    extern __shared__ float2 xs[];                                // [2 n2][RC_KB]
    float *gs = reinterpret_cast<float *>(xs + 2 * n2 * RC_KB);   // [n2][RC_KB]
    const int k3b = blockIdx.x * RC_KB;
    const int nk = min(RC_KB, h3 - k3b);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float2 *Sp = S + (int64_t)blockIdx.y * n2 * h3 + k3b;
    // load: the column tile (twice) and the kernels, 8 independent loads in flight per thread
    constexpr int LB = 8;
    const int total = n2 * RC_KB;
    for (int t0 = threadIdx.x; t0 < total; t0 += LB * RC_WARPS * 32) {
        float2 v[LB];
        float gv[LB];
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            const int t = t0 + u * RC_WARPS * 32;
            const int j = t / RC_KB, kk = t - j * RC_KB;
            const bool ok = t < total && kk < nk;
            v[u] = ok ? Sp[(int64_t)j * h3 + kk] : make_float2(0.f, 0.f);
            gv[u] = ok ? __ldg(G + (int64_t)j * h3 + k3b + kk) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            const int t = t0 + u * RC_WARPS * 32;
            if (t < total) {
                const int j = t / RC_KB, kk = t - j * RC_KB;
                xs[j * RC_KB + kk] = v[u];
                xs[(j + n2) * RC_KB + kk] = v[u];
                gs[j * RC_KB + kk] = gv[u];
            }
        }
    }
    __syncthreads();
    // rows m0 .. m0 + 8 of a thread need x[m0 + r - dd]: as dd grows the window
    // shifts by one, so it lives in a rotating register buffer, slot (r - dd) mod 9,
    // and each tap loads one new x (smem tile index m - dd + n2 stays in [1, 2 n2))
    for (int m0 = warp * RC_ROWS; m0 < n2; m0 += RC_ROWS * RC_WARPS) {
        float2 acc[RC_ROWS], buf[RC_ROWS];
#pragma unroll
        for (int r = 0; r < RC_ROWS; ++r) {
            acc[r] = make_float2(0.f, 0.f);
            // rows past n2 - 1 start from row n2 - 1 (inside the tile) and are never stored
            buf[r] = xs[(min(m0 + r, n2 - 1) + n2) * RC_KB + lane];
        }
        for (int d0 = 0; d0 < n2; d0 += RC_ROWS) {
#pragma unroll
            for (int u = 0; u < RC_ROWS; ++u) {
                const int dd = d0 + u;
                if (dd < n2) {
                    if (dd > 0) buf[(RC_ROWS - u) % RC_ROWS] = xs[(m0 - dd + n2) * RC_KB + lane];
                    const float g = gs[dd * RC_KB + lane];
#pragma unroll
                    for (int r = 0; r < RC_ROWS; ++r) {
                        const float2 x = buf[(r - u + RC_ROWS) % RC_ROWS];
                        acc[r].x = fmaf(g, x.x, acc[r].x);
                        acc[r].y = fmaf(g, x.y, acc[r].y);
                    }
                }
            }
        }
#pragma unroll
        for (int r = 0; r < RC_ROWS; ++r) {
            const int m = m0 + r;
            if (m < n2 && lane < nk) Sp[(int64_t)m * h3 + lane] = acc[r];
        }
    }
}

// Real transforms along n3 = N as Bluestein convolutions through the pencil's FFT
// pipeline: X[k] = sum_n x[n] e^{-2 pi i k n / N}
// = conj(w_k) sum_n (x_n conj(w_n)) w_{k-n} with w_m = e^{i pi m^2 / N}, a circular
// convolution of length M >= 2N - 1, taken as undo(FWD(u) . V) with V the
// transform of v (v_m = w_m for m < N, v_{M-m} = w_m for 0 < m < N, zero between),
// divided by M and stored in DIF position order.  The inverse uses conj(w) in
// place of w.  M = 1458 (the compile-time pipeline, fused outer stages) for
// 365 <= N <= 729; otherwise M = the next 2,3,5-smooth even length >= 2N - 1 on
// the runtime pipeline (same fused outer stages, FIXED = false), used for N >= 128
// with a prime factor above 7, where cuFFT slows down.  Two real rows travel as one
// complex row (a + i b), three complex rows per CTA; the spectra keep the R2C
// layout [row][N/2 + 1].
constexpr int kBlueM = 1458;
constexpr int kBlueHalf = 729;
constexpr int kBlueMaxM = 4096;

struct BlueR2CRows {
    const float *x;
    int64_t nrows, q0;
    int N, hm;  // hm: M / 2, the stride of zb
    const float2 *chirp;
    float2 *zb;  // 3 x M/2 results in shared memory
    __device__ __forceinline__ float2 get(int c, int i) const {
        const int64_t r = 2 * (q0 + c);
        if (i >= N || r >= nrows) return make_float2(0.f, 0.f);
        const float a = x[r * N + i], b = r + 1 < nrows ? x[(r + 1) * N + i] : 0.f;
        return c_mulc(make_float2(a, b), __ldg(chirp + i));
    }
    __device__ __forceinline__ bool want(int i) const { return i < N; }
    __device__ __forceinline__ void put(int c, int i, float2 v) const {
        zb[c * hm + i] = c_mulc(v, __ldg(chirp + i));
    }
};

// FWD(u), the pointwise product with V, undo: rows loaded and stored by `rows`
template <bool FIXED, class Rows>
__device__ __forceinline__ void blue_convolve(const Rows &rows, const FftLen &F, const float2 *__restrict__ V,
                                              const float2 *__restrict__ tw, float2 *sm, int M) {
    if constexpr (FIXED) {
        fft1458_load(rows, tw, sm, threadIdx.x);
        __syncthreads();
        ct_forward<kBlueM, 2>(sm, 3, kBlueM, tw, threadIdx.x, blockDim.x);
    } else {
        fftlead_any<false>(rows, F, sm, M, threadIdx.x, blockDim.x);
        __syncthreads();
        fft_forward(sm, 3, M, F, 2, threadIdx.x, blockDim.x);
    }
    for (int p = threadIdx.x; p < M; p += blockDim.x) {
        const float2 v = __ldg(V + p);
#pragma unroll
        for (int c = 0; c < 3; ++c) sm[c * M + p] = c_mul(sm[c * M + p], v);
    }
    __syncthreads();
    if constexpr (FIXED) {
        ct_inverse<kBlueM, 3, 2>(sm, 3, kBlueM, tw, threadIdx.x, blockDim.x);
        fft1458_store(rows, tw, sm, threadIdx.x);
    } else {
        fft_inverse(sm, 3, M, F, 2, threadIdx.x, blockDim.x);
        fftlead_any<true>(rows, F, sm, M, threadIdx.x, blockDim.x);
    }
}

template <bool FIXED>
__global__ void __launch_bounds__(256, 4) k_blue_r2c(const float *__restrict__ x, int64_t nrows, int N,
                                                     const float2 *__restrict__ chirp,
                                                     const float2 *__restrict__ V,
                                                     const float2 *__restrict__ tw, FftLen F,
                                                     float2 *__restrict__ S) {
    extern __shared__ float2 sm[];  // 3 transform rows of M, then 3 x M/2 results
    const int M = FIXED ? kBlueM : F.n, hm = M / 2;
    const int h = N / 2 + 1;
    const int64_t q0 = (int64_t)blockIdx.x * 3;
    const BlueR2CRows rows{x, nrows, q0, N, hm, chirp, sm + 3 * M};
    blue_convolve<FIXED>(rows, F, V, tw, sm, M);
    __syncthreads();
    // A = (Z_k + conj Z_{N-k}) / 2, B = (Z_k - conj Z_{N-k}) / 2i
    const float2 *zb = sm + 3 * M;
    for (int t = threadIdx.x; t < 3 * h; t += blockDim.x) {
        const int c = t / h, k = t - c * h;
        const int64_t r = 2 * (q0 + c);
        if (r >= nrows) continue;
        const float2 zk = zb[c * hm + k];
        const float2 zm = zb[c * hm + (k == 0 ? 0 : N - k)];
        S[r * h + k] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
        if (r + 1 < nrows) S[(r + 1) * h + k] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    }
}

struct BlueC2RRows {
    const float2 *S;
    float *y;
    int64_t nrows, q0;
    int N, h;
    const float2 *chirp;
    __device__ __forceinline__ float2 get(int c, int i) const {
        const int64_t r = 2 * (q0 + c);
        if (i >= N || r >= nrows) return make_float2(0.f, 0.f);
        const bool lo = i < h;
        const int k = lo ? i : N - i;
        float2 A = S[r * h + k];
        float2 B = r + 1 < nrows ? S[(r + 1) * h + k] : make_float2(0.f, 0.f);
        if (k == 0 || 2 * k == N) A.y = B.y = 0.f;  // as a C2R reads them: real
        if (!lo) {
            A.y = -A.y;
            B.y = -B.y;
        }
        return c_mul(make_float2(A.x - B.y, A.y + B.x), __ldg(chirp + i));  // (A + i B) w
    }
    __device__ __forceinline__ bool want(int i) const { return i < N; }
    __device__ __forceinline__ void put(int c, int i, float2 v) const {
        const int64_t r = 2 * (q0 + c);
        if (r >= nrows) return;
        const float2 z = c_mul(v, __ldg(chirp + i));
        y[r * N + i] = z.x;
        if (r + 1 < nrows) y[(r + 1) * N + i] = z.y;
    }
};

template <bool FIXED>
__global__ void __launch_bounds__(256, FIXED ? 5 : 4) k_blue_c2r(const float2 *__restrict__ S, int64_t nrows, int N,
                                                     const float2 *__restrict__ chirp,
                                                     const float2 *__restrict__ V,
                                                     const float2 *__restrict__ tw, FftLen F,
                                                     float *__restrict__ y) {
    extern __shared__ float2 sm[];  // 3 transform rows of M
    const int M = FIXED ? kBlueM : F.n;
    const BlueC2RRows rows{S, y, nrows, (int64_t)blockIdx.x * 3, N, N / 2 + 1, chirp};
    blue_convolve<FIXED>(rows, F, V, tw, sm, M);
}

// chirp w_n = e^{i pi n^2 / N}, the convolution kernels' spectra in DIF position
// order (forward: v; inverse: conj v; both / M) and the M-point twiddles, in FP64
static void blue_tables(int N, int M, std::vector<float2> &chirp, std::vector<float2> &vf, std::vector<float2> &vi,
                        std::vector<float2> &tw) {
    std::vector<double> wc(N), ws(N);
    for (int64_t n = 0; n < N; ++n) {
        const double a = M_PI * (double)((n * n) % (2 * (int64_t)N)) / (double)N;
        wc[n] = std::cos(a);
        ws[n] = std::sin(a);
    }
    chirp.resize(N);
    for (int n = 0; n < N; ++n) chirp[n] = make_float2((float)wc[n], (float)ws[n]);
    std::vector<double> vr(M, 0.0), vim(M, 0.0);
    for (int m = 0; m < N; ++m) {
        vr[m] = wc[m];
        vim[m] = ws[m];
        if (m > 0) {
            vr[M - m] = wc[m];
            vim[M - m] = ws[m];
        }
    }
    std::vector<double> cs(M), sn(M);
    for (int e = 0; e < M; ++e) {
        cs[e] = std::cos(-2.0 * M_PI * e / M);
        sn[e] = std::sin(-2.0 * M_PI * e / M);
    }
    const std::vector<int> pos = fft_positions(M, fft_schedule(M, true));
    vf.assign(M, make_float2(0.f, 0.f));
    vi.assign(M, make_float2(0.f, 0.f));
    std::vector<double> Fr(M), Fi(M);
    for (int k = 0; k < M; ++k) {
        double re = 0.0, im = 0.0;
        for (int m = 0; m < M; ++m) {
            if (vr[m] == 0.0 && vim[m] == 0.0) continue;
            const int e = (int)(((int64_t)k * m) % M);
            re += vr[m] * cs[e] - vim[m] * sn[e];
            im += vr[m] * sn[e] + vim[m] * cs[e];
        }
        Fr[k] = re;
        Fi[k] = im;
    }
    for (int k = 0; k < M; ++k) {
        // transform of conj v at k = conj(transform of v at -k)
        const int km = (M - k) % M;
        vf[pos[k]] = make_float2((float)(Fr[k] / M), (float)(Fi[k] / M));
        vi[pos[k]] = make_float2((float)(Fr[km] / M), (float)(-Fi[km] / M));
    }
    tw.resize(M);
    for (int e = 0; e < M; ++e) tw[e] = make_float2((float)cs[e], (float)sn[e]);
}

// largest prime factor of n
static int64_t largest_prime_factor(int64_t n) {
    int64_t p = 1;
    for (int64_t q = 2; q * q <= n; ++q)
        while (n % q == 0) {
            p = q;
            n /= q;
        }
    return n > 1 ? std::max(p, n) : p;
}

// schedule of the runtime Bluestein length M (lead 2) over the device twiddles
static FftLen blue_len(int M, const float2 *tw_dev) {
    const std::vector<int> r = fft_schedule(M, true);
    FftLen F{};
    F.n = M;
    F.ns = (int)r.size();
    int b = M;
    for (int s = 0; s < F.ns; ++s) {
        F.radix[s] = r[s];
        F.bsz[s] = b;
        F.dm[s] = FastDiv::make((uint32_t)(b / r[s]));
        F.dnb[s] = FastDiv::make((uint32_t)(M / r[s]));
        F.dblk[s] = FastDiv::make((uint32_t)(M / b));
        b /= r[s];
    }
    F.tw = tw_dev;
    return F;
}

RampPrecond::RampPrecond(Dims3 dd) : d(dd) {
    int64_t n2 = d.n2, n3 = d.n3, h3 = n3 / 2 + 1;
    std::vector<float> xf(h3), yf(n2), f(n2 * h3);
    for (int64_t i = 0; i < h3; ++i) xf[i] = (float)i / (float)n3;
    for (int64_t i = 0; i < n2; ++i) yf[i] = (i <= n2 / 2) ? (float)i / (float)n2 : (float)(i - n2) / (float)n2;
    // the 1/(n2 n3) normalisation of the c2r is folded into the filter
    float scale = (float)(1.0 / (double)(n2 * n3));
    for (int64_t j = 0; j < n2; ++j)
        for (int64_t i = 0; i < h3; ++i) f[j * h3 + i] = std::sqrt(xf[i] * xf[i] + yf[j] * yf[j]) * scale;
    spec.alloc(3 * d.n1 * n2 * h3);
    cols = n2 <= kRampConvMaxN2 && 3 * d.n1 <= 65535;
    if (cols) {
        // G[dd * h3 + k3] = sum_k2 f(k2, k3) cos(2 pi k2 dd / n2), in double
        std::vector<double> cs(n2);
        for (int64_t t = 0; t < n2; ++t) cs[t] = std::cos(2.0 * M_PI * (double)t / (double)n2);
        std::vector<float> g(n2 * h3);
        for (int64_t dd2 = 0; dd2 < n2; ++dd2)
            for (int64_t i = 0; i < h3; ++i) {
                double acc = 0.0;
                for (int64_t j = 0; j < n2; ++j) acc += (double)f[j * h3 + i] * cs[(j * dd2) % n2];
                g[dd2 * h3 + i] = (float)acc;
            }
        filt.alloc(n2 * h3);
        upload(filt.p, g.data(), g.size());
        const bool fixed = n3 >= 365 && n3 <= kBlueHalf;
        const int64_t mrt = next_smooth_even(2 * n3 - 1);
        blue = fixed || (n3 >= 128 && largest_prime_factor(n3) > 7 && mrt <= kBlueMaxM);
        blue_fixed = fixed;
        if (blue) {
            const int M = fixed ? kBlueM : (int)mrt;
            std::vector<float2> hc, hvf, hvi, htw;
            blue_tables((int)n3, M, hc, hvf, hvi, htw);
            chirp.alloc(hc.size());
            upload(chirp.p, hc.data(), hc.size());
            vfwd.alloc(hvf.size());
            upload(vfwd.p, hvf.data(), hvf.size());
            vinv.alloc(hvi.size());
            upload(vinv.p, hvi.data(), hvi.size());
            tw.alloc(htw.size());
            upload(tw.p, htw.data(), htw.size());
            blue_f = blue_len(M, tw.p);
            raise_smem_limit((const void *)k_blue_r2c<true>, (int)(3 * (kBlueM + kBlueHalf) * sizeof(float2)));
            raise_smem_limit((const void *)k_blue_c2r<true>, (int)(3 * kBlueM * sizeof(float2)));
            raise_smem_limit((const void *)k_blue_r2c<false>, (int)(3 * (M + M / 2) * sizeof(float2)));
            raise_smem_limit((const void *)k_blue_c2r<false>, (int)(3 * M * sizeof(float2)));
        } else {
            int n[1] = {(int)n3};
            r2c.make(1, n, CUFFT_R2C, (int)(3 * d.n1 * n2));
            c2r.make(1, n, CUFFT_C2R, (int)(3 * d.n1 * n2));
        }
        raise_smem_limit((const void *)k_ramp_cols, (int)(n2 * RC_KB * (2 * sizeof(float2) + sizeof(float))));
    } else {
        filt.alloc(n2 * h3);
        upload(filt.p, f.data(), f.size());
        int n[2] = {(int)n2, (int)n3};
        r2c.make(2, n, CUFFT_R2C, (int)(3 * d.n1));
        c2r.make(2, n, CUFFT_C2R, (int)(3 * d.n1));
    }
}

void RampPrecond::apply3(const float *r3, float *z3, cudaStream_t s) {
    int64_t h3 = d.n3 / 2 + 1, plane = d.n2 * h3;
    const int64_t nrows = 3 * d.n1 * d.n2;
    const unsigned gblue = (unsigned)(((nrows + 1) / 2 + 2) / 3);
    const int M = blue_f.n;
    if (blue && blue_fixed) {
        k_blue_r2c<true><<<gblue, 256, 3 * (kBlueM + kBlueHalf) * sizeof(float2), s>>>(
            r3, nrows, (int)d.n3, chirp.p, vfwd.p, tw.p, blue_f, spec.p);
        LAMINO_LAUNCH("k_blue_r2c");
    } else if (blue) {
        k_blue_r2c<false><<<gblue, 256, 3 * (M + M / 2) * sizeof(float2), s>>>(r3, nrows, (int)d.n3, chirp.p,
                                                                              vfwd.p, tw.p, blue_f, spec.p);
        LAMINO_LAUNCH("k_blue_r2c");
    } else {
        LAMINO_CUFFT(cufftSetStream(r2c.h, s));
        LAMINO_CUFFT(cufftExecR2C(r2c.h, const_cast<float *>(r3), (cufftComplex *)spec.p));
    }
    if (cols) {
        const dim3 grid((unsigned)((h3 + RC_KB - 1) / RC_KB), (unsigned)(3 * d.n1));
        const int smem = (int)(d.n2 * RC_KB * (2 * sizeof(float2) + sizeof(float)));
        k_ramp_cols<<<grid, RC_WARPS * 32, smem, s>>>(spec.p, filt.p, (int)d.n2, (int)h3);
        LAMINO_LAUNCH("k_ramp_cols");
    } else {
        k_filter_mul<<<grid_for(3 * d.n1 * plane, 256), 256, 0, s>>>(spec.p, filt.p, plane, 3 * d.n1 * plane);
        LAMINO_LAUNCH("k_filter_mul");
    }
    if (blue && blue_fixed) {
        k_blue_c2r<true><<<gblue, 256, 3 * kBlueM * sizeof(float2), s>>>(spec.p, nrows, (int)d.n3, chirp.p,
                                                                         vinv.p, tw.p, blue_f, z3);
        LAMINO_LAUNCH("k_blue_c2r");
    } else if (blue) {
        k_blue_c2r<false><<<gblue, 256, 3 * M * sizeof(float2), s>>>(spec.p, nrows, (int)d.n3, chirp.p, vinv.p,
                                                                     tw.p, blue_f, z3);
        LAMINO_LAUNCH("k_blue_c2r");
    } else {
        LAMINO_CUFFT(cufftSetStream(c2r.h, s));
        LAMINO_CUFFT(cufftExecC2R(c2r.h, (cufftComplex *)spec.p, z3));
    }
}

// ---------------------------------------------------------------------------
// CG (src/conjgrad.cpp:37-117)
// ---------------------------------------------------------------------------

__global__ void k_cg_update(float *__restrict__ x, float *__restrict__ r, const float *__restrict__ p,
                            const float *__restrict__ Ap, float alpha, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += p[i] * alpha;
        r[i] -= Ap[i] * alpha;
    }
}
__global__ void k_cg_dir(float *__restrict__ p, const float *__restrict__ z, float beta, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + p[i] * beta;
}

CgStats cgsolver(const OpFn &A, const float *y3, float *x3, Dims3 d, int max_iter, float tol, cudaStream_t s) {
    CgWork w(d);
    CgStats st = cgsolver(A, y3, x3, w, max_iter, tol, s);
    LAMINO_CUDA(cudaStreamSynchronize(s));
    return st;
}

CgStats cgsolver(const OpFn &A, const float *y3, float *x3, CgWork &w, int max_iter, float tol, cudaStream_t s) {
    const Dims3 d = w.d;
    const int64_t n = 3 * d.size();
    DevBuf<float> &r = w.r, &p = w.p, &z = w.z, &Ap = w.Ap;
    RampPrecond &M = w.M;
    Reducer &red = w.red;
    CgStats st;
    A(x3, Ap.p, s);
    vec_lin2(r.p, 1.f, y3, -1.f, Ap.p, n, s);
    M.apply3(r.p, z.p, s);
    LAMINO_CUDA(cudaMemcpyAsync(p.p, z.p, n * 4, cudaMemcpyDeviceToDevice, s));
    red.zero(1, s);
    vec_dot(z.p, r.p, n, red.d, s);
    red.fetch(1, s);
    double rs_old = red.h[0];
    for (int it = 0; it < max_iter; ++it) {
        A(p.p, Ap.p, s);
        red.zero(2, s);
        vec_dot(p.p, Ap.p, n, red.d, s);
        red.fetch(1, s);
        double pAp = red.h[0];
        if (std::fabs(pAp) < 1e-10) break;
        float alpha = (float)(rs_old / pAp);
        k_cg_update<<<grid_for(n, 256), 256, 0, s>>>(x3, r.p, p.p, Ap.p, alpha, n);
        LAMINO_LAUNCH("k_cg_update");
        M.apply3(r.p, z.p, s);
        red.zero(1, s);
        vec_dot(z.p, r.p, n, red.d, s);
        red.fetch(1, s);
        double rs_new = red.h[0];
        st.iters = it + 1;
        st.last_res = std::sqrt(std::fabs(rs_new));
        if (std::sqrt(std::fabs(rs_new)) < tol) break;
        float beta = (float)(rs_new / rs_old);
        k_cg_dir<<<grid_for(n, 256), 256, 0, s>>>(p.p, z.p, beta, n);
        LAMINO_LAUNCH("k_cg_dir");
        rs_old = rs_new;
    }
    return st;
}

CgStats cgsolver_refined(const OpFn &A_hi, const OpFn &A_lo, const float *y3, float *x3, Dims3 d, int inner,
                         int refinements, float tol, cudaStream_t s) {
    CgWork w(d);
    CgStats st = cgsolver_refined(A_hi, A_lo, y3, x3, w, inner, refinements, tol, s);
    LAMINO_CUDA(cudaStreamSynchronize(s));
    return st;
}

CgStats cgsolver_refined(const OpFn &A_hi, const OpFn &A_lo, const float *y3, float *x3, CgWork &w, int inner,
                         int refinements, float tol, cudaStream_t s) {
    const int64_t n = 3 * w.d.size();
    if (w.e1.n != (size_t)n) w.e1.alloc(n);
    if (w.e2.n != (size_t)n) w.e2.alloc(n);
    DevBuf<float> &r = w.e1, &dx = w.e2;
    Reducer &red = w.red;
    CgStats st;
    for (int k = 0; k < refinements; ++k) {
        A_hi(x3, r.p, s);
        vec_lin2(r.p, 1.f, y3, -1.f, r.p, n, s);  // r = y - A_hi x
        red.zero(1, s);
        vec_dot(r.p, r.p, n, red.d, s);
        red.fetch(1, s);
        st.last_res = std::sqrt(red.h[0]);
        if (st.last_res < tol) break;
        LAMINO_CUDA(cudaMemsetAsync(dx.p, 0, dx.bytes(), s));
        CgStats in = cgsolver(A_lo, r.p, dx.p, w, inner, tol, s);
        st.iters += in.iters;
        vec_lin2(x3, 1.f, x3, 1.f, dx.p, n, s);
    }
    return st;
}

// ---------------------------------------------------------------------------
// split Bregman (src/bregman.cpp:39-134)
// ---------------------------------------------------------------------------

int split_bregman(const OpFn &A, const float *yT3, float *x3, Dims3 d, float lam, float mu, int outer_max,
                  int inner_max, float tol, float xtol, cudaStream_t s) {
    return split_bregman_refined(A, OpFn(), 0, yT3, x3, d, lam, mu, outer_max, inner_max, tol, xtol, s);
}

int split_bregman_refined(const OpFn &A, const OpFn &A_lo, int refinements, const float *yT3, float *x3, Dims3 d,
                          float lam, float mu, int outer_max, int inner_max, float tol, float xtol, cudaStream_t s) {
    const int64_t V = d.size(), n = 3 * V;
    DevBuf<float> xold(n), dd(9 * V), bb(9 * V), rhs(n);
    LAMINO_CUDA(cudaMemcpyAsync(xold.p, x3, n * 4, cudaMemcpyDeviceToDevice, s));
    LAMINO_CUDA(cudaMemsetAsync(dd.p, 0, dd.bytes(), s));
    LAMINO_CUDA(cudaMemsetAsync(bb.p, 0, bb.bytes(), s));
    OpFn Ap = [&](const float *u, float *out, cudaStream_t st) {
        A(u, out, st);
        laplacian_axpy(out, mu, u, d, st);
    };
    OpFn Ap_lo = [&](const float *u, float *out, cudaStream_t st) {
        A_lo(u, out, st);
        laplacian_axpy(out, mu, u, d, st);
    };
    Reducer red(8);
    CgWork work(d);
    int it = 0;
    for (; it < outer_max; ++it) {
        sb_rhs(yT3, dd.p, bb.p, mu, d, rhs.p, s);
        // x = cgsolver(Ap, rhs, x_old, ...)
        LAMINO_CUDA(cudaMemcpyAsync(x3, xold.p, n * 4, cudaMemcpyDeviceToDevice, s));
        if (A_lo && refinements > 0)
            cgsolver_refined(Ap, Ap_lo, rhs.p, x3, work, inner_max, refinements, tol, s);
        else
            cgsolver(Ap, rhs.p, x3, work, inner_max, tol, s);
        sb_shrink(x3, dd.p, bb.p, lam, mu, d, s);
        red.zero(6, s);
        vec_sqdist3(x3, xold.p, V, red.d, s);
        vec_sqdist3(xold.p, nullptr, V, red.d + 3, s);
        red.fetch(6, s);
        double nd = 0.0;
        for (int i = 0; i < 3; ++i) nd += std::sqrt(red.h[i]) / (std::sqrt(red.h[3 + i]) + 1e-8);
        LAMINO_CUDA(cudaMemcpyAsync(xold.p, x3, n * 4, cudaMemcpyDeviceToDevice, s));
        if (nd < xtol) { ++it; break; }
    }
    LAMINO_CUDA(cudaStreamSynchronize(s));
    return it;
}

// ---------------------------------------------------------------------------
// Nesterov (src/nagopt.cpp:116-209)
// ---------------------------------------------------------------------------

__global__ void k_extrap(float *__restrict__ y, const float *__restrict__ x, const float *__restrict__ xo, float beta,
                         int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = x[i] + (x[i] - xo[i]) * beta;
}

// One host read per line-search step: the losses of x and y, |g| and the
// x-change norms (used when the step is accepted) are reduced on the device
// into one buffer and fetched together, where the reference reads each as it
// goes; the values and the decisions are the same.  The reference evaluates
// loss(x) once more after each line search (src/nagopt.cpp); x has not changed
// since the line search's last evaluation, so that value is reused.
NagSolve::NagSolve(GradFn grad, LossTerms loss, float *x3, Dims3 d, int max_iters, float lipschitz, float tol,
                   float xtol, int max_inner, cudaStream_t s)
    : grad_(std::move(grad)), loss_(std::move(loss)), x_(x3), d_(d), max_iters_(max_iters), max_inner_(max_inner),
      tol_(tol), xtol_(xtol), s_(s), xold_(3 * d.size()), y_(3 * d.size()), g_(3 * d.size()),
      red_(2 * loss_.nterms + 9) {
    step_ = step_prev_ = (float)(0.1 / lipschitz);
    LAMINO_CUDA(cudaMemcpyAsync(xold_.p, x_, 3 * d.size() * 4, cudaMemcpyDeviceToDevice, s_));
    done_ = max_iters_ <= 0 || max_inner_ <= 0;
}

// slots: [loss terms of x][loss terms of y][|g_c|^2][|x_c - xold_c|^2][|x_c|^2]
void NagSolve::enqueue() {
    const int64_t V = d_.size(), n = 3 * V;
    const int M = loss_.nterms;
    double *const gsl = red_.d + 2 * M;
    const float beta = (float)(tnew_ * (1.0 / t_ - 1.0));
    tnew_ = 0.5 * (std::sqrt(std::pow(t_, 4) + 4 * std::pow(t_, 2)) - std::pow(t_, 2));
    k_extrap<<<grid_for(n, 256), 256, 0, s_>>>(y_.p, x_, xold_.p, beta, n);
    LAMINO_LAUNCH("k_extrap");
    grad_(y_.p, g_.p, s_);
    vec_lin2(x_, 1.f, y_.p, -step_, g_.p, n, s_);
    red_.zero(2 * M + 9, s_);
    loss_.enqueue(x_, red_.d, s_);
    loss_.enqueue(y_.p, red_.d + M, s_);
    vec_sqdist3(g_.p, nullptr, V, gsl, s_);
    vec_sqdist3(x_, xold_.p, V, gsl + 3, s_);
    vec_sqdist3(x_, nullptr, V, gsl + 6, s_);
    LAMINO_CUDA(cudaMemcpyAsync(red_.h, red_.d, sizeof(double) * (2 * M + 9), cudaMemcpyDeviceToHost, s_));
}

bool NagSolve::finish() {
    const int M = loss_.nterms;
    const double *h = red_.h;
    const double ex = loss_.value(h), ey = loss_.value(h + M);
    double gy = 0.0;
    for (int i = 0; i < 3; ++i) gy += std::sqrt(h[2 * M + i]);
    gy *= 0.5 * step_;
    bool line_search_over = false;
    if (ex > ey + gy) {
        step_ *= 0.9f;
    } else {
        step_ = step_prev_;
        t_ = tnew_;
        double xe = 0, xn = 0;
        for (int i = 0; i < 3; ++i) {
            xe += std::sqrt(h[2 * M + 3 + i]);
            xn += std::sqrt(h[2 * M + 6 + i]);
        }
        xerr_ = xe / xn;
        if (xerr_ < xtol_) {
            ++it_;
            done_ = true;
            return true;
        }
        LAMINO_CUDA(cudaMemcpyAsync(xold_.p, x_, 3 * d_.size() * 4, cudaMemcpyDeviceToDevice, s_));
        line_search_over = true;
    }
    if (!line_search_over && ++inner_ < max_inner_) return false;
    // end of an outer iteration: its loss is ex (x unchanged since)
    inner_ = 0;
    ++it_;
    if (ex < tol_ || it_ >= max_iters_) done_ = true;
    return done_;
}

int nagopt(const GradFn &grad, const LossTerms &loss, float *x, Dims3 d, int max_iters, float lipschitz, float tol,
           float xtol, int max_inner, cudaStream_t s) {
    NagSolve nag(grad, loss, x, d, max_iters, lipschitz, tol, xtol, max_inner, s);
    while (!nag.done()) {
        nag.enqueue();
        LAMINO_CUDA(cudaStreamSynchronize(s));
        nag.finish();
    }
    LAMINO_CUDA(cudaStreamSynchronize(s));
    return nag.iterations();
}

// ---------------------------------------------------------------------------
// power iteration
// ---------------------------------------------------------------------------

__global__ void k_uniform(float *__restrict__ x, int64_t n, unsigned long long seed) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        x[i] = (float)((z >> 40) * (1.0 / 16777216.0));
    }
}

// x = Ax / sqrt(*sq) with the factor formed in double and rounded to float, as
// the host does in the loop below
__global__ void k_scale_inv_norm(float *__restrict__ out, const float *__restrict__ x, const double *sq, int64_t n) {
    const float a = (float)(1.0 / sqrt(*sq));
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a * x[i] + 0.f;
}

double lipschitz(const OpFn &A, Dims3 d, int max_iters, double tol, unsigned long long seed, cudaStream_t s) {
    const int64_t n = 3 * d.size();
    DevBuf<float> x(n), Ax(n);
    if (tol == 0.0 && max_iters > 0) {
        // no early stop: the whole iteration stays on the device (the norms into
        // one slot each, the normalisation read from the slot) and the norms are
        // fetched once; same arithmetic as the loop below
        Reducer red(max_iters + 1);
        red.zero(max_iters + 1, s);
        k_uniform<<<grid_for(n, 256), 256, 0, s>>>(x.p, n, seed);
        LAMINO_LAUNCH("k_uniform");
        vec_dot(x.p, x.p, n, red.d, s);
        k_scale_inv_norm<<<grid_for(n, 256), 256, 0, s>>>(x.p, x.p, red.d, n);
        LAMINO_LAUNCH("k_scale_inv_norm");
        for (int i = 0; i < max_iters; ++i) {
            A(x.p, Ax.p, s);
            vec_dot(Ax.p, Ax.p, n, red.d + 1 + i, s);
            k_scale_inv_norm<<<grid_for(n, 256), 256, 0, s>>>(x.p, Ax.p, red.d + 1 + i, n);
            LAMINO_LAUNCH("k_scale_inv_norm");
        }
        red.fetch(max_iters + 1, s);
        double L = 0.0;
        for (int i = 0; i < max_iters; ++i) {
            const double nA = std::sqrt(red.h[1 + i]);
            if (nA < 1e-12) return 0.0;
            L = nA;
        }
        return L;
    }
    Reducer red(2);
    k_uniform<<<grid_for(n, 256), 256, 0, s>>>(x.p, n, seed);
    LAMINO_LAUNCH("k_uniform");
    red.zero(1, s);
    vec_dot(x.p, x.p, n, red.d, s);
    red.fetch(1, s);
    vec_scale(x.p, (float)(1.0 / std::sqrt(red.h[0])), x.p, n, s);
    double L = 0.0;
    for (int i = 0; i < max_iters; ++i) {
        A(x.p, Ax.p, s);
        red.zero(1, s);
        vec_dot(Ax.p, Ax.p, n, red.d, s);
        red.fetch(1, s);
        double nA = std::sqrt(red.h[0]);
        if (nA < 1e-12) return 0.0;
        vec_scale(x.p, (float)(1.0 / nA), Ax.p, n, s);
        if (std::fabs(nA - L) < tol) { L = nA; break; }
        L = nA;
    }
    LAMINO_CUDA(cudaStreamSynchronize(s));
    return L;
}

}  // namespace lamino
