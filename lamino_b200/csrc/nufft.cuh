// ES-kernel 3-D NUFFT on the laminography planes (type 1 / type 2), plus the
// projection-space stages of the forward and adjoint operators.
#pragma once

#include <memory>
#include <vector>

#include "common.cuh"
#include "geometry.cuh"

namespace lamino {

// Width / shape of the exponential-of-semicircle kernel for a tolerance at
// oversampling 2 (Barnett, Magland, af Klinteberg, SIAM J. Sci. Comput. 2019).
inline int es_width(double eps) {
    int w = (int)std::ceil(std::log10(10.0 / eps));
    return w < 2 ? 2 : w;
}
int64_t next_smooth_even(int64_t n);

// Partition of the fine grid into bins of b1 x b2 x b3 cells.  A point belongs
// to the bin holding the first cell of its kernel footprint, so its w^3 taps
// stay inside the bin's tile of (b + w - 1) cells per dimension, which one CTA
// stages in shared memory.  Tile rows are r3 >= t3 cells apart with
// r3 = w (mod 16): the w x w (t2, t3) taps that consecutive lanes take then fall
// in distinct shared-memory banks.
struct BinLayout {
    int b1 = 8, b2 = 8, b3 = 8;
    int nb1 = 0, nb2 = 0, nb3 = 0;
    int t1 = 0, t2 = 0, t3 = 0, r3 = 0;
    __host__ __device__ int64_t nbins() const { return (int64_t)nb1 * nb2 * nb3; }
    __host__ __device__ int64_t tile_cells() const { return (int64_t)t1 * t2 * r3; }
};

// Point ids of one geometry grouped by bin (counting sort), with bin offsets.
struct SortedPoints {
    uint64_t uid = 0;
    bool paired = false;     // ids of antipodal pairs (the adjoint), else of points
    uint64_t last_use = 0;
    DevBuf<uint32_t> perm;   // npts
    DevBuf<uint32_t> start;  // nbins + 1
};

struct NufftPlan {
    Dims3 vol;                // recon volume (n1, n2, n3), n3 fastest
    int64_t nf1, nf2, nf3;    // fine grid paired with n1 (z), n2 (y), n3 (x)
    int w = 7;
    float beta = 16.1f;
    double eps = 1.2e-6;
    DevBuf<float> ip1, ip2, ip3;   // 1 / p(k) per mode index along each dim
    DevBuf<float2> gin;            // 3 fine grids: deconvolved modes (zero elsewhere)
    DevBuf<float2> gwork;          // 3 fine grids: FFT outputs / spread accumulators
    FftPlan fft3;                  // batched 3 x C2C 3-D on the fine grid
    // projection-space workspace (largest geometry seen), with its 2-D plan
    DevBuf<float2> pbuf;
    FftPlan fft2;
    int64_t f2_np = -1, f2_nr = -1, f2_nc = -1;
    // bin-sorted point orders of the geometries used with this plan (bounded LRU)
    BinLayout bins;
    std::vector<std::unique_ptr<SortedPoints>> sorted;
    uint64_t use_clock = 0;
    static constexpr int kMaxSorted = 16;

    NufftPlan(Dims3 d, double eps);
    int64_t nf() const { return nf1 * nf2 * nf3; }
    void ensure_proj(const Geom &g, cudaStream_t s);
    // bin layout for b1 x b2 x b3 bins (drops cached point orders)
    void set_bins(int b1, int b2, int b3);
    // the geometry's bin-sorted order of points, or of antipodal point pairs
    // (built on first use, then cached)
    const SortedPoints &sort_points(const Geom &g, cudaStream_t s, bool paired = false);
    const SortedPoints *find_sorted(const Geom &g, bool paired = false) const;
    // time candidate bin layouts and keep the fastest for objective 0 (adjoint of
    // the first geometry, including its sort: a setup pass) or 1 (the sum over
    // the geometries of sysmat, sorted orders reused: a solver's operator);
    // cached per (fine grid, width, objective, points) for the process.  Returns
    // the best time in ms (0 when taken from the cache).
    double autotune_bins(const std::vector<const Geom *> &gs, int objective, cudaStream_t s);
    void drop_sorted() { sorted.clear(); }

    // --- operators (device pointers; volumes are 3 contiguous components) ---
    // forward projection (src/projection.cpp:42-77)
    void forward(const Geom &g, const float *m3, float *proj, cudaStream_t s);
    // adjoint (src/projection.cpp:90-126); accumulate adds into m3
    void adjoint(const Geom &g, const float *proj, float *m3, bool accumulate, cudaStream_t s);
    // sum over geometries of sysmat (src/gradient.cpp:34-89), NUFFT form
    void normal(const std::vector<const Geom *> &gs, const float *x3, float *y3, cudaStream_t s);
    // same sum over geometries given as a pointer array (no host containers)
    void normal_ptrs(const Geom *const *gs, int ng, const float *x3, float *y3, cudaStream_t s);
    // raw transforms on one geometry (FINUFFT-level boundary, complex data)
    void type2(const Geom &g, const float2 *modes, float2 *c, cudaStream_t s);
    void type1(const Geom &g, const float2 *c, float2 *modes, cudaStream_t s);

    // internals
    void normal_impl(const Geom *const *gs, int ng, bool may_sort, const float *x3, float *y3, cudaStream_t s);
    void normal_points(const Geom *const *gs, int ng, bool may_sort, cudaStream_t s);
    void pad_real(const float *x3, int ncomp, cudaStream_t s);
    void pad_complex(const float2 *f, cudaStream_t s);
    void fft_fine(int sign, int ncomp, cudaStream_t s);
    void extract_real(float *y3, int ncomp, float scale, bool accumulate, cudaStream_t s);
};

}  // namespace lamino
