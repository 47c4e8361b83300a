// MBIR drivers (src/mbir_cg.cpp, src/mbir_sb.cpp, src/mbir3.cpp) on the GPU path.
#pragma once

#include <array>
#include <memory>
#include <vector>

#include "common.cuh"
#include "geometry.cuh"
#include "nufft.cuh"
#include "solvers.cuh"
#include "toeplitz.cuh"

namespace lamino {

// Toeplitz with FP32 spectra, with FP16 spectra, the NUFFT form, or Toeplitz with
// both spectra (FP16 correction solves inside FP32-residual refinement cycles).
enum OpKind : int { OP_TOEPLITZ_FP32 = 0, OP_TOEPLITZ_FP16 = 1, OP_NUFFT = 2, OP_TOEPLITZ_MIXED = 3 };

struct ReconParams {  // include/config.h:146-158 defaults
    int max_iters = 50;
    int inner_iters = 3;
    float sigma = 1000.f, p = 1.2f, lambda = 0.1f, mu = 10.f, tol = 1e-5f, xtol = 1e-5f;
    float pad_factor = 1.4142f;
    int op_kind = OP_TOEPLITZ_FP32;
    double eps = 1.2e-6;
    int refinements = 3;  // refinement cycles per linear solve with OP_TOEPLITZ_MIXED
    int use_graphs = 1;   // replay each solver iteration's operator work as a CUDA graph
    int autotune = 1;     // pick launch shapes / bin layouts by timing (cached per size)
};

struct Dataset {
    const float *proj;  // device, (nproj, nrows, ncols)
    int64_t nproj, nrows, ncols;
    const float *angles;  // host
    float gamma;
};

// Padded volume dims n + 2 floor(n (PAD-1) / 2) (src/mbir_sb.cpp:50-60).
int64_t pad_dim(int64_t n, float factor_minus_one);

// pad2d (include/padding.h:94-131) fused with the 1/max normalisation; returns new
// dims; `out` is reallocated only when smaller than the padded projections
void normalize_pad2d(const float *proj, int64_t np, int64_t nr, int64_t nc, float inv_max, float factor,
                     DevBuf<float> &out, int64_t &onr, int64_t &onc, cudaStream_t s);
// crop3d (include/padding.h:207-232, symmetric), 3 components
void crop3d3(const float *in, Dims3 from, Dims3 to, float *out, cudaStream_t s);

// Estimated peak device bytes of one mbir() call (admission control).
int64_t mbir_footprint(int method, const std::vector<std::array<int64_t, 3>> &proj_dims, Dims3 recon,
                       const ReconParams &prm);

// Host wall-clock seconds of the last mbir() call on this thread: setup
// (normalisation, padding, grids, adjoints), operator build, solve; and the
// number of normal-operator applications of the solve.
struct MbirPhases {
    double setup_s = 0, build_s = 0, solve_s = 0;
    int64_t applies = 0;
    double plan_s = 0, adjoint_s = 0, tune_s = 0;  // parts: NUFFT plan, setup adjoints, autotuning
};
MbirPhases &last_mbir_phases();

// method 1 = CG, 2 = split Bregman, 3 = NAG + qGGMRF.  out3: recon dims, device.
void mbir(int method, const std::vector<Dataset> &data, Dims3 recon, const ReconParams &prm, float *out3,
          cudaStream_t s);

class GraphedOp;
// One reconstruction in three parts: prepare() (normalisation, padding, grids,
// setup adjoints, operators; for MBIR3 also the Lipschitz constant and the NAG
// state), the solve, finish() (crop into out3, phase times).  mbir() runs the
// three in a row; the batched form steps several MBIR3 solves together.
// prepare() runs on stream s; the solve and finish() on solve_stream (s when
// null), which waits for the end of prepare().  Buffers allocated while an
// AllocStreamScope is active are freed on their allocation stream when the
// job is destroyed, after finish() has synchronised the solve stream.
class MbirJob {
  public:
    MbirJob(int method, const std::vector<Dataset> &data, Dims3 recon, const ReconParams &prm, float *out3,
            cudaStream_t s, cudaStream_t solve_stream = nullptr);
    ~MbirJob();
    MbirJob(const MbirJob &) = delete;
    MbirJob &operator=(const MbirJob &) = delete;
    void prepare();
    void solve();
    void finish();
    int method() const { return method_; }
    NagSolve *nag() { return nag_.get(); }
    cudaStream_t solve_stream() const { return ss_; }

  private:
    int method_;
    std::vector<Dataset> data_;
    Dims3 recon_, od_;
    ReconParams prm_;
    float *out3_;
    cudaStream_t s_, ss_;
    int64_t V_ = 0, n_ = 0;
    std::unique_ptr<NufftPlan> plan_;
    std::vector<std::unique_ptr<Geom>> geoms_;
    std::vector<const Geom *> gptr_;
    DevBuf<float> yT_, x_, Sx_;
    std::unique_ptr<Toeplitz> T_;
    std::vector<std::unique_ptr<Toeplitz>> Tg_;
    std::vector<const Toeplitz *> parts_;
    OpFn A_raw_, A_lo_raw_;
    std::vector<OpFn> Ag_;
    std::unique_ptr<GraphedOp> gA_, gA_lo_, gGrad_, gLoss_;
    std::unique_ptr<NagSolve> nag_;
    int64_t extra_applies_ = 0;
    double t0_ = 0, t_plan_ = 0, t_setup_ = 0, t_build_ = 0, t_adj_ = 0, t_tune_ = 0;
};


}  // namespace lamino
