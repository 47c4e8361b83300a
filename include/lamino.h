/*
 * lamino_b200 C ABI: the GPU (sm_100a) laminography operator and solvers.
 *
 * Drop-in boundary for the reference's FINUFFT/OpenMP path.  Every entry point
 * names the reference interface it replaces (paths relative to the reference
 * project root).  Conventions:
 *   - All functions return 0 on success or a LAMINO_ERR_* code; the message of
 *     the last failure on the calling thread is lamino_last_error().  No C++
 *     exception crosses this boundary.
 *   - Array pointers may be host or device memory (detected per call); host
 *     buffers are staged through device memory inside the call.
 *   - Volumes are 3 contiguous float32 components [3][n1][n2][n3] (n3 fastest),
 *     in the reference's internal order (n1, n2, n3) = (W, T, H).
 *   - Projections are float32 [nproj][nrows][ncols] (ncols fastest).
 *   - `stream` is a cudaStream_t (NULL = default stream).  Calls with host
 *     buffers synchronise the stream before returning.
 *   - Handles are thread-compatible: one thread at a time per handle.
 */
#ifndef LAMINO_H
#define LAMINO_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LAMINO_OK 0
#define LAMINO_ERR_ARG 1
#define LAMINO_ERR_OOM 2
#define LAMINO_ERR_CUDA 3
#define LAMINO_ERR_CUFFT 4
#define LAMINO_ERR_TIMEOUT 5
#define LAMINO_ERR_NONFINITE 6
#define LAMINO_ERR_STATE 7

typedef struct lamino_geom_s *lamino_geom_t;     /* one gamma dataset's polar grid */
typedef struct lamino_plan_s *lamino_plan_t;     /* NUFFT plan for one volume size */
typedef struct lamino_normal_s *lamino_normal_t; /* Toeplitz sum_gamma sysmat */
typedef struct lamino_op_s *lamino_op_t;         /* any normal operator, for the solvers */

/* Message of the last failure on this thread ("" if none). */
const char *lamino_last_error(void);
/* Library version string. */
const char *lamino_version(void);

/* ---- geometry ------------------------------------------------------------
 * Replaces tomocam::PolarGrid<float>::PolarGrid(angles, nrows, ncols, gamma)
 * (include/polar_grid.h:44-75).  `angles` (radians) and `gamma` are host values.
 */
int lamino_geom_create(const float *angles, int64_t nproj, int64_t nrows, int64_t ncols, float gamma,
                       lamino_geom_t *out);
/* Materialises the PolarGrid x, y, z arrays (each nproj*nrows*ncols floats). */
int lamino_geom_points(lamino_geom_t g, float *x, float *y, float *z, void *stream);
int lamino_geom_destroy(lamino_geom_t g);

/* ---- NUFFT plan -----------------------------------------------------------
 * Replaces tomocam::nufft::plans::cache<float> / FinufftPlanWrapper<float>
 * (include/finufft_plan_cache.h:34-72, include/finufft_plan.h:93-129): one
 * plan per volume size (n1, n2, n3) and tolerance instead of one per process.
 * eps = 1.2e-6 reproduces the reference's float tolerance (finufft_plan.h:66).
 */
int lamino_plan_create(int64_t n1, int64_t n2, int64_t n3, double eps, lamino_plan_t *out);
int lamino_plan_destroy(lamino_plan_t p);
/* Fine-grid bins of b1 x b2 x b3 cells for the plan's spreading and
 * interpolation (each bin's tile of (b + w - 1)^3 cells per component is staged
 * in shared memory); default 4 x 8 x 16.  Drops the plan's cached point orders.
 * No reference counterpart (FINUFFT's opts.gpu_binsize* play this role in
 * cuFINUFFT). */
int lamino_plan_set_bins(lamino_plan_t p, int b1, int b2, int b3);
/* Autotuner: times candidate bin layouts on the given geometries and keeps the
 * fastest for objective 0 (adjoint of geoms[0] including its bin sort, a setup
 * pass) or 1 (sum over geoms of sysmat with cached sorts, a solver's operator).
 * The choice is cached per fine grid, kernel width, objective and point count
 * for the process.  bins[3] (may be NULL) receives the layout, *best_ms (may be
 * NULL) its time (0 when taken from the cache). */
int lamino_plan_autotune(lamino_plan_t p, const lamino_geom_t *geoms, int ngeom, int objective, int *bins,
                         double *best_ms, void *stream);
/* Type 2, iflag -1: c[j] = sum_k modes[k] e^{-i k.x_j} (include/nufft.h:52-64).
 * modes: complex64 interleaved [n1][n2][n3]; c: complex64 [nproj][nrows][ncols]. */
int lamino_nufft3d2(lamino_plan_t p, lamino_geom_t g, const float *modes, float *c, void *stream);
/* Type 1, iflag +1: modes[k] = sum_j c[j] e^{+i k.x_j} (include/nufft.h:37-49). */
int lamino_nufft3d1(lamino_plan_t p, lamino_geom_t g, const float *c, float *modes, void *stream);

/* ---- operators ------------------------------------------------------------ */
/* tomocam::forward (include/projection.h:52-54, src/projection.cpp:42-77):
 * m3 [3][n1][n2][n3] -> proj [nproj][nrows][ncols]. */
int lamino_forward(lamino_plan_t p, lamino_geom_t g, const float *m3, float *proj, void *stream);
/* tomocam::adjoint (include/projection.h:64-66, src/projection.cpp:90-126). */
int lamino_adjoint(lamino_plan_t p, lamino_geom_t g, const float *proj, float *m3, void *stream);
/* sum over geometries of tomocam::sysmat (include/tomocam.h:50-52, src/gradient.cpp:34-89),
 * evaluated with the NUFFT (interp -> weight -> spread) on the GPU. */
int lamino_sysmat(lamino_plan_t p, const lamino_geom_t *geoms, int ngeom, const float *x3, float *y3,
                  void *stream);
/* tomocam::gradient (include/tomocam.h:64-67, src/gradient.cpp:98-105): sysmat(f) - yT. */
int lamino_gradient(lamino_plan_t p, lamino_geom_t g, const float *f3, const float *yT3, float *out3,
                    void *stream);
/* tomocam::residual (include/tomocam.h:79-82, src/gradient.cpp:117-127). */
int lamino_residual(lamino_plan_t p, lamino_geom_t g, const float *f3, const float *yT3, float yTy, double *out,
                    void *stream);

/* Allocation-free variant of lamino_residual (no counterpart in the reference).
 * For callers that cannot allocate device memory: a service overlapping several
 * reconstructions on one GPU evaluates this residual (the MBIR3 loss) inside its
 * line search, where a cudaMalloc/cudaFree would stall the other requests
 * (cudaFree waits for the whole device), and a caller whose device memory is
 * owned by another allocator may get none at all.  It calls no cudaMalloc,
 * cudaFree or allocating library routine: A f and the FP64 reduction slots live
 * in a 96 MiB static device array, held by every GPU that loads this library
 * until exit, so the volume may hold at most 8,388,586 voxels (n1*n2*n3);
 * larger volumes are rejected with LAMINO_ERR_ARG.  f3 and yT3 must be device
 * pointers (host pointers are rejected); res is host memory.  The first call on
 * a device resolves the array's device address (with that device current) and
 * should come before any stream capture; the address is kept for the life of
 * the process, so after cudaDeviceReset (which ends the context the address
 * belongs to) this entry point must not be called again in that process.  A
 * plan that has not sorted the geometry (no earlier lamino_residual /
 * lamino_sysmat with it) uses an unsorted point kernel, which needs no buffer
 * either.  Every call shares the array and it
 * keeps the last call's contents (the reduction slots are cleared at the start
 * of each call); calls that overlap on the GPU, on any stream, race. */
int lamino_residual_noalloc(lamino_plan_t p, lamino_geom_t g, const float *f3, const float *yT3, float yTy,
                            double *res, void *stream);

/* ---- Toeplitz normal operator ----------------------------------------------
 * sum_gamma sysmat as a 3x3 block convolution (no reference counterpart; it
 * replaces the MBIR `A` closures src/mbir_cg.cpp:97-105, src/mbir_sb.cpp:89-97).
 * precision: 0 = FP32 spectra, 1 = FP16 spectra with a power-of-two scale per
 * (k2, k3) pencil, 2 = both.
 */
#define LAMINO_PREC_FP32 0
#define LAMINO_PREC_FP16 1
#define LAMINO_PREC_MIXED 2 /* both spectra; lamino_normal_apply uses the FP32 ones */
int lamino_normal_create(const lamino_geom_t *geoms, int ngeom, int64_t n1, int64_t n2, int64_t n3, int precision,
                         lamino_normal_t *out, void *stream);
int lamino_normal_apply(lamino_normal_t op, const float *x3, float *y3, void *stream);
/* count independent applies y3s[i] = A x3s[i] on HOST buffers (no reference
 * counterpart; it serves callers that stream volumes through the operator, e.g.
 * the MBIR closures of many reconstructions sharing one geometry).  The inputs
 * are staged through two device buffers on a copy-in stream and the results
 * through two on a copy-out stream, so the copy-in of volume i+1 and the
 * copy-out of result i-1 overlap apply i (PCIe is full duplex); pinned
 * (page-locked) host buffers are needed for the overlap, pageable ones work but
 * serialise.  Returns when every result is in host memory.  Device pointers are
 * rejected (use lamino_normal_apply). */
int lamino_normal_apply_many(lamino_normal_t op, int count, const float *const *x3s, float *const *y3s,
                             void *stream);
/* Embedding-grid sizes L[3] = (L1, L2, L3) and device bytes held by the operator. */
int lamino_normal_info(lamino_normal_t op, int64_t *L, int64_t *bytes);
int lamino_normal_destroy(lamino_normal_t op);
/* Autotuner: times the valid launch shapes (rows per CTA of the n3 transforms,
 * k3 values per CTA of the n2 transforms) and keeps the fastest; cached per
 * embedding size and precision for the process.  Outputs may be NULL. */
int lamino_normal_autotune(lamino_normal_t op, int *rows, int *kb, double *best_ms, void *stream);
/* Quadratic forms out[3 g + i] = x_i . (S_g x)_i (double, host) for the
 * operators parts[g] (FP32 or mixed spectra, op's volume size), computed from
 * one forward half-spectrum of x with op's buffers (Parseval) instead of one
 * apply per part; the x_i . sysmat_g(x)_i terms of residual()
 * (src/gradient.cpp:117-127) and of the MBIR3 loss (src/mbir3.cpp:108-116). */
int lamino_normal_quadforms(lamino_normal_t op, const lamino_normal_t *parts, int nparts, const float *x3,
                            double *out, void *stream);
/* Per-stage CUDA-event timing of lamino_normal_apply on the launching stream
 * (measurement hook; no reference counterpart).  enable != 0 records events for
 * up to max_applies subsequent applies. */
int lamino_normal_profile(lamino_normal_t op, int enable, int max_applies);
/* Stage timings accumulated since lamino_normal_profile: nstages (<= 8) stages in
 * the order r2c_rows, dim2_fwd, pencil, dim2_inv, c2r_rows (one kernel each);
 * ms[k] summed milliseconds; bytes[k] the
 * algorithmic bytes of one apply of stage k; napplies profiled applies;
 * kernels_per_apply this library's kernel launches in one apply.  Any output
 * pointer except nstages may be NULL. */
int lamino_normal_stage_times(lamino_normal_t op, int *nstages, double *ms, int64_t *bytes, int *napplies,
                              int *kernels_per_apply);

/* ---- regularisers / finite differences (one component of dims n1,n2,n3) ---- */
/* tomocam::opt::qggmrf (include/optimize.h:146-153, src/qggmrf.cpp:60-95): g += prior gradient. */
int lamino_qggmrf(float *g, const float *x, int64_t n1, int64_t n2, int64_t n3, float sigma, float p,
                  void *stream);
/* tomocam::opt::grad_u (src/finitediff.cpp:8-47): out3 = 3 directional central differences. */
int lamino_grad_u(const float *u, int64_t n1, int64_t n2, int64_t n3, float *out3, void *stream);
/* tomocam::opt::divergence (src/finitediff.cpp:54-71): negative divergence of du3. */
int lamino_divergence(const float *du3, int64_t n1, int64_t n2, int64_t n3, float *out, void *stream);
/* tomocam::opt::laplacian (include/bregman.h:34-36): divergence(grad_u(u)). */
int lamino_laplacian(const float *u, int64_t n1, int64_t n2, int64_t n3, float *out, void *stream);
/* tomocam::opt::demag (include/demag.h:13-79): the demagnetizing field
 * h3 = F^-1[-k (k . F m) / |k|^2] / N of m3, both [3][n1][n2][n3]; k = 0 gives 0.
 * The reference defines it for the CG solver's constraint hook
 * (src/conjgrad.cpp:46-52), where its use is switched off; so is it here. */
int lamino_demag(const float *m3, int64_t n1, int64_t n2, int64_t n3, float *h3, void *stream);
/* tomocam::opt::RampPreconditioner::apply (include/precond.h:72-86), all 3 components. */
int lamino_ramp_precond(const float *r3, int64_t n1, int64_t n2, int64_t n3, float *z3, void *stream);

/* ---- solvers over a normal operator ---------------------------------------- */
/* Operator handles: the Toeplitz operator, or the NUFFT form over geometries. */
int lamino_op_from_normal(lamino_normal_t n, lamino_op_t *out);
int lamino_op_from_plan(lamino_plan_t p, const lamino_geom_t *geoms, int ngeom, lamino_op_t *out);
int lamino_op_apply(lamino_op_t op, const float *x3, float *y3, void *stream);
int lamino_op_destroy(lamino_op_t op);
/* tomocam::opt::cgsolver (include/optimize.h:101-103, src/conjgrad.cpp:37-117).
 * x3: x0 on entry, solution on exit.  iters (may be NULL): iterations run. */
int lamino_cgsolver(lamino_op_t A, const float *y3, float *x3, int64_t n1, int64_t n2, int64_t n3, int max_iter,
                    float tol, int *iters, void *stream);
/* tomocam::opt::split_bregman (include/optimize.h:85-88, src/bregman.cpp:39-134). */
int lamino_split_bregman(lamino_op_t A, const float *yT3, float *x3, int64_t n1, int64_t n2, int64_t n3,
                         float lambda, float mu, int outer_max, int inner_max, float tol, float xtol, int *iters,
                         void *stream);
/* tomocam::opt::lipschitz (include/optimize.h:135-137, src/lipschitz.cpp:31-53):
 * power-iteration estimate of ||A|| with FP64 norms and a seeded start. */
int lamino_lipschitz(lamino_op_t A, int64_t n1, int64_t n2, int64_t n3, int max_iters, double tol, uint64_t seed,
                     double *L, void *stream);

/* ---- MBIR drivers ------------------------------------------------------------
 * tomocam::MBIR1 / MBIR2 / MBIR3 (include/tomocam.h:101-154; src/mbir_cg.cpp:48-128,
 * src/mbir_sb.cpp:47-114, src/mbir3.cpp:47-135).  Fields default as
 * tomocam::ReconParams (include/config.h:146-158); lamino_recon_params_default fills them.
 * op_kind: 0 Toeplitz FP32, 1 Toeplitz FP16 spectra, 2 NUFFT form, 3 mixed (FP16
 * correction solves inside `refinements` FP32-residual refinement cycles per
 * linear solve; MBIR1 and MBIR2).  MBIR3 uses mu as the Lipschitz constant of
 * its gradient (src/mbir3.cpp:124); mu <= 0 estimates it instead with 30 power
 * iterations of the normal operator (FP64 norms), as lamino_lipschitz.
 */
typedef struct {
    int max_iters, inner_iters;
    float sigma, p, lambda, mu, tol, xtol, pad_factor;
    int op_kind;
    double eps;
    int refinements;
    int use_graphs; /* replay each solver iteration's operator work as a CUDA graph (non-default streams) */
    int autotune;   /* pick launch shapes / bin layouts by timing (cached per size) */
} lamino_recon_params;
void lamino_recon_params_default(lamino_recon_params *p);
/* method 1, 2 or 3.  projs[i]: [proj_dims[3i]][proj_dims[3i+1]][proj_dims[3i+2]];
 * angles[i]: proj_dims[3i] radians (host); out3: [3][r1][r2][r3]. */
int lamino_mbir(int method, int ndatasets, const float *const *projs, const int64_t *proj_dims,
                const float *const *angles, const float *gammas, int64_t r1, int64_t r2, int64_t r3,
                const lamino_recon_params *params, float *out3, void *stream);

/* Host wall-clock seconds of the calling thread's last lamino_mbir: setup
 * (normalisation, padding, grids, adjoints), operator build and solve, the
 * number of normal-operator applications in the solve, and parts[3] = seconds
 * in the NUFFT plan creation, the setup adjoints and autotuning (any pointer may
 * be NULL). */
int lamino_mbir_phases(double *setup_s, double *build_s, double *solve_s, int64_t *applies, double *parts);

/* Estimated peak device bytes of one lamino_mbir call (used for admission control). */
int lamino_mbir_footprint(int method, int ndatasets, const int64_t *proj_dims, int64_t r1, int64_t r2, int64_t r3,
                          const lamino_recon_params *params, int64_t *bytes);

/* ---- batched MBIR3 (no reference counterpart; each request is tomocam::MBIR3,
 * src/mbir3.cpp:47-135) -------------------------------------------------------------
 * nreq reconstructions of any sizes solved together on the calling device, from
 * host buffers to host buffers.  Request r has nds[r] datasets; the datasets of
 * all requests follow one another in projs / proj_dims (3 per dataset) / angles /
 * gammas, request by request.  recon_dims: 3 per request; params: nreq entries;
 * out3[r]: [3][recon_dims[3r]][recon_dims[3r+1]][recon_dims[3r+2]] (host).
 * Preparer threads (`threads`) set requests up, largest estimated footprint
 * first, while the sum of their estimated footprints (lamino_mbir_footprint)
 * fits in `budget` bytes; the
 * calling thread drives all prepared NAG solves, each with one line-search step
 * in flight on its own stream, deciding a step as soon as its reductions have
 * landed.  Optional outputs: times[2r], times[2r+1] = seconds
 * after the call started when request r was prepared and finished; counts[2r],
 * counts[2r+1] = its NAG iterations and normal-operator applications; stats[4] =
 * peak estimated bytes held, peak requests solving at once, line-search steps,
 * wall-clock microseconds.  Each result equals lamino_mbir(3, ...) of the same
 * request. */
int lamino_mbir3_batch(int nreq, const int *nds, const float *const *projs, const int64_t *proj_dims,
                       const float *const *angles, const float *gammas, const int64_t *recon_dims,
                       const lamino_recon_params *params, float *const *out3, int64_t budget, int threads,
                       double *times, int64_t *counts, int64_t *stats);

/* ---- continuous-batching server (no reference counterpart) ----------------------
 * Requests are MBIR1/2/3 problems as for lamino_mbir (inputs copied at submit).
 * A request is admitted in arrival order as soon as one of `slots` workers is free
 * and its estimated footprint fits in `budget_bytes` next to the running ones; each
 * worker runs on its own CUDA stream, so admitted reconstructions overlap on the
 * device and keep their iterates there until they finish.  flags & 1: dry run
 * (workers hold each request for dry_run_ms without touching the GPU; for tests
 * of the admission logic). */
typedef struct lamino_server_s *lamino_server_t;
int lamino_server_create(int64_t budget_bytes, int slots, int flags, double dry_run_ms, lamino_server_t *out);
int lamino_server_submit(lamino_server_t srv, int method, int ndatasets, const float *const *projs,
                         const int64_t *proj_dims, const float *const *angles, const float *gammas, int64_t r1,
                         int64_t r2, int64_t r3, const lamino_recon_params *params, int64_t *id);
/* Waits for request `id` (timeout_s < 0: no limit; returns LAMINO_ERR_TIMEOUT on
 * expiry), copies the reconstruction to out3 (host, may be NULL), reports the time
 * queued and running and the total latency in seconds and, in phases[7], the
 * request's lamino_mbir_phases figures (setup, build, solve seconds, applies,
 * plan, adjoints, tuning seconds), then forgets the request.  Every output
 * pointer may be NULL. */
int lamino_server_wait(lamino_server_t srv, int64_t id, double timeout_s, float *out3, double *queue_s,
                       double *run_s, double *latency_s, double *phases);
/* stats[10] = submitted, completed, failed, bytes in use, peak bytes in use, budget,
 * active, peak active, queued, slots. */
int lamino_server_stats(lamino_server_t srv, int64_t *stats);
/* Shuts the server down: requests still queued fail (their waiters return
 * LAMINO_ERR_STATE), running ones finish, and the call returns once every other
 * call on this server has returned.  No call may start on it after this one. */
int lamino_server_destroy(lamino_server_t srv);

#ifdef __cplusplus
}
#endif
#endif /* LAMINO_H */
