#!/usr/bin/env python
"""Benchmark: A^H A (normal-operator) applies/s of the laminography operator.

Workload (the reference's README-size reconstruction): recon 3 x 51 x 511 x 511
float32, padded internally to (W, T, H) = (721, 71, 721); 4 gamma datasets
(0/45/90/135 deg) x 361 angles uniform in [0, 2 pi) (seeded); 511 x 511
detector padded to 1233 x 1233 (MBIR2 padding).  One step = one sum-over-gamma
A^H A apply (src/gradient.cpp:34-89 summed as src/mbir_sb.cpp:89-97) through
the Toeplitz operator, inputs resident in HBM.  Inputs (443 MB) and spectra
(GBs) exceed the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs N independent replicas (one per rank, launched by torchrun); the
operator has no cross-GPU exchange.  Rank 0 prints one JSON line.  At N = 1 the
line also carries `nufft`: the NUFFT form's adjoint / forward / sysmat times and
FP32 rates at half the full size (--no-nufft skips it), and `served`: p50/p99
reconstruction latency and saturated reconstructions/s of the continuous-
batching server and the batched form against the plain one-at-a-time FP32 loop
on a 100-request stream of uneven NAG + qGGMRF reconstructions (--no-served
skips it).

Other forms (their own JSON line): --form served (the full plain-vs-served
sweep), --form nufft (NUFFT-form forward / adjoint / sysmat times), --form recon
(README-size split-Bregman reconstruction end to end, FP32 and mixed).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "A^H A applies/s at 3x51x511x511"
RECON = (51, 511, 511)              # (T, H, W) as in the reference's config
PADDED = (721, 71, 721)             # internal (W, T, H) after MBIR2 padding
GAMMAS_DEG = (0.0, 45.0, 90.0, 135.0)
NPROJ = 361
DET_PADDED = 1233
# smaller cases of the same geometry, for profiler captures only (not bench lines)
SCALES = {"full": ((721, 71, 721), 361, 1233), "half": ((361, 36, 361), 181, 617),
          "quarter": ((181, 18, 181), 91, 309),
          # same n1 (FFT length 1458) as the full case, thin in n2/n3: > L2 but < 1 GB
          "pencil": ((721, 18, 360), 45, 309),
          # n1 = 721, n2 = 71 as the full case (compile-time n1 / n2 FFT lengths), n3 thin: < 2 GB
          "pencil2": ((721, 71, 180), 45, 309),
          # n2 = 71, n3 = 721 as the full case (compile-time n2 / n3 lengths), n1 thin: < 2 GB
          "rows": ((181, 71, 721), 45, 309)}


def workload_config(precision: str, n: int):
    return {
        "workload": "toeplitz normal operator, 3x51x511x511 recon (padded 721x71x721), "
                    "4 gammas x 361 angles, 1233x1233 padded projections",
        "recon_dims": list(RECON), "padded_dims": list(PADDED), "gammas_deg": list(GAMMAS_DEG),
        "angles_per_gamma": NPROJ, "projection_grid": [DET_PADDED, DET_PADDED],
        "kernel_spectra": precision, "parallelism": f"replicas{n}" if n > 1 else "single",
        "l2": "inputs larger than L2 (x 443 MB, spectra > 1 GB); no flush",
    }


# ---------------------------------------------------------------------------
# CPU baseline and reference arm: the reference's own sysmat, compiled
# (oracle/_ref), on a bounded sample of the workload
# ---------------------------------------------------------------------------

REF_GAMMA = 0.7853981852531433  # float32(pi / 4): the 45 deg dataset
REF_NPROJ = (1, 4)               # projections per sample call (two counts, to fit F and P)
_REF_STATE: dict = {}


def reference_sample(nproj: int):
    """One call of the reference's own tomocam::sysmat<float> (src/gradient.cpp:34-89,
    compiled unmodified into oracle/_ref against this project's FINUFFT-API and
    FFTW-API shims) on the full 721 x 71 x 721 volume and `nproj` projections of
    the 1233 x 1233 padded detector.  Returns host seconds."""
    import numpy as np
    from oracle import refpath as R
    if "x" not in _REF_STATE:  # inputs, outside the timed call
        rng = np.random.default_rng(11)
        _REF_STATE["x"] = rng.standard_normal((3,) + PADDED).astype(np.float32)
        _REF_STATE["th"] = rng.uniform(0, 2 * np.pi, 8).astype(np.float32)
    t = time.perf_counter()
    R.sysmat(_REF_STATE["x"], _REF_STATE["th"][:nproj], DET_PADDED, DET_PADDED, np.float32(REF_GAMMA),
             dtype=np.float32)
    return time.perf_counter() - t


def reference_model(samples):
    """Fit t(p) = F + p P to (projections, seconds) samples (F: the per-call
    fine-grid FFTs and deconvolution, P: the per-projection gridding and array
    work) and extrapolate one sum-over-gamma apply: 4 gammas x (F + 361 P)."""
    import numpy as np
    p = np.array([s[0] for s in samples], float)
    t = np.array([s[1] for s in samples], float)
    if len(set(p.tolist())) < 2:
        raise RuntimeError("the reference model needs samples at two projection counts")
    A = np.stack([np.ones_like(p), p], axis=1)
    (F, P), *_ = np.linalg.lstsq(A, t, rcond=None)
    F, P = max(float(F), 0.0), max(float(P), 0.0)
    return F, P, len(GAMMAS_DEG) * (F + NPROJ * P)


def reference_threads():
    from oracle import oracle as O
    return O.num_threads()


def reference_description(F, P, apply_s):
    return (f"reference's own tomocam::sysmat<float> (oracle/_ref: src/gradient.cpp and src/projection.cpp "
            f"compiled unmodified against this project's FINUFFT-API / FFTW-API shims) on the full 721x71x721 "
            f"volume, 1 or 4 projections of 1233x1233 per call; fit t = F + p P: F = {F:.2f} s per call "
            f"(fine-grid FFTs), P = {P:.3f} s per projection; one sum-over-gamma apply extrapolated as "
            f"4 x (F + 361 P) = {apply_s:.1f} s")


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from oracle import refpath as R
    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtomocam_ref.so is not built "
                          "(oracle/Makefile needs the reference tree)"}), flush=True)
        return 0
    # steps alternate 1 and 4 projections so the timed samples fit F and P
    for w in range(args.warmup):
        reference_sample(REF_NPROJ[w % 2])
    t_start = time.perf_counter()
    samples = []
    for k in range(args.steps):
        p = REF_NPROJ[k % 2]
        samples.append((p, reference_sample(p)))
    wall = time.perf_counter() - t_start
    if args.steps < 2:
        samples.append((REF_NPROJ[1], reference_sample(REF_NPROJ[1])))
    F, P, apply_s = reference_model(samples)
    v = 1.0 / apply_s
    threads = reference_threads()
    ms_step = 1e3 * sum(t for _, t in samples[:args.steps]) / args.steps
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "applies/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.precision, args.gpus),
        "cpu_baseline": {"value": v, "unit": "applies/s", "cores": threads, "kind": "reference",
                         "sample": reference_description(F, P, apply_s) +
                         "; ms_per_step is the measured time of one sample call"},
        "e2e": {"value": v, "unit": "applies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "wall_s": wall,
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# clocks sampling during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "50", "-i", str(gpu_index)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if "Active" in r[5 + i] and "Not" not in r[5 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


class UtilSampler:
    """nvidia-smi utilization.gpu (share of time a kernel was running) sampled
    every 100 ms while a phase runs; mean of the samples."""

    def __init__(self, gpu_index: int = 0):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=utilization.gpu", "--format=csv,noheader,nounits",
                                       "-lms", "100", "-i", str(gpu_index)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
        self.f.flush()
        self.f.seek(0)
        vals = [float(v) for v in self.f.read().split() if v.replace(".", "").isdigit()]
        os.unlink(self.f.name)
        return statistics.mean(vals) if vals else None


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def synthetic_magnetization_gpu(torch, dims, seed=1234, sigma=5.0, lateral_frac=0.8):
    """Unit vectors i.i.d. per voxel, Gaussian-smoothed (sigma voxels, reflect),
    renormalised, zeroed outside a full-thickness x central-80% lateral slab."""
    import torch.nn.functional as F
    g = torch.Generator(device="cuda").manual_seed(seed)
    m = torch.randn((3,) + tuple(dims), device="cuda", generator=g)
    m = m / (torch.linalg.vector_norm(m, dim=0, keepdim=True) + 1e-12)
    v = m.unsqueeze(1)  # (3, 1, n1, n2, n3)
    for ax in range(3):
        # Gaussian truncated at 3 sigma, or at the axis length for thin axes (reflect padding)
        r = min(int(3 * sigma), dims[ax] - 1)
        k = torch.exp(-0.5 * (torch.arange(-r, r + 1, device="cuda", dtype=torch.float32) / sigma) ** 2)
        k = k / k.sum()
        shape = [1, 1, 1, 1, 1]
        shape[2 + ax] = 2 * r + 1
        pad = [0, 0, 0, 0, 0, 0]
        pad[2 * (2 - ax)] = pad[2 * (2 - ax) + 1] = r
        v = F.conv3d(F.pad(v, pad, mode="reflect"), k.view(shape))
    m = v.squeeze(1)
    m = m / (torch.linalg.vector_norm(m, dim=0, keepdim=True) + 1e-12)
    n1, n2, n3 = dims
    a1, a3 = round(n1 * (1 - lateral_frac) / 2), round(n3 * (1 - lateral_frac) / 2)
    mask = torch.zeros(dims, device="cuda")
    mask[a1:n1 - a1, :, a3:n3 - a3] = 1
    return (m * mask).contiguous()


def read_traffic(stage: str):
    """DRAM bytes per launch of a stage's kernel from the committed ncu summary, if any."""
    import glob
    import re
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(path) as f:
            txt = f.read()
        m = re.search(rf"traffic\[{re.escape(stage)}\]:\s*([0-9.eE+]+)", txt)
        if m:
            return float(m.group(1))
    return None


def max_over_ranks(ms: float, dist=None) -> float:
    """The slowest rank's time (every rank takes part; NCCL reduces a CUDA
    tensor, gloo a host one)."""
    if dist is None:
        return ms
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args):
    import numpy as np
    import torch
    import lamino_b200 as L

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    L.lib()

    dims, nproj, det = SCALES[args.scale]
    rng = np.random.default_rng(2026)
    pgs = [L.PolarGrid(rng.uniform(0, 2 * np.pi, nproj).astype(np.float32), det, det,
                       np.float32(np.deg2rad(g))) for g in GAMMAS_DEG]
    t0 = time.perf_counter()
    op = L.ToeplitzNormal(pgs, dims, args.precision)
    build_s = time.perf_counter() - t0
    shape = op.autotune()  # launch shapes by timing (untimed setup)
    x = synthetic_magnetization_gpu(torch, dims)
    y = torch.empty_like(x)
    stream = torch.cuda.current_stream()

    for _ in range(args.warmup):
        op(x, out=y)
    torch.cuda.synchronize()

    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    phys = int(visible.split(",")[local]) if visible else local
    op.profile(True, args.steps)
    sampler = ClockSampler(phys) if rank == 0 else None
    time.sleep(0.2 if sampler else 0)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        op(x, out=y)
    e1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = sampler.stop() if sampler else None
    ms = e0.elapsed_time(e1)
    stages, napplies, kpa = op.stage_times()
    op.profile(False)
    ms = max_over_ranks(ms, dist)
    value = world * args.steps / (ms / 1e3)

    # e2e: the same apply through the C ABI on pinned HOST buffers, every step
    # copying its input volume in and its result out.  lamino_normal_apply_many
    # streams the K volumes: the copy-in of step i+1 and the copy-out of step i-1
    # overlap apply i.  Timed on the host clock around the whole call (it returns
    # when the last result is in host memory).  The serial form (one
    # lamino_normal_apply per step: copy in, apply, copy out) is reported beside it.
    xh = [x.cpu().pin_memory(), (x * 0.5).cpu().pin_memory()]
    yh = [torch.empty_like(xh[0]).pin_memory() for _ in range(2)]
    k_e2e = args.steps
    xs = [xh[i % 2] for i in range(k_e2e)]
    ys = [yh[i % 2] for i in range(k_e2e)]
    op.apply_many(xs[:2], ys[:2])  # staging buffers and streams
    for _ in range(2):
        op(xh[0], out=yh[0])
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    op.apply_many(xs, ys)
    ms_e2e = (time.perf_counter() - t0) * 1e3
    ms_e2e = max_over_ranks(ms_e2e, dist)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(k_e2e):
        op(xh[0], out=yh[0])
    f1.record(stream)
    torch.cuda.synchronize()
    ms_serial = max_over_ranks(f0.elapsed_time(f1), dist)
    nbytes = x.numel() * 4

    # roofline of the dominant stage
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        with open(peaks_path) as f:
            peak = float(json.load(f)["hbm_gbs"])
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    dom = max(stages, key=lambda k: stages[k][0])
    dom_ms = stages[dom][0] / max(napplies, 1)
    dom_bytes = stages[dom][1]
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    # whole-apply algorithmic bytes: x and y (3V floats each), 6 real FP32 half-spectra
    # and 3 forward + 3 product complex spectra written and read, S = 2n1 2n2 (n3+1)
    n1, n2, n3 = dims
    S_alg = (2 * n1) * (2 * n2) * (n3 + 1)
    V = n1 * n2 * n3
    b_apply = 2 * 3 * V * 4 + 6 * S_alg * (2 if args.precision == "fp16" else 4) + 12 * S_alg * 8
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_src, "traffic": read_traffic(dom),
                "apply_algorithmic_bytes": b_apply,
                "apply_achieved": b_apply / (ms / args.steps / 1e3) / 1e9,
                "apply_frac": b_apply / (ms / args.steps / 1e3) / 1e9 / peak,
                "stages_ms_per_apply": {k: v[0] / max(napplies, 1) for k, v in stages.items()},
                "stages_algorithmic_bytes": {k: v[1] for k, v in stages.items()}}

    line = {
        "metric": METRIC, "value": value, "unit": "applies/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded smoothed unit-vector magnetization, "
                                                     "seeded angles)",
        "config": workload_config(args.precision, world) if args.scale == "full" else
        {"workload": f"profiling case {args.scale}: padded {dims}, 4 gammas x {nproj} angles, {det}^2"},
        "e2e": {"value": world * k_e2e / (ms_e2e / 1e3), "unit": "applies/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes, "api": "lamino_normal_apply_many (pinned host buffers, "
                "copy-in / apply / copy-out overlapped across steps)",
                "serial_value": world * k_e2e / (ms_serial / 1e3),
                "serial_api": "lamino_normal_apply per step (copy in, apply, copy out)"},
        "gpu_launches": kpa * args.steps,
        "roofline": roofline,
        "clocks": clocks,
        "operator_build_s": build_s,
        "launch_shape": {"rows_per_cta": shape[0], "k3_per_cta": shape[1], "tuned_apply_ms": shape[2]},
    }
    if rank == 0 and world == 1 and not args.no_nufft:
        # the NUFFT form's spreading and interpolation (setup adjoints, plain
        # sysmat) with their FP32 rate, at half the full size
        nu = nufft_measure(torch, L, "half", 2, 3)
        line["nufft"] = {k: nu[k] for k in ("workload", "points_per_gamma", "adjoint_ms", "forward_ms",
                                            "sysmat_sum_gamma_ms", "fp32_tflops", "fp32_peak_tflops",
                                            "fp32_frac", "fp32_peak_source", "flop_count")}
    if rank == 0 and world == 1 and not args.no_served:
        # the served form against the plain loop on a request stream (one GPU)
        sv = serve_compare(torch, L, SERVE_LINE_REQUESTS, [0.5, 1.0, 1.5], SERVE_SLOTS)
        line["served"] = {
            "workload": f"{SERVE_LINE_REQUESTS} requests of the mixed-size NAG + qGGMRF stream (thickness "
                        "8-32, lateral 64-256, 2 gammas x 60-240 angles, 40 iterations), Poisson arrivals at "
                        "0.5 / 1.0 / 1.5 x the plain loop's saturated throughput, 3 slots, 150 GB budget; "
                        "plain = one at a time, eager launches, default shapes; plain_tuned = one at a time "
                        "with the served form's graphs and tuned shapes; batched = all requests through "
                        "lamino_mbir3_batch at once (4 preparer threads, one solver thread); all FP32 with "
                        "FP64 reductions",
            "rates": [{"rate_x_plain_capacity": r["rate_x_plain_capacity"],
                       "served_p50_s": r["served"]["p50_s"], "served_p99_s": r["served"]["p99_s"],
                       "plain_p50_s": r["plain"]["p50_s"], "plain_p99_s": r["plain"]["p99_s"],
                       **({"plain_tuned_p50_s": r["plain_tuned"]["p50_s"],
                           "plain_tuned_p99_s": r["plain_tuned"]["p99_s"]} if "plain_tuned" in r else {})}
                      for r in sv["sweep"]],
            "saturated_recon_per_s": sv["saturated"]["served"]["recon_per_s"],
            "plain_saturated_recon_per_s": sv["saturated"]["plain"]["recon_per_s"],
            "plain_tuned_saturated_recon_per_s": sv["saturated"]["plain_tuned"]["recon_per_s"],
            "max_rel_err_vs_plain": sv["max_rel_err_served_vs_plain"],
            **({"batched_saturated_recon_per_s": sv["saturated"]["batched"]["recon_per_s"],
                "batched_max_rel_err_vs_plain": sv["saturated"]["batched"]["max_rel_err_vs_plain"]}
               if "batched" in sv["saturated"] else {}),
            "gpu_utilization_pct_saturated": sv["gpu_utilization_pct_saturated"]}
        at1 = [r for r in sv["sweep"] if r["rate_x_plain_capacity"] == 1.0][0]
        line["served"].update({"p50_s": at1["served"]["p50_s"], "p99_s": at1["served"]["p99_s"],
                               "plain_p50_s": at1["plain"]["p50_s"], "plain_p99_s": at1["plain"]["p99_s"]})
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import refpath as R
        if R.available():
            samples = [(p, reference_sample(p)) for p in REF_NPROJ]
            F, P, apply_s = reference_model(samples)
            line["cpu_baseline"] = {"value": 1.0 / apply_s, "unit": "applies/s", "cores": reference_threads(),
                                    "kind": "reference", "sample": reference_description(F, P, apply_s)}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# served and batched forms: many uneven reconstructions
# ---------------------------------------------------------------------------

SERVE_BUDGET = 150 * 10**9   # HBM bytes the served form may admit at once
SERVE_ITERS = 40             # NAG + qGGMRF iterations of a mix request
SERVE_LINE_REQUESTS = 100    # requests of the served summary in the default bench line
SERVE_BATCH_THREADS = 4      # preparer threads of the batched form
SERVE_SLOTS = 3              # server slots (requests running at once) of the served line


def serve_mix(n: int, seed: int = 7, big_frac: float = 0.0):
    """Seeded request specs.  Mix requests: thickness from {8,16,24,32}, square
    lateral size from {64,128,192,256}, 2 datasets of 60-240 angles each; the
    first at gamma 0, the second at gamma = a tilt drawn from [20, 50] deg (the
    reference geometry has no separate tilt angle); NAG + qGGMRF (sigma 1000,
    p 1.2) for 40 iterations.  With probability big_frac a request is instead
    the README-size split-Bregman reconstruction (51x511x511, 4 gammas x 361
    angles, 50 outer iterations)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for r in range(n):
        if big_frac > 0 and rng.random() < big_frac:
            out.append(dict(kind="readme", method=2, recon=(511, 51, 511), det=(511, 511), nproj=[NPROJ] * 4,
                            gammas=list(GAMMAS_DEG), seed=1234 + r, sigma=5.0))
        else:
            t = int(rng.choice([8, 16, 24, 32]))
            h = int(rng.choice([64, 128, 192, 256]))
            out.append(dict(kind="mix", method=3, recon=(h, t, h), det=(h, h),
                            nproj=[int(rng.integers(60, 241)) for _ in range(2)],
                            gammas=[0.0, float(rng.uniform(20.0, 50.0))], seed=1234 + r, sigma=3.0))
    return out


def serve_data(torch, L, spec):
    """Host projections of one request: forward model of a seeded smoothed
    unit-vector magnetization plus Gaussian noise at 1% of the signal RMS."""
    import numpy as np
    m = synthetic_magnetization_gpu(torch, spec["recon"], seed=spec["seed"], sigma=spec["sigma"])
    rng = np.random.default_rng(spec["seed"])
    g = torch.Generator(device="cuda").manual_seed(spec["seed"] + 1)
    plan = L.NufftPlan(spec["recon"])
    data = []
    for n, gd in zip(spec["nproj"], spec["gammas"]):
        th = rng.uniform(0, 2 * np.pi, n).astype(np.float32)
        gam = np.float32(np.deg2rad(gd))
        y = L.forward(m, L.PolarGrid(th, spec["det"][0], spec["det"][1], gam), plan=plan)
        y = y + 0.01 * y.pow(2).mean().sqrt() * torch.randn(y.shape, device="cuda", generator=g)
        data.append((y.cpu().numpy(), th, gam))
    del plan
    return data


def serve_params(L, spec, form: str):
    # plain: eager launches, default launch shapes; plain_tuned and served: graphs, tuned shapes
    kw = dict(op_kind="toeplitz", use_graphs=False, autotune=False) if form == "plain" else \
        dict(op_kind="toeplitz", use_graphs=True, autotune=True)
    if spec["method"] == 3:  # mu = 0: Lipschitz constant from 30 power iterations
        return L.ReconParams(maxIters=SERVE_ITERS, sigma=1000.0, p=1.2, mu=0.0, **kw)
    return L.ReconParams(maxIters=50, innerIters=3, lam=0.1, mu=10.0, **kw)


def _pct(v, q):
    import numpy as np
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def run_plain_loop(L, specs, data, arrivals, form: str = "plain"):
    """One reconstruction at a time in arrival order (FP32 Toeplitz; eager
    launches and default shapes, or with form "plain_tuned" the served form's
    graphs and tuned shapes): returns results, latencies (arrival -> done),
    service times and applies."""
    fns = {1: L.MBIR1, 2: L.MBIR2, 3: L.MBIR3}
    res, lat, svc, app, ph = [], [], [], [], []
    t0 = time.perf_counter()
    for i, (sp, d) in enumerate(zip(specs, data)):
        now = time.perf_counter() - t0
        if arrivals[i] > now:
            time.sleep(arrivals[i] - now)
        a = time.perf_counter()
        res.append(fns[sp["method"]](d, sp["recon"], serve_params(L, sp, form)))
        b = time.perf_counter()
        svc.append(b - a)
        lat.append(b - t0 - arrivals[i])
        ph.append(L.mbir_phases())
        app.append(ph[-1]["applies"])
    return res, lat, svc, app, time.perf_counter() - t0, ph


def run_served(L, specs, data, arrivals, slots: int):
    """Requests submitted to the continuous-batching server at their arrival
    times (a submitting thread); latency = server-measured submit -> done."""
    import threading
    srv = L.ReconServer(SERVE_BUDGET, slots)
    ids = [None] * len(specs)
    ready = [threading.Event() for _ in specs]
    t0 = time.perf_counter()

    def feeder():
        for i, (sp, d) in enumerate(zip(specs, data)):
            now = time.perf_counter() - t0
            if arrivals[i] > now:
                time.sleep(arrivals[i] - now)
            ids[i] = srv.submit(sp["method"], d, sp["recon"], serve_params(L, sp, "served"))
            ready[i].set()

    th = threading.Thread(target=feeder)
    th.start()
    res, lat, app, info = [], [], [], []
    for i in range(len(specs)):
        ready[i].wait()
        vol, t = srv.wait(ids[i])
        res.append(vol)
        lat.append(t["latency_s"])
        app.append(t["applies"])
        info.append(t)
    span = time.perf_counter() - t0
    th.join()
    st = srv.stats()
    srv.close()
    return res, lat, app, span, st, info


def run_batched(L, specs, data):
    """All requests (MBIR3) through the batched form at once (lamino_mbir3_batch:
    preparer threads under the HBM budget, one thread driving the NAG solves); returns the
    results, the call's info and its host wall time."""
    reqs = [(d, sp["recon"], serve_params(L, sp, "served")) for sp, d in zip(specs, data)]
    t0 = time.perf_counter()
    res, info = L.mbir3_batch(reqs, SERVE_BUDGET, SERVE_BATCH_THREADS)
    return res, info, time.perf_counter() - t0


def _gpu_index() -> int:
    visible = os.environ.get("CUDA_VISIBLE_DEVICES")
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return int(visible.split(",")[local]) if visible else local


def serve_compare(torch, L, n: int, rates, slots: int, big_frac: float = 0.0, seed: int = 7):
    """Plain one-at-a-time loop against the served form on the same request
    stream: saturating throughput (all requests at t = 0), then Poisson
    arrivals at each multiple of the plain loop's saturating throughput."""
    import numpy as np
    specs = serve_mix(n, seed, big_frac)
    data = [serve_data(torch, L, sp) for sp in specs]
    torch.cuda.synchronize()
    # warm-up: one request of each distinct size through each form (module load,
    # kernel attributes, memory pools, the autotuner's per-size cache)
    seen, warm = set(), []
    for i, sp in enumerate(specs):
        if (sp["method"], tuple(sp["recon"])) not in seen:
            seen.add((sp["method"], tuple(sp["recon"])))
            warm.append(i)
    run_plain_loop(L, [specs[i] for i in warm], [data[i] for i in warm], [0.0] * len(warm))
    run_plain_loop(L, [specs[i] for i in warm], [data[i] for i in warm], [0.0] * len(warm), "plain_tuned")
    run_served(L, [specs[i] for i in warm], [data[i] for i in warm], [0.0] * len(warm), slots)
    if all(sp["method"] == 3 for sp in specs):
        run_batched(L, [specs[i] for i in warm], [data[i] for i in warm])
    zeros = [0.0] * n
    util = {}
    u = UtilSampler(_gpu_index())
    p_res, p_lat, p_svc, p_app, p_span, p_ph = run_plain_loop(L, specs, data, zeros)
    util["plain"] = u.stop()
    u = UtilSampler(_gpu_index())
    _, _, _, t_app, t_span, _ = run_plain_loop(L, specs, data, zeros, "plain_tuned")
    util["plain_tuned"] = u.stop()
    u = UtilSampler(_gpu_index())
    s_res, s_lat, s_app, s_span, s_st, s_info = run_served(L, specs, data, zeros, slots)
    util["served"] = u.stop()
    b_out = None
    if all(sp["method"] == 3 for sp in specs):
        u = UtilSampler(_gpu_index())
        b_res, b_info, b_span = run_batched(L, specs, data)
        util["batched"] = u.stop()
        b_err = max(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)) for a, b in zip(b_res, p_res))
        b_out = {"recon_per_s": n / b_span, "applies_per_s": sum(b_info["applies"]) / b_span, "makespan_s": b_span,
                 "threads": SERVE_BATCH_THREADS, "peak_live": b_info["peak_live"],
                 "peak_bytes": b_info["peak_in_use"], "steps": b_info["steps"],
                 "max_rel_err_vs_plain": b_err}
    errs = [float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)) for a, b in zip(s_res, p_res)]
    nonfinite = sum(int(not np.all(np.isfinite(a))) + int(not np.all(np.isfinite(b))) for a, b in zip(s_res, p_res))
    err = max(errs)
    mu_plain = n / p_span

    def phase_means(rows):
        return {k: float(np.mean([r[k] for r in rows]))
                for k in ("setup_s", "plan_s", "adjoint_s", "build_s", "tune_s", "solve_s", "applies")}
    out = {
        "requests": n, "slots": slots, "budget_bytes": SERVE_BUDGET,
        "mix": {"readme_size": sum(sp["kind"] == "readme" for sp in specs),
                "voxels_total": int(sum(3 * np.prod(sp["recon"]) for sp in specs))},
        "saturated": {
            "plain": {"recon_per_s": mu_plain, "applies_per_s": sum(p_app) / p_span, "makespan_s": p_span},
            "plain_tuned": {"recon_per_s": n / t_span, "applies_per_s": sum(t_app) / t_span, "makespan_s": t_span},
            "served": {"recon_per_s": n / s_span, "applies_per_s": sum(s_app) / s_span, "makespan_s": s_span,
                       "peak_active": s_st["peak_active"], "peak_bytes": s_st["peak_in_use"]},
            **({"batched": b_out} if b_out else {}),
        },
        "max_rel_err_served_vs_plain": err,
        "gpu_utilization_pct_saturated": util,
        "nonfinite_results": nonfinite,
        "mean_phases": {"plain": phase_means(p_ph), "served": phase_means(s_info)},
        "sweep": [],
    }
    rng = np.random.default_rng(seed + 1)
    for f in rates:
        lam = f * mu_plain
        arr = list(np.cumsum(rng.exponential(1.0 / lam, n)) - 0.0)
        arr = [a - arr[0] for a in arr]
        _, pl, psvc, _, pspan, _ = run_plain_loop(L, specs, data, arr)
        sres, sl, _, sspan, _, sinfo = run_served(L, specs, data, arr, slots)
        tuned = None
        if f == 1.0:  # one rate for the tuned loop: graphs and tuning without the batching
            _, tl, tsvc, _, tspan, _ = run_plain_loop(L, specs, data, arr, "plain_tuned")
            tuned = {"p50_s": _pct(tl, 50), "p99_s": _pct(tl, 99), "mean_s": float(np.mean(tl)),
                     "recon_per_s": n / tspan, "service_mean_s": float(np.mean(tsvc))}
        out["sweep"].append({
            "rate_x_plain_capacity": f, "arrivals_per_s": lam, "arrival_span_s": float(arr[-1]),
            "plain": {"p50_s": _pct(pl, 50), "p99_s": _pct(pl, 99), "mean_s": float(np.mean(pl)),
                      "recon_per_s": n / pspan, "service_mean_s": float(np.mean(psvc))},
            "served": {"p50_s": _pct(sl, 50), "p99_s": _pct(sl, 99), "mean_s": float(np.mean(sl)),
                       "recon_per_s": n / sspan, "run_mean_s": float(np.mean([t["run_s"] for t in sinfo]))},
            **({"plain_tuned": tuned} if tuned else {}),
        })
    return out


def fp32_peak_tflops(torch) -> float:
    """Nominal FP32 FMA peak of the device: SMs x 128 lanes x 2 FLOP x the
    maximum SM clock (148 x 128 x 2 x 1.965 GHz = 74.4 TFLOP/s on B200)."""
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    mhz = 1965.0
    try:
        import pynvml
        pynvml.nvmlInit()
        mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(pynvml.nvmlDeviceGetHandleByIndex(_gpu_index()),
                                                      pynvml.NVML_CLOCK_SM))
    except Exception:
        pass
    return props.multi_processor_count * 128 * 2 * mhz * 1e6 / 1e12


def nufft_measure(torch, L, scale: str, warmup: int, steps: int, bins=None):
    """The plain NUFFT form of the operator at a bench scale: forward and adjoint
    projection of one gamma dataset and the sum-over-gamma sysmat (interp ->
    weight -> spread per point), CUDA-event timed with inputs in HBM, with the
    FP32 rate of the taps.  The first call of each geometry includes its bin
    sort (cached afterwards)."""
    import numpy as np
    dims, nproj, det = SCALES[scale]
    rng = np.random.default_rng(2026)
    pgs = [L.PolarGrid(rng.uniform(0, 2 * np.pi, nproj).astype(np.float32), det, det,
                       np.float32(np.deg2rad(g))) for g in GAMMAS_DEG]
    plan = L.NufftPlan(dims)
    if bins:
        plan.set_bins(*bins)
    x = synthetic_magnetization_gpu(torch, dims)
    proj = torch.rand((nproj, det, det), device="cuda", generator=torch.Generator(device="cuda").manual_seed(3))
    stream = torch.cuda.current_stream()

    def timed(fn, k):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k

    t_sort = time.perf_counter()
    L.adjoint(proj, pgs[0], dims, plan=plan)  # includes the bin sort of pgs[0]
    torch.cuda.synchronize()
    t_sort = time.perf_counter() - t_sort
    k = max(1, steps)
    ms_adj = timed(lambda: L.adjoint(proj, pgs[0], dims, plan=plan), k)
    ms_fwd = timed(lambda: L.forward(x, pgs[0], plan=plan), k)
    ms_sys = timed(lambda: L.sysmat(x, pgs, plan=plan), k)
    M = nproj * det * det
    w = 7
    # one spread or one interpolation: 3 components x w^3 taps x 2 FMA (real weight x complex) per point
    flop_pass = 3 * w ** 3 * 2 * 2 * M
    peak = fp32_peak_tflops(torch)
    rate = {"adjoint": flop_pass / (ms_adj / 1e3) / 1e12, "forward": flop_pass / (ms_fwd / 1e3) / 1e12,
            "sysmat": 2 * len(pgs) * flop_pass / (ms_sys / 1e3) / 1e12}
    return {"workload": f"padded volume {dims}, {len(pgs)} gammas x {nproj} angles, {det}^2 projections",
            "bins": list(bins or (4, 8, 16)), "points_per_gamma": M, "first_adjoint_incl_sort_s": t_sort,
            "adjoint_ms": ms_adj, "forward_ms": ms_fwd, "sysmat_sum_gamma_ms": ms_sys,
            "sysmat_applies_per_s": 1e3 / ms_sys,
            "fp32_tflops": rate, "fp32_peak_tflops": peak,
            "fp32_frac": {kk: v / peak for kk, v in rate.items()},
            "fp32_peak_source": "nominal: SMs x 128 FP32 lanes x 2 FLOP x max SM clock",
            "flop_count": "4116 FLOP per point per spread or interpolation (343 taps x 3 components x 2 FMA)"}


def run_nufft_form(args):
    import torch
    import lamino_b200 as L
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    L.lib()
    bins = tuple(int(b) for b in args.bins.split(",")) if args.bins else None
    res = nufft_measure(torch, L, args.scale, args.warmup, args.steps, bins)
    line = {"form": "nufft", "metric": "NUFFT-form operator times", "unit": "ms", "higher_is_better": False,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": res.pop("workload"), "bins": res.pop("bins")}, **res,
            "sysmat_tflops_fp32": res["fp32_tflops"]["sysmat"]}
    print(json.dumps(line), flush=True)
    return 0


def run_recon_form(args):
    """One README-size reconstruction end to end through the C ABI with host
    buffers (split Bregman, lambda 0.1, mu 10, 50 outer x 3 inner iterations on
    51x511x511 from 4 gammas x 361 angles of 511^2 projections): the FP32 form
    and the mixed-precision form (FP16 correction solves inside 3 FP32-residual
    refinement cycles per linear solve), with their relative difference."""
    import numpy as np
    import torch
    import lamino_b200 as L
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    L.lib()
    spec = dict(kind="readme", method=2, recon=(511, 51, 511), det=(511, 511), nproj=[NPROJ] * 4,
                gammas=list(GAMMAS_DEG), seed=1234, sigma=5.0)
    t0 = time.perf_counter()
    data = serve_data(torch, L, spec)
    t_data = time.perf_counter() - t0
    out = {"form": "recon", "metric": "README-size MBIR2 reconstruction seconds", "unit": "s",
           "higher_is_better": False, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "MBIR2 (split Bregman, 50 x 3), recon 3x51x511x511, 4 gammas x 361 angles, "
                                  "511^2 projections, host buffers through lamino_mbir"},
           "data_generation_s": t_data}
    vols = {}
    forms = [f for f in (("fp32", "toeplitz"), ("mixed", "mixed")) if f[0] in args.recon_forms.split(",")]
    for name, kind in forms:
        p = L.ReconParams(maxIters=args.iters, innerIters=3, lam=0.1, mu=10.0, op_kind=kind)
        torch.cuda.synchronize()
        a = time.perf_counter()
        vols[name] = L.MBIR2(data, spec["recon"], p)
        b = time.perf_counter()
        out[name] = {"seconds": b - a, **L.mbir_phases()}
    if len(vols) == 2:
        d = vols["mixed"].astype(np.float64) - vols["fp32"]
        out["mixed_vs_fp32_rel_l2"] = float(np.linalg.norm(d) / np.linalg.norm(vols["fp32"]))
    out["config"]["outer_iterations"] = args.iters
    print(json.dumps(out), flush=True)
    return 0


def run_serve_form(args):
    import torch
    import lamino_b200 as L
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    L.lib()
    rates = [float(r) for r in args.rates.split(",")]
    t0 = time.perf_counter()
    res = serve_compare(torch, L, args.requests, rates, args.slots, args.big_frac)
    res["wall_s"] = time.perf_counter() - t0
    line = {"form": args.form, "metric": "reconstruction latency p50/p99 and recon/s, served vs plain",
            "unit": "s", "higher_is_better": False, "dtype": "f32", "data": "synthetic", **res}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp32", "fp16"], default="fp32")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-served", action="store_true", help="skip the served-form summary of the apply line")
    ap.add_argument("--no-nufft", action="store_true", help="skip the NUFFT-form summary of the apply line")
    ap.add_argument("--scale", choices=sorted(SCALES), default="full",
                    help="smaller cases of the same geometry for profiler captures")
    ap.add_argument("--form", choices=["apply", "served", "nufft", "recon"], default="apply",
                    help="apply: the operator metric; served: plain loop vs continuous-batching server; "
                         "nufft: the NUFFT-form forward / adjoint / sysmat; recon: README-size MBIR2 end to end")
    ap.add_argument("--bins", default="", help="nufft form: fine-grid bin size b1,b2,b3")
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--slots", type=int, default=SERVE_SLOTS)
    ap.add_argument("--rates", default="0.5,1.0,1.5", help="arrival rates, x the plain loop's capacity")
    ap.add_argument("--big-frac", type=float, default=0.0, help="share of README-size requests")
    ap.add_argument("--iters", type=int, default=50, help="recon form: split-Bregman outer iterations")
    ap.add_argument("--recon-forms", default="fp32,mixed", help="recon form: fp32, mixed or both")
    args = ap.parse_args()
    if args.form == "served":
        return run_serve_form(args)
    if args.form == "nufft":
        return run_nufft_form(args)
    if args.form == "recon":
        return run_recon_form(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
