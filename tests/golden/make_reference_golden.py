"""Golden fixtures from the reference's OWN operator and solver code.

The reference's src/projection.cpp, src/gradient.cpp, src/conjgrad.cpp,
src/bregman.cpp, src/nagopt.cpp, src/qggmrf.cpp, src/finitediff.cpp and the MBIR
drivers are compiled unmodified into oracle/_ref/libtomocam_ref.so (oracle/Makefile)
against this project's FINUFFT-API and FFTW-API shims.  This script runs them in
double precision (the reference's double FINUFFT tolerance, 1e-14) on seeded
inputs, each case in its own process (the reference sizes its global NUFFT plan
by the first call), and writes:

  reference_path_ops.npz      forward, adjoint, sysmat, normal (sum over gamma),
                              gradient, residual, the ramp preconditioner, and the
                              float build's sysmat / forward, on small inputs
  reference_path_solvers.npz  cgsolver and split_bregman on the normal operator,
                              MBIR1 / MBIR2 / MBIR3 on small datasets
  reference_path_config0.npz  MBIR1 (CG, 20 iterations) at config 0: recon
                              16 x 128 x 128, 2 gammas x 90 angles, 128 x 128
                              projections; its inputs come from
                              oracle.config0_datasets() (seeded), fingerprinted

Run from the repository root:  python tests/golden/make_reference_golden.py [ops|solvers|config0]
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402
from oracle import refpath as R  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

# small operator case: volume (n1, n2, n3), two gamma datasets
OPS_DIMS = (9, 5, 11)
OPS_GEOMS = ((7, 13, 15, 0.3), (5, 11, 13, np.pi / 4))   # (nproj, nrows, ncols, gamma)
SOLVER_DIMS = (10, 6, 12)
SOLVER_GEOMS = ((8, 15, 17, 0.0), (6, 13, 15, 0.8))
MBIR_RECON = (8, 5, 9)
MBIR_NPROJ = (6, 5)
MBIR_DET = (9, 11)
MBIR_GAMMAS = (0.0, 0.8)


def fingerprint(arrs) -> str:
    h = hashlib.sha256()
    for a in arrs:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def ops_inputs(seed=20261203):
    rng = np.random.default_rng(seed)
    geoms = []
    for n, nr, nc, g in OPS_GEOMS:
        geoms.append((rng.uniform(0, 2 * np.pi, n).astype(np.float32), nr, nc, np.float32(g)))
    x = O.synthetic_magnetization(OPS_DIMS, seed=seed, sigma=1.0).astype(np.float64)
    x += 0.1 * rng.standard_normal(x.shape)
    yT = rng.standard_normal((3,) + OPS_DIMS)
    proj = rng.standard_normal((OPS_GEOMS[0][0], OPS_GEOMS[0][1], OPS_GEOMS[0][2]))
    ramp_even = rng.standard_normal((5, 8, 12))
    ramp_odd = rng.standard_normal((5, 7, 13))
    return geoms, x, yT, proj, ramp_even, ramp_odd


def make_ops():
    geoms, x, yT, proj, re, ro = ops_inputs()
    d = {"x": x, "yT": yT, "proj": proj, "ramp_even_in": re, "ramp_odd_in": ro,
         "dims": np.array(OPS_DIMS)}
    gd = [(th.astype(np.float64), nr, nc, float(g)) for th, nr, nc, g in geoms]
    for i, (th, nr, nc, g) in enumerate(gd):
        d[f"angles{i}"] = geoms[i][0]
        d[f"geom{i}"] = np.array([nr, nc, g])
        d[f"forward{i}"] = R.isolated("forward", x, th, nr, nc, g)
        d[f"sysmat{i}"] = R.isolated("sysmat", x, th, nr, nc, g)
        d[f"gradient{i}"] = R.isolated("gradient", x, yT, th, nr, nc, g)
        yTy = float(np.sum(yT * yT)) * 4.0
        d[f"yTy{i}"] = np.array(yTy)
        d[f"residual{i}"] = np.array(R.isolated("residual", x, yT, th, nr, nc, yTy, g))
        # the float build (the reference as it runs by default: float plans at 1.2e-6)
        thf = geoms[i][0]
        d[f"sysmat{i}_f32"] = R.isolated("sysmat", x, thf, nr, nc, np.float32(g), dtype=np.float32)
        d[f"forward{i}_f32"] = R.isolated("forward", x, thf, nr, nc, np.float32(g), dtype=np.float32)
    th, nr, nc, g = gd[0]
    d["adjoint0"] = R.isolated("adjoint", proj, th, g, OPS_DIMS)
    d["normal"] = R.isolated("normal", x, gd)
    d["ramp_even"] = R.isolated("ramp", re)
    d["ramp_odd"] = R.isolated("ramp", ro)
    np.savez_compressed(os.path.join(OUT, "reference_path_ops.npz"), **d)


def mbir_datasets(seed=3):
    """Small MBIR datasets: oracle forward model (exact NUDFT) + offset, float32."""
    rng = np.random.default_rng(seed)
    m = O.synthetic_magnetization(MBIR_RECON, seed=seed, sigma=1.0).astype(np.float64)
    plan = O.NufftPlan(MBIR_RECON, exact=True)
    data = []
    for n, g in zip(MBIR_NPROJ, MBIR_GAMMAS):
        th = rng.uniform(0, 2 * np.pi, n).astype(np.float32)
        pg = O.PolarGrid(th, MBIR_DET[0], MBIR_DET[1], np.float32(g))
        proj = O.forward(m, pg, pg.gamma, plan) + 0.05
        data.append((proj.astype(np.float32), th, np.float32(g)))
    return data


MBIR_PARAMS = {1: dict(max_iters=6, inner_iters=2), 2: dict(max_iters=4, inner_iters=2),
               3: dict(max_iters=6, inner_iters=2)}


def solver_inputs(seed=7):
    rng = np.random.default_rng(seed)
    geoms = [(rng.uniform(0, 2 * np.pi, n).astype(np.float32), nr, nc, np.float32(g))
             for n, nr, nc, g in SOLVER_GEOMS]
    b = rng.standard_normal((3,) + SOLVER_DIMS)
    return geoms, b


def make_solvers():
    geoms, b = solver_inputs()
    gd = [(th.astype(np.float64), nr, nc, float(g)) for th, nr, nc, g in geoms]
    x0 = np.zeros_like(b)
    d = {"b": b, "dims": np.array(SOLVER_DIMS)}
    for i, (th, nr, nc, g) in enumerate(geoms):
        d[f"angles{i}"] = th
        d[f"geom{i}"] = np.array([nr, nc, float(g)])
    d["cg"] = R.isolated("cgsolver", b, x0, gd, 8, 0.0)
    d["sb"] = R.isolated("split_bregman", b, x0, gd, 0.1, 10.0, 3, 3, 0.0, 0.0)
    data = mbir_datasets()
    for i, (p, th, g) in enumerate(data):
        d[f"mbir_proj{i}"] = p
        d[f"mbir_angles{i}"] = th
        d[f"mbir_gamma{i}"] = np.array(g)
    dd = [(p.astype(np.float64), th.astype(np.float64), float(g)) for p, th, g in data]
    for k, kw in MBIR_PARAMS.items():
        d[f"mbir{k}"] = R.isolated("mbir", k, dd, MBIR_RECON, **kw)
    np.savez_compressed(os.path.join(OUT, "reference_path_solvers.npz"), **d)


def make_config0():
    data = O.config0_datasets()
    dd = [(p.astype(np.float64), th.astype(np.float64), float(g)) for p, th, g in data]
    t = time.time()
    x = R.isolated("mbir", 1, dd, O.CONFIG0_RECON, max_iters=20)
    secs = time.time() - t
    np.savez_compressed(os.path.join(OUT, "reference_path_config0.npz"),
                        mbir1=x.astype(np.float32),
                        inputs_sha256=np.array(fingerprint([a for p in data for a in p])),
                        seconds_fp64=np.array(secs))
    print(f"config0 MBIR1 (reference, FP64): {secs:.1f} s")


if __name__ == "__main__":
    what = sys.argv[1:] or ["ops", "solvers", "config0"]
    for w in what:
        t = time.time()
        {"ops": make_ops, "solvers": make_solvers, "config0": make_config0}[w]()
        print(w, f"{time.time() - t:.1f} s")
