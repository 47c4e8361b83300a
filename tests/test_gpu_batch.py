"""The batched MBIR3 form (lamino_mbir3_batch) against direct MBIR3 calls.

Requests of uneven size (thickness 8-24, lateral 48-128, two datasets of
50-120 angles) run together through the batched form: preparer threads set
them up under an HBM budget small enough that they wait for one another, and
the calling thread drives their NAG + qGGMRF solves (src/mbir3.cpp:47-135),
one line-search step in flight per request.  Each result must equal the direct MBIR3 call of the same
request (same operators, same arithmetic, the Lipschitz constant estimated by
30 power iterations in both) to relative L2 1e-5; the direct calls themselves
are checked against the FP64 oracle in test_gpu_served_parity.py.
"""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu
TOL = 1e-5

SIZES = [(8, 64, 60, 90), (16, 96, 75, 50), (24, 48, 120, 100), (8, 128, 64, 70), (16, 64, 80, 80)]


def _requests(L, O, iters):
    reqs = []
    for i, (t, h, na, nb) in enumerate(SIZES):
        recon = (h, t, h)
        m = O.synthetic_magnetization(recon, seed=300 + i, sigma=3.0).astype(np.float32)
        rng = np.random.default_rng(400 + i)
        plan = L.NufftPlan(recon)
        data = []
        for n, g in ((na, 0.0), (nb, float(np.deg2rad(rng.uniform(20.0, 50.0))))):
            th = rng.uniform(0, 2 * np.pi, n).astype(np.float32)
            y = np.asarray(L.forward(m, L.PolarGrid(th, h, h, np.float32(g)), plan=plan))
            y = y + 0.01 * np.sqrt(np.mean(y ** 2)) * rng.standard_normal(y.shape).astype(np.float32)
            data.append((y.astype(np.float32), th, np.float32(g)))
        p = L.ReconParams(maxIters=iters, sigma=1000.0, p=1.2, mu=0.0, op_kind="toeplitz", use_graphs=True,
                          autotune=True)
        reqs.append((data, recon, p))
    return reqs


def test_batch_equals_direct_mbir3(L, O):
    reqs = _requests(L, O, iters=8)
    direct = [L.MBIR3(d, r, p) for d, r, p in reqs]
    fps = [L.mbir_footprint(3, [x[0].shape for x in d], r, p) for d, r, p in reqs]
    budget = max(fps) + min(fps)  # at most two requests held at once: the others wait for memory
    vols, info = L.mbir3_batch(reqs, budget_bytes=budget, threads=2)
    errs = [rel(v, w) for v, w in zip(vols, direct)]
    print("batched vs direct:", ", ".join(f"{e:.1e}" for e in errs), info)
    assert max(errs) < TOL
    assert all(np.all(np.isfinite(v)) for v in vols)
    assert info["peak_in_use"] <= budget
    assert info["peak_live"] >= 1 and info["steps"] >= sum(info["iterations"])
    assert all(0 < a <= b for a, b in zip(info["ready_s"], info["done_s"]))


def test_batch_many_at_once_and_zero_iterations(L, O):
    reqs = _requests(L, O, iters=5)
    # one request with no iterations: its result is the zero start
    d0, r0, p0 = reqs[0]
    p0 = L.ReconParams(maxIters=0, sigma=1000.0, p=1.2, mu=0.0, op_kind="toeplitz")
    reqs[0] = (d0, r0, p0)
    vols, info = L.mbir3_batch(reqs, threads=4)
    assert np.all(vols[0] == 0.0) and info["iterations"][0] == 0
    direct = [L.MBIR3(d, r, p) for d, r, p in reqs[1:]]
    errs = [rel(v, w) for v, w in zip(vols[1:], direct)]
    print("batched vs direct:", ", ".join(f"{e:.1e}" for e in errs), info)
    assert max(errs) < TOL
    assert 1 <= info["peak_live"] <= len(reqs)  # how many overlap depends on the timing
