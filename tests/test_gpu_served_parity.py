"""The served and batched forms at the sizes they serve, against the FP64 oracle.

The two smallest requests of the batched / served mix (NAG + qGGMRF, recon
thickness 8 and 16 x lateral 64, two datasets of 60 angles at gamma 0 and a
tilt, 64 x 64 projections) run through the continuous-batching server
(lamino_server_*), the batched form (lamino_mbir3_batch) and as direct MBIR3
calls, and all three are compared with the
oracle's double-precision MBIR3 (src/mbir3.cpp:47-135) in its Toeplitz form
(oracle.MBIR3_toeplitz, pinned to the reference's own MBIR3 on the CPU).  The
Lipschitz constant is the oracle's 30-step power iteration, passed to both as
`mu`, so the comparison covers the solver and not the estimate.  Tolerance:
relative L2 1e-4 on the final volume.
"""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu
TOL_VOLUME = 1e-4
ITERS = 6


def _request(O, thickness, seed):
    """recon (n1, n2, n3) = (64, thickness, 64) internal order; data from the
    FP64 forward model plus 1% Gaussian noise."""
    recon = (64, thickness, 64)
    rng = np.random.default_rng(seed)
    m = O.synthetic_magnetization(recon, seed=seed, sigma=3.0)
    plan = O.NufftPlan(recon, eps=1e-9)
    data = []
    for g in (0.0, float(np.deg2rad(rng.uniform(20.0, 50.0)))):
        th = rng.uniform(0, 2 * np.pi, 60).astype(np.float32)
        pg = O.PolarGrid(th, 64, 64, np.float32(g))
        y = O.forward(m, pg, pg.gamma, plan)
        y = y + 0.01 * np.sqrt(np.mean(y ** 2)) * rng.standard_normal(y.shape)
        data.append((y.astype(np.float32), th, np.float32(g)))
    return recon, data


@pytest.mark.parametrize("thickness,seed", [(8, 1234), (16, 1235)])
def test_served_and_direct_mbir3_vs_fp64_oracle(L, O, thickness, seed):
    recon, data = _request(O, thickness, seed)
    po = O.ReconParams(maxIters=ITERS, innerIters=3, sigma=1000.0, p=1.2)
    want, lip = O.MBIR3_toeplitz(data, recon, po, eps=1e-9, lipschitz_iters=30)
    p = L.ReconParams(maxIters=ITERS, innerIters=3, sigma=1000.0, p=1.2, mu=float(lip), op_kind="toeplitz",
                      use_graphs=True, autotune=True)
    direct = L.MBIR3(data, recon, p)
    with L.ReconServer(budget_bytes=8 << 30, slots=2) as srv:
        rid = srv.submit(3, data, recon, p)
        served, _ = srv.wait(rid)
    (batched,), info = L.mbir3_batch([(data, recon, p)], budget_bytes=8 << 30, threads=1)
    e_direct, e_served, e_batched = rel(direct, want), rel(served, want), rel(batched, want)
    print(f"thickness {thickness}: direct {e_direct:.2e}, served {e_served:.2e}, batched {e_batched:.2e} "
          f"vs FP64 oracle (L = {lip:.4g})")
    assert e_direct < TOL_VOLUME
    assert e_served < TOL_VOLUME
    assert e_batched < TOL_VOLUME
    assert info["iterations"] == [ITERS]
