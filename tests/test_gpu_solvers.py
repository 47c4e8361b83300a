"""GPU parity tests for the solver path (regularisers, CG, split Bregman, NAG,
power iteration, MBIR drivers), through the C ABI."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu


def test_qggmrf_vs_reference(L, gold_ref):
    g = gold_ref["qg_g0"].copy()
    L.opt.qggmrf(g, gold_ref["qg_x"], 1000.0, 1.2)
    assert rel(g, gold_ref["qg_g"]) < 1e-6


@pytest.mark.parametrize("dims", [(37, 29, 70), (300, 40, 100)])
def test_qggmrf_tiles_and_plane_runs(L, O, dims):
    """qGGMRF at sizes with several CTA tiles (12 x 32 columns plus halo) and
    runs of planes per CTA, against the oracle (src/qggmrf.cpp:60-95, pinned to
    the reference's compiled code); includes equal neighbours (delta = 0, where
    both sides of a pair take rho'(0))."""
    rng = np.random.default_rng(7)
    x = rng.standard_normal(dims).astype(np.float32)
    x[5:9, 3:6, 10:20] = 0.25  # a flat patch: delta = 0 pairs
    g = np.zeros(dims, np.float32)  # the increments alone (they are small beside O(1) values)
    want = O.qggmrf(g, x, 1000.0, 1.2)
    L.opt.qggmrf(g, x, 1000.0, 1.2)
    assert rel(g, want) < 1e-6
    assert not g[0].any() and not g[:, :, -1].any()  # borders untouched


def test_laplacian_plane_runs(L, O):
    """A volume large enough that each thread of the Laplacian marches through
    runs of several planes (sizes of the 51x511x511 case's padded n2, n3)."""
    rng = np.random.default_rng(21)
    u = rng.standard_normal((20, 71, 721)).astype(np.float32)
    assert np.allclose(L.opt.laplacian(u), O.laplacian(u.astype(np.float64)), rtol=0, atol=2e-6)


def test_finite_differences_vs_reference(L, gold_ref):
    assert np.allclose(L.opt.grad_u(gold_ref["fd_u"]), gold_ref["fd_grad"], rtol=0, atol=1e-6)
    assert np.allclose(L.opt.divergence(gold_ref["fd_du"]), gold_ref["fd_div"], rtol=0, atol=1e-6)
    assert np.allclose(L.opt.laplacian(gold_ref["fd_u"]), gold_ref["fd_lap"], rtol=0, atol=2e-6)


@pytest.mark.parametrize("dims", [(9, 5, 11), (15, 7, 13)])
def test_demag_vs_oracle(L, O, dims):
    """Demagnetizing field (include/demag.h:13-79) against the FP64 restatement, on
    odd sizes (the reference's padded volumes are odd), its linearity, and
    demag(demag(m)) = -demag(m) (H is minus a projection)."""
    rng = np.random.default_rng(7)
    m = rng.standard_normal((3,) + dims).astype(np.float32)
    h = L.opt.demag(m)
    want = O.demag(m)
    assert rel(h, want) < 1e-5
    m2 = rng.standard_normal((3,) + dims).astype(np.float32)
    assert rel(L.opt.demag(2.0 * m + m2), 2.0 * want + O.demag(m2)) < 1e-5
    # H = -P m with P the projection on the longitudinal (curl-free) part: demag(H) = -H
    assert rel(L.opt.demag(h), -want) < 1e-5


@pytest.mark.parametrize("dims", [(5, 9, 12), (3, 71, 721), (3, 5, 400), (1, 3, 365), (2, 128, 400), (2, 5, 179),
                                  (1, 3, 1001), (2, 130, 6)])
def test_ramp_preconditioner_vs_oracle(L, O, dims):
    """Every form: n2 <= 128 runs 1-D transforms along n3 and a circulant
    convolution along n2, the n3 transforms as Bluestein convolutions of 1458
    when 365 <= n3 <= 729 (odd and even n3, an odd number of rows; n2 = 128 takes
    the column kernel's second pass over rows) and as Bluestein convolutions of a
    runtime length for n3 with a prime factor above 7 (179 -> 360, 1001 -> 2048),
    larger n2 the 2-D transforms."""
    rng = np.random.default_rng(1)
    r = rng.standard_normal((3,) + dims).astype(np.float32)
    M = O.RampPreconditioner(dims)
    want = np.stack([M.apply(r[i]) for i in range(3)])
    assert rel(L.opt.ramp_precond(r), want) < 1e-5


def _problem(L, O, dims=(14, 6, 12), geoms=((8, 21, 19, 0.0), (6, 21, 19, 0.7)), seed=2):
    rng = np.random.default_rng(seed)
    pgs, opgs = [], []
    for np_, nr, nc, g in geoms:
        th = rng.uniform(0, 2 * np.pi, np_).astype(np.float32)
        pgs.append(L.PolarGrid(th, nr, nc, np.float32(g)))
        opgs.append(O.PolarGrid(th, nr, nc, np.float32(g)))
    return pgs, opgs


def test_cgsolver_vs_oracle(L, O):
    dims = (14, 6, 12)
    pgs, opgs = _problem(L, O, dims)
    plan_o = O.NufftPlan(dims, eps=1e-12)
    A_o = lambda v: O.normal(v, opgs, [p.gamma for p in opgs], plan_o)
    xt = O.synthetic_magnetization(dims, seed=9, sigma=1.5).astype(np.float64)
    y = A_o(xt)
    want = O.cgsolver(A_o, y, np.zeros_like(y), 8, 1e-12)
    T = L.ToeplitzNormal(pgs, dims)
    got = L.opt.cgsolver(T, y.astype(np.float32), np.zeros_like(y, np.float32), 8, 1e-12)
    assert rel(got, want) < 1e-4
    got_n = L.opt.cgsolver((L.NufftPlan(dims), pgs), y.astype(np.float32), np.zeros_like(y, np.float32), 8, 1e-12)
    assert rel(got_n, want) < 1e-4


def test_split_bregman_vs_oracle(L, O):
    dims = (14, 6, 12)
    pgs, opgs = _problem(L, O, dims)
    plan_o = O.NufftPlan(dims, eps=1e-12)
    A_o = lambda v: O.normal(v, opgs, [p.gamma for p in opgs], plan_o)
    yT = A_o(O.synthetic_magnetization(dims, seed=10, sigma=1.5).astype(np.float64))
    want = O.split_bregman(A_o, yT, np.zeros_like(yT), 0.1, 10.0, 4, 3, 1e-12, 1e-12)
    got = L.opt.split_bregman(L.ToeplitzNormal(pgs, dims), yT.astype(np.float32),
                              np.zeros_like(yT, np.float32), 0.1, 10.0, 4, 3, 1e-12, 1e-12)
    assert rel(got, want) < 1e-4


def test_lipschitz_vs_oracle(L, O):
    dims = (14, 6, 12)
    pgs, opgs = _problem(L, O, dims)
    plan_o = O.NufftPlan(dims, eps=1e-12)
    A_o = lambda v: O.normal(v, opgs, [p.gamma for p in opgs], plan_o)
    Lo = O.lipschitz(A_o, (3,) + dims, max_iters=60, tol=1e-9)
    Lg = L.opt.lipschitz(L.ToeplitzNormal(pgs, dims), dims, max_iters=60, tol=1e-9)
    assert Lg == pytest.approx(Lo, rel=1e-3)
    # without an early stop (tol 0, as MBIR3 calls it) the iteration runs on the
    # device with one host read at the end: the same arithmetic as the loop with a
    # read per step, which tol = -1 (a stop that never triggers) still takes
    T = L.ToeplitzNormal(pgs, dims)
    a = L.opt.lipschitz(T, dims, max_iters=30, tol=0.0)
    b = L.opt.lipschitz(T, dims, max_iters=30, tol=-1.0)
    assert a == b
    assert a == pytest.approx(O.lipschitz(A_o, (3,) + dims, max_iters=30, tol=0.0), rel=1e-3)


def _datasets(L, O, recon=(8, 5, 9), nproj=(6, 5), det=(9, 11), gammas=(0.0, 0.8), seed=3):
    """Synthetic projections from the oracle forward model on the padded grid."""
    rng = np.random.default_rng(seed)
    m = O.synthetic_magnetization(recon, seed=seed, sigma=1.0).astype(np.float64)
    plan = O.NufftPlan(recon, exact=True)
    data = []
    for n, g in zip(nproj, gammas):
        th = rng.uniform(0, 2 * np.pi, n).astype(np.float32)
        pg = O.PolarGrid(th, det[0], det[1], np.float32(g))
        proj = O.forward(m, pg, pg.gamma, plan) + 0.05
        data.append((proj.astype(np.float32), th, np.float32(g)))
    return data


@pytest.mark.parametrize("method", [1, 2, 3])
def test_mbir_vs_oracle(L, O, method):
    recon = (8, 5, 9)
    data = _datasets(L, O, recon)
    po = O.ReconParams(maxIters=4, innerIters=2)
    fn_o = {1: O.MBIR1, 2: O.MBIR2, 3: O.MBIR3}[method]
    want = fn_o(data, recon, po, exact=True)
    for kind in ("toeplitz", "nufft"):
        pl = L.ReconParams(maxIters=4, innerIters=2, op_kind=kind)
        fn = {1: L.MBIR1, 2: L.MBIR2, 3: L.MBIR3}[method]
        got = fn(data, recon, pl)
        assert got.shape == (3,) + recon
        assert rel(got, want) < 1e-4, kind


@pytest.mark.parametrize("method", [1, 2])
def test_mbir_mixed_precision_vs_oracle(L, O, method):
    """Mixed form (FP16 spectra in the correction solves, FP32-residual refinement
    cycles, FP64 reductions) against the FP64 oracle running the same refined
    algorithm with the exact operator in both roles.  Bar: 1e-4 (final volume)."""
    recon = (8, 5, 9)
    data = _datasets(L, O, recon)
    R = 3
    po = O.ReconParams(maxIters=6, innerIters=3)
    fn_o = {1: O.MBIR1, 2: O.MBIR2}[method]
    want = fn_o(data, recon, po, exact=True, refinements=R)
    got = {1: L.MBIR1, 2: L.MBIR2}[method](data, recon, L.ReconParams(maxIters=6, innerIters=3, op_kind="mixed",
                                                                        refinements=R))
    err = rel(got, want)
    print(f"MBIR{method} mixed vs FP64 oracle: {err:.2e}")
    assert err < 1e-4
