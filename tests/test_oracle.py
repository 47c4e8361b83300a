"""CPU tests: the oracle pinned against the reference's own compiled code and
golden fixtures, plus the definitional properties the reference's smoke
programs print (tests/test_grad.cpp, tests/test_loss.cpp, tests/test_cg.cpp,
tests/test_fft_r2c.cpp of the reference)."""
import ctypes

import numpy as np
import pytest

from conftest import rel


# ---------------------------------------------------------------- pinned pieces

@pytest.mark.parametrize("tag", ["odd", "even"])
def test_polar_grid_matches_reference(O, gold_ref, tag):
    th = gold_ref[f"grid_{tag}_theta"]
    np_, nr, nc, g = gold_ref[f"grid_{tag}_meta"]
    pg = O.PolarGrid(th, int(nr), int(nc), np.float32(g))
    x, y, z = gold_ref[f"grid_{tag}_xyz"]
    assert np.array_equal(pg.x, x) and np.array_equal(pg.y, y) and np.array_equal(pg.z, z)


@pytest.mark.parametrize("tag", ["odd", "even"])
def test_beam_dir_vector(O, gold_ref, tag):
    th = gold_ref[f"grid_{tag}_theta"]
    g = gold_ref[f"grid_{tag}_meta"][3]
    c = O.beam_dir_vector(np.float32(g), th.astype(np.float64)).T
    assert np.allclose(c, gold_ref[f"grid_{tag}_coeff"], rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("tag", ["odd", "even"])
def test_shifts_match_reference(O, gold_ref, tag):
    a = gold_ref[f"shift_{tag}_in"]
    assert np.array_equal(O.fftshift2(a), gold_ref[f"shift_{tag}_f"])
    assert np.array_equal(O.ifftshift2(a), gold_ref[f"shift_{tag}_i"])


def test_padding_matches_reference(O, gold_ref):
    a = gold_ref["pad2d_in"]
    assert np.array_equal(O.pad2d(a, np.float32(0.4142)), gold_ref["pad2d_p04"])
    assert np.array_equal(O.pad2d(a, np.float32(1.4142)), gold_ref["pad2d_p14"])
    assert np.array_equal(O.crop3d(gold_ref["crop3d_in"], (7, 5, 9)), gold_ref["crop3d_out"])


def test_finite_differences_match_reference(O, gold_ref):
    u = gold_ref["fd_u"]
    assert np.allclose(O.grad_u(u), gold_ref["fd_grad"], rtol=0, atol=1e-6)
    assert np.allclose(O.divergence(gold_ref["fd_du"]), gold_ref["fd_div"], rtol=0, atol=1e-6)
    assert np.allclose(O.laplacian(u), gold_ref["fd_lap"], rtol=0, atol=2e-6)


def test_qggmrf_matches_reference(O, gold_ref):
    g = O.qggmrf(gold_ref["qg_g0"], gold_ref["qg_x"], 1000.0, 1.2)
    assert rel(g, gold_ref["qg_g"]) < 1e-6
    # delta == 0 contributes q / (sigma^q C), not 0 (src/qggmrf.cpp:53-55)
    assert O.d_potential(np.array([0.0]), 1e6, 1000 ** 0.8, 1.2)[0] == pytest.approx(2e-3)


def test_nagopt_matches_reference(O, gold_ref):
    dg, b = gold_ref["nag_diag"].astype(np.float64), gold_ref["nag_b"].astype(np.float64)
    grad = lambda x: dg * x - b
    loss = lambda x: float(0.5 * np.sum(dg * x * x) - np.sum(b * x) + 10.0)
    x = O.nagopt(grad, loss, np.zeros_like(dg), 25, 6.0, 1e-9, 1e-9, 5)
    assert rel(x, gold_ref["nag_x"]) < 1e-4


def test_padded_dims():
    from oracle import oracle as O
    assert O.padded_volume_dims((16, 128, 128)) == (22, 180, 180)
    assert O.padded_volume_dims((51, 511, 511)) == (71, 721, 721)
    assert O.pad2d(np.zeros((1, 511, 511), np.float32), np.float32(1.4142)).shape == (1, 1233, 1233)
    assert O.pad2d(np.zeros((1, 128, 128), np.float32), np.float32(0.4142)).shape == (1, 180, 180)


# ---------------------------------------------------------------- NUFFT semantics

def test_es_nufft_vs_nudft(O):
    rng = np.random.default_rng(3)
    dims = (9, 5, 11)
    pg = O.PolarGrid(rng.uniform(0, 6.28, 3).astype(np.float32), 13, 15, np.float32(0.8))
    pe, pn = O.NufftPlan(dims, exact=True), O.NufftPlan(dims, eps=1e-12)
    f = rng.standard_normal(dims) + 1j * rng.standard_normal(dims)
    c = rng.standard_normal(pg.dims()) + 1j * rng.standard_normal(pg.dims())
    assert rel(O.nufft3d2(f, pg, pn), O.nufft3d2(f, pg, pe)) < 1e-10
    assert rel(O.nufft3d1(c, pg, pn), O.nufft3d1(c, pg, pe)) < 1e-10
    # type 1 is the adjoint of type 2
    lhs = np.vdot(c, O.nufft3d2(f, pg, pe))
    rhs = np.vdot(O.nufft3d1(c, pg, pe), f)
    assert abs(lhs - rhs) < 1e-9 * abs(lhs)


def test_golden_operators(O, gold_orc):
    th = gold_orc["op_theta"]
    nr, nc, g = gold_orc["op_meta"]
    pg = O.PolarGrid(th, int(nr), int(nc), np.float32(g))
    pe = O.NufftPlan((9, 5, 11), exact=True)
    assert rel(O.nufft3d2(gold_orc["op_f"], pg, pe), gold_orc["op_nudft2"]) < 1e-12
    assert rel(O.forward(gold_orc["op_m"], pg, np.float32(g), pe), gold_orc["op_forward"]) < 1e-12
    assert rel(O.sysmat(gold_orc["op_m"], pg, np.float32(g), pe), gold_orc["op_sysmat"]) < 1e-12


@pytest.mark.parametrize("nr,nc", [(31, 29), (26, 34), (180, 180), (462, 462), (1233, 1233)])
def test_detector_points_pair_up_antipodally(O, nr, nc):
    """The adjoint spreads points i and N-1-i of a projection (N = nrows ncols)
    through one footprint: on the reference's detector grids, odd and even,
    x_{N-1-i} = -x_i to within float rounding (here 1e-6 of [-pi, pi))."""
    th = np.linspace(0, 2 * np.pi, 5, endpoint=False).astype(np.float32)
    pg = O.PolarGrid(th, nr, nc, np.float32(0.6))
    for a in (pg.x, pg.y, pg.z):
        f = a.reshape(len(th), -1).astype(np.float64)
        assert np.abs(f + f[:, ::-1]).max() < 2e-6


def test_adjoint_pair_rule(O):
    """Re sum_i f_i e^{i k.x_i} over all points equals the sum over pairs
    (q, N-1-q), q < (N+1)/2, of f_q at x_q plus conj(f_{N-1-q}) at -x_{N-1-q},
    the middle point of an odd N taken once: the rule the GPU adjoint spreads by."""
    rng = np.random.default_rng(3)
    th = rng.uniform(0, 2 * np.pi, 3).astype(np.float32)
    for nr, nc in ((7, 5), (6, 4), (5, 6)):
        pg = O.PolarGrid(th, nr, nc, np.float32(0.4))
        N = nr * nc
        pts = np.stack([a.reshape(len(th), N).astype(np.float64) for a in (pg.z, pg.y, pg.x)], -1)
        f = rng.standard_normal((len(th), N)) + 1j * rng.standard_normal((len(th), N))
        k = np.stack(np.meshgrid(*(np.arange(-3, 3),) * 3, indexing="ij"), -1).reshape(-1, 3)
        full = np.einsum("pn,kpn->k", f, np.exp(1j * np.einsum("kd,pnd->kpn", k, pts))).real
        H = (N + 1) // 2
        q = np.arange(H)
        g = np.conj(f[:, N - 1 - q])
        g[:, q == N - 1 - q] = 0
        second = -pts[:, N - 1 - q]
        paired = (np.einsum("pn,kpn->k", f[:, :H], np.exp(1j * np.einsum("kd,pnd->kpn", k, pts[:, :H])))
                  + np.einsum("pn,kpn->k", g, np.exp(1j * np.einsum("kd,pnd->kpn", k, second)))).real
        assert np.allclose(paired, full, rtol=1e-12, atol=1e-10)


def test_gridded_pair_rule(O):
    """The pair rule holds for the ES-gridded transforms the GPU kernels compute,
    not only for the exact sums: on the periodic fine grid (m -> -m, the kernel
    even) the real part of a type-1 sum over all points equals that over the
    pairs (f_q at x_q, conj(f_{N-1-q}) at -x_{N-1-q}), and the type-2 value of a
    real volume at -x is the conjugate of its value at x.  FP64 oracle at the
    GPU's kernel width (eps 1.2e-6, w = 7)."""
    rng = np.random.default_rng(5)
    dims = (9, 5, 11)
    plan = O.NufftPlan(dims, eps=1.2e-6)
    th = rng.uniform(0, 2 * np.pi, 3).astype(np.float32)
    for nr, nc in ((7, 5), (6, 8)):
        pg = O.PolarGrid(th, nr, nc, np.float32(0.7))
        N = nr * nc
        xs = [a.reshape(len(th), N).astype(np.float64) for a in (pg.x, pg.y, pg.z)]
        f = rng.standard_normal((len(th), N)) + 1j * rng.standard_normal((len(th), N))
        full = plan.type1(f, *xs).real
        H = (N + 1) // 2
        q = np.arange(H)
        g = np.conj(f[:, N - 1 - q])
        g[:, q == N - 1 - q] = 0
        pts = [np.concatenate([a[:, :H], -a[:, N - 1 - q]], 1) for a in xs]
        paired = plan.type1(np.concatenate([f[:, :H], g], 1), *pts).real
        assert np.abs(paired - full).max() < 1e-10 * np.abs(full).max()
        m = rng.standard_normal(dims)
        c = plan.type2(m, *xs)
        cm = plan.type2(m, *(-a for a in xs))
        assert np.abs(cm - np.conj(c)).max() < 1e-10 * np.abs(c).max()


def test_sysmat_equals_adjoint_forward_odd_grid(O):
    """tests/test_grad.cpp:15-55 of the reference: adjoint(forward(f)) vs gradient(f, 0)."""
    rng = np.random.default_rng(5)
    dims = (7, 5, 9)
    pg = O.PolarGrid(rng.uniform(-1.2, 0.1, 6).astype(np.float32), 13, 15, np.float32(np.pi / 4))
    pe = O.NufftPlan(dims, exact=True)
    f = rng.random((3,) + dims)
    g1 = O.adjoint(O.forward(f, pg, pg.gamma, pe), pg, dims, pg.gamma, pe)
    g2 = O.sysmat(f, pg, pg.gamma, pe)
    assert rel(g1, g2) < 1e-10


def test_residual_identity(O):
    """tests/test_loss.cpp pattern: ||P f - y||^2 = f.AAf - 2 f.P^T y + y.y per component sum."""
    rng = np.random.default_rng(6)
    dims = (7, 5, 9)
    pg = O.PolarGrid(rng.uniform(0, 6.28, 5).astype(np.float32), 11, 13, np.float32(0.4))
    pe = O.NufftPlan(dims, exact=True)
    f = rng.standard_normal((3,) + dims)
    yT = rng.standard_normal((3,) + dims)
    AAf = O.sysmat(f, pg, pg.gamma, pe)
    yTy = float(np.sum(yT * yT))
    want = sum(np.sqrt(np.sum(f[i] * AAf[i]) - 2 * np.sum(f[i] * yT[i]) + yTy) for i in range(3))
    assert O.residual(f, yT, pg, yTy, pg.gamma, pe) == pytest.approx(want, rel=1e-12)


def test_toeplitz_kernel_is_the_normal_operator(O):
    rng = np.random.default_rng(7)
    dims = (9, 4, 8)
    ths = [rng.uniform(0, 6.28, 5).astype(np.float32), rng.uniform(0, 6.28, 3).astype(np.float32)]
    gms = [0.0, 0.9]
    pgs = [O.PolarGrid(t, 12, 11, g, dtype=np.float64) for t, g in zip(ths, gms)]
    pe = O.NufftPlan(dims, exact=True)
    x = rng.standard_normal((3,) + dims)
    T = O.toeplitz_kernel(dims, ths, gms, 12, 11)
    assert rel(O.toeplitz_apply(x, T), O.normal(x, pgs, gms, pe)) < 1e-12


# ---------------------------------------------------------------- solvers

def test_cg_diagonal_system(O):
    """tests/test_cg.cpp:16-55 pattern: CG on diag(1..N) (identity preconditioner)."""
    N = 100
    d = np.arange(1, N + 1, dtype=np.float64).reshape(1, 1, N)
    xt = np.random.default_rng(1).random((1, 1, N))
    b = np.stack([d * xt] * 3)

    class Ident:
        def apply(self, r):
            return r

    x = O.cgsolver(lambda v: d * v, b, np.zeros_like(b), 1000, 1e-10, precond=Ident())
    assert rel(x, np.stack([xt] * 3)) < 1e-8


def test_ramp_preconditioner_roundtrip_zero_dc(O):
    """include/precond.h: filter(0,0) = 0, so constant slices map to zero."""
    M = O.RampPreconditioner((3, 6, 8))
    assert M.filter[0, 0] == 0.0
    assert np.allclose(M.apply(np.ones((3, 6, 8))), 0.0, atol=1e-12)


def test_fft_roundtrip():
    """tests/test_fft_r2c.cpp: 2-D r2c -> c2r / n recovers the input (1e-10 double)."""
    a = np.random.default_rng(2).random((3, 5, 7))
    c = np.fft.irfft2(np.fft.rfft2(a), s=(5, 7))
    assert np.max(np.abs(a - c)) < 1e-10
