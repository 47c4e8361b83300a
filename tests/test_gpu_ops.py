"""GPU parity tests for the operator path, through the C ABI (ctypes).

Tolerances: single operator applies within relative L2 1e-5 of the oracle
(FP64, eps 1e-12, the reference's float coordinates); the Toeplitz FP16
storage variant within 2e-3 of the FP32 one.
"""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu
TOL = 1e-5


def test_geometry_points_bitexact(L, gold_ref):
    for tag in ("odd", "even"):
        th = gold_ref[f"grid_{tag}_theta"]
        _, nr, nc, g = gold_ref[f"grid_{tag}_meta"]
        pg = L.PolarGrid(th, int(nr), int(nc), np.float32(g))
        x, y, z = pg.points()
        gx, gy, gz = gold_ref[f"grid_{tag}_xyz"]
        assert np.array_equal(x, gx) and np.array_equal(y, gy) and np.array_equal(z, gz)


def _golden_grid(L, gold_orc):
    th = gold_orc["op_theta"]
    nr, nc, g = gold_orc["op_meta"]
    return L.PolarGrid(th, int(nr), int(nc), np.float32(g)), np.float32(g)


def test_nufft_vs_golden_nudft(L, gold_orc):
    pg, _ = _golden_grid(L, gold_orc)
    assert rel(L.nufft3d2(gold_orc["op_f"], pg), gold_orc["op_nudft2"]) < TOL
    assert rel(L.nufft3d1(gold_orc["op_c"], pg, (9, 5, 11)), gold_orc["op_nudft1"]) < TOL


def test_operators_vs_golden(L, gold_orc):
    pg, g = _golden_grid(L, gold_orc)
    assert rel(L.forward(gold_orc["op_m"], pg, g), gold_orc["op_forward"]) < TOL
    assert rel(L.adjoint(gold_orc["op_proj"], pg, (9, 5, 11), g), gold_orc["op_adjoint"]) < TOL
    assert rel(L.sysmat(gold_orc["op_m"], pg, g), gold_orc["op_sysmat"]) < TOL


CASES = [
    # volume dims, [(nproj, nrows, ncols, gamma)]
    ((22, 6, 20), [(7, 31, 29, 0.0), (5, 31, 29, np.pi / 4)]),
    ((17, 9, 24), [(6, 26, 34, 1.1)]),
]


@pytest.mark.parametrize("dims,geoms", CASES)
def test_operators_vs_oracle(L, O, dims, geoms):
    rng = np.random.default_rng(11)
    plan_o = O.NufftPlan(dims, eps=1e-12)
    pgs, opgs = [], []
    for np_, nr, nc, g in geoms:
        th = rng.uniform(0, 2 * np.pi, np_).astype(np.float32)
        pgs.append(L.PolarGrid(th, nr, nc, np.float32(g)))
        opgs.append(O.PolarGrid(th, nr, nc, np.float32(g)))
    m = O.synthetic_magnetization(dims, seed=5, sigma=1.5)
    for pg, opg in zip(pgs, opgs):
        assert rel(L.forward(m, pg), O.forward(m, opg, opg.gamma, plan_o)) < TOL
        proj = rng.standard_normal(opg.dims()).astype(np.float32)
        assert rel(L.adjoint(proj, pg, dims), O.adjoint(proj, opg, dims, opg.gamma, plan_o)) < TOL
    want = O.normal(m, opgs, [p.gamma for p in opgs], plan_o)
    assert rel(L.sysmat(m, pgs), want) < TOL
    # random (white) input exercises high frequencies
    xr = rng.standard_normal((3,) + dims).astype(np.float32)
    assert rel(L.sysmat(xr, pgs), O.normal(xr, opgs, [p.gamma for p in opgs], plan_o)) < TOL


@pytest.mark.parametrize("bins", [(8, 8, 8), (4, 4, 4), (16, 2, 8), (3, 5, 7), (4, 16, 4)])
def test_bin_layouts_vs_oracle(L, O, bins):
    """Spreading / interpolation give the oracle's result for any bin layout,
    including bins larger than the fine grid (tiles wrapping onto themselves)."""
    dims, geoms = CASES[0]
    rng = np.random.default_rng(21)
    plan_o = O.NufftPlan(dims, eps=1e-12)
    plan = L.NufftPlan(dims).set_bins(*bins)
    pgs, opgs = [], []
    for np_, nr, nc, g in geoms:
        th = rng.uniform(0, 2 * np.pi, np_).astype(np.float32)
        pgs.append(L.PolarGrid(th, nr, nc, np.float32(g)))
        opgs.append(O.PolarGrid(th, nr, nc, np.float32(g)))
    m = rng.standard_normal((3,) + dims).astype(np.float32)
    for pg, opg in zip(pgs, opgs):
        assert rel(L.forward(m, pg, plan=plan), O.forward(m, opg, opg.gamma, plan_o)) < TOL
        proj = rng.standard_normal(opg.dims()).astype(np.float32)
        assert rel(L.adjoint(proj, pg, dims, plan=plan), O.adjoint(proj, opg, dims, opg.gamma, plan_o)) < TOL
    assert rel(L.sysmat(m, pgs, plan=plan), O.normal(m, opgs, [p.gamma for p in opgs], plan_o)) < TOL
    f = (rng.standard_normal(dims) + 1j * rng.standard_normal(dims)).astype(np.complex64)
    c = L.nufft3d2(f, pgs[1], plan=plan)
    assert rel(c, O.nufft3d2(f.astype(np.complex128), opgs[1], plan_o)) < TOL
    assert rel(L.nufft3d1(c, pgs[1], dims, plan=plan),
               O.nufft3d1(c.astype(np.complex128), opgs[1], plan_o)) < TOL


def test_autotuners_keep_results(L, O):
    """The tuned launch shapes and bin layouts give the oracle's results, and a
    second tuning of the same size comes from the cache."""
    dims, geoms = CASES[0]
    rng = np.random.default_rng(41)
    pgs, opgs = [], []
    for np_, nr, nc, g in geoms:
        th = rng.uniform(0, 2 * np.pi, np_).astype(np.float32)
        pgs.append(L.PolarGrid(th, nr, nc, np.float32(g)))
        opgs.append(O.PolarGrid(th, nr, nc, np.float32(g)))
    plan_o = O.NufftPlan(dims, eps=1e-12)
    x = rng.standard_normal((3,) + dims).astype(np.float32)
    want = O.normal(x, opgs, [p.gamma for p in opgs], plan_o)
    plan = L.NufftPlan(dims)
    bins, ms = plan.autotune(pgs, "normal")
    assert len(bins) == 3 and ms > 0
    assert rel(L.sysmat(x, pgs, plan=plan), want) < TOL
    bins2, ms2 = L.NufftPlan(dims).autotune(pgs, "normal")
    assert bins2 == bins and ms2 == 0.0
    T = L.ToeplitzNormal(pgs, dims)
    rows, kb, ms = T.autotune()
    assert rows >= 1 and kb >= 1 and ms > 0
    assert rel(T(x), want) < TOL
    assert L.ToeplitzNormal(pgs, dims).autotune()[2] == 0.0


def test_bin_layout_rejects_bad_sizes(L):
    plan = L.NufftPlan((8, 6, 8))
    with pytest.raises(L.LaminoError):
        plan.set_bins(0, 8, 8)
    with pytest.raises(L.LaminoError):
        plan.set_bins(40, 40, 40)  # tile beyond shared memory


@pytest.mark.parametrize("dims,geoms", CASES)
def test_toeplitz_vs_oracle(L, O, dims, geoms):
    rng = np.random.default_rng(12)
    pgs, opgs, ths = [], [], []
    for np_, nr, nc, g in geoms:
        th = rng.uniform(0, 2 * np.pi, np_).astype(np.float32)
        ths.append(th)
        pgs.append(L.PolarGrid(th, nr, nc, np.float32(g)))
        opgs.append(O.PolarGrid(th, nr, nc, np.float32(g)))
    plan_o = O.NufftPlan(dims, eps=1e-12)
    T = L.ToeplitzNormal(pgs, dims, "fp32")
    for x in (O.synthetic_magnetization(dims, seed=6, sigma=1.5),
              rng.standard_normal((3,) + dims).astype(np.float32)):
        want = O.normal(x, opgs, [p.gamma for p in opgs], plan_o)
        assert rel(T(x), want) < TOL
        assert rel(T(x), L.sysmat(x, pgs)) < TOL
    T16 = L.ToeplitzNormal(pgs, dims, "fp16")
    x = O.synthetic_magnetization(dims, seed=7, sigma=1.5)
    assert rel(T16(x), T(x)) < 2e-3


def test_toeplitz_matches_analytic_oracle(L, O):
    rng = np.random.default_rng(13)
    dims = (9, 4, 8)
    ths = [rng.uniform(0, 6.28, 5).astype(np.float32), rng.uniform(0, 6.28, 3).astype(np.float32)]
    gms = [0.0, 0.9]
    T = L.ToeplitzNormal([L.PolarGrid(t, 12, 11, g) for t, g in zip(ths, gms)], dims)
    Tk = O.toeplitz_kernel(dims, [t.astype(np.float64) for t in ths],
                           [float(np.float32(g)) for g in gms], 12, 11)
    x = rng.standard_normal((3,) + dims).astype(np.float32)
    assert rel(T(x), O.toeplitz_apply(x.astype(np.float64), Tk)) < TOL


@pytest.mark.parametrize("dims,geoms", CASES)
def test_toeplitz_quadforms_match_applies(L, O, dims, geoms):
    """Parseval quadratic forms x_i . S_g x_i equal the dot products with applies
    of each per-gamma operator, and the summed operator's form is their sum."""
    rng = np.random.default_rng(31)
    pgs = [L.PolarGrid(rng.uniform(0, 2 * np.pi, n).astype(np.float32), nr, nc, np.float32(g))
           for n, nr, nc, g in geoms]
    parts = [L.ToeplitzNormal([pg], dims) for pg in pgs]
    total = L.ToeplitzNormal(pgs, dims)
    x = rng.standard_normal((3,) + dims).astype(np.float32)
    q = total.quadforms(x, parts)
    for gi, T in enumerate(parts):
        y = T(x)
        want = [float(np.dot(x[i].ravel().astype(np.float64), y[i].ravel())) for i in range(3)]
        assert np.allclose(q[gi], want, rtol=1e-5, atol=1e-6 * max(abs(w) for w in want)), (gi, q[gi], want)
    qs = total.quadforms(x, [total])[0]
    assert np.allclose(qs, q.sum(axis=0), rtol=1e-5)


def test_edge_sizes(L, O):
    """Degenerate shapes: single projection, single row, thin volume."""
    rng = np.random.default_rng(14)
    dims = (3, 1, 2)
    th = np.array([0.3], np.float32)
    pg = L.PolarGrid(th, 1, 3, 0.5)
    opg = O.PolarGrid(th, 1, 3, np.float32(0.5))
    pe = O.NufftPlan(dims, exact=True)
    m = rng.standard_normal((3,) + dims).astype(np.float32)
    assert rel(L.forward(m, pg), O.forward(m, opg, opg.gamma, pe)) < TOL
    assert rel(L.sysmat(m, pg), O.sysmat(m, opg, opg.gamma, pe)) < TOL
    T = L.ToeplitzNormal([pg], dims)
    assert rel(T(m), O.sysmat(m, opg, opg.gamma, pe)) < TOL


def test_invalid_arguments_raise(L):
    with pytest.raises(L.LaminoError) as e:
        L.PolarGrid(np.zeros(0, np.float32), 5, 5, 0.0)
    assert e.value.code == 1
    with pytest.raises(L.LaminoError):
        L.NufftPlan((0, 4, 4))
    pg = L.PolarGrid([0.1], 4, 4, 0.0)
    with pytest.raises(L.LaminoError):
        L.ToeplitzNormal([pg], (4, -1, 4))


def test_device_tensors_in_place(L, O):
    """torch CUDA tensors go through the same C ABI without host staging."""
    import torch
    dims = (12, 5, 10)
    th = np.linspace(0, 3, 6, dtype=np.float32)
    pg = L.PolarGrid(th, 17, 15, 0.4)
    x = O.synthetic_magnetization(dims, seed=3, sigma=1.5)
    xd = torch.from_numpy(x).cuda()
    T = L.ToeplitzNormal([pg], dims)
    yd = T(xd)
    torch.cuda.synchronize()
    assert yd.is_cuda
    assert rel(yd.cpu().numpy(), T(x)) < 1e-6


def test_full_size_toeplitz_properties(L):
    """51x511x511 reconstruction size (padded 721x71x721), 4 gammas x 361 angles,
    1233x1233 padded projections: symmetry, linearity, agreement with the NUFFT form."""
    import torch
    dims = (721, 71, 721)
    rng = np.random.default_rng(15)
    pgs = [L.PolarGrid(rng.uniform(0, 2 * np.pi, 361).astype(np.float32), 1233, 1233, g)
           for g in np.deg2rad([0.0, 45.0, 90.0, 135.0]).astype(np.float32)]
    T = L.ToeplitzNormal(pgs, dims, "fp32")
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((3,) + dims, device="cuda", generator=g)
    y = torch.randn((3,) + dims, device="cuda", generator=g)
    Ax, Ay = T(x), T(y)
    lhs = torch.sum(Ax.double() * y.double()).item()
    rhs = torch.sum(x.double() * Ay.double()).item()
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs)
    assert torch.sum(x.double() * Ax.double()).item() > 0
    Axy = T(2.0 * x - 0.5 * y)
    assert (torch.linalg.norm(Axy - (2.0 * Ax - 0.5 * Ay)) / torch.linalg.norm(Axy)).item() < 1e-5
    # smooth input: agreement with the NUFFT-form sum_gamma sysmat.  At this size
    # both FP32 forms carry rounding at the 1e-5 level: the NUFFT form accumulates
    # 2.2e9 points x 343 taps with float atomics on float coordinates (its spread
    # against the Toeplitz form measured 2.6e-5 at w=7 and 3.7e-5 at w=8, i.e. not
    # kernel-width limited), so the bar here is 1e-4.
    k = torch.arange(721, device="cuda", dtype=torch.float32)
    s = torch.exp(-((k - 360) / 120.0) ** 2)
    xs = (s[:, None, None] * torch.ones(71, device="cuda")[None, :, None] * s[None, None, :])
    xs = torch.stack([xs, 0.5 * xs, -0.25 * xs]).contiguous()
    ys = T(xs)
    yn = L.sysmat(xs, pgs)
    assert (torch.linalg.norm(ys - yn) / torch.linalg.norm(yn)).item() < 1e-4


@pytest.mark.parametrize("dims", [(721, 3, 8), (5, 71, 9), (4, 3, 721), (721, 71, 9), (90, 3, 8), (180, 3, 8),
                                  (270, 3, 8), (362, 3, 8), (4, 10, 90), (4, 22, 180), (4, 32, 270),
                                  (4, 44, 362)])
def test_toeplitz_compiled_fft_lengths(L, O, dims):
    """Thin volumes whose FFT lengths hit the compile-time schedules (n1 = 721 ->
    1458, n2 = 71 -> 144, n3 = 721 -> packed 729; n1 = 90 / 180 / 270 / 362 ->
    180 / 360 / 540 / 750, n2 = 10 / 22 / 32 / 44 -> 20 / 48 / 64 / 90 and n3 =
    90 / 180 / 270 / 362 -> packed 90 / 180 / 270 / 375, the lengths of the
    batched mix) against the oracle.  The
    Toeplitz form evaluates the exact lattice, so the oracle here uses FP64
    points (the reference's double path): with white input on a 721-long axis
    the float32 points of the float path move the highest modes' phases by about
    k * ulp and differ from it by 2.5e-5."""
    rng = np.random.default_rng(16)
    th = rng.uniform(0, 2 * np.pi, 4).astype(np.float32)
    pg = L.PolarGrid(th, 13, 11, np.float32(0.7))
    opg = O.PolarGrid(th, 13, 11, np.float32(0.7), dtype=np.float64)
    x = rng.standard_normal((3,) + dims).astype(np.float32)
    want = O.sysmat(x, opg, opg.gamma, O.NufftPlan(dims, exact=True))
    T = L.ToeplitzNormal([pg], dims)
    y = T(x)
    assert rel(y, want) < TOL
    assert rel(L.ToeplitzNormal([pg], dims, "fp16")(x), want) < 2e-3
    # the quadratic forms read the spectra in the same storage order as the apply
    q = T.quadforms(x, [T])[0]
    dots = [float(np.dot(x[i].ravel().astype(np.float64), y[i].ravel())) for i in range(3)]
    assert np.allclose(q, dots, rtol=1e-5, atol=1e-6 * max(abs(d) for d in dots)), (q, dots)


def test_toeplitz_apply_many_matches_single_applies(L, O):
    """lamino_normal_apply_many on host volumes (pageable numpy and pinned
    tensors; odd and even counts) gives each volume's single-apply result
    bit for bit, and rejects device buffers."""
    import torch
    rng = np.random.default_rng(3)
    dims = (17, 6, 15)
    pgs = [L.PolarGrid(rng.uniform(0, 2 * np.pi, 5).astype(np.float32), 23, 21, np.float32(g)) for g in (0.0, 0.9)]
    T = L.ToeplitzNormal(pgs, dims)
    xs = [rng.standard_normal((3,) + dims).astype(np.float32) for _ in range(5)]
    want = [T(x) for x in xs]
    for n in (1, 2, 5):
        outs = [np.empty_like(x) for x in xs[:n]]
        T.apply_many(xs[:n], outs)
        for o, w in zip(outs, want):
            assert np.array_equal(o, w)
    xp = [torch.from_numpy(x).pin_memory() for x in xs[:3]]
    yp = [torch.empty_like(x).pin_memory() for x in xp]
    T.apply_many(xp, yp)
    for o, w in zip(yp, want):
        assert np.array_equal(o.numpy(), w)
    xd = torch.from_numpy(xs[0]).cuda()
    with pytest.raises(ValueError):
        T.apply_many([xd], [torch.empty_like(xd)])
