"""GPU parity against the reference's OWN code: the fixtures
tests/golden/reference_path_*.npz were produced by the reference's
src/projection.cpp, src/gradient.cpp, include/precond.h, src/conjgrad.cpp,
src/bregman.cpp, src/nagopt.cpp and MBIR drivers compiled unmodified (double
precision) against this project's FINUFFT-API / FFTW-API shims
(tests/golden/make_reference_golden.py).  Everything runs through the C ABI.

Tolerances: a single operator apply within relative L2 1e-5, a solver or
reconstruction (final volume) within 1e-4.
"""
import hashlib
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel

pytestmark = pytest.mark.gpu
TOL_APPLY = 1e-5
TOL_VOLUME = 1e-4


@pytest.fixture(scope="module")
def ops():
    return dict(np.load(os.path.join(GOLDEN, "reference_path_ops.npz")))


@pytest.fixture(scope="module")
def solvers():
    return dict(np.load(os.path.join(GOLDEN, "reference_path_solvers.npz")))


def _grids(L, d):
    out = []
    for i in range(2):
        nr, nc, g = d[f"geom{i}"]
        out.append(L.PolarGrid(d[f"angles{i}"], int(nr), int(nc), np.float32(g)))
    return out


def test_operators_vs_reference(L, ops):
    dims = tuple(int(v) for v in ops["dims"])
    x = ops["x"].astype(np.float32)
    yT = ops["yT"].astype(np.float32)
    pgs = _grids(L, ops)
    for i, pg in enumerate(pgs):
        assert rel(L.forward(x, pg), ops[f"forward{i}"]) < TOL_APPLY
        assert rel(L.sysmat(x, pg), ops[f"sysmat{i}"]) < TOL_APPLY
        assert rel(L.gradient(x, yT, pg), ops[f"gradient{i}"]) < TOL_APPLY
        r = L.residual(x, yT, pg, float(ops[f"yTy{i}"]))
        assert r == pytest.approx(float(ops[f"residual{i}"]), rel=TOL_APPLY)
    assert rel(L.adjoint(ops["proj"].astype(np.float32), pgs[0], dims), ops["adjoint0"]) < TOL_APPLY
    assert rel(L.sysmat(x, pgs), ops["normal"]) < TOL_APPLY
    T = L.ToeplitzNormal(pgs, dims, "fp32")
    assert rel(T(x), ops["normal"]) < TOL_APPLY


@pytest.mark.parametrize("tag", ["even", "odd"])
def test_ramp_preconditioner_vs_reference(L, ops, tag):
    v = ops[f"ramp_{tag}_in"].astype(np.float32)
    got = L.opt.ramp_precond(np.stack([v, 2 * v, -v]))
    want = ops[f"ramp_{tag}"]
    assert rel(got, np.stack([want, 2 * want, -want])) < TOL_APPLY


def test_solvers_vs_reference(L, solvers):
    dims = tuple(int(v) for v in solvers["dims"])
    pgs = _grids(L, solvers)
    T = L.ToeplitzNormal(pgs, dims)
    b = solvers["b"].astype(np.float32)
    x0 = np.zeros_like(b)
    assert rel(L.opt.cgsolver(T, b, x0, 8, 0.0), solvers["cg"]) < TOL_VOLUME
    assert rel(L.opt.split_bregman(T, b, x0, 0.1, 10.0, 3, 3, 0.0, 0.0), solvers["sb"]) < TOL_VOLUME


@pytest.mark.parametrize("method", [1, 2, 3])
@pytest.mark.parametrize("kind", ["toeplitz", "nufft"])
def test_mbir_vs_reference(L, solvers, method, kind):
    from make_reference_golden import MBIR_PARAMS, MBIR_RECON
    data = [(solvers[f"mbir_proj{i}"], solvers[f"mbir_angles{i}"], np.float32(solvers[f"mbir_gamma{i}"]))
            for i in range(2)]
    kw = MBIR_PARAMS[method]
    p = L.ReconParams(maxIters=kw["max_iters"], innerIters=kw["inner_iters"], op_kind=kind)
    got = {1: L.MBIR1, 2: L.MBIR2, 3: L.MBIR3}[method](data, MBIR_RECON, p)
    err = rel(got, solvers[f"mbir{method}"])
    print(f"MBIR{method} {kind} vs reference: {err:.2e}")
    assert err < TOL_VOLUME


@pytest.mark.parametrize("kind", ["toeplitz", "nufft"])
def test_config0_mbir1_vs_reference(L, O, kind):
    """Config 0 end to end: recon 16 x 128 x 128 (internal 128 x 16 x 128,
    padded 180 x 22 x 180), 2 gammas x 90 angles, 128 x 128 projections, 20 CG
    iterations (src/mbir_cg.cpp:48-128), against the reference's own MBIR1 in
    double precision."""
    gold = np.load(os.path.join(GOLDEN, "reference_path_config0.npz"))
    data = O.config0_datasets()
    h = hashlib.sha256()
    for d in data:
        for a in d:
            h.update(np.ascontiguousarray(a).tobytes())
    same_inputs = h.hexdigest() == str(gold["inputs_sha256"])
    got = L.MBIR1(data, O.CONFIG0_RECON, L.ReconParams(maxIters=20, op_kind=kind))
    err = rel(got, gold["mbir1"])
    print(f"config0 MBIR1 {kind} vs reference FP64: {err:.2e} (inputs bit-identical: {same_inputs})")
    assert err < TOL_VOLUME
