"""CPU tests: the oracle's restatement of the operator and solver compositions
pinned to the reference's OWN code.

The fixtures tests/golden/reference_path_*.npz come from the reference's
src/projection.cpp, src/gradient.cpp, include/precond.h, src/conjgrad.cpp,
src/bregman.cpp, src/nagopt.cpp, src/qggmrf.cpp and the MBIR drivers compiled
unmodified against this project's FINUFFT-API / FFTW-API shims, run in double
precision (tests/golden/make_reference_golden.py).  Each composition of the
oracle (shift and scale order, the sysmat weights, the ramp filter and its
1 / (n2 n3), the CG stopping rule, the split-Bregman outer loop, the MBIR
normalisation and padding) must reproduce them; tolerances are those of two
FP64 NUFFTs (eps 1e-12 vs 1e-14).
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, rel

OPS = os.path.join(GOLDEN, "reference_path_ops.npz")
SOLVERS = os.path.join(GOLDEN, "reference_path_solvers.npz")


@pytest.fixture(scope="module")
def ops():
    return dict(np.load(OPS))


@pytest.fixture(scope="module")
def solvers():
    return dict(np.load(SOLVERS))


def _grid(O, d, i, dtype=np.float64):
    nr, nc, g = d[f"geom{i}"]
    return O.PolarGrid(d[f"angles{i}"], int(nr), int(nc), np.float32(g), dtype=dtype), float(np.float32(g))


def test_operators_match_reference(O, ops):
    dims = tuple(int(v) for v in ops["dims"])
    plan = O.NufftPlan(dims, eps=1e-12)
    x, yT = ops["x"], ops["yT"]
    grids = []
    for i in range(2):
        pg, g = _grid(O, ops, i)
        grids.append((pg, g))
        assert rel(O.forward(x, pg, g, plan), ops[f"forward{i}"]) < 1e-10
        assert rel(O.sysmat(x, pg, g, plan), ops[f"sysmat{i}"]) < 1e-10
        assert rel(O.gradient(x, yT, pg, g, plan), ops[f"gradient{i}"]) < 1e-10
        r = O.residual(x, yT, pg, float(ops[f"yTy{i}"]), g, plan)
        assert r == pytest.approx(float(ops[f"residual{i}"]), rel=1e-10)
    pg, g = grids[0]
    assert rel(O.adjoint(ops["proj"], pg, dims, g, plan), ops["adjoint0"]) < 1e-10
    want = ops["normal"]
    assert rel(O.normal(x, [p for p, _ in grids], [g for _, g in grids], plan), want) < 1e-10


def test_reference_float_build_accuracy(O, ops):
    """The reference as it runs by default (float plans, tol 1.2e-6, float
    points) is within a few 1e-6 of its double build: the scale of the 1e-5
    single-apply tolerance."""
    for i in range(2):
        assert rel(ops[f"sysmat{i}_f32"], ops[f"sysmat{i}"]) < 5e-6
        assert rel(ops[f"forward{i}_f32"], ops[f"forward{i}"]) < 5e-6


@pytest.mark.parametrize("tag", ["even", "odd"])
def test_ramp_preconditioner_matches_reference(O, ops, tag):
    v = ops[f"ramp_{tag}_in"]
    assert rel(O.RampPreconditioner(v.shape).apply(v), ops[f"ramp_{tag}"]) < 1e-12


def _solver_problem(O, s):
    dims = tuple(int(v) for v in s["dims"])
    plan = O.NufftPlan(dims, eps=1e-12)
    grids = [_grid(O, s, i) for i in range(2)]
    A = lambda v: O.normal(v, [p for p, _ in grids], [g for _, g in grids], plan)
    return dims, A


def test_cgsolver_matches_reference(O, solvers):
    _, A = _solver_problem(O, solvers)
    b = solvers["b"]
    got = O.cgsolver(A, b, np.zeros_like(b), 8, 0.0)
    assert rel(got, solvers["cg"]) < 1e-9


def test_split_bregman_matches_reference(O, solvers):
    _, A = _solver_problem(O, solvers)
    b = solvers["b"]
    got = O.split_bregman(A, b, np.zeros_like(b), 0.1, 10.0, 3, 3, 0.0, 0.0)
    assert rel(got, solvers["sb"]) < 1e-9


@pytest.mark.parametrize("method", [1, 2, 3])
def test_mbir_matches_reference(O, solvers, method):
    from make_reference_golden import MBIR_PARAMS, MBIR_RECON
    data = [(solvers[f"mbir_proj{i}"], solvers[f"mbir_angles{i}"], np.float32(solvers[f"mbir_gamma{i}"]))
            for i in range(2)]
    kw = MBIR_PARAMS[method]
    po = O.ReconParams(maxIters=kw["max_iters"], innerIters=kw["inner_iters"])
    fn = {1: O.MBIR1, 2: O.MBIR2, 3: O.MBIR3}[method]
    got = fn(data, MBIR_RECON, po, eps=1e-12, grid_dtype=np.float64)
    assert rel(got, solvers[f"mbir{method}"]) < 1e-8


def test_mbir3_toeplitz_form_matches_reference(O, solvers):
    """The oracle's MBIR3 with FP64 Toeplitz operators (used where the NUFFT
    form is too slow on the CPU) reproduces the reference's own MBIR3."""
    from make_reference_golden import MBIR_PARAMS, MBIR_RECON
    data = [(solvers[f"mbir_proj{i}"], solvers[f"mbir_angles{i}"], np.float32(solvers[f"mbir_gamma{i}"]))
            for i in range(2)]
    kw = MBIR_PARAMS[3]
    po = O.ReconParams(maxIters=kw["max_iters"], innerIters=kw["inner_iters"])
    got, L = O.MBIR3_toeplitz(data, MBIR_RECON, po, grid_dtype=np.float64)
    assert L == po.mu
    assert rel(got, solvers["mbir3"]) < 1e-6


def test_reference_fixture_inputs_regenerate(O, ops, solvers):
    """The fixtures' inputs are reproducible from their seeds (the GPU tests
    rebuild them the same way)."""
    from make_reference_golden import mbir_datasets, ops_inputs, solver_inputs
    geoms, x, yT, proj, re, ro = ops_inputs()
    assert np.array_equal(x, ops["x"]) and np.array_equal(proj, ops["proj"])
    assert np.array_equal(geoms[1][0], ops["angles1"])
    g2, b = solver_inputs()
    assert np.array_equal(b, solvers["b"])
    for i, (p, th, g) in enumerate(mbir_datasets()):
        assert np.allclose(p, solvers[f"mbir_proj{i}"], rtol=0, atol=1e-6)


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "..", "..", "oracle", "_ref", "libtomocam_ref.so")),
                    reason="compiled reference path not built")
def test_reference_live_sysmat_random_case(O):
    """A fresh random case through the compiled reference (its own process,
    since the reference fixes one NUFFT size per process) against the oracle."""
    from oracle import refpath as R
    rng = np.random.default_rng(99)
    dims = (7, 4, 9)
    th = rng.uniform(0, 2 * np.pi, 4)
    x = rng.standard_normal((3,) + dims)
    pg = O.PolarGrid(th, 9, 11, 1.3, dtype=np.float64)
    want = O.sysmat(x, pg, 1.3, O.NufftPlan(dims, eps=1e-12))
    assert rel(R.isolated("sysmat", x, th, 9, 11, 1.3), want) < 1e-10
