"""The reference's C++ operator surface over the C ABI (include/lamino_tomocam.hpp).

tests/cpp/shim_test.cpp includes the header together with the reference's own
polar_grid.h / array.h (compiled by tests/cpp/Makefile) and calls
tomocam::gpu::forward / adjoint / sysmat / gradient / residual, the summed
normal operator and MBIR1 / MBIR3 on Array<float> data.  Its results are
compared with the outputs of the reference's own code in double precision
(tests/golden/reference_path_*.npz): a single operator apply within relative L2
1e-5, a reconstruction within 1e-4.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT, rel

pytestmark = pytest.mark.gpu
BIN = os.path.join(ROOT, "tests", "cpp", "_build", "shim_test")
TOL_APPLY = 1e-5
TOL_VOLUME = 1e-4


def _put(d, name, a, dtype):
    np.ascontiguousarray(a, dtype=dtype).tofile(os.path.join(d, name))


def _get(d, name, shape):
    return np.fromfile(os.path.join(d, f"out_{name}.f32"), np.float32).reshape(shape)


def test_cpp_shim_vs_reference(L, tmp_path):
    from make_reference_golden import MBIR_PARAMS, MBIR_RECON
    assert os.path.exists(BIN), "tests/cpp/_build/shim_test is not built (tests/cpp/Makefile)"
    ops = dict(np.load(os.path.join(GOLDEN, "reference_path_ops.npz")))
    sol = dict(np.load(os.path.join(GOLDEN, "reference_path_solvers.npz")))
    d = str(tmp_path)
    dims = [int(v) for v in ops["dims"]]
    geoms = [ops["geom0"], ops["geom1"]]
    mp = [sol["mbir_proj0"], sol["mbir_proj1"]]
    meta = dims + [len(ops["angles0"]), int(geoms[0][0]), int(geoms[0][1]),
                   len(ops["angles1"]), int(geoms[1][0]), int(geoms[1][1])]
    meta += list(mp[0].shape) + list(mp[1].shape) + list(MBIR_RECON)
    meta += [MBIR_PARAMS[1]["max_iters"], MBIR_PARAMS[3]["max_iters"]]
    _put(d, "meta.i64", meta, np.int64)
    _put(d, "gammas.f32", [geoms[0][2], geoms[1][2], sol["mbir_gamma0"], sol["mbir_gamma1"]], np.float32)
    for g in range(2):
        _put(d, f"angles{g}.f32", ops[f"angles{g}"], np.float32)
        _put(d, f"mproj{g}.f32", mp[g], np.float32)
        _put(d, f"mangles{g}.f32", sol[f"mbir_angles{g}"], np.float32)
    for k in ("x", "yT", "proj"):
        _put(d, f"{k}.f32", ops[k], np.float32)
    _put(d, "yTy.f32", [ops["yTy0"]], np.float32)

    r = subprocess.run([BIN, d], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "invalid_argument on a grid without projections: yes" in r.stdout, r.stdout

    vol = (3,) + tuple(dims)
    for g in range(2):
        assert rel(_get(d, f"forward{g}", ops[f"forward{g}"].shape), ops[f"forward{g}"]) < TOL_APPLY
        assert rel(_get(d, f"sysmat{g}", vol), ops[f"sysmat{g}"]) < TOL_APPLY
        assert rel(_get(d, f"gradient{g}", vol), ops[f"gradient{g}"]) < TOL_APPLY
    assert rel(_get(d, "adjoint0", vol), ops["adjoint0"]) < TOL_APPLY
    assert float(_get(d, "residual0", (1,))[0]) == pytest.approx(float(ops["residual0"]), rel=TOL_APPLY)
    assert rel(_get(d, "normal", vol), ops["normal"]) < TOL_APPLY
    rvol = (3,) + tuple(MBIR_RECON)
    for k in (1, 3):
        err = rel(_get(d, f"mbir{k}", rvol), sol[f"mbir{k}"])
        print(f"C++ shim MBIR{k} vs reference: {err:.2e}")
        assert err < TOL_VOLUME
