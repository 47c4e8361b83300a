"""lamino_residual_noalloc: the allocation-free residual.

It exists for callers that cannot allocate device memory (a service overlapping
reconstructions on one GPU, whose line search must not stall other requests on
a cudaMalloc/cudaFree; a caller whose device memory belongs to another
allocator).  This test calls it through the C ABI on device tensors and checks
it against lamino_residual on two calls in a row, so the second call runs on
the static scratch the first one left behind.  The file is named to be
collected last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bind(L):
    lib = L.lib()
    fn = lib.lamino_residual_noalloc
    vp = ctypes.c_void_p
    fn.argtypes = [vp, vp, vp, vp, ctypes.c_float, ctypes.POINTER(ctypes.c_double), vp]
    fn.restype = ctypes.c_int
    return fn


def test_residual_noalloc_matches_residual(L, O):
    import torch
    fn = _bind(L)
    dims = (20, 8, 18)
    rng = np.random.default_rng(21)
    th = rng.uniform(0, 2 * np.pi, 7).astype(np.float32)
    pg = L.PolarGrid(th, 27, 25, np.float32(0.6))
    plan = L.NufftPlan(dims)
    f = torch.from_numpy(O.synthetic_magnetization(dims, seed=4, sigma=1.5)).cuda()
    yT = torch.from_numpy(rng.standard_normal((3,) + dims).astype(np.float32)).cuda()
    yTy = float(torch.sum(yT.double() * yT.double()).item())
    want = L.residual(f, yT, pg, yTy, plan=plan)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        got = ctypes.c_double()
        rc = fn(plan._h, pg._h, ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(yT.data_ptr()),
                yTy, ctypes.byref(got), stream)
        assert rc == 0, L.lib().lamino_last_error().decode()
        assert got.value == pytest.approx(want, rel=1e-5)


def test_residual_noalloc_rejects_host_pointers(L):
    fn = _bind(L)
    dims = (6, 4, 5)
    pg = L.PolarGrid(np.array([0.2, 1.0], np.float32), 9, 9, 0.3)
    plan = L.NufftPlan(dims)
    f = np.zeros((3,) + dims, np.float32)
    got = ctypes.c_double()
    rc = fn(plan._h, pg._h, ctypes.c_void_p(f.ctypes.data), ctypes.c_void_p(f.ctypes.data), 0.0,
            ctypes.byref(got), None)
    assert rc == 1
    assert b"device pointers" in L.lib().lamino_last_error()
