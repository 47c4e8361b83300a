"""lamino_residual_noalloc: the allocation-free residual.

It exists for callers that cannot allocate device memory (a service overlapping
reconstructions on one GPU, whose line search must not stall other requests on
a cudaMalloc/cudaFree; a caller whose device memory belongs to another
allocator).  These tests call it through the C ABI on device tensors, on two
calls in a row (the second runs on the static scratch the first one left
behind), and check it against the FP64 oracle and against lamino_residual.  The
first test uses a plan that has never sorted its geometry, so the normal
operator takes the unsorted point kernel; the device's free memory and the
default memory pool's usage must not change across a call.  The file is named
to be collected last.
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


def _pool_used():
    """Bytes in use in the device's default stream-ordered pool (None if the
    runtime bindings are not importable)."""
    try:
        from cuda.bindings import runtime as rt
    except ImportError:
        try:
            from cuda import cudart as rt
        except ImportError:
            return None
    err, dev = rt.cudaGetDevice()
    err, pool = rt.cudaDeviceGetDefaultMemPool(dev)
    err, used = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
    return int(used)


def _problem(L, O, dims, seed):
    import torch
    rng = np.random.default_rng(seed)
    th = rng.uniform(0, 2 * np.pi, 7).astype(np.float32)
    pg = L.PolarGrid(th, 27, 25, np.float32(0.6))
    opg = O.PolarGrid(th, 27, 25, np.float32(0.6))
    f = O.synthetic_magnetization(dims, seed=4, sigma=1.5)
    yT = rng.standard_normal((3,) + dims).astype(np.float32)
    yTy = float(np.sum(yT.astype(np.float64) ** 2))
    want = O.residual(f.astype(np.float64), yT.astype(np.float64), opg, yTy, opg.gamma,
                      O.NufftPlan(dims, eps=1e-12))
    return pg, torch.from_numpy(f).cuda(), torch.from_numpy(yT).cuda(), yTy, want


def _call(L, fn, plan, pg, f, yT, yTy):
    import torch
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    got = ctypes.c_double()
    rc = fn(plan._h, pg._h, ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(yT.data_ptr()), yTy,
            ctypes.byref(got), stream)
    assert rc == 0, L.lib().lamino_last_error().decode()
    return got.value


def test_residual_noalloc_unsorted_plan_vs_oracle(L, O):
    """A plan that never sorted its geometry (unsorted point kernel), two calls
    in a row, against the FP64 oracle (src/gradient.cpp:117-127) at 1e-5, with
    no change in device memory across the second call."""
    import torch
    fn = _bind(L)
    dims = (20, 8, 18)
    pg, f, yT, yTy, want = _problem(L, O, dims, seed=21)
    plan = L.NufftPlan(dims)
    first = _call(L, fn, plan, pg, f, yT, yTy)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    pool0 = _pool_used()
    second = _call(L, fn, plan, pg, f, yT, yTy)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert _pool_used() == pool0
    for got in (first, second):
        assert got == pytest.approx(want, rel=1e-5)


def test_residual_noalloc_matches_residual(L, O):
    """After lamino_residual sorted the geometry (binned kernel): the same value
    as lamino_residual and as the oracle, on two calls in a row."""
    fn = _bind(L)
    dims = (20, 8, 18)
    pg, f, yT, yTy, want = _problem(L, O, dims, seed=22)
    plan = L.NufftPlan(dims)
    ref = L.residual(f, yT, pg, yTy, plan=plan)
    assert ref == pytest.approx(want, rel=1e-5)
    for _ in range(2):
        assert _call(L, fn, plan, pg, f, yT, yTy) == pytest.approx(ref, rel=1e-5)


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


def test_residual_noalloc_rejects_volumes_above_the_limit(L):
    """3 x V floats + 256 bytes must fit the 96 MiB static scratch: at most
    8,388,586 voxels.  A 256 x 256 x 129 volume (8,454,144 voxels) is refused
    before any pointer is used."""
    import torch
    fn = _bind(L)
    dims = (256, 256, 129)
    pg = L.PolarGrid(np.array([0.2, 1.0], np.float32), 9, 9, 0.3)
    plan = L.NufftPlan(dims)
    f = torch.zeros(3, device="cuda")
    got = ctypes.c_double()
    rc = fn(plan._h, pg._h, ctypes.c_void_p(f.data_ptr()), ctypes.c_void_p(f.data_ptr()), 0.0,
            ctypes.byref(got), None)
    assert rc == 1
    msg = L.lib().lamino_last_error()
    assert b"exceeds the static scratch" in msg and b"8388586" in msg
