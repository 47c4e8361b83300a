"""lamino_b200: B200-native laminography NUFFT operator and solvers.

Python mirror of the reference's operator surface (``tomocam::PolarGrid``,
``forward``, ``adjoint``, ``sysmat``, ``gradient``, ``residual``, ``MBIR1-3``
and ``tomocam::opt::*``) over the C ABI of ``liblamino_b200.so``
(include/lamino.h).  Arrays may be numpy arrays (host; staged through device
memory by the library) or torch CUDA tensors (device; used in place).  There is
no CPU fallback: every call goes through the CUDA library and raises if it is
missing or fails.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

__all__ = [
    "LaminoError", "lib", "PolarGrid", "NufftPlan", "ToeplitzNormal", "beam_dir_vector",
    "forward", "adjoint", "sysmat", "gradient", "residual", "nufft3d1", "nufft3d2",
    "MBIR1", "MBIR2", "MBIR3", "ReconParams", "opt", "padded_volume_dims", "mbir_footprint",
    "mbir_phases", "mbir3_batch",
    "ReconServer",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblamino_b200.so")
_lib = None


class LaminoError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"lamino error {code}: {msg}")
        self.code = code


def lib():
    """Load liblamino_b200.so (building it first if it is missing and nvcc exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _b
        _b.build()
    L = ctypes.CDLL(LIB_PATH)
    vp, i64, i32, f32, f64 = (ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_float,
                              ctypes.c_double)
    P = ctypes.POINTER
    sig = {
        "lamino_last_error": ([], ctypes.c_char_p),
        "lamino_version": ([], ctypes.c_char_p),
        "lamino_geom_create": ([vp, i64, i64, i64, f32, P(vp)], i32),
        "lamino_geom_points": ([vp, vp, vp, vp, vp], i32),
        "lamino_geom_destroy": ([vp], i32),
        "lamino_plan_create": ([i64, i64, i64, f64, P(vp)], i32),
        "lamino_plan_destroy": ([vp], i32),
        "lamino_plan_set_bins": ([vp, i32, i32, i32], i32),
        "lamino_plan_autotune": ([vp, P(vp), i32, i32, P(i32), P(f64), vp], i32),
        "lamino_normal_autotune": ([vp, P(i32), P(i32), P(f64), vp], i32),
        "lamino_nufft3d2": ([vp, vp, vp, vp, vp], i32),
        "lamino_nufft3d1": ([vp, vp, vp, vp, vp], i32),
        "lamino_forward": ([vp, vp, vp, vp, vp], i32),
        "lamino_adjoint": ([vp, vp, vp, vp, vp], i32),
        "lamino_sysmat": ([vp, P(vp), i32, vp, vp, vp], i32),
        "lamino_gradient": ([vp, vp, vp, vp, vp, vp], i32),
        "lamino_residual": ([vp, vp, vp, vp, f32, P(f64), vp], i32),
        "lamino_normal_create": ([P(vp), i32, i64, i64, i64, i32, P(vp), vp], i32),
        "lamino_normal_apply": ([vp, vp, vp, vp], i32),
        "lamino_normal_apply_many": ([vp, i32, vp, vp, vp], i32),
        "lamino_normal_info": ([vp, P(i64), P(i64)], i32),
        "lamino_normal_destroy": ([vp], i32),
        "lamino_normal_quadforms": ([vp, P(vp), i32, vp, P(f64), vp], i32),
        "lamino_normal_profile": ([vp, i32, i32], i32),
        "lamino_normal_stage_times": ([vp, P(i32), P(f64), P(i64), P(i32), P(i32)], i32),
        "lamino_qggmrf": ([vp, vp, i64, i64, i64, f32, f32, vp], i32),
        "lamino_grad_u": ([vp, i64, i64, i64, vp, vp], i32),
        "lamino_divergence": ([vp, i64, i64, i64, vp, vp], i32),
        "lamino_laplacian": ([vp, i64, i64, i64, vp, vp], i32),
        "lamino_demag": ([vp, i64, i64, i64, vp, vp], i32),
        "lamino_ramp_precond": ([vp, i64, i64, i64, vp, vp], i32),
        "lamino_op_from_normal": ([vp, P(vp)], i32),
        "lamino_op_from_plan": ([vp, P(vp), i32, P(vp)], i32),
        "lamino_op_apply": ([vp, vp, vp, vp], i32),
        "lamino_op_destroy": ([vp], i32),
        "lamino_cgsolver": ([vp, vp, vp, i64, i64, i64, i32, f32, P(i32), vp], i32),
        "lamino_split_bregman": ([vp, vp, vp, i64, i64, i64, f32, f32, i32, i32, f32, f32, P(i32), vp], i32),
        "lamino_lipschitz": ([vp, i64, i64, i64, i32, f64, ctypes.c_uint64, P(f64), vp], i32),
        "lamino_recon_params_default": ([vp], None),
        "lamino_mbir": ([i32, i32, P(vp), P(i64), P(vp), P(f32), i64, i64, i64, vp, vp, vp], i32),
        "lamino_mbir_footprint": ([i32, i32, P(i64), i64, i64, i64, vp, P(i64)], i32),
        "lamino_mbir3_batch": ([i32, P(i32), P(vp), P(i64), P(vp), P(f32), P(i64), vp, P(vp), i64, i32, P(f64),
                                P(i64), P(i64)], i32),
        "lamino_server_create": ([i64, i32, i32, f64, P(vp)], i32),
        "lamino_server_submit": ([vp, i32, i32, P(vp), P(i64), P(vp), P(f32), i64, i64, i64, vp, P(i64)], i32),
        "lamino_server_wait": ([vp, i64, f64, vp, P(f64), P(f64), P(f64), P(f64)], i32),
        "lamino_mbir_phases": ([P(f64), P(f64), P(f64), P(i64), P(f64)], i32),
        "lamino_server_stats": ([vp, P(i64)], i32),
        "lamino_server_destroy": ([vp], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        raise LaminoError(rc, lib().lamino_last_error().decode())


def version() -> str:
    return lib().lamino_version().decode()


# ---------------------------------------------------------------------------
# array plumbing: numpy (host) or torch CUDA tensors (device)
# ---------------------------------------------------------------------------

def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _ptr(a):
    if _is_torch(a):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return ctypes.c_void_p(a.data_ptr())
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return ctypes.c_void_p(a.ctypes.data)


def _as_f32(a):
    if _is_torch(a):
        import torch
        if a.dtype != torch.float32:
            raise TypeError("expected a float32 tensor")
        return a.contiguous()
    return np.ascontiguousarray(a, dtype=np.float32)


def _empty_like_kind(ref, shape, dtype="float32"):
    if _is_torch(ref):
        import torch
        tdt = {"float32": torch.float32, "complex64": torch.complex64}[dtype]
        return torch.empty(shape, dtype=tdt, device=ref.device)
    return np.empty(shape, dtype=dtype)


def _stream(a=None):
    if a is not None and _is_torch(a) and a.is_cuda:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream(a.device).cuda_stream)
    return ctypes.c_void_p(0)


# ---------------------------------------------------------------------------
# geometry / plans / operators
# ---------------------------------------------------------------------------

def beam_dir_vector(gamma: float, alpha: float):
    """include/projection.h:37-41 in float32."""
    g, a = np.float32(gamma), np.float32(alpha)
    return (np.sin(g) * np.sin(a), np.cos(a), np.cos(g) * np.sin(a))


class PolarGrid:
    """tomocam::PolarGrid<float> (include/polar_grid.h:44-75).  Points are not stored:
    the GPU kernels regenerate them from per-row/column/angle factors."""

    def __init__(self, angles, nrows: int, ncols: int, gamma: float):
        self.theta = np.ascontiguousarray(angles, dtype=np.float32)
        self.nrows, self.ncols, self.gamma = int(nrows), int(ncols), float(np.float32(gamma))
        h = ctypes.c_void_p()
        _check(lib().lamino_geom_create(_ptr(self.theta), len(self.theta), self.nrows, self.ncols,
                                        self.gamma, ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.lamino_geom_destroy(self._h)
            self._h = None

    def dims(self):
        return (len(self.theta), self.nrows, self.ncols)

    def nprojs(self):
        return len(self.theta)

    def size(self):
        return len(self.theta) * self.nrows * self.ncols

    def points(self):
        """Materialise (x, y, z), each (nproj, nrows, ncols) float32, on the host."""
        out = [np.empty(self.dims(), np.float32) for _ in range(3)]
        _check(lib().lamino_geom_points(self._h, *[_ptr(a) for a in out], ctypes.c_void_p(0)))
        return out


class NufftPlan:
    """One GPU NUFFT plan per volume size (replaces the process-global FINUFFT plan
    cache of include/finufft_plan_cache.h:34-72)."""

    def __init__(self, dims, eps: float = 1.2e-6):
        self.dims = tuple(int(d) for d in dims)
        h = ctypes.c_void_p()
        _check(lib().lamino_plan_create(*self.dims, float(eps), ctypes.byref(h)))
        self._h = h

    def set_bins(self, b1: int, b2: int, b3: int):
        """Fine-grid bin size of the shared-memory spreading / interpolation."""
        _check(lib().lamino_plan_set_bins(self._h, int(b1), int(b2), int(b3)))
        return self

    def autotune(self, grids, objective: str = "normal"):
        """Time candidate bin layouts on `grids` and keep the fastest for
        'adjoint' (one setup pass incl. the sort) or 'normal' (repeated sysmat);
        returns (bins, best_ms)."""
        arr = (ctypes.c_void_p * len(grids))(*[g._h.value for g in grids])
        b = (ctypes.c_int * 3)()
        ms = ctypes.c_double()
        _check(lib().lamino_plan_autotune(self._h, arr, len(grids), {"adjoint": 0, "normal": 1}[objective], b,
                                          ctypes.byref(ms), ctypes.c_void_p(0)))
        return tuple(b), ms.value

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.lamino_plan_destroy(self._h)
            self._h = None


_plans: dict = {}


def _plan_for(dims, eps=1.2e-6) -> NufftPlan:
    key = (tuple(int(d) for d in dims), float(eps))
    if key not in _plans:
        _plans[key] = NufftPlan(key[0], key[1])
    return _plans[key]


def nufft3d2(modes, pg: PolarGrid, plan: NufftPlan | None = None):
    """include/nufft.h:52-64: complex64 modes (n1,n2,n3) -> complex64 (nproj,nrows,ncols)."""
    plan = plan or _plan_for(modes.shape)
    if _is_torch(modes):
        out = _empty_like_kind(modes, pg.dims(), "complex64")
        m = modes.contiguous()
    else:
        m = np.ascontiguousarray(modes, dtype=np.complex64)
        out = np.empty(pg.dims(), np.complex64)
    _check(lib().lamino_nufft3d2(plan._h, pg._h, _ptr(m), _ptr(out), _stream(modes)))
    return out


def nufft3d1(c, pg: PolarGrid, recon_dims, plan: NufftPlan | None = None):
    """include/nufft.h:37-49: complex64 points -> complex64 modes recon_dims."""
    plan = plan or _plan_for(recon_dims)
    if _is_torch(c):
        out = _empty_like_kind(c, tuple(recon_dims), "complex64")
        cc = c.contiguous()
    else:
        cc = np.ascontiguousarray(c, dtype=np.complex64)
        out = np.empty(tuple(recon_dims), np.complex64)
    _check(lib().lamino_nufft3d1(plan._h, pg._h, _ptr(cc), _ptr(out), _stream(c)))
    return out


def forward(m, pg: PolarGrid, gamma=None, plan: NufftPlan | None = None):
    """tomocam::forward (src/projection.cpp:42-77).  m: (3, n1, n2, n3)."""
    m = _as_f32(m)
    plan = plan or _plan_for(m.shape[1:])
    out = _empty_like_kind(m, pg.dims())
    _check(lib().lamino_forward(plan._h, pg._h, _ptr(m), _ptr(out), _stream(m)))
    return out


def adjoint(proj, pg: PolarGrid, recon_dims, gamma=None, plan: NufftPlan | None = None):
    """tomocam::adjoint (src/projection.cpp:90-126) -> (3, *recon_dims)."""
    proj = _as_f32(proj)
    plan = plan or _plan_for(recon_dims)
    out = _empty_like_kind(proj, (3,) + tuple(recon_dims))
    _check(lib().lamino_adjoint(plan._h, pg._h, _ptr(proj), _ptr(out), _stream(proj)))
    return out


def _geom_array(grids):
    arr = (ctypes.c_void_p * len(grids))(*[g._h.value for g in grids])
    return ctypes.cast(arr, ctypes.POINTER(ctypes.c_void_p)), arr


def sysmat(x, grid, gamma=None, plan: NufftPlan | None = None):
    """tomocam::sysmat (src/gradient.cpp:34-89) in NUFFT form; `grid` may be a list
    of PolarGrids, in which case the sum over them is returned."""
    grids = grid if isinstance(grid, (list, tuple)) else [grid]
    x = _as_f32(x)
    plan = plan or _plan_for(x.shape[1:])
    out = _empty_like_kind(x, tuple(x.shape))
    gp, keep = _geom_array(grids)
    _check(lib().lamino_sysmat(plan._h, gp, len(grids), _ptr(x), _ptr(out), _stream(x)))
    return out


def gradient(f, yT, grid, gamma=None, plan=None):
    """tomocam::gradient (src/gradient.cpp:98-105): sysmat(f) - yT."""
    f, yT = _as_f32(f), _as_f32(yT)
    plan = plan or _plan_for(f.shape[1:])
    out = _empty_like_kind(f, tuple(f.shape))
    _check(lib().lamino_gradient(plan._h, grid._h, _ptr(f), _ptr(yT), _ptr(out), _stream(f)))
    return out


def residual(f, yT, grid, yTy: float, gamma=None, plan=None) -> float:
    """tomocam::residual (src/gradient.cpp:117-127)."""
    f, yT = _as_f32(f), _as_f32(yT)
    plan = plan or _plan_for(f.shape[1:])
    r = ctypes.c_double()
    _check(lib().lamino_residual(plan._h, grid._h, _ptr(f), _ptr(yT), float(yTy), ctypes.byref(r),
                                 _stream(f)))
    return r.value


class ToeplitzNormal:
    """sum_gamma sysmat as a Toeplitz (block-convolution) operator; precision
    'fp32' or 'fp16' (spectra stored in half precision with per-plane scales)."""

    def __init__(self, grids: Sequence[PolarGrid], dims, precision: str = "fp32", stream=None):
        self.dims = tuple(int(d) for d in dims)
        self.grids = list(grids)
        gp, keep = _geom_array(self.grids)
        h = ctypes.c_void_p()
        prec = {"fp32": 0, "fp16": 1, "mixed": 2}[precision]
        _check(lib().lamino_normal_create(gp, len(self.grids), *self.dims, prec, ctypes.byref(h),
                                          stream or ctypes.c_void_p(0)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.lamino_normal_destroy(self._h)
            self._h = None

    def __call__(self, x, out=None):
        x = _as_f32(x)
        if out is None:
            out = _empty_like_kind(x, tuple(x.shape))
        _check(lib().lamino_normal_apply(self._h, _ptr(x), _ptr(out), _stream(x)))
        return out

    def apply_many(self, xs, outs):
        """outs[i] = A xs[i] for host volumes (numpy arrays or CPU tensors, pinned
        for the overlap): the copy-in of the next volume and the copy-out of the
        previous result overlap the current apply (lamino_normal_apply_many)."""
        n = len(xs)
        if len(outs) != n:
            raise ValueError("xs and outs must have the same length")
        shape = (3,) + self.dims
        for a in list(xs) + list(outs):
            if tuple(a.shape) != shape:
                raise ValueError(f"every volume must have shape {shape}")
            if _is_torch(a) and (a.is_cuda or str(a.dtype) != "torch.float32" or not a.is_contiguous()):
                raise ValueError("apply_many takes contiguous float32 host tensors")
            if not _is_torch(a) and (a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"]):
                raise ValueError("apply_many takes contiguous float32 host arrays")
        xp = (ctypes.c_void_p * max(n, 1))(*[_ptr(a).value for a in xs])
        yp = (ctypes.c_void_p * max(n, 1))(*[_ptr(a).value for a in outs])
        _check(lib().lamino_normal_apply_many(self._h, n, xp, yp, ctypes.c_void_p(0)))
        return outs

    def profile(self, enable: bool, max_applies: int = 64):
        _check(lib().lamino_normal_profile(self._h, int(bool(enable)), int(max_applies)))

    def stage_times(self):
        """{stage: (total_ms, bytes_per_apply)}, applies profiled, own kernels per apply."""
        n = ctypes.c_int()
        ms = (ctypes.c_double * 8)()
        by = (ctypes.c_int64 * 8)()
        na, kp = ctypes.c_int(), ctypes.c_int()
        _check(lib().lamino_normal_stage_times(self._h, ctypes.byref(n), ms, by, ctypes.byref(na),
                                               ctypes.byref(kp)))
        names = ["r2c_rows", "dim2_fwd", "pencil", "dim2_inv", "c2r_rows", "s5", "s6", "s7"]
        return ({names[k]: (ms[k], by[k]) for k in range(n.value)}, na.value, kp.value)

    def info(self):
        L = (ctypes.c_int64 * 3)()
        b = ctypes.c_int64()
        _check(lib().lamino_normal_info(self._h, L, ctypes.byref(b)))
        return tuple(L), b.value

    def autotune(self):
        """Time the launch shapes and keep the fastest; returns (rows, kb, best_ms)."""
        r, k, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        _check(lib().lamino_normal_autotune(self._h, ctypes.byref(r), ctypes.byref(k), ctypes.byref(ms),
                                            ctypes.c_void_p(0)))
        return r.value, k.value, ms.value

    def quadforms(self, x, parts) -> np.ndarray:
        """(len(parts), 3) array of x_i . (S_g x)_i for the operators `parts`
        (same volume size), from one forward half-spectrum of x."""
        x = _as_f32(x)
        arr = (ctypes.c_void_p * len(parts))(*[p._h.value for p in parts])
        out = (ctypes.c_double * (3 * len(parts)))()
        _check(lib().lamino_normal_quadforms(self._h, arr, len(parts), _ptr(x), out, _stream(x)))
        return np.array(out[:], dtype=np.float64).reshape(len(parts), 3)


def _pad_n(n: int, f) -> int:
    return int(n) + 2 * (int(np.float32(n) * np.float32(f)) // 2)


def padded_volume_dims(recon_dims, method: int = 2, pad_factor=np.float32(1.4142)):
    """Volume padding of MBIR1 (T(PAD-1.0)) and MBIR2/3 (T(PAD)-1 in float)."""
    if method == 1:
        f = np.float32(float(np.float32(pad_factor)) - 1.0)
    else:
        f = np.float32(pad_factor) - np.float32(1.0)
    return tuple(_pad_n(n, f) for n in recon_dims)


# ---------------------------------------------------------------------------
# solvers (tomocam::opt)
# ---------------------------------------------------------------------------

class _Op:
    def __init__(self, A, dims):
        self.dims = tuple(int(d) for d in dims)
        h = ctypes.c_void_p()
        if isinstance(A, ToeplitzNormal):
            _check(lib().lamino_op_from_normal(A._h, ctypes.byref(h)))
        else:
            plan, grids = A
            gp, keep = _geom_array(grids)
            _check(lib().lamino_op_from_plan(plan._h, gp, len(grids), ctypes.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.lamino_op_destroy(self._h)


class opt:  # namespace mirroring tomocam::opt
    @staticmethod
    def qggmrf(g, x, sigma: float, p: float):
        """src/qggmrf.cpp:60-95: g += prior gradient (in place; returns g)."""
        x = _as_f32(x)
        _check(lib().lamino_qggmrf(_ptr(g), _ptr(x), *x.shape, float(sigma), float(p), _stream(x)))
        return g

    @staticmethod
    def grad_u(u):
        u = _as_f32(u)
        out = _empty_like_kind(u, (3,) + tuple(u.shape))
        _check(lib().lamino_grad_u(_ptr(u), *u.shape, _ptr(out), _stream(u)))
        return out

    @staticmethod
    def divergence(du):
        du = _as_f32(du)
        out = _empty_like_kind(du, tuple(du.shape[1:]))
        _check(lib().lamino_divergence(_ptr(du), *du.shape[1:], _ptr(out), _stream(du)))
        return out

    @staticmethod
    def laplacian(u):
        u = _as_f32(u)
        out = _empty_like_kind(u, tuple(u.shape))
        _check(lib().lamino_laplacian(_ptr(u), *u.shape, _ptr(out), _stream(u)))
        return out

    @staticmethod
    def demag(m3):
        """tomocam::opt::demag (include/demag.h:13-79): the demagnetizing field of
        m3 (3, n1, n2, n3)."""
        m3 = _as_f32(m3)
        if m3.ndim != 4 or m3.shape[0] != 3:
            raise ValueError("expected a (3, n1, n2, n3) magnetization")
        out = _empty_like_kind(m3, tuple(m3.shape))
        _check(lib().lamino_demag(_ptr(m3), *m3.shape[1:], _ptr(out), _stream(m3)))
        return out

    @staticmethod
    def ramp_precond(r3):
        r3 = _as_f32(r3)
        out = _empty_like_kind(r3, tuple(r3.shape))
        _check(lib().lamino_ramp_precond(_ptr(r3), *r3.shape[1:], _ptr(out), _stream(r3)))
        return out

    @staticmethod
    def cgsolver(A, y, x0, max_iter: int, tol: float):
        """src/conjgrad.cpp:37-117.  A: ToeplitzNormal or (NufftPlan, [PolarGrid])."""
        y = _as_f32(y)
        x = _as_f32(x0).clone() if _is_torch(x0) else np.array(x0, dtype=np.float32)
        op = _Op(A, y.shape[1:])
        it = ctypes.c_int()
        _check(lib().lamino_cgsolver(op._h, _ptr(y), _ptr(x), *op.dims, int(max_iter), float(tol),
                                     ctypes.byref(it), _stream(y)))
        return x

    @staticmethod
    def split_bregman(A, yT, x0, lam, mu, outer_max, inner_max, tol, xtol):
        """src/bregman.cpp:39-134."""
        yT = _as_f32(yT)
        x = _as_f32(x0).clone() if _is_torch(x0) else np.array(x0, dtype=np.float32)
        op = _Op(A, yT.shape[1:])
        it = ctypes.c_int()
        _check(lib().lamino_split_bregman(op._h, _ptr(yT), _ptr(x), *op.dims, float(lam), float(mu),
                                          int(outer_max), int(inner_max), float(tol), float(xtol),
                                          ctypes.byref(it), _stream(yT)))
        return x

    @staticmethod
    def lipschitz(A, dims, max_iters: int = 30, tol: float = 1e-5, seed: int = 0) -> float:
        op = _Op(A, dims)
        L = ctypes.c_double()
        _check(lib().lamino_lipschitz(op._h, *op.dims, int(max_iters), float(tol), int(seed),
                                      ctypes.byref(L), ctypes.c_void_p(0)))
        return L.value


# ---------------------------------------------------------------------------
# MBIR drivers
# ---------------------------------------------------------------------------

class _ReconParamsC(ctypes.Structure):
    _fields_ = [("max_iters", ctypes.c_int), ("inner_iters", ctypes.c_int),
                ("sigma", ctypes.c_float), ("p", ctypes.c_float), ("lam", ctypes.c_float),
                ("mu", ctypes.c_float), ("tol", ctypes.c_float), ("xtol", ctypes.c_float),
                ("pad_factor", ctypes.c_float), ("op_kind", ctypes.c_int), ("eps", ctypes.c_double),
                ("refinements", ctypes.c_int), ("use_graphs", ctypes.c_int), ("autotune", ctypes.c_int)]


class ReconParams:
    """tomocam::ReconParams defaults (include/config.h:146-158) plus the operator
    form: op_kind 'toeplitz' (FP32 spectra), 'toeplitz_fp16', 'nufft' or 'mixed'
    (FP16 correction solves in `refinements` FP32-residual cycles), and
    use_graphs (replay each solver iteration's operator work as a CUDA graph) and
    autotune (launch shapes / bin layouts picked by timing, cached per size)."""

    def __init__(self, **kw):
        c = _ReconParamsC()
        lib().lamino_recon_params_default(ctypes.byref(c))
        self.maxIters, self.innerIters = c.max_iters, c.inner_iters
        self.sigma, self.p, self.lam, self.mu = c.sigma, c.p, c.lam, c.mu
        self.tol, self.xtol, self.PAD_FACTOR = c.tol, c.xtol, c.pad_factor
        self.op_kind, self.eps, self.refinements = "toeplitz", c.eps, c.refinements
        self.use_graphs = bool(c.use_graphs)
        self.autotune = bool(c.autotune)
        for k, v in kw.items():
            setattr(self, k, v)

    def _c(self):
        kind = {"toeplitz": 0, "toeplitz_fp16": 1, "nufft": 2, "mixed": 3}[self.op_kind]
        return _ReconParamsC(int(self.maxIters), int(self.innerIters), float(self.sigma), float(self.p),
                             float(self.lam), float(self.mu), float(self.tol), float(self.xtol),
                             float(self.PAD_FACTOR), kind, float(self.eps), int(self.refinements),
                             int(bool(self.use_graphs)), int(bool(self.autotune)))


def _datasets_c(datasets):
    """ctypes arrays (projection pointers, dims, angle pointers, gammas) of a list of
    (projections, angles, gamma) triples, plus the arrays they point into."""
    n = len(datasets)
    if n == 0:
        raise ValueError("no datasets")
    keep = []
    projs = (ctypes.c_void_p * n)()
    angs = (ctypes.c_void_p * n)()
    dims = (ctypes.c_int64 * (3 * n))()
    gam = (ctypes.c_float * n)()
    for i, (proj, angles, gamma) in enumerate(datasets):
        p = _as_f32(proj)
        a = np.ascontiguousarray(angles, dtype=np.float32)
        if p.ndim != 3 or a.shape != (p.shape[0],):
            raise ValueError("projections must be (nproj, nrows, ncols) with one angle per projection")
        keep += [p, a]
        projs[i] = _ptr(p).value
        angs[i] = _ptr(a).value
        dims[3 * i:3 * i + 3] = list(p.shape)
        gam[i] = float(gamma)
    return n, projs, dims, angs, gam, keep


def _mbir(method, datasets, recon_dims, params):
    params = params or ReconParams()
    n, projs, dims, angs, gam, keep = _datasets_c(datasets)
    ref = keep[0]
    out = _empty_like_kind(ref, (3,) + tuple(recon_dims))
    pc = params._c()
    _check(lib().lamino_mbir(method, n, projs, dims, angs, gam, *[int(d) for d in recon_dims],
                             ctypes.byref(pc), _ptr(out), _stream(ref)))
    return out


def mbir_phases() -> dict:
    """Phases of this thread's last MBIR call: setup, operator build and solve
    seconds (host wall clock) and the solve's normal-operator applications."""
    a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    n = ctypes.c_int64()
    parts = (ctypes.c_double * 3)()
    _check(lib().lamino_mbir_phases(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(n), parts))
    return {"setup_s": a.value, "build_s": b.value, "solve_s": c.value, "applies": n.value,
            "plan_s": parts[0], "adjoint_s": parts[1], "tune_s": parts[2]}


def mbir_footprint(method: int, proj_shapes, recon_dims, params: ReconParams | None = None) -> int:
    """Estimated peak device bytes of one MBIR{method} call with datasets of the
    given (nproj, nrows, ncols) shapes (the server's admission figure)."""
    params = params or ReconParams()
    n = len(proj_shapes)
    dims = (ctypes.c_int64 * (3 * n))(*[int(v) for sh in proj_shapes for v in sh])
    out = ctypes.c_int64()
    pc = params._c()
    _check(lib().lamino_mbir_footprint(method, n, dims, *[int(d) for d in recon_dims], ctypes.byref(pc),
                                       ctypes.byref(out)))
    return out.value


def mbir3_batch(requests, budget_bytes: int = 150 * 10**9, threads: int = 4):
    """Batched MBIR3 (no reference counterpart; each request is tomocam::MBIR3,
    src/mbir3.cpp:47-135): ``requests`` is a list of (datasets, recon_dims,
    params or None).  Preparer threads set requests up in order under the HBM
    budget while the calling thread drives every prepared NAG solve, one
    line-search step in flight per request.  Returns (volumes, info): the (3, r1, r2, r3) results in request order
    and {"ready_s", "done_s", "iterations", "applies" (per request),
    "peak_in_use", "peak_live", "steps", "wall_s"}."""
    nreq = len(requests)
    keep, outs = [], []
    all_sets = []
    nds = (ctypes.c_int * max(nreq, 1))()
    rdims = (ctypes.c_int64 * max(3 * nreq, 1))()
    prm = (_ReconParamsC * max(nreq, 1))()
    outp = (ctypes.c_void_p * max(nreq, 1))()
    for r, (datasets, recon_dims, params) in enumerate(requests):
        if len(datasets) == 0:
            raise ValueError("no datasets")
        nds[r] = len(datasets)
        all_sets += list(datasets)
        rdims[3 * r:3 * r + 3] = [int(d) for d in recon_dims]
        prm[r] = (params or ReconParams())._c()
        o = np.empty((3,) + tuple(int(d) for d in recon_dims), dtype=np.float32)
        outs.append(o)
        outp[r] = o.ctypes.data
    if all_sets:
        _, projs, dims, angs, gam, keep = _datasets_c(all_sets)
    else:
        projs, dims, angs, gam = (ctypes.c_void_p * 1)(), (ctypes.c_int64 * 3)(), (ctypes.c_void_p * 1)(), \
            (ctypes.c_float * 1)()
    for p in keep:
        if _is_torch(p) and p.is_cuda:
            raise TypeError("mbir3_batch takes host inputs (numpy arrays or CPU tensors)")
    times = (ctypes.c_double * max(2 * nreq, 1))()
    counts = (ctypes.c_int64 * max(2 * nreq, 1))()
    stats = (ctypes.c_int64 * 4)()
    _check(lib().lamino_mbir3_batch(nreq, nds, projs, dims, angs, gam, rdims, prm, outp, int(budget_bytes),
                                    int(threads), times, counts, stats))
    info = {"ready_s": [times[2 * r] for r in range(nreq)], "done_s": [times[2 * r + 1] for r in range(nreq)],
            "iterations": [counts[2 * r] for r in range(nreq)], "applies": [counts[2 * r + 1] for r in range(nreq)],
            "peak_in_use": stats[0], "peak_live": stats[1], "steps": stats[2], "wall_s": stats[3] * 1e-6}
    return outs, info


class ReconServer:
    """Continuous-batching MBIR server (no reference counterpart).

    Requests are admitted in arrival order while a worker slot is free and the
    sum of their estimated device footprints stays within ``budget_bytes``; each
    worker runs on its own CUDA stream.  ``dry_run_ms`` (not None) makes the
    workers hold each request that long without touching the GPU, which tests
    the admission logic on any machine."""

    STAT_KEYS = ("submitted", "completed", "failed", "in_use", "peak_in_use", "budget", "active",
                 "peak_active", "queued", "slots")

    def __init__(self, budget_bytes: int, slots: int = 4, dry_run_ms: float | None = None):
        h = ctypes.c_void_p()
        flags = 1 if dry_run_ms is not None else 0
        _check(lib().lamino_server_create(int(budget_bytes), int(slots), flags, float(dry_run_ms or 0.0),
                                          ctypes.byref(h)))
        self._h = h
        self._dims = {}

    def submit(self, method: int, datasets, recon_dims, params: ReconParams | None = None) -> int:
        """Queue MBIR{method} on the datasets (inputs are copied); returns the request id."""
        params = params or ReconParams()
        n, projs, dims, angs, gam, keep = _datasets_c(datasets)
        rid = ctypes.c_int64()
        pc = params._c()
        _check(lib().lamino_server_submit(self._h, method, n, projs, dims, angs, gam,
                                          *[int(d) for d in recon_dims], ctypes.byref(pc), ctypes.byref(rid)))
        self._dims[rid.value] = tuple(int(d) for d in recon_dims)
        return rid.value

    def wait(self, rid: int, timeout: float | None = None):
        """Block until request `rid` finished; returns (volume (3, r1, r2, r3) numpy,
        {"queue_s", "run_s", "latency_s", "setup_s", "build_s", "solve_s", "applies"}).
        Raises LaminoError on failure or timeout."""
        if rid not in self._dims:
            raise LaminoError(1, "unknown request id")
        shape = (3,) + self._dims[rid]
        out = np.empty(shape, dtype=np.float32)
        q, r, l = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        ph = (ctypes.c_double * 7)()
        rc = lib().lamino_server_wait(self._h, int(rid), -1.0 if timeout is None else float(timeout),
                                      ctypes.c_void_p(out.ctypes.data), ctypes.byref(q), ctypes.byref(r),
                                      ctypes.byref(l), ph)
        if rc != 5:  # LAMINO_ERR_TIMEOUT: the request stays queryable
            self._dims.pop(rid, None)
        _check(rc)
        return out, {"queue_s": q.value, "run_s": r.value, "latency_s": l.value, "setup_s": ph[0],
                     "build_s": ph[1], "solve_s": ph[2], "applies": int(ph[3]), "plan_s": ph[4],
                     "adjoint_s": ph[5], "tune_s": ph[6]}

    def stats(self) -> dict:
        st = (ctypes.c_int64 * 10)()
        _check(lib().lamino_server_stats(self._h, st))
        return dict(zip(self.STAT_KEYS, list(st)))

    def close(self):
        if self._h:
            _check(lib().lamino_server_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def MBIR1(datasets, recon_dims, params: ReconParams | None = None):
    """tomocam::MBIR1 (src/mbir_cg.cpp:48-128): CG on sum_gamma sysmat."""
    return _mbir(1, datasets, recon_dims, params)


def MBIR2(datasets, recon_dims, params: ReconParams | None = None):
    """tomocam::MBIR2 (src/mbir_sb.cpp:47-114): split-Bregman isotropic TV."""
    return _mbir(2, datasets, recon_dims, params)


def MBIR3(datasets, recon_dims, params: ReconParams | None = None):
    """tomocam::MBIR3 (src/mbir3.cpp:47-135): Nesterov + qGGMRF."""
    return _mbir(3, datasets, recon_dims, params)
