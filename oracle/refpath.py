"""ctypes access to the reference's own compiled operator and solver path
(oracle/_ref/libtomocam_ref.so, built by oracle/Makefile from the reference's
src/projection.cpp, src/gradient.cpp, src/conjgrad.cpp, src/bregman.cpp,
src/nagopt.cpp, src/qggmrf.cpp, src/finitediff.cpp and the MBIR drivers against
this project's FINUFFT-API and FFTW-API shims).

TEST INFRASTRUCTURE ONLY: the golden fixtures under tests/golden/ and the bench's
reference arm use it; nothing in the product imports it.

The reference keeps one FINUFFT plan per precision for the whole process, sized
by its first call (include/finufft_plan_cache.h:50-66).  ``isolated(name, ...)``
therefore runs one call in a fresh spawned process; direct calls are only safe
when every call in the process uses the same volume size per precision.
"""
from __future__ import annotations

import ctypes
import multiprocessing as mp
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libtomocam_ref.so")

_LIB = None

_I64 = ctypes.c_int64
_INT = ctypes.c_int
_DBL = ctypes.c_double


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _LIB
    if _LIB is None:
        if not available():
            raise RuntimeError(f"compiled reference path missing: {LIB_PATH} (build with oracle/Makefile)")
        L = ctypes.CDLL(LIB_PATH)
        for s, real in (("_f", ctypes.c_float), ("_d", ctypes.c_double)):
            P = ctypes.POINTER(real)
            PI = ctypes.POINTER(_I64)
            getattr(L, "ref_forward" + s).argtypes = [P, _I64, _I64, _I64, P, _I64, _I64, _I64, real, P]
            getattr(L, "ref_adjoint" + s).argtypes = [P, _I64, _I64, _I64, P, real, _I64, _I64, _I64, P]
            getattr(L, "ref_sysmat" + s).argtypes = [P, _I64, _I64, _I64, P, _I64, _I64, _I64, real, P]
            getattr(L, "ref_normal" + s).argtypes = [P, _I64, _I64, _I64, _INT, PI, PI, PI, P, P, P]
            getattr(L, "ref_gradient" + s).argtypes = [P, P, _I64, _I64, _I64, P, _I64, _I64, _I64, real, P]
            getattr(L, "ref_residual" + s).argtypes = [P, P, _I64, _I64, _I64, P, _I64, _I64, _I64, real, real, P]
            getattr(L, "ref_ramp" + s).argtypes = [P, _I64, _I64, _I64, P]
            getattr(L, "ref_cgsolver" + s).argtypes = [P, P, _I64, _I64, _I64, _INT, PI, PI, PI, P, P, _I64, real,
                                                       _INT, P]
            getattr(L, "ref_split_bregman" + s).argtypes = [P, P, _I64, _I64, _I64, _INT, PI, PI, PI, P, P, real,
                                                            real, _I64, _I64, real, real, _INT, P]
            getattr(L, "ref_mbir" + s).argtypes = [_INT, _INT, P, PI, PI, PI, P, P, _I64, _I64, _I64, _I64, _I64,
                                                   _DBL, _DBL, _DBL, _DBL, _DBL, _DBL, _INT, P]
        _LIB = L
    return _LIB


def _t(dtype):
    return ("_f", ctypes.c_float, np.float32) if np.dtype(dtype) == np.float32 else ("_d", ctypes.c_double, np.float64)


def _p(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def _c(a, npt):
    return np.ascontiguousarray(a, dtype=npt)


def _check(rc, name):
    if rc != 0:
        raise RuntimeError(f"reference {name} failed (status {rc})")


def _geoms(geoms, npt):
    """geoms: list of (angles, nrows, ncols, gamma)."""
    nproj = np.array([len(g[0]) for g in geoms], np.int64)
    nrows = np.array([g[1] for g in geoms], np.int64)
    ncols = np.array([g[2] for g in geoms], np.int64)
    angles = _c(np.concatenate([np.asarray(g[0]) for g in geoms]), npt)
    gammas = _c([g[3] for g in geoms], npt)
    return nproj, nrows, ncols, angles, gammas


def forward(m3, angles, nrows, ncols, gamma, dtype=np.float64):
    s, ct, npt = _t(dtype)
    m3 = _c(m3, npt)
    _, n1, n2, n3 = m3.shape
    a = _c(angles, npt)
    out = np.zeros((a.size, nrows, ncols), npt)
    _check(getattr(lib(), "ref_forward" + s)(_p(m3, ct), n1, n2, n3, _p(a, ct), a.size, nrows, ncols, ct(gamma),
                                              _p(out, ct)), "forward")
    return out


def adjoint(proj, angles, gamma, dims, dtype=np.float64):
    s, ct, npt = _t(dtype)
    proj = _c(proj, npt)
    a = _c(angles, npt)
    out = np.zeros((3,) + tuple(dims), npt)
    _check(getattr(lib(), "ref_adjoint" + s)(_p(proj, ct), *proj.shape, _p(a, ct), ct(gamma), *dims, _p(out, ct)),
           "adjoint")
    return out


def sysmat(x3, angles, nrows, ncols, gamma, dtype=np.float64):
    s, ct, npt = _t(dtype)
    x3 = _c(x3, npt)
    a = _c(angles, npt)
    out = np.zeros_like(x3)
    _check(getattr(lib(), "ref_sysmat" + s)(_p(x3, ct), *x3.shape[1:], _p(a, ct), a.size, nrows, ncols, ct(gamma),
                                             _p(out, ct)), "sysmat")
    return out


def normal(x3, geoms, dtype=np.float64):
    s, ct, npt = _t(dtype)
    x3 = _c(x3, npt)
    nproj, nrows, ncols, angles, gammas = _geoms(geoms, npt)
    out = np.zeros_like(x3)
    PI = ctypes.POINTER(_I64)
    _check(getattr(lib(), "ref_normal" + s)(_p(x3, ct), *x3.shape[1:], len(geoms), _p(nproj, _I64),
                                             _p(nrows, _I64), _p(ncols, _I64), _p(angles, ct), _p(gammas, ct),
                                             _p(out, ct)), "normal")
    return out


def gradient(x3, yT3, angles, nrows, ncols, gamma, dtype=np.float64):
    s, ct, npt = _t(dtype)
    x3, yT3 = _c(x3, npt), _c(yT3, npt)
    a = _c(angles, npt)
    out = np.zeros_like(x3)
    _check(getattr(lib(), "ref_gradient" + s)(_p(x3, ct), _p(yT3, ct), *x3.shape[1:], _p(a, ct), a.size, nrows,
                                               ncols, ct(gamma), _p(out, ct)), "gradient")
    return out


def residual(x3, yT3, angles, nrows, ncols, yTy, gamma, dtype=np.float64):
    s, ct, npt = _t(dtype)
    x3, yT3 = _c(x3, npt), _c(yT3, npt)
    a = _c(angles, npt)
    out = np.zeros(1, npt)
    _check(getattr(lib(), "ref_residual" + s)(_p(x3, ct), _p(yT3, ct), *x3.shape[1:], _p(a, ct), a.size, nrows,
                                               ncols, ct(yTy), ct(gamma), _p(out, ct)), "residual")
    return float(out[0])


def ramp(v, dtype=np.float64):
    s, ct, npt = _t(dtype)
    v = _c(v, npt)
    out = np.zeros_like(v)
    _check(getattr(lib(), "ref_ramp" + s)(_p(v, ct), *v.shape, _p(out, ct)), "ramp")
    return out


def cgsolver(b3, x03, geoms, max_iter, tol, dtype=np.float64, quiet=True):
    s, ct, npt = _t(dtype)
    b3, x03 = _c(b3, npt), _c(x03, npt)
    nproj, nrows, ncols, angles, gammas = _geoms(geoms, npt)
    out = np.zeros_like(b3)
    _check(getattr(lib(), "ref_cgsolver" + s)(_p(b3, ct), _p(x03, ct), *b3.shape[1:], len(geoms), _p(nproj, _I64),
                                               _p(nrows, _I64), _p(ncols, _I64), _p(angles, ct), _p(gammas, ct),
                                               max_iter, ct(tol), int(quiet), _p(out, ct)), "cgsolver")
    return out


def split_bregman(yT3, x03, geoms, lam, mu, outer, inner, tol, xtol, dtype=np.float64, quiet=True):
    s, ct, npt = _t(dtype)
    yT3, x03 = _c(yT3, npt), _c(x03, npt)
    nproj, nrows, ncols, angles, gammas = _geoms(geoms, npt)
    out = np.zeros_like(yT3)
    _check(getattr(lib(), "ref_split_bregman" + s)(
        _p(yT3, ct), _p(x03, ct), *yT3.shape[1:], len(geoms), _p(nproj, _I64), _p(nrows, _I64), _p(ncols, _I64),
        _p(angles, ct), _p(gammas, ct), ct(lam), ct(mu), outer, inner, ct(tol), ct(xtol), int(quiet),
        _p(out, ct)), "split_bregman")
    return out


def mbir(which, datasets, recon_dims, max_iters=50, inner_iters=3, sigma=1000.0, p=1.2, lam=0.1, mu=10.0,
         tol=1e-5, xtol=1e-5, dtype=np.float64, quiet=True):
    """tomocam::MBIR1/2/3 (which = 1, 2, 3) on datasets [(proj, angles, gamma)]
    (gamma in radians), recon_dims (n1, n2, n3) internal order."""
    s, ct, npt = _t(dtype)
    proj = _c(np.concatenate([np.ravel(d[0]) for d in datasets]), npt)
    nproj = np.array([d[0].shape[0] for d in datasets], np.int64)
    nrows = np.array([d[0].shape[1] for d in datasets], np.int64)
    ncols = np.array([d[0].shape[2] for d in datasets], np.int64)
    angles = _c(np.concatenate([np.asarray(d[1]) for d in datasets]), npt)
    gammas = _c([d[2] for d in datasets], npt)
    out = np.zeros((3,) + tuple(recon_dims), npt)
    _check(getattr(lib(), "ref_mbir" + s)(which, len(datasets), _p(proj, ct), _p(nproj, _I64), _p(nrows, _I64),
                                           _p(ncols, _I64), _p(angles, ct), _p(gammas, ct), *recon_dims,
                                           max_iters, inner_iters, sigma, p, lam, mu, tol, xtol, int(quiet),
                                           _p(out, ct)), f"MBIR{which}")
    return out


def _child(name, args, kwargs, q):
    try:
        q.put(("ok", globals()[name](*args, **kwargs)))
    except BaseException as e:  # noqa: BLE001 - reported to the parent
        q.put(("err", repr(e)))


def isolated(name, *args, **kwargs):
    """Run one function of this module in a fresh spawned process (one volume
    size per process, as the reference's global plan cache requires)."""
    import queue

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_child, args=(name, args, kwargs, q))
    p.start()
    while True:
        try:
            status, val = q.get(timeout=0.5)
            break
        except queue.Empty:
            if not p.is_alive():
                raise RuntimeError(f"reference {name}: child process exited with code {p.exitcode}")
    p.join()
    if status != "ok":
        raise RuntimeError(f"reference {name} failed in child: {val}")
    return val
