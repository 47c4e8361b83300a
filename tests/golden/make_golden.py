"""Generate the committed golden fixtures in tests/golden/ (seeded, small).

Two sources:
  * the reference's own code, compiled from its sources into
    oracle/_ref/libtomocam_ref.so (PolarGrid, shifts, padding, finite
    differences, qGGMRF, nagopt) -- the fixtures that pin the oracle;
  * the oracle (oracle/oracle.py) with the exact FP64 NUDFT for the
    NUFFT-composed operators (forward, adjoint, sysmat), which the reference
    cannot build here (FINUFFT/FFTW absent).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
fp = ctypes.POINTER(ctypes.c_float)
dp = ctypes.POINTER(ctypes.c_double)
i64 = ctypes.c_int64


def P(a, t=fp):
    return a.ctypes.data_as(t)


def ref_fixtures(ref):
    rng = np.random.default_rng(20260101)
    out = {}
    # PolarGrid: odd and even detector sizes
    for tag, (np_, nr, nc, g) in {"odd": (5, 13, 15, 0.7), "even": (4, 12, 16, 1.1)}.items():
        th = rng.uniform(0, 2 * np.pi, np_).astype(np.float32)
        x, y, z = (np.zeros((np_, nr, nc), np.float32) for _ in range(3))
        ref.ref_polar_grid_f.argtypes = [fp, i64, i64, i64, ctypes.c_float, fp, fp, fp]
        ref.ref_polar_grid_f(P(th), np_, nr, nc, np.float32(g), P(x), P(y), P(z))
        out[f"grid_{tag}_theta"] = th
        out[f"grid_{tag}_meta"] = np.array([np_, nr, nc, g], np.float64)
        out[f"grid_{tag}_xyz"] = np.stack([x, y, z])
        coeff = np.zeros((np_, 3), np.float32)
        ref.ref_beam_dir_f.argtypes = [ctypes.c_float, ctypes.c_float, fp]
        for i in range(np_):
            ref.ref_beam_dir_f(np.float32(g), th[i], P(coeff[i]))
        out[f"grid_{tag}_coeff"] = coeff
    # shifts on odd and even planes (complex)
    for tag, shp in {"odd": (2, 5, 7), "even": (2, 4, 6)}.items():
        a = (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)).astype(np.complex64)
        f, fi = np.zeros_like(a), np.zeros_like(a)
        ref.ref_fftshift2_c.argtypes = [fp, i64, i64, i64, fp]
        ref.ref_ifftshift2_c.argtypes = [fp, i64, i64, i64, fp]
        ref.ref_fftshift2_c(P(a.view(np.float32)), *shp, P(f.view(np.float32)))
        ref.ref_ifftshift2_c(P(a.view(np.float32)), *shp, P(fi.view(np.float32)))
        out[f"shift_{tag}_in"], out[f"shift_{tag}_f"], out[f"shift_{tag}_i"] = a, f, fi
    # padding
    a = rng.standard_normal((3, 11, 9)).astype(np.float32)
    od = np.zeros(3, np.int64)
    ref.ref_pad2d_f.argtypes = [fp, i64, i64, i64, ctypes.c_float, fp, ctypes.POINTER(i64)]
    for tag, fac in {"p04": 0.4142, "p14": 1.4142}.items():
        ref.ref_pad2d_f(P(a), 3, 11, 9, np.float32(fac), None, od.ctypes.data_as(ctypes.POINTER(i64)))
        b = np.zeros(tuple(od), np.float32)
        ref.ref_pad2d_f(P(a), 3, 11, 9, np.float32(fac), P(b), od.ctypes.data_as(ctypes.POINTER(i64)))
        out[f"pad2d_{tag}"] = b
    out["pad2d_in"] = a
    v = rng.standard_normal((10, 7, 12)).astype(np.float32)
    c = np.zeros((7, 5, 9), np.float32)
    ref.ref_crop3d_f.argtypes = [fp, i64, i64, i64, i64, i64, i64, fp]
    ref.ref_crop3d_f(P(v), 10, 7, 12, 7, 5, 9, P(c))
    out["crop3d_in"], out["crop3d_out"] = v, c
    # finite differences and qGGMRF on a seeded cube
    u = rng.standard_normal((6, 7, 8)).astype(np.float32)
    g3 = np.zeros((3, 6, 7, 8), np.float32)
    ref.ref_grad_u_f.argtypes = [fp, i64, i64, i64, fp]
    ref.ref_grad_u_f(P(u), 6, 7, 8, P(g3))
    dv = np.zeros((6, 7, 8), np.float32)
    du = rng.standard_normal((3, 6, 7, 8)).astype(np.float32)
    ref.ref_divergence_f.argtypes = [fp, i64, i64, i64, fp]
    ref.ref_divergence_f(P(du), 6, 7, 8, P(dv))
    lp = np.zeros((6, 7, 8), np.float32)
    ref.ref_laplacian_f.argtypes = [fp, i64, i64, i64, fp]
    ref.ref_laplacian_f(P(u), 6, 7, 8, P(lp))
    out.update(fd_u=u, fd_grad=g3, fd_du=du, fd_div=dv, fd_lap=lp)
    xq = (rng.standard_normal((6, 7, 8)) * 50).astype(np.float32)
    xq[2, 3, 4] = xq[2, 3, 5]  # a zero difference exercises the delta == 0 branch
    gq = rng.standard_normal((6, 7, 8)).astype(np.float32)
    gout = gq.copy()
    ref.ref_qggmrf_f.argtypes = [fp, fp, i64, i64, i64, ctypes.c_float, ctypes.c_float]
    ref.ref_qggmrf_f(P(gout), P(xq), 6, 7, 8, np.float32(1000.0), np.float32(1.2))
    out.update(qg_x=xq, qg_g0=gq, qg_g=gout)
    # nagopt (reference code) on a quadratic 0.5 x'Dx - b'x with D diagonal
    dims = (1, 1, 6)
    dg = (np.arange(18, dtype=np.float32) % 6 + 1).reshape(3, *dims)
    bq = rng.standard_normal((3, *dims)).astype(np.float32)

    @ctypes.CFUNCTYPE(None, fp, fp, ctypes.c_void_p)
    def gcb(x, g, ctx):
        xa = np.ctypeslib.as_array(x, (18,))
        ga = np.ctypeslib.as_array(g, (18,))
        ga[:] = (dg.ravel() * xa - bq.ravel()).astype(np.float32)

    @ctypes.CFUNCTYPE(ctypes.c_float, fp, ctypes.c_void_p)
    def lcb(x, ctx):
        xa = np.ctypeslib.as_array(x, (18,)).astype(np.float64)
        return float(0.5 * np.sum(dg.ravel() * xa * xa) - np.sum(bq.ravel() * xa) + 10.0)

    x0 = np.zeros((3, *dims), np.float32)
    ref.ref_nagopt_f.argtypes = [type(gcb), type(lcb), ctypes.c_void_p, fp, i64, i64, i64, i64,
                                 ctypes.c_float, ctypes.c_float, ctypes.c_float, i64]
    xs = x0.copy()
    ref.ref_nagopt_f(gcb, lcb, None, P(xs), *dims, 25, np.float32(6.0), np.float32(1e-9),
                     np.float32(1e-9), 5)
    out.update(nag_diag=dg, nag_b=bq, nag_x=xs)
    return out


def oracle_fixtures():
    rng = np.random.default_rng(777)
    out = {}
    dims = (9, 5, 11)
    th = rng.uniform(0, 2 * np.pi, 4).astype(np.float32)
    gamma = np.float32(0.6)
    pg = O.PolarGrid(th, 13, 15, gamma)
    pe = O.NufftPlan(dims, exact=True)
    m = rng.standard_normal((3,) + dims)
    f = rng.standard_normal(dims) + 1j * rng.standard_normal(dims)
    c = rng.standard_normal(pg.dims()) + 1j * rng.standard_normal(pg.dims())
    out.update(op_theta=th, op_meta=np.array([13, 15, gamma], np.float64), op_m=m.astype(np.float32),
               op_f=f.astype(np.complex64), op_c=c.astype(np.complex64))
    out["op_nudft2"] = O.nufft3d2(f.astype(np.complex64), pg, pe)
    out["op_nudft1"] = O.nufft3d1(c.astype(np.complex64), pg, pe)
    out["op_forward"] = O.forward(m.astype(np.float32), pg, gamma, pe)
    proj = rng.standard_normal(pg.dims())
    out["op_proj"] = proj.astype(np.float32)
    out["op_adjoint"] = O.adjoint(proj.astype(np.float32), pg, dims, gamma, pe)
    out["op_sysmat"] = O.sysmat(m.astype(np.float32), pg, gamma, pe)
    return out


def main():
    ref = O.ref_lib()
    if ref is None:
        raise SystemExit("oracle/_ref/libtomocam_ref.so missing: run make -f oracle/Makefile")
    np.savez_compressed(os.path.join(OUT, "reference_small.npz"), **ref_fixtures(ref))
    np.savez_compressed(os.path.join(OUT, "oracle_small.npz"), **oracle_fixtures())
    print("wrote", os.listdir(OUT))


if __name__ == "__main__":
    main()
