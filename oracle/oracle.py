"""CPU oracle for the laminography operator and its solvers.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this module, and only as the
checker.  The product (``lamino_b200``) never imports it.

It restates, in numpy (FP64 by default) plus the C gridding kernels of
``nufft_oracle.c``, the reference's algorithm for the hot path.  Each function
cites the reference file:line it follows (paths relative to the reference
project root).  FINUFFT and FFTW are third-party and absent from the reference
tree: the non-uniform transforms follow their published definitions
(exact NUDFT for tiny cases, the ES-kernel method of Barnett et al. 2019
otherwise) and uniform FFTs use numpy / scipy.fft.

Parity pinning.  The reference ships no golden vectors.  The parts of the path
that the reference can compile without external libraries (PolarGrid,
beam_dir_vector, padding, shifts, finite differences, qGGMRF, nagopt) are
compiled from the reference sources into ``oracle/_ref/libtomocam_ref.so`` and
the tests check this module against them.  The NUFFT-composed operators
(forward / adjoint / sysmat) are pinned against the exact NUDFT only.
"""
from __future__ import annotations

import ctypes
import math
import os
from typing import Callable, Sequence

import numpy as np

try:  # multithreaded FFTs for the CPU baseline; numpy's pocketfft otherwise
    import scipy.fft as _sfft

    def _fftn(a, axes=None):
        return _sfft.fftn(a, axes=axes, workers=-1)

    def _ifftn_unnorm(a, axes=None):
        return _sfft.ifftn(a, axes=axes, workers=-1, norm="forward")
except Exception:  # pragma: no cover
    def _fftn(a, axes=None):
        return np.fft.fftn(a, axes=axes)

    def _ifftn_unnorm(a, axes=None):
        return np.fft.ifftn(a, axes=axes, norm="forward")

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so missing: run `make -f oracle/Makefile`")
        lib = ctypes.CDLL(path)
        d, f, i64, i32 = (ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float),
                          ctypes.c_int64, ctypes.c_int)
        lib.oracle_nudft3d2.argtypes = [i64, d, d, d, i32, i64, i64, i64, d, d]
        lib.oracle_nudft3d1.argtypes = [i64, d, d, d, d, i32, i64, i64, i64, d]
        lib.oracle_es_interp.argtypes = [i64, d, d, d, i64, i64, i64, d, i32, ctypes.c_double, d]
        lib.oracle_es_spread.argtypes = [i64, d, d, d, d, i64, i64, i64, d, i32, ctypes.c_double]
        lib.oracle_es_interp_f.argtypes = [i64, f, f, f, i64, i64, i64, f, i32, ctypes.c_float, f]
        lib.oracle_es_spread_f.argtypes = [i64, f, f, f, f, i64, i64, i64, f, i32, ctypes.c_float]
        lib.oracle_num_threads.restype = ctypes.c_int
        _LIB = lib
    return _LIB


def ref_lib():
    """The reference's own sources behind a C shim (None when not built)."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libtomocam_ref.so")
        if not os.path.exists(path):
            return None
        _REF = ctypes.CDLL(path)
    return _REF


def _p(a, ct=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def num_threads() -> int:
    return int(_lib().oracle_num_threads())


# ---------------------------------------------------------------------------
# geometry
# ---------------------------------------------------------------------------

class PolarGrid:
    """Non-uniform frequency points of one gamma dataset.

    Restates ``PolarGrid::PolarGrid`` (include/polar_grid.h:44-75) in the
    arithmetic of ``T`` (float32 reproduces the reference float path):
        dX = T(2 pi / ncols);  qX = T(k*dX - pi + dX/2)   (middle term in double)
        z = -qX sin(g) + qY cos(th) cos(g);  y = -qY sin(th);  x = qX cos(g) + qY cos(th) sin(g)
    Arrays x, y, z have shape (nproj, nrows, ncols).
    """

    def __init__(self, angles, nrows: int, ncols: int, gamma, dtype=np.float32):
        T = np.dtype(dtype).type
        self.dtype = np.dtype(dtype)
        self.theta = np.asarray(angles, dtype=dtype)
        self.gamma = T(gamma)
        self.nrows, self.ncols = int(nrows), int(ncols)
        dX = T((2 * math.pi) / float(T(ncols)))
        dY = T((2 * math.pi) / float(T(nrows)))
        k = np.arange(ncols)
        j = np.arange(nrows)
        # k*dX in T, then (double) - M_PI + (double)(dX/2), then back to T
        qX = ((k.astype(dtype) * dX).astype(np.float64) - math.pi
              + np.float64(T(dX / T(2)))).astype(dtype)
        qY = ((j.astype(dtype) * dY).astype(np.float64) - math.pi
              + np.float64(T(dY / T(2)))).astype(dtype)
        # sinf/cosf of the C library are correctly rounded on these inputs; numpy's
        # float32 SIMD trig is not, so evaluate in double and round once.
        sg = np.sin(np.float64(self.gamma)).astype(dtype)
        cg = np.cos(np.float64(self.gamma)).astype(dtype)
        st = np.sin(self.theta.astype(np.float64)).astype(dtype)
        ct = np.cos(self.theta.astype(np.float64)).astype(dtype)
        qXb = qX[None, None, :]
        qYb = qY[None, :, None]
        ctb = ct[:, None, None]
        stb = st[:, None, None]
        self.z = ((-qXb) * sg + (qYb * ctb) * cg).astype(dtype)
        self.y = np.broadcast_to(-qYb * stb, (len(self.theta), nrows, ncols)).astype(dtype)
        self.x = (qXb * cg + (qYb * ctb) * sg).astype(dtype)
        self.qX, self.qY = qX, qY

    def dims(self):
        return (len(self.theta), self.nrows, self.ncols)

    def nprojs(self):
        return len(self.theta)

    def size(self):
        return len(self.theta) * self.nrows * self.ncols


def beam_dir_vector(gamma, alpha, dtype=np.float64):
    """include/projection.h:37-41: {sin g sin a, cos a, cos g sin a}."""
    g = np.asarray(gamma, dtype=dtype)
    a = np.asarray(alpha, dtype=dtype)
    return np.stack([np.sin(g) * np.sin(a), np.cos(a) + 0 * g, np.cos(g) * np.sin(a)])


# ---------------------------------------------------------------------------
# NUFFT (FINUFFT semantics as called by include/nufft.h:37-64)
# ---------------------------------------------------------------------------

def next_smooth_even(n: int) -> int:
    """Smallest even 2,3,5-smooth integer >= n (fine-grid sizes)."""
    n = max(2, int(n))
    if n % 2:
        n += 1
    while True:
        m = n
        for p in (2, 3, 5):
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 2


def es_params(eps: float, upsampfac: float = 2.0):
    """ES kernel width and shape for a requested tolerance (Barnett et al. 2019,
    sigma = 2): w = ceil(log10(10/eps)), beta = 2.30 w."""
    assert upsampfac == 2.0
    w = int(math.ceil(math.log10(10.0 / eps)))
    w = max(2, min(w, 16))
    return w, 2.30 * w


def es_fourier(nf: int, N: int, w: int, beta: float, nquad: int = 200):
    """Kernel Fourier factors p(k) = (w/2) int_{-1}^{1} phi(t) cos(k pi w t / nf) dt
    for centred modes k = -floor(N/2) .. ceil(N/2)-1 (Gauss-Legendre)."""
    t, wq = np.polynomial.legendre.leggauss(nquad)
    phi = np.exp(beta * (np.sqrt(1.0 - t * t) - 1.0))
    k = np.arange(N) - N // 2
    return (w / 2.0) * (np.cos(np.outer(k, t) * (math.pi * w / nf)) @ (wq * phi))


class NufftPlan:
    """3-D type-1/2 transform for a volume of shape (n1, n2, n3) (modes N1=n3 pairs
    with x, N2=n2 with y, N3=n1 with z), mirroring FinufftPlanWrapper
    (include/finufft_plan.h:93-129, upsampfac 2).  ``exact`` selects the NUDFT."""

    def __init__(self, dims, eps: float = 1e-12, exact: bool = False, single: bool = False):
        self.dims = tuple(int(d) for d in dims)
        self.exact = exact
        self.single = single
        self.w, self.beta = es_params(eps)
        n1, n2, n3 = self.dims
        self.nf = tuple(next_smooth_even(max(2 * n, 2 * self.w)) for n in (n1, n2, n3))
        self.p = [es_fourier(nf, n, self.w, self.beta) for nf, n in zip(self.nf, self.dims)]
        self.idx = [np.arange(n) - n // 2 for n in self.dims]

    def _corr(self):
        pz, py, px = self.p
        return pz[:, None, None] * py[None, :, None] * px[None, None, :]

    def _fine_index(self):
        return np.ix_(*[k % nf for k, nf in zip(self.idx, self.nf)])

    def type2(self, f, x, y, z):
        """c_j = sum_k f[k] exp(-i k.x_j); f complex (n1,n2,n3); returns complex (M,)."""
        x, y, z = (np.ascontiguousarray(np.ravel(a), dtype=np.float64) for a in (x, y, z))
        M = x.size
        f = np.asarray(f, dtype=np.complex128)
        n1, n2, n3 = self.dims
        if self.exact:
            c = np.zeros(M, np.complex128)
            fc = np.ascontiguousarray(f)
            _lib().oracle_nudft3d2(M, _p(x), _p(y), _p(z), -1, n3, n2, n1,
                                   _p(fc.view(np.float64)), _p(c.view(np.float64)))
            return c
        g = np.zeros(self.nf, np.complex128)
        g[self._fine_index()] = f / self._corr()
        G = _fftn(g)  # exponent -1 (iflag -1)
        return self._interp(G, x, y, z)

    def type1(self, c, x, y, z):
        """f[k] = sum_j c_j exp(+i k.x_j); returns complex (n1,n2,n3)."""
        x, y, z = (np.ascontiguousarray(np.ravel(a), dtype=np.float64) for a in (x, y, z))
        M = x.size
        c = np.ascontiguousarray(np.ravel(c), dtype=np.complex128)
        n1, n2, n3 = self.dims
        if self.exact:
            f = np.zeros(self.dims, np.complex128)
            _lib().oracle_nudft3d1(M, _p(x), _p(y), _p(z), _p(c.view(np.float64)), 1,
                                   n3, n2, n1, _p(f.view(np.float64)))
            return f
        G = self._spread(c, x, y, z)
        F = _ifftn_unnorm(G)  # exponent +1, unnormalised
        return F[self._fine_index()] / self._corr()

    def _interp(self, G, x, y, z):
        nfz, nfy, nfx = self.nf
        M = x.size
        if self.single:
            G32 = np.ascontiguousarray(G, dtype=np.complex64)
            c = np.zeros(M, np.complex64)
            xf, yf, zf = (a.astype(np.float32) for a in (x, y, z))
            fp = ctypes.c_float
            _lib().oracle_es_interp_f(M, _p(xf, fp), _p(yf, fp), _p(zf, fp), nfx, nfy, nfz,
                                      _p(G32.view(np.float32), fp), self.w, self.beta,
                                      _p(c.view(np.float32), fp))
            return c.astype(np.complex128)
        Gc = np.ascontiguousarray(G, dtype=np.complex128)
        c = np.zeros(M, np.complex128)
        _lib().oracle_es_interp(M, _p(x), _p(y), _p(z), nfx, nfy, nfz,
                                _p(Gc.view(np.float64)), self.w, self.beta,
                                _p(c.view(np.float64)))
        return c

    def _spread(self, c, x, y, z):
        nfz, nfy, nfx = self.nf
        M = x.size
        if self.single:
            G = np.zeros(self.nf, np.complex64)
            cf = c.astype(np.complex64)
            xf, yf, zf = (a.astype(np.float32) for a in (x, y, z))
            fp = ctypes.c_float
            _lib().oracle_es_spread_f(M, _p(xf, fp), _p(yf, fp), _p(zf, fp),
                                      _p(cf.view(np.float32), fp), nfx, nfy, nfz,
                                      _p(G.view(np.float32), fp), self.w, self.beta)
            return G.astype(np.complex128)
        G = np.zeros(self.nf, np.complex128)
        _lib().oracle_es_spread(M, _p(x), _p(y), _p(z), _p(c.view(np.float64)),
                                nfx, nfy, nfz, _p(G.view(np.float64)), self.w, self.beta)
        return G


def nufft3d2(f, pg: PolarGrid, plan: NufftPlan):
    """include/nufft.h:52-64 (type 2, iflag -1) on a PolarGrid; returns (nproj,nrows,ncols)."""
    return plan.type2(f, pg.x, pg.y, pg.z).reshape(pg.dims())


def nufft3d1(c, pg: PolarGrid, plan: NufftPlan):
    """include/nufft.h:37-49 (type 1, iflag +1); returns complex recon volume."""
    return plan.type1(c, pg.x, pg.y, pg.z)


# ---------------------------------------------------------------------------
# uniform FFT helpers (include/fftutils.h, include/fft.h)
# ---------------------------------------------------------------------------

def fftshift2(a):
    """include/fftutils.h:85-103: out[.., j, k] = in[.., (j+n2//2)%n2, (k+n3//2)%n3]."""
    n2, n3 = a.shape[-2:]
    return np.roll(a, (-(n2 // 2), -(n3 // 2)), axis=(-2, -1))


def ifftshift2(a):
    """include/fftutils.h:148-168: shift by n//2 (+1 when n is odd)."""
    n2, n3 = a.shape[-2:]
    d1 = n2 // 2 + (n2 % 2)
    d2 = n3 // 2 + (n3 % 2)
    return np.roll(a, (-d1, -d2), axis=(-2, -1))


def fft2(a):
    """include/fft.h:35-74: batched 2-D forward c2c over the last two axes, unnormalised."""
    return _fftn(a, axes=(-2, -1))


def ifft2(a):
    """include/fft.h:77-114: batched 2-D backward c2c, unnormalised."""
    return _ifftn_unnorm(a, axes=(-2, -1))


def fftfreq(n: int):
    """include/fftutils.h:37-52."""
    n2 = n // 2 if n % 2 == 0 else n // 2 + 1
    i = np.arange(n)
    return np.where(i < n2, i, i - n) * (2 * math.pi / n)


# ---------------------------------------------------------------------------
# operators (src/projection.cpp, src/gradient.cpp)
# ---------------------------------------------------------------------------

def _coeffs(pg: PolarGrid, gamma):
    return beam_dir_vector(float(gamma), pg.theta.astype(np.float64))  # (3, nproj)


def forward(m, pg: PolarGrid, gamma, plan: NufftPlan):
    """src/projection.cpp:42-77.  m: (3, n1, n2, n3) real -> (nproj, nrows, ncols) real."""
    coeff = _coeffs(pg, gamma)
    proj = np.zeros(pg.dims(), np.complex128)
    for i in range(3):
        c = nufft3d2(np.asarray(m[i], np.complex128), pg, plan)
        proj += coeff[i][:, None, None] * c
    proj = ifftshift2(ifft2(fftshift2(proj)))
    return proj.real / float(pg.nrows * pg.ncols)


def adjoint(proj, pg: PolarGrid, recon_dims, gamma, plan: NufftPlan):
    """src/projection.cpp:90-126.  proj real (nproj,nrows,ncols) -> (3, *recon_dims) real."""
    c = ifftshift2(fft2(fftshift2(np.asarray(proj, np.complex128))))
    coeff = _coeffs(pg, gamma)
    scale = float(pg.size() // pg.nprojs())
    out = np.zeros((3,) + tuple(recon_dims))
    for i in range(3):
        out[i] = nufft3d1(coeff[i][:, None, None] * c, pg, plan).real / scale
    return out


def sysmat(x, pg: PolarGrid, gamma, plan: NufftPlan):
    """src/gradient.cpp:34-89: y_i = Re(N1(sum_k c_i c_k N2(x_k))) / (nrows*ncols)."""
    coeff = _coeffs(pg, gamma)
    scale = float(pg.size() // pg.nprojs())
    ck = [nufft3d2(np.asarray(x[k], np.complex128), pg, plan) for k in range(3)]
    out = np.zeros(np.shape(x))
    for i in range(3):
        r = sum((coeff[i] * coeff[k])[:, None, None] * ck[k] for k in range(3))
        out[i] = nufft3d1(r, pg, plan).real / scale
    return out


def normal(x, grids: Sequence[PolarGrid], gammas, plan: NufftPlan):
    """The MBIR `A` closure: sum over gamma of sysmat (src/mbir_sb.cpp:89-97)."""
    out = sysmat(x, grids[0], gammas[0], plan)
    for pg, g in zip(grids[1:], gammas[1:]):
        out += sysmat(x, pg, g, plan)
    return out


def gradient(f, yT, pg, gamma, plan):
    """src/gradient.cpp:98-105."""
    return sysmat(f, pg, gamma, plan) - yT


def residual(f, yT, pg, yTy, gamma, plan):
    """src/gradient.cpp:117-127: sum_i sqrt(f_i.AAf_i - 2 f_i.yT_i + yTy)."""
    AAx = sysmat(f, pg, gamma, plan)
    err = 0.0
    for i in range(3):
        xAAx = float(np.dot(np.ravel(f[i]), np.ravel(AAx[i])))
        yTx = float(np.dot(np.ravel(f[i]), np.ravel(yT[i])))
        err += math.sqrt(xAAx - 2.0 * yTx + yTy)
    return err


# ---------------------------------------------------------------------------
# Toeplitz form of the normal operator (this project's design, checked
# against `normal` above)
# ---------------------------------------------------------------------------

def dirichlet(s, n: int):
    """sum_{c<n} exp(i s (c-(n-1)/2) 2 pi/n) = sin(pi s)/sin(pi s/n) (limit where 0/0)."""
    s = np.asarray(s, dtype=np.float64)
    den = np.sin(np.pi * s / n)
    num = np.sin(np.pi * s)
    m = np.rint(s / n)
    near = np.abs(s - m * n) < 1e-9
    lim = n * np.where((m * (n - 1)) % 2 == 0, 1.0, -1.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        out = np.where(near, lim, num / np.where(near, 1.0, den))
    return out


def toeplitz_kernel(dims, thetas_per_gamma, gammas, nrows, ncols):
    """T_ik[d] = (1/(nrows ncols)) sum_gamma sum_theta c_i c_k D_ncols(d.a) D_nrows(d.b)
    for d in [-(n-1), n-1]^3, with a = (cos g, 0, -sin g), b = (cos th sin g, -sin th,
    cos th cos g) in (x, y, z) order.  Returns (6, 2n1-1, 2n2-1, 2n3-1) for the pairs
    (00, 11, 22, 01, 02, 12); index d + (n-1)."""
    n1, n2, n3 = dims
    dz = np.arange(-(n1 - 1), n1)[:, None, None].astype(np.float64)
    dy = np.arange(-(n2 - 1), n2)[None, :, None].astype(np.float64)
    dx = np.arange(-(n3 - 1), n3)[None, None, :].astype(np.float64)
    pairs = [(0, 0), (1, 1), (2, 2), (0, 1), (0, 2), (1, 2)]
    T = np.zeros((6, 2 * n1 - 1, 2 * n2 - 1, 2 * n3 - 1))
    for th, g in zip(thetas_per_gamma, gammas):
        g = float(g)
        Da = dirichlet(dx * math.cos(g) - dz * math.sin(g), ncols)
        u = dx * math.sin(g) + dz * math.cos(g)
        for t in np.asarray(th, np.float64):
            c = beam_dir_vector(g, t)
            Db = dirichlet(math.cos(t) * u - dy * math.sin(t), nrows)
            P = Da * Db
            for q, (i, k) in enumerate(pairs):
                T[q] += c[i] * c[k] * P
    return T / float(nrows * ncols)


def toeplitz_apply(x, T):
    """y_i = sum_k T_ik * x_k (linear convolution, outputs cropped to x's shape)."""
    n1, n2, n3 = x.shape[1:]
    L = (2 * n1 - 1, 2 * n2 - 1, 2 * n3 - 1)
    K = _fftn(np.fft.ifftshift(T, axes=(1, 2, 3)), axes=(1, 2, 3))  # centre d=0 at index 0
    X = _fftn(np.pad(x, ((0, 0), (0, L[0] - n1), (0, L[1] - n2), (0, L[2] - n3))), axes=(1, 2, 3))
    idx = {(0, 0): 0, (1, 1): 1, (2, 2): 2, (0, 1): 3, (0, 2): 4, (1, 2): 5}
    y = np.zeros_like(x, dtype=np.float64)
    for i in range(3):
        acc = sum(K[idx[tuple(sorted((i, k)))]] * X[k] for k in range(3))
        y[i] = _ifftn_unnorm(acc, axes=(0, 1, 2)).real[:n1, :n2, :n3] / np.prod(L)
    return y


# ---------------------------------------------------------------------------
# padding / cropping (include/padding.h) and array ops (include/array_ops.h)
# ---------------------------------------------------------------------------

def _npad(n: int, factor) -> int:
    """2 * (size_t(n * factor) / 2) with the product in float (padding.h:98-101)."""
    return 2 * (int(np.float32(n) * np.float32(factor)) // 2)


def pad2d(arr, factor):
    """include/padding.h:94-131 (symmetric)."""
    if np.float32(factor) < 1e-6:
        return arr.copy()
    n1, n2, n3 = arr.shape
    p2, p3 = _npad(n2, factor), _npad(n3, factor)
    out = np.zeros((n1, n2 + p2, n3 + p3), arr.dtype)
    out[:, p2 // 2:p2 // 2 + n2, p3 // 2:p3 // 2 + n3] = arr
    return out


def crop2d(arr, new_dims):
    """include/padding.h:134-166 (symmetric)."""
    n1, m2, m3 = new_dims
    d2 = (arr.shape[1] - m2) // 2
    d3 = (arr.shape[2] - m3) // 2
    return arr[:n1, d2:d2 + m2, d3:d3 + m3].copy()


def pad3d(arr, factor):
    """include/padding.h:169-204 (symmetric)."""
    if np.float32(factor) < 1e-6:
        return arr.copy()
    p = [_npad(n, factor) for n in arr.shape]
    out = np.zeros(tuple(n + q for n, q in zip(arr.shape, p)), arr.dtype)
    sl = tuple(slice(q // 2, q // 2 + n) for n, q in zip(arr.shape, p))
    out[sl] = arr
    return out


def crop3d(arr, new_dims):
    """include/padding.h:207-232 (symmetric)."""
    d = [(a - b) // 2 for a, b in zip(arr.shape, new_dims)]
    return arr[tuple(slice(o, o + n) for o, n in zip(d, new_dims))].copy()


def padded_volume_dims(recon_dims, pad_factor=np.float32(1.4142)):
    """Volume padding of MBIR1/2/3 (src/mbir_sb.cpp:50-60): n + 2*floor(n*(PAD-1)/2)."""
    f = np.float32(pad_factor) - np.float32(1.0)
    return tuple(int(n) + 2 * (int(np.float32(n) * f) // 2) for n in recon_dims)


# ---------------------------------------------------------------------------
# solvers (src/conjgrad.cpp, include/precond.h, src/bregman.cpp, src/finitediff.cpp,
# src/qggmrf.cpp, src/nagopt.cpp, src/lipschitz.cpp)
# ---------------------------------------------------------------------------

class RampPreconditioner:
    """include/precond.h:33-87: per-n1-slice 2-D ramp |k| filter via r2c/c2r."""

    def __init__(self, dims):
        n1, n2, n3 = dims
        xf = np.arange(n3 // 2 + 1) / n3
        j = np.arange(n2)
        yf = np.where(j <= n2 // 2, j, j - n2) / n2
        self.filter = np.sqrt(xf[None, :] ** 2 + yf[:, None] ** 2)
        self.dims = dims

    def apply(self, a):
        n1, n2, n3 = a.shape
        F = np.fft.rfft2(a, axes=(1, 2)) * self.filter[None]
        return np.fft.irfft2(F, s=(n2, n3), axes=(1, 2))  # irfft2 includes 1/(n2 n3)


def _vdot(a, b):
    return sum(float(np.dot(np.ravel(a[i]), np.ravel(b[i]))) for i in range(3))


def cgsolver(A: Callable, y, x0, max_iter: int, tol: float, precond=None, log=None):
    """src/conjgrad.cpp:37-117 (PCG with the ramp preconditioner)."""
    x = np.array(x0, dtype=np.float64)
    M = precond if precond is not None else RampPreconditioner(x.shape[1:])
    r = y - A(x)
    z = np.stack([M.apply(r[i]) for i in range(3)])
    p = z.copy()
    rs_old = _vdot(z, r)
    for it in range(max_iter):
        Ap = A(p)
        pAp = _vdot(p, Ap)
        if abs(pAp) < 1e-10:
            break
        alpha = rs_old / pAp
        x += alpha * p
        r -= alpha * Ap
        z = np.stack([M.apply(r[i]) for i in range(3)])
        rs_new = _vdot(z, r)
        if log is not None:
            log.append(math.sqrt(max(rs_new, 0.0)))
        if math.sqrt(max(rs_new, 0.0)) < tol:
            break
        p = z + p * (rs_new / rs_old)
        rs_old = rs_new
    return x


def cgsolver_refined(A_hi: Callable, A_lo: Callable, y, x0, inner: int, refinements: int, tol: float):
    """Iterative refinement around PCG (this project's mixed-precision form):
    r = y - A_hi x; d = PCG(A_lo, r, 0, inner); x += d, `refinements` times."""
    x = np.array(x0, dtype=np.float64)
    for _ in range(refinements):
        r = y - A_hi(x)
        if math.sqrt(float(np.sum(r * r))) < tol:
            break
        x += cgsolver(A_lo, r, np.zeros_like(x), inner, tol)
    return x


def grad_u(u):
    """src/finitediff.cpp:8-47: central differences / 2 on interior voxels, zero border."""
    g = np.zeros((3,) + u.shape, dtype=np.float64)
    c = (slice(1, -1),) * 3
    g[0][c] = (u[2:, 1:-1, 1:-1] - u[:-2, 1:-1, 1:-1]) / 2.0
    g[1][c] = (u[1:-1, 2:, 1:-1] - u[1:-1, :-2, 1:-1]) / 2.0
    g[2][c] = (u[1:-1, 1:-1, 2:] - u[1:-1, 1:-1, :-2]) / 2.0
    return g


def divergence(du):
    """src/finitediff.cpp:54-71: NEGATIVE central-difference divergence, zero border."""
    out = np.zeros(du[0].shape, dtype=np.float64)
    out[1:-1, 1:-1, 1:-1] = (-(du[0][2:, 1:-1, 1:-1] - du[0][:-2, 1:-1, 1:-1]) / 2.0
                             - (du[1][1:-1, 2:, 1:-1] - du[1][1:-1, :-2, 1:-1]) / 2.0
                             - (du[2][1:-1, 1:-1, 2:] - du[2][1:-1, 1:-1, :-2]) / 2.0)
    return out


def laplacian(u):
    """include/bregman.h:34-36: divergence(grad_u(u)) (= -div grad, PSD)."""
    return divergence(grad_u(u))


def _fftfreq_ref(n: int) -> np.ndarray:
    """include/fftutils.h:36-51: 0..ceil(n/2)-1, then negatives, times 2 pi / n."""
    half = n // 2 if n % 2 == 0 else n // 2 + 1
    return np.array([i if i < half else i - n for i in range(n)], np.float64) * (2 * np.pi / n)


def demag(m3):
    """include/demag.h:13-79 in FP64: H = irfftn(-k (k . rfftn(m)) / |k|^2), the k = 0
    term set to 0 (the reference's frequency grids: fftfreq along n1, n2, rfftfreq
    along n3, each times 2 pi / n)."""
    m = np.asarray(m3, dtype=np.float64)
    n1, n2, n3 = m.shape[1:]
    kx, ky = _fftfreq_ref(n1), _fftfreq_ref(n2)
    kz = np.arange(n3 // 2 + 1, dtype=np.float64) * (2 * np.pi / n3)
    K = np.meshgrid(kx, ky, kz, indexing="ij")
    M = np.fft.rfftn(m, axes=(1, 2, 3))
    kk = K[0] ** 2 + K[1] ** 2 + K[2] ** 2
    kk[0, 0, 0] = 1.0
    kdm = K[0] * M[0] + K[1] * M[1] + K[2] * M[2]
    H = np.stack([-kdm * K[c] / kk for c in range(3)])
    H[:, 0, 0, 0] = 0
    return np.fft.irfftn(H, s=(n1, n2, n3), axes=(1, 2, 3))


def split_bregman(A: Callable, yT, x0, lam, mu, outer_max, inner_max, tol, xtol, log=None,
                  A_lo: Callable | None = None, refinements: int = 0):
    """src/bregman.cpp:39-134 (isotropic TV, inner PCG on A + mu*laplacian).  With
    A_lo and refinements > 0 the inner solve is cgsolver_refined (mixed form)."""
    eps = 1e-8
    x = np.array(x0, dtype=np.float64)
    x_old = x.copy()
    d = np.zeros((3, 3) + x.shape[1:])
    b = np.zeros((3, 3) + x.shape[1:])

    def Ap(u):
        du = A(u)
        return du + mu * np.stack([laplacian(u[i]) for i in range(3)])

    def Ap_lo(u):
        return A_lo(u) + mu * np.stack([laplacian(u[i]) for i in range(3)])

    for it in range(outer_max):
        rhs = np.stack([yT[i] + divergence(d[i] - b[i]) * mu for i in range(3)])
        if A_lo is not None and refinements > 0:
            x = cgsolver_refined(Ap, Ap_lo, rhs, x_old, inner_max, refinements, tol)
        else:
            x = cgsolver(Ap, rhs, x_old, inner_max, tol)
        gx = np.stack([grad_u(x[i]) for i in range(3)])
        sk = np.sqrt(eps + ((gx + b) ** 2).sum(axis=(0, 1)))
        d = np.maximum(sk - lam / mu, 0.0) * ((gx + b) / sk)
        b = b + gx - d
        nd = sum(np.linalg.norm(x[i] - x_old[i]) / (np.linalg.norm(x_old[i]) + eps)
                 for i in range(3))
        if log is not None:
            log.append(nd)
        x_old = x.copy()
        if nd < xtol:
            break
    return x


# qGGMRF neighbour weights (src/qggmrf.cpp:25-29), index (dx+1)*9 + (dy+1)*3 + (dz+1);
# entry 12 (0.0532) differs from its mirror entry 14 (0.0523) in the reference.
QGGMRF_WEIGHT = np.array([0.0302, 0.037, 0.0302, 0.037, 0.0523, 0.037,
                          0.0302, 0.037, 0.0302, 0.037, 0.0523, 0.037,
                          0.0532, 0.0, 0.0523, 0.037, 0.0523, 0.037,
                          0.0302, 0.037, 0.0302, 0.037, 0.0523, 0.037,
                          0.0302, 0.037, 0.0302], dtype=np.float32)
MRF_Q = 2.0
MRF_C = 0.001


def d_potential(delta, sigma_q, sigma_qp, p):
    """src/qggmrf.cpp:42-57 (note the non-zero value q/(sigma^q C) at delta == 0)."""
    ad = np.abs(delta)
    t1 = np.power(ad, MRF_Q - p) / sigma_qp
    t3 = MRF_C + t1
    with np.errstate(divide="ignore", invalid="ignore"):
        v = (delta / (t3 * sigma_q)) * (MRF_Q - ((MRF_Q - p) * t1) / t3)
    return np.where(ad > 0, v, MRF_Q / (sigma_q * MRF_C))


def qggmrf(g, x, sigma, p):
    """src/qggmrf.cpp:60-95: g[interior] += sum_26 w * rho'(x_nbr - x); returns new g."""
    x = np.asarray(x, np.float64)
    sigma_q = float(np.float32(sigma)) ** MRF_Q
    sigma_qp = float(np.float32(sigma)) ** (MRF_Q - float(np.float32(p)))
    p = float(np.float32(p))
    n1, n2, n3 = x.shape
    u = x[1:-1, 1:-1, 1:-1]
    acc = np.zeros_like(u)
    for dx in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dz in (-1, 0, 1):
                if dx == 0 and dy == 0 and dz == 0:
                    continue
                v = x[1 + dx:n1 - 1 + dx, 1 + dy:n2 - 1 + dy, 1 + dz:n3 - 1 + dz]
                w = float(QGGMRF_WEIGHT[(dx + 1) * 9 + (dy + 1) * 3 + (dz + 1)])
                acc += w * d_potential(v - u, sigma_q, sigma_qp, p)
    out = np.array(g, dtype=np.float64)
    out[1:-1, 1:-1, 1:-1] += acc
    return out


def nagopt(grad: Callable, loss: Callable, x, max_iters, lipschitz, tol, xtol,
           max_inner_iters=20, log=None):
    """src/nagopt.cpp:116-209 (vector form).  Acceptance test uses the norm (not
    its square) of g; the line search keeps the overwritten x on rejection."""
    x = np.array(x, dtype=np.float64)
    xold = x.copy()
    t = 1.0
    tnew = 1.0
    step = 0.1 / lipschitz
    step_prev = step
    xerr = float("inf")
    for it in range(max_iters):
        for inner in range(max_inner_iters):
            beta = tnew * (1.0 / t - 1.0)
            tnew = 0.5 * (math.sqrt(t ** 4 + 4 * t ** 2) - t ** 2)
            y = x + (x - xold) * beta
            g = grad(y)
            x = y - g * step
            ex = loss(x)
            ey = loss(y)
            gy = 0.5 * step * sum(float(np.linalg.norm(g[i])) for i in range(3))
            if ex > ey + gy:
                step *= 0.9
            else:
                step = step_prev
                t = tnew
                xe = sum(float(np.linalg.norm(x[i] - xold[i])) for i in range(3))
                xn = sum(float(np.linalg.norm(x[i])) for i in range(3))
                xerr = xe / xn
                if xerr < xtol:
                    return x
                xold = x.copy()
                break
        e = loss(x)
        if log is not None:
            log.append((e, xerr))
        if e < tol:
            break
    return x


def lipschitz(A: Callable, shape, max_iters=30, tol=1e-5, seed=0):
    """Power iteration of src/lipschitz.cpp:31-53 (which does not compile in the
    reference: Array::random_like is missing); seeded start, FP64 norms."""
    rng = np.random.default_rng(seed)
    x = rng.random(shape)
    x /= np.linalg.norm(x)
    L = 0.0
    for _ in range(max_iters):
        Ax = A(x)
        nA = float(np.linalg.norm(Ax))
        if abs(nA) < 1e-12:
            return 0.0
        x = Ax / nA
        if abs(nA - L) < tol:
            L = nA
            break
        L = nA
    return L


# ---------------------------------------------------------------------------
# MBIR drivers (src/mbir_cg.cpp, src/mbir_sb.cpp, src/mbir3.cpp)
# ---------------------------------------------------------------------------

class ReconParams:
    """include/config.h:146-158 defaults."""

    def __init__(self, **kw):
        self.maxIters = 50
        self.innerIters = 3
        self.sigma = 1000.0
        self.p = 1.2
        self.lam = 0.1
        self.mu = 10.0
        self.tol = 1e-5
        self.xtol = 1e-5
        self.PAD_FACTOR = np.float32(1.4142)
        for k, v in kw.items():
            setattr(self, k, v)


def mbir_setup(datasets, recon_dims, params, proj_pad, eps=1e-12, exact=False,
               grid_dtype=np.float32):
    """Common setup of MBIR1/2/3: normalise by max, pad2d, PolarGrid, yT += adjoint."""
    out_dims = padded_volume_dims(recon_dims, params.PAD_FACTOR)
    plan = NufftPlan(out_dims, eps=eps, exact=exact)
    grids, gammas = [], []
    yT = np.zeros((3,) + out_dims)
    for proj, angles, gamma in datasets:
        y = np.asarray(proj, np.float64) / float(np.max(proj))
        y = pad2d(y, proj_pad)
        pg = PolarGrid(angles, y.shape[1], y.shape[2], gamma, dtype=grid_dtype)
        grids.append(pg)
        gammas.append(gamma)
        yT += adjoint(y, pg, out_dims, gamma, plan)
    return out_dims, plan, grids, gammas, yT


def MBIR1(datasets, recon_dims, params, eps=1e-12, exact=False, refinements=0, grid_dtype=np.float32):
    """src/mbir_cg.cpp:48-128 (projections padded by PAD_FACTOR-1).  refinements > 0
    runs the mixed form's algorithm (cgsolver_refined, maxIters // refinements inner
    iterations per cycle) with the exact operator in both roles.  grid_dtype: the
    precision of the PolarGrid points (float32 as the reference's float build,
    float64 as its double build)."""
    pad = np.float32(params.PAD_FACTOR - 1.0)
    out_dims, plan, grids, gammas, yT = mbir_setup(datasets, recon_dims, params, pad, eps, exact, grid_dtype)
    A = lambda v: normal(v, grids, gammas, plan)
    if refinements > 0:
        x = cgsolver_refined(A, A, yT, np.zeros((3,) + out_dims), max(1, params.maxIters // refinements),
                             refinements, params.tol)
    else:
        x = cgsolver(A, yT, np.zeros((3,) + out_dims), params.maxIters, params.tol)
    return np.stack([crop3d(x[i], recon_dims) for i in range(3)])


def MBIR2(datasets, recon_dims, params, eps=1e-12, exact=False, refinements=0, grid_dtype=np.float32):
    """src/mbir_sb.cpp:47-114 (projections padded by PAD_FACTOR itself); refinements
    > 0 as in MBIR1 for each inner linear solve."""
    out_dims, plan, grids, gammas, yT = mbir_setup(datasets, recon_dims, params,
                                                   params.PAD_FACTOR, eps, exact, grid_dtype)
    A = lambda v: normal(v, grids, gammas, plan)
    x = split_bregman(A, yT, np.zeros((3,) + out_dims), params.lam, params.mu,
                      params.maxIters, params.innerIters, params.tol, params.xtol,
                      A_lo=A if refinements > 0 else None, refinements=refinements)
    return np.stack([crop3d(x[i], recon_dims) for i in range(3)])


def MBIR3(datasets, recon_dims, params, eps=1e-12, exact=False, grid_dtype=np.float32):
    """src/mbir3.cpp:47-135 (NAG + qGGMRF; `mu` passed as the Lipschitz constant)."""
    out_dims, plan, grids, gammas, yT = mbir_setup(datasets, recon_dims, params,
                                                   params.PAD_FACTOR, eps, exact, grid_dtype)

    def grad(x):
        g = sum(gradient(x, yT, pg, gm, plan) for pg, gm in zip(grids, gammas))
        return np.stack([qggmrf(g[i], x[i], params.sigma, params.p) for i in range(3)])

    yTy = sum(float(np.dot(np.ravel(yT[i]), np.ravel(yT[i]))) for i in range(3))

    def loss(x):
        return sum(residual(x, yT, pg, yTy, gm, plan) for pg, gm in zip(grids, gammas))

    x = nagopt(grad, loss, np.zeros((3,) + out_dims), params.maxIters, params.mu,
               params.tol, params.xtol, params.innerIters)
    return np.stack([crop3d(x[i], recon_dims) for i in range(3)])


def MBIR3_toeplitz(datasets, recon_dims, params, eps=1e-12, grid_dtype=np.float32, lipschitz_iters=0):
    """MBIR3 (src/mbir3.cpp:47-135) with each dataset's sysmat in its FP64
    Toeplitz form (toeplitz_kernel / toeplitz_apply: the same operator up to the
    float rounding of the grid points), for volumes where 40 iterations of the
    NUFFT form would take too long on the CPU; the setup adjoints stay NUFFT.
    Gradient sum_g (S_g x - yT) (yT subtracted once per dataset, src/mbir3.cpp:93-96)
    plus qGGMRF; loss sum_g residual_g.  lipschitz_iters > 0 replaces `mu` by the
    power-iteration estimate of sum_g S_g (seed 0).  Returns (volume, L used)."""
    out_dims, plan, grids, gammas, yT = mbir_setup(datasets, recon_dims, params,
                                                   params.PAD_FACTOR, eps, False, grid_dtype)
    Ts = [toeplitz_kernel(out_dims, [pg.theta], [float(gm)], pg.nrows, pg.ncols) for pg, gm in zip(grids, gammas)]
    S = [lambda v, T=T: toeplitz_apply(v, T) for T in Ts]
    yTy = sum(float(np.dot(np.ravel(yT[i]), np.ravel(yT[i]))) for i in range(3))

    def grad(x):
        g = sum(Sg(x) - yT for Sg in S)
        return np.stack([qggmrf(g[i], x[i], params.sigma, params.p) for i in range(3)])

    def loss(x):
        err = 0.0
        for Sg in S:
            AAx = Sg(x)
            for i in range(3):
                xAAx = float(np.dot(np.ravel(x[i]), np.ravel(AAx[i])))
                yTx = float(np.dot(np.ravel(x[i]), np.ravel(yT[i])))
                err += math.sqrt(xAAx - 2.0 * yTx + yTy)
        return err

    L = params.mu
    if lipschitz_iters > 0:
        L = lipschitz(lambda v: sum(Sg(v) for Sg in S), (3,) + out_dims, lipschitz_iters)
    x = nagopt(grad, loss, np.zeros((3,) + out_dims), params.maxIters, L, params.tol, params.xtol,
               params.innerIters)
    return np.stack([crop3d(x[i], recon_dims) for i in range(3)]), L


# ---------------------------------------------------------------------------
# synthetic inputs (seeded; no public dataset exists for this path)
# ---------------------------------------------------------------------------

def synthetic_magnetization(dims, seed=1234, sigma=3.0, lateral_frac=0.8):
    """Unit vectors i.i.d. per voxel, Gaussian-smoothed (reflect), renormalised,
    zeroed outside a full-thickness x central-80%-lateral slab.  dims = (n1, n2, n3)
    in the internal (W, T, H) order; thickness is n2."""
    from scipy.ndimage import gaussian_filter
    rng = np.random.default_rng(seed)
    m = rng.standard_normal((3,) + tuple(dims))
    m /= np.linalg.norm(m, axis=0, keepdims=True) + 1e-12
    for i in range(3):
        m[i] = gaussian_filter(m[i], sigma, mode="reflect")
    m /= np.linalg.norm(m, axis=0, keepdims=True) + 1e-12
    n1, n2, n3 = dims
    mask = np.zeros(dims, bool)
    a1 = int(round(n1 * (1 - lateral_frac) / 2))
    a3 = int(round(n3 * (1 - lateral_frac) / 2))
    mask[a1:n1 - a1, :, a3:n3 - a3] = True
    return (m * mask).astype(np.float32)


# Config 0 of the workload set (the reference's small CPU-runnable case):
# recon (T, H, W) = 16 x 128 x 128 (internal (n1, n2, n3) = (W, T, H) =
# (128, 16, 128)), 2 gamma datasets (0, 45 deg) x 90 angles uniform in
# [0, 2 pi), 128 x 128 detector, data = forward model + 1% Gaussian noise,
# 20 CG iterations (MBIR1).
CONFIG0_RECON = (128, 16, 128)
CONFIG0_GAMMAS = (0.0, math.pi / 4)
CONFIG0_NPROJ = 90
CONFIG0_DET = (128, 128)


def config0_datasets(seed: int = 1234):
    """Seeded config-0 datasets [(proj float32 (90, 128, 128), angles float32, gamma float32)].

    Data follow the reference's forward tool (src/forward.cpp:132-177): the
    magnetization is padded by pad3d(sqrt(2) - 1), projected with the forward
    model on the detector padded likewise, and cropped to 128 x 128 (crop2d);
    then N(0, (0.01 RMS)^2) noise is added.  The forward model runs in FP64 with
    ES gridding at eps 1e-6 (data generation only)."""
    rng = np.random.default_rng(seed)
    m = synthetic_magnetization(CONFIG0_RECON, seed=seed, sigma=3.0).astype(np.float64)
    fpad = np.float32(math.sqrt(2.0) - 1.0)
    mp = np.stack([pad3d(m[i], fpad) for i in range(3)])
    det_p = tuple(n + _npad(n, fpad) for n in CONFIG0_DET)
    plan = NufftPlan(mp.shape[1:], eps=1e-6)
    out = []
    for g in CONFIG0_GAMMAS:
        th = rng.uniform(0, 2 * np.pi, CONFIG0_NPROJ).astype(np.float32)
        pg = PolarGrid(th, det_p[0], det_p[1], np.float32(g), dtype=np.float64)
        p = forward(mp, pg, float(np.float32(g)), plan)
        p = crop2d(p, (CONFIG0_NPROJ,) + CONFIG0_DET)
        rms = float(np.sqrt(np.mean(p * p)))
        p = p + rng.normal(0.0, 0.01 * rms, p.shape)
        out.append((p.astype(np.float32), th, np.float32(g)))
    return out
