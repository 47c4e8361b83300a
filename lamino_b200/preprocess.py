"""Host-side array preparation around the GPU operators, as the reference's
tools do it: NaN/Inf masking and the rectangular support mask
(include/mask.h:29-91), symmetric 3-D padding and 2-D cropping
(include/padding.h:134-204) and axis permutation (include/array_ops.h).
These run once per dataset on the host, as in the reference, before the data
go to the device."""
from __future__ import annotations

import math

import numpy as np

__all__ = ["mask_infs_nans", "mask_support", "pad3d", "crop2d", "transpose"]


def mask_infs_nans(projs) -> np.ndarray:
    """A copy with every NaN and infinity set to 0 (include/mask.h:29-40)."""
    out = np.array(projs, dtype=np.float32, copy=True)
    out[~np.isfinite(out)] = 0.0
    return out


def mask_support(projs, dims, theta, gamma) -> np.ndarray:
    """Zero the detector pixels that cannot see a rectangular sample of
    (n1, n2, n3) = dims voxels (include/mask.h:42-91): pixel (y, x) of projection
    p, relative to the detector centre, is kept when its un-rotated position
    ((x cos g cos t + y sin g) / cos t, (-x sin g cos t + y cos g) / cos t) lies
    within (n3 / 2, n2 / 2).  Raises when a projection angle is within 1e-6 (in
    cosine) of 90 degrees, where the mask is undefined."""
    p = np.asarray(projs, dtype=np.float32)
    npj, nr, nc = p.shape
    f = np.float32
    cg, sg = f(math.cos(float(gamma))), f(math.sin(float(gamma)))
    xcen, ycen = f(nc // 2), f(nr // 2)
    ylim, xlim = f(int(dims[1]) // 2), f(int(dims[2]) // 2)
    x = np.arange(nc, dtype=np.float32) - xcen
    y = np.arange(nr, dtype=np.float32) - ycen
    X, Y = np.meshgrid(x, y)
    out = p.copy()
    for i, t in enumerate(np.asarray(theta, dtype=np.float32)):
        ct = f(math.cos(float(t)))
        if abs(ct) < 1e-6:
            raise ValueError("projection angle too close to 90 degrees: the support mask is undefined")
        xc = (X * cg * ct + Y * sg) / ct
        yc = (-X * sg * ct + Y * cg) / ct
        out[i][(np.abs(xc) > xlim) | (np.abs(yc) > ylim)] = 0.0
    return out


def _npad(n: int, factor: float) -> int:
    """2 * (size_t(n * factor) / 2) with the product in float (include/padding.h:173-178)."""
    return 2 * (int(np.float32(n) * np.float32(factor)) // 2)


def pad3d(arr, factor: float) -> np.ndarray:
    """Zero padding of every axis by 2 floor(n factor / 2), centred (SYMMETRIC)."""
    a = np.asarray(arr, dtype=np.float32)
    if np.float32(factor) < 1e-6:
        return a.copy()
    pads = [_npad(n, factor) for n in a.shape]
    out = np.zeros(tuple(n + q for n, q in zip(a.shape, pads)), np.float32)
    out[tuple(slice(q // 2, q // 2 + n) for n, q in zip(a.shape, pads))] = a
    return out


def crop2d(arr, new_dims) -> np.ndarray:
    """The centred (m2, m3) window of every slice, first m1 slices (SYMMETRIC)."""
    a = np.asarray(arr)
    m1, m2, m3 = (int(v) for v in new_dims)
    d2, d3 = (a.shape[1] - m2) // 2, (a.shape[2] - m3) // 2
    if d2 < 0 or d3 < 0 or m1 > a.shape[0]:
        raise ValueError("crop window larger than the array")
    return np.ascontiguousarray(a[:m1, d2:d2 + m2, d3:d3 + m3])


def transpose(arr, axes) -> np.ndarray:
    """Axis permutation: output axis i is input axis axes[i]."""
    return np.ascontiguousarray(np.transpose(np.asarray(arr), tuple(int(a) for a in axes)))
