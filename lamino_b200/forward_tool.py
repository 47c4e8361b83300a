"""Synthetic projections from a magnetization volume, the reference's
``forward`` tool (src/forward.cpp:19-183) on the GPU forward operator:

    python -m lamino_b200.forward_tool config.toml

config.toml:  [input] data_path, component_1, component_2, component_3 (TIFF
stacks of the x, y, z components, (thickness, rows, cols) each);
[angles] filename (text, degrees or radians); [orientation] gamma (degrees);
[output] filename, basedir, dims = [rows, cols] of the detector.

The volume is permuted to (cols, thickness, rows), zero-padded by sqrt(2) - 1
in every axis, projected onto a detector padded the same way and cropped back
to dims, as the reference does."""
from __future__ import annotations

import math
import os
import sys

import numpy as np

from . import config as cfg
from . import tiffio
from .preprocess import crop2d, pad3d, transpose

__all__ = ["project", "main"]

PADDING = 1.41421356237  # sqrt(2): the corners of the sample stay inside the detector


def _padded(dim: int) -> int:
    """dim + 2 int(dim (PADDING - 1) / 2), in double (src/forward.cpp:146-149)."""
    return int(dim + 2 * int(dim * (PADDING - 1) / 2))


def project(m3, angles, gamma: float, out_dims) -> np.ndarray:
    """Projections (nproj, out_dims[0], out_dims[1]) of m3 = 3 arrays (T, H, W)."""
    import lamino_b200 as L
    f = np.float32(PADDING - 1)
    vol = np.stack([pad3d(transpose(np.asarray(m3[i], np.float32), (2, 0, 1)), f) for i in range(3)])
    nr, nc = _padded(int(out_dims[0])), _padded(int(out_dims[1]))
    pg = L.PolarGrid(np.asarray(angles, np.float32), nr, nc, np.float32(gamma))
    proj = L.forward(vol, pg)
    return crop2d(proj, (len(angles), int(out_dims[0]), int(out_dims[1])))


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if not argv:
        print("usage: python -m lamino_b200.forward_tool config.toml", file=sys.stderr)
        return 1
    t = cfg.read_toml_file(argv[0])
    try:
        inp = t["input"]
        base = inp["data_path"]
        comps = [inp["component_1"], inp["component_2"], inp["component_3"]]
        angles_file = t["angles"]["filename"]
        gamma = np.float32(float(np.float32(t["orientation"]["gamma"])) * math.pi / 180.0)
        out_file, out_dir = t["output"]["filename"], t["output"]["basedir"]
        dims = t["output"]["dims"]
    except (KeyError, TypeError) as e:
        print(f"missing entry in {argv[0]}: {e}", file=sys.stderr)
        return 1
    if not isinstance(dims, list) or len(dims) != 2 or not all(isinstance(v, int) for v in dims):
        print("Output dimensions must be an array of two integers", file=sys.stderr)
        return 1
    os.makedirs(out_dir, exist_ok=True)
    paths = [os.path.join(base, c) for c in comps]
    if not all(os.path.exists(p) for p in paths):
        print(f"One or more components do not exist in data path: {base}", file=sys.stderr)
        return 1
    angles = cfg.read_angles_file(angles_file)
    m3 = [tiffio.read(p) for p in paths]
    print(f"Data dimensions: {list(m3[0].shape)}; angles [{angles.min():g}, {angles.max():g}] with "
          f"{len(angles)} steps; gamma {float(gamma):g}", file=sys.stderr)
    proj = project(m3, angles, gamma, dims)
    out = os.path.join(out_dir, out_file)
    tiffio.write(out, proj)
    print(f"Projections {list(proj.shape)} written to {out}", file=sys.stderr)
    return 0


if __name__ == "__main__":
    sys.exit(main())
