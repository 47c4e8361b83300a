"""Reconstruction from a TOML file, the reference's ``recon`` tool
(src/recon.cpp:31-112) on the GPU path:

    python -m lamino_b200.recon config.toml

Reads the datasets, runs MBIR1 (no regularizer), MBIR2 (split Bregman) or
MBIR3 (qGGMRF) on the reconstruction size given as (thickness, rows, cols) —
internally (cols, thickness, rows), as the reference reorders it — and writes
the three components as TIFF stacks (<base>0.tiff ...) and/or one .vti file.
Without an argument it prints the usage and writes an example config.toml."""
from __future__ import annotations

import os
import sys
import time

import numpy as np

from . import config as cfg
from . import tiffio, vti
from .preprocess import transpose

__all__ = ["reconstruct", "main"]


def _elapsed(sec: float) -> str:
    if sec > 3600:
        h = int(sec // 3600)
        m = int((sec - 3600 * h) // 60)
        return f"Reconstruction completed in {h} hours, {m} minutes, and {sec - 3600 * h - 60 * m:.2f} seconds."
    if sec > 60:
        m = int(sec // 60)
        return f"Reconstruction completed in {m} minutes and {sec - 60 * m:.2f} seconds."
    return f"Reconstruction completed in {sec:.2f} seconds."


def reconstruct(datasets, rc: "cfg.ReconConfig", gpu: "cfg.GpuParams | None" = None) -> np.ndarray:
    """(3, T, H, W) reconstruction of rc.recon_dims = (T, H, W) from
    [(projections, angles, gamma)], in the reference's axis conventions."""
    import lamino_b200 as L
    gpu = gpu or cfg.GpuParams()
    d = rc.recon_dims
    internal = (d[2], d[0], d[1])  # src/recon.cpp:60: (W, T, H)
    p = L.ReconParams(maxIters=rc.max_iters, innerIters=rc.inner_iters, sigma=rc.sigma, p=rc.p, lam=rc.lam,
                      mu=rc.mu, tol=rc.tol, xtol=rc.xtol, op_kind=gpu.operator, use_graphs=gpu.use_graphs,
                      autotune=gpu.autotune)
    fn = {1: L.MBIR1, 2: L.MBIR2, 3: L.MBIR3}[rc.method]
    vol = fn(datasets, internal, p)  # (3, W, T, H)
    return np.stack([transpose(vol[i], (1, 2, 0)) for i in range(3)])  # src/recon.cpp:76-78


def main(argv=None) -> int:
    argv = sys.argv[1:] if argv is None else argv
    if not argv:
        print("Usage: python -m lamino_b200.recon <input.toml>\n"
              "Please see config.toml (written now) for an example input file.", file=sys.stderr)
        cfg.dump_config()
        return 1
    table = cfg.read_toml_file(argv[0])
    datasets = cfg.parse_input_datasets(table)
    rc = cfg.ReconConfig.from_toml(table)
    out = cfg.OutputParams.from_toml(table)
    gpu = cfg.GpuParams.from_toml(table)
    print(rc.describe())
    import torch
    torch.cuda.set_device(gpu.device)
    t0 = time.perf_counter()
    recon = reconstruct(datasets, rc, gpu)
    print(_elapsed(time.perf_counter() - t0))
    base_dir = os.path.dirname(out.filepath)
    if base_dir:
        os.makedirs(base_dir, exist_ok=True)
    if out.has_format("tiff"):
        tiffio.write3(out.filepath, recon)
    if out.has_format("vti"):
        vti.write_vectors(out.filepath, recon)
        print(f"Reconstruction saved to {out.filepath}.")
    return 0


if __name__ == "__main__":
    sys.exit(main())
