"""TOML front end of a reconstruction, as the reference's ``recon`` tool reads
it (include/config.h:37-367): the ``[[input]]`` datasets (TIFF projection stack,
text file of angles, gamma in degrees), ``[recon_params]`` (dimensions,
iterations, tolerances, regularizer) and ``[output]`` (file name, formats).

One table is added for this library, ``[gpu]``, absent from the reference:
``operator`` = "toeplitz" (default) | "toeplitz_fp16" | "nufft" | "mixed",
``device`` (CUDA ordinal, default 0), ``use_graphs`` and ``autotune`` (bools,
default true).
"""
from __future__ import annotations

import math
import os
import sys
import tomllib
from dataclasses import dataclass, field

import numpy as np

from . import tiffio
from .preprocess import mask_infs_nans

__all__ = ["read_toml_file", "read_angles_file", "parse_input_datasets", "ReconConfig", "OutputParams",
           "GpuParams", "dump_config"]

UNCONSTRAINED, SPLIT_BREGMAN, QGGMRF = "unconstrained", "split_bregman", "qGGMRF"


def read_toml_file(path: str) -> dict:
    """The parsed TOML table; RuntimeError when the file is missing or malformed."""
    if not os.path.exists(path):
        raise RuntimeError(f"TOML file does not exist: {path}")
    try:
        with open(path, "rb") as f:
            return tomllib.load(f)
    except tomllib.TOMLDecodeError as e:
        raise RuntimeError(f"Failed to parse TOML file '{path}': {e}") from None


def read_angles_file(path: str) -> np.ndarray:
    """Whitespace-separated angles; converted from degrees to radians when the
    largest one exceeds 2 pi in magnitude (include/config.h:55-79)."""
    if not os.path.exists(path):
        raise RuntimeError(f"Could not open angles file: {path}")
    vals = []
    with open(path) as f:
        for tok in f.read().split():
            try:
                vals.append(float(tok))
            except ValueError:
                break  # the reference's stream extraction stops at the first non-number
    if not vals:
        raise RuntimeError(f"No angles found in file: {path}")
    a = np.array(vals, dtype=np.float32)
    if abs(float(a.max())) > 2 * math.pi:
        a = (a.astype(np.float64) * math.pi / 180.0).astype(np.float32)
    return a


def parse_input_datasets(config: dict) -> list:
    """[(projections float32 (nproj, nrows, ncols), angles float32, gamma float32 radians)]
    from the [[input]] array (include/config.h:82-140); NaN / Inf pixels become 0."""
    inputs = config.get("input")
    if not isinstance(inputs, list):
        raise RuntimeError("Missing [[input]] array in TOML file")
    out = []
    for entry in inputs:
        if not isinstance(entry, dict):
            raise RuntimeError("Invalid [[input]] entry")
        if not all(k in entry for k in ("filename", "angles", "gamma")):
            raise RuntimeError("[[input]] entry must have 'filename', 'angles', and 'gamma' fields")
        fn, af, g = entry["filename"], entry["angles"], entry["gamma"]
        if not isinstance(fn, str):
            raise RuntimeError("[[input]] 'filename' must be a string")
        if not os.path.exists(fn):
            raise RuntimeError(f"Projection file does not exist: {fn}")
        if not isinstance(af, str):
            raise RuntimeError("[[input]] 'angles' must be a string")
        if not os.path.exists(af):
            raise RuntimeError(f"Angles file does not exist: {af}")
        if isinstance(g, bool) or not isinstance(g, (int, float)):
            raise RuntimeError("[[input]] 'gamma' field must be a number")
        projs = mask_infs_nans(tiffio.read(fn))
        angles = read_angles_file(af)
        if angles.shape[0] != projs.shape[0]:
            raise RuntimeError(f"{af}: {angles.shape[0]} angles for {projs.shape[0]} projections in {fn}")
        gamma = np.float32(float(np.float32(g)) * math.pi / 180.0)
        out.append((projs, angles, gamma))
    return out


@dataclass
class ReconConfig:
    """[recon_params] with the reference's defaults (include/config.h:145-258)."""
    regularizer: str = UNCONSTRAINED
    recon_dims: tuple = (0, 0, 0)
    max_iters: int = 50
    inner_iters: int = 3
    sigma: float = 1000.0
    p: float = 1.2
    lam: float = 0.1
    mu: float = 10.0
    tol: float = 1e-5
    xtol: float = 1e-5

    @classmethod
    def from_toml(cls, config: dict) -> "ReconConfig":
        rp = config.get("recon_params")
        if not isinstance(rp, dict):
            raise RuntimeError("Missing [recon_params] section in config file")
        c = cls()
        c.max_iters = int(rp.get("max_iters", 50))
        dims = rp.get("recon_dims")
        if not isinstance(dims, list) or len(dims) != 3:
            raise RuntimeError("[recon_params] 'recon_dims' must be an array of three integers")
        d = []
        for i, v in enumerate(dims):
            if isinstance(v, bool) or not isinstance(v, int) or v <= 0:
                raise RuntimeError(f"[recon_params] 'recon_dims[{i}]' must be a positive integer")
            d.append(v - 1 if v % 2 == 0 else v)  # odd sizes, as the reference
        c.recon_dims = tuple(d)
        if d[0] / d[2] > 0.15:
            print(f"Warning: recon_dims[0] / recon_dims[2] = {d[0] / d[2]:.2f} > 0.15. In laminography, the "
                  "thickness (recon_dims[0]) is expected to be much smaller than the in-plane dimensions "
                  "(recon_dims[1], recon_dims[2]). This may lead to increased memory usage.", file=sys.stderr)
        c.tol = float(rp.get("tol", 1e-5))
        c.xtol = float(rp.get("xtol", 1e-5))
        reg = rp.get("regularizer")
        if isinstance(reg, dict):
            method = reg.get("method", SPLIT_BREGMAN)
            if method == QGGMRF:
                prm = reg.get(QGGMRF)
                if not isinstance(prm, dict):
                    raise RuntimeError("Missing [recon_params.regularizer.qGGMRF] section in config file")
                c.regularizer = QGGMRF
                c.sigma = float(prm.get("sigma", 1000.0))
                c.p = float(prm.get("p", 1.2))
            elif method == SPLIT_BREGMAN:
                prm = reg.get(SPLIT_BREGMAN)
                if not isinstance(prm, dict):
                    raise RuntimeError("Missing [recon_params.regularizer.split_bregman] section in config file")
                c.regularizer = SPLIT_BREGMAN
                c.lam = float(prm.get("lambda", 0.1))
                c.mu = float(prm.get("mu", 10.0))
                c.inner_iters = int(prm.get("inner_iters", 3))
            else:
                raise RuntimeError("[recon_params] 'regularizer' must be either 'qGGMRF' or 'split_bregman'")
        return c

    @property
    def method(self) -> int:
        """MBIR1 (CG), MBIR2 (split Bregman) or MBIR3 (NAG + qGGMRF), as src/recon.cpp:65-73."""
        return {UNCONSTRAINED: 1, SPLIT_BREGMAN: 2, QGGMRF: 3}[self.regularizer]

    def describe(self) -> str:
        name = {QGGMRF: "qGGMRF", SPLIT_BREGMAN: "Split-Bregman"}.get(self.regularizer, "Unconstrained")
        s = ["Reconstruction Parameters:", f"  max_outer_iters: {self.max_iters}",
             f"  inner_iters: {self.inner_iters}",
             f"  recon_dims: [{self.recon_dims[0]}, {self.recon_dims[1]}, {self.recon_dims[2]}]",
             f"  tol: {self.tol:g}", f"  xtol: {self.xtol:g}", f"  regularizer: {name}"]
        if self.regularizer == QGGMRF:
            s += [f"    sigma: {self.sigma:g}", f"    p: {self.p:g}"]
        elif self.regularizer == SPLIT_BREGMAN:
            s += [f"    lambda: {self.lam:g}", f"    mu: {self.mu:g}"]
        return "\n".join(s)


@dataclass
class OutputParams:
    """[output] (include/config.h:260-310): file path and formats, "tiff" and/or "vti"."""
    filepath: str = "./recon.tiff"
    formats: list = field(default_factory=lambda: ["tiff", "vti"])

    @classmethod
    def from_toml(cls, config: dict) -> "OutputParams":
        o = config.get("output")
        if not isinstance(o, dict):
            raise RuntimeError("Missing [output] section in config file")
        out = cls(filepath=str(o.get("filename", "./recon.tiff")))
        if "formats" in o:
            fmts = []
            for f in o["formats"]:
                if not isinstance(f, str):
                    raise RuntimeError("[output] 'formats' array must contain strings")
                if f not in ("tiff", "vti"):
                    raise RuntimeError(f"[output] invalid format '{f}'. Must be 'tiff' or 'vti'")
                if f not in fmts:
                    fmts.append(f)
            out.formats = fmts
        return out

    def has_format(self, fmt: str) -> bool:
        return fmt in self.formats


@dataclass
class GpuParams:
    """[gpu] (this library only): operator form, device and the tuning switches."""
    operator: str = "toeplitz"
    device: int = 0
    use_graphs: bool = True
    autotune: bool = True

    @classmethod
    def from_toml(cls, config: dict) -> "GpuParams":
        g = config.get("gpu", {})
        if not isinstance(g, dict):
            raise RuntimeError("[gpu] must be a table")
        p = cls(operator=str(g.get("operator", "toeplitz")), device=int(g.get("device", 0)),
                use_graphs=bool(g.get("use_graphs", True)), autotune=bool(g.get("autotune", True)))
        if p.operator not in ("toeplitz", "toeplitz_fp16", "nufft", "mixed"):
            raise RuntimeError("[gpu] 'operator' must be 'toeplitz', 'toeplitz_fp16', 'nufft' or 'mixed'")
        return p


TEMPLATE = """[[input]]
filename = "/path/to/gamma0_stack.tiff"
angles = "/path/to/gamma0_angles.txt"
gamma = 0

[[input]]
filename = "/path/to/gamma45_stack.tiff"
angles = "/path/to/gamma45_angles.txt"
gamma = 45

[output]
filename = "output.tiff"
formats = ["tiff", "vti"]  # available: "tiff", "vti"

[recon_params]
max_iters = 50
tol = 1e-5
xtol = 1e-5
recon_dims = [51, 511, 511]

[recon_params.regularizer]
method = "split_bregman"

[recon_params.regularizer.split_bregman]
lambda = 0.1
mu = 10.0

# alternatively, for qGGMRF regularization:
# [recon_params.regularizer]
# method = "qGGMRF"
# [recon_params.regularizer.qGGMRF]
# sigma = 1000.0
# p = 1.2

# GPU backend (this library): operator = "toeplitz" | "toeplitz_fp16" | "nufft" | "mixed"
[gpu]
operator = "toeplitz"
device = 0
"""


def dump_config(path: str = "config.toml") -> None:
    """Write an example configuration (include/config.h:312-366, plus [gpu])."""
    with open(path, "w") as f:
        f.write(TEMPLATE)
