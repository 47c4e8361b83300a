"""The tools around the operator path: TIFF / VTI I/O, the TOML front end, the
host-side preparation helpers (pinned to the reference's compiled code), and —
on a GPU — the ``recon`` and ``forward`` command-line tools end to end."""
import ctypes
import math
import os
import struct
import subprocess
import sys

import numpy as np
import pytest

from conftest import ROOT, rel

sys.path.insert(0, ROOT)
from lamino_b200 import config as cfg  # noqa: E402
from lamino_b200 import preprocess as pp  # noqa: E402
from lamino_b200 import tiffio, vti  # noqa: E402


# ---------------------------------------------------------------------------
# TIFF
# ---------------------------------------------------------------------------

def test_tiff_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    a = rng.standard_normal((4, 7, 9)).astype(np.float32)
    for comp in ("none", "lzw"):
        fn = str(tmp_path / f"a_{comp}.tif")
        tiffio.write(fn, a, compression=comp)
        assert np.array_equal(tiffio.read(fn), a)
    # compressible data long enough to grow the LZW code width and clear the table
    b = rng.integers(0, 7, (2, 160, 250)).astype(np.float32)
    fn = str(tmp_path / "b.tif")
    tiffio.write(fn, b, compression="lzw")
    assert os.path.getsize(fn) < b.nbytes / 3
    assert np.array_equal(tiffio.read(fn, odd=False), b)


def test_tiff_odd_crop_rule(tmp_path):
    """As include/tiff.h:49-56: a row is dropped when the WIDTH is even and a column
    when the HEIGHT is even."""
    a = np.arange(2 * 6 * 9, dtype=np.float32).reshape(2, 6, 9)  # h 6 (even), w 9 (odd)
    fn = str(tmp_path / "c.tif")
    tiffio.write(fn, a)
    got = tiffio.read(fn)
    assert got.shape == (2, 6, 8) and np.array_equal(got, a[:, :6, :8])
    b = np.ones((1, 7, 10), np.float32)  # w even -> rows 6
    tiffio.write(fn, b)
    assert tiffio.read(fn).shape == (1, 6, 10)
    assert tiffio.read(fn, odd=False).shape == (1, 7, 10)


def test_tiff_big_endian_integer_samples(tmp_path):
    """A big-endian, 16-bit unsigned, two-strip page written by hand."""
    h, w = 3, 4
    pix = (np.arange(h * w).reshape(h, w) * 100).astype(">u2")
    strips = [pix[:2].tobytes(), pix[2:].tobytes()]
    ifd_off = 8 + sum(len(s) for s in strips)
    entries = [(256, 3, 1, w), (257, 3, 1, h), (258, 3, 1, 16), (259, 3, 1, 1), (262, 3, 1, 1),
               (273, 4, 2, None), (277, 3, 1, 1), (278, 3, 1, 2), (279, 4, 2, None), (339, 3, 1, 1)]
    extra_off = ifd_off + 2 + 12 * len(entries) + 4
    offs = [8, 8 + len(strips[0])]
    cnts = [len(s) for s in strips]
    extra = struct.pack(">II", *offs) + struct.pack(">II", *cnts)
    ifd = struct.pack(">H", len(entries))
    for tag, typ, cnt, val in entries:
        if tag == 273:
            ifd += struct.pack(">HHII", tag, typ, cnt, extra_off)
        elif tag == 279:
            ifd += struct.pack(">HHII", tag, typ, cnt, extra_off + 8)
        else:
            ifd += struct.pack(">HHI", tag, typ, cnt) + struct.pack(">H", val) + b"\0\0"
    ifd += struct.pack(">I", 0)
    fn = str(tmp_path / "be.tif")
    with open(fn, "wb") as f:
        f.write(b"MM" + struct.pack(">HI", 42, ifd_off) + b"".join(strips) + ifd + extra)
    got = tiffio.read(fn, odd=False)
    assert got.dtype == np.float32 and got.shape == (1, h, w)
    assert np.array_equal(got[0], pix.astype(np.float32))


def test_tiff_vectors_and_write3(tmp_path):
    rng = np.random.default_rng(1)
    v = [rng.standard_normal((3, 5, 7)).astype(np.float32) for _ in range(3)]
    fn = str(tmp_path / "v.tif")
    tiffio.write_vectors(fn, v)
    got = tiffio.read(fn, odd=False)
    assert got.shape == (3, 5, 7, 3)
    for i in range(3):
        assert np.array_equal(got[..., i], v[i])
    names = tiffio.write3(str(tmp_path / "rec.tiff"), v)
    assert [os.path.basename(n) for n in names] == ["rec0.tiff", "rec1.tiff", "rec2.tiff"]
    for i, n in enumerate(names):
        assert np.array_equal(tiffio.read(n, odd=False), v[i])


def test_tiff_rejects_non_tiff(tmp_path):
    fn = tmp_path / "x.tif"
    fn.write_bytes(b"not a tiff at all")
    with pytest.raises(ValueError):
        tiffio.read(str(fn))


# ---------------------------------------------------------------------------
# VTI
# ---------------------------------------------------------------------------

def test_vti_roundtrip(tmp_path):
    rng = np.random.default_rng(2)
    v = [rng.standard_normal((3, 4, 5)).astype(np.float32) for _ in range(3)]
    path = vti.write_vectors(str(tmp_path / "out.tiff"), v)
    assert path.endswith("out.vti")
    comps, origin = vti.read_vectors(path)
    assert origin == (-2.5, -2.0, -1.5)
    for i in range(3):
        assert np.array_equal(comps[i], v[i].astype(np.float64))
    txt = open(path, "rb").read()
    assert b'NumberOfComponents="3"' in txt and b'Vectors="magnetization"' in txt


# ---------------------------------------------------------------------------
# TOML front end
# ---------------------------------------------------------------------------

def _write(p, text):
    p.write_text(text)
    return str(p)


def test_config_recon_params(tmp_path, capsys):
    t = cfg.read_toml_file(_write(tmp_path / "c.toml", """
[recon_params]
recon_dims = [20, 255, 256]
max_iters = 7
tol = 1e-4
[recon_params.regularizer]
method = "split_bregman"
[recon_params.regularizer.split_bregman]
lambda = 0.2
mu = 5.0
inner_iters = 4
"""))
    rc = cfg.ReconConfig.from_toml(t)
    assert rc.recon_dims == (19, 255, 255) and rc.method == 2
    assert (rc.max_iters, rc.inner_iters, rc.lam, rc.mu, rc.tol, rc.xtol) == (7, 4, 0.2, 5.0, 1e-4, 1e-5)
    assert "Warning" not in capsys.readouterr().err
    t = cfg.read_toml_file(_write(tmp_path / "d.toml", """
[recon_params]
recon_dims = [41, 101, 101]
[recon_params.regularizer]
method = "qGGMRF"
[recon_params.regularizer.qGGMRF]
sigma = 500.0
"""))
    rc = cfg.ReconConfig.from_toml(t)
    assert rc.method == 3 and rc.sigma == 500.0 and rc.p == 1.2 and rc.max_iters == 50
    assert "0.41 > 0.15" in capsys.readouterr().err
    t = cfg.read_toml_file(_write(tmp_path / "e.toml", "[recon_params]\nrecon_dims = [5, 9, 9]\n"))
    assert cfg.ReconConfig.from_toml(t).method == 1  # no regularizer: MBIR1


@pytest.mark.parametrize("text,msg", [
    ("x = 1\n", "Missing [recon_params]"),
    ("[recon_params]\nrecon_dims = [5, 9]\n", "array of three integers"),
    ("[recon_params]\nrecon_dims = [5, 0, 9]\n", "recon_dims[1]"),
    ("[recon_params]\nrecon_dims = [5, 9, 9]\n[recon_params.regularizer]\nmethod = 'tv'\n", "either 'qGGMRF'"),
    ("[recon_params]\nrecon_dims = [5, 9, 9]\n[recon_params.regularizer]\nmethod = 'qGGMRF'\n",
     "Missing [recon_params.regularizer.qGGMRF]"),
])
def test_config_errors(tmp_path, text, msg):
    t = cfg.read_toml_file(_write(tmp_path / "bad.toml", text))
    with pytest.raises(RuntimeError) as e:
        cfg.ReconConfig.from_toml(t)
    assert msg in str(e.value)


def test_config_output_and_gpu(tmp_path):
    t = cfg.read_toml_file(_write(tmp_path / "o.toml", """
[output]
filename = "out/rec.tiff"
formats = ["vti", "vti", "tiff"]
[gpu]
operator = "mixed"
use_graphs = false
"""))
    o = cfg.OutputParams.from_toml(t)
    assert o.filepath == "out/rec.tiff" and o.formats == ["vti", "tiff"]
    g = cfg.GpuParams.from_toml(t)
    assert (g.operator, g.device, g.use_graphs, g.autotune) == ("mixed", 0, False, True)
    assert cfg.OutputParams.from_toml({"output": {}}).formats == ["tiff", "vti"]
    with pytest.raises(RuntimeError):
        cfg.OutputParams.from_toml({"output": {"formats": ["png"]}})
    with pytest.raises(RuntimeError):
        cfg.GpuParams.from_toml({"gpu": {"operator": "fft"}})
    with pytest.raises(RuntimeError):
        cfg.read_toml_file(_write(tmp_path / "broken.toml", "[[input\n"))
    with pytest.raises(RuntimeError):
        cfg.read_toml_file(str(tmp_path / "missing.toml"))


def test_angles_and_datasets(tmp_path):
    deg = np.array([0.0, 90.0, 180.0, 359.0])
    af = _write(tmp_path / "deg.txt", " ".join(f"{v}" for v in deg))
    a = cfg.read_angles_file(af)
    assert np.allclose(a, np.deg2rad(deg), rtol=1e-6) and a.dtype == np.float32
    rad = _write(tmp_path / "rad.txt", "0.1\n0.2\n6.0\n")
    assert np.allclose(cfg.read_angles_file(rad), [0.1, 0.2, 6.0])
    with pytest.raises(RuntimeError):
        cfg.read_angles_file(_write(tmp_path / "empty.txt", "\n"))
    proj = np.ones((4, 5, 5), np.float32)
    proj[1, 2, 3] = np.nan
    proj[2, 0, 0] = np.inf
    tiffio.write(str(tmp_path / "p.tif"), proj)
    t = {"input": [{"filename": str(tmp_path / "p.tif"), "angles": af, "gamma": 45}]}
    (p, th, g), = cfg.parse_input_datasets(t)
    assert p[1, 2, 3] == 0 and p[2, 0, 0] == 0 and np.isfinite(p).all() and p.sum() == 4 * 25 - 2
    assert g == np.float32(45 * math.pi / 180) and th.shape == (4,)
    for bad in ({"input": [{"filename": "x"}]}, {"input": [{"filename": str(tmp_path / "none.tif"),
                                                               "angles": af, "gamma": 0}]}, {}):
        with pytest.raises(RuntimeError):
            cfg.parse_input_datasets(bad)


def test_dump_config_parses(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    from lamino_b200 import recon
    assert recon.main([]) == 1  # usage; writes the example
    t = cfg.read_toml_file("config.toml")
    rc = cfg.ReconConfig.from_toml(t)
    assert rc.recon_dims == (51, 511, 511) and rc.method == 2
    assert cfg.OutputParams.from_toml(t).formats == ["tiff", "vti"]
    assert len(t["input"]) == 2


# ---------------------------------------------------------------------------
# host-side preparation vs the reference's compiled code
# ---------------------------------------------------------------------------

def _f(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def test_preprocess_vs_reference(REF):
    i64 = ctypes.c_int64
    rng = np.random.default_rng(3)
    a = rng.standard_normal((5, 6, 7)).astype(np.float32)
    # transpose: output axis i = input axis axes[i]
    for axes in [(2, 0, 1), (1, 2, 0)]:
        out = np.empty(a.size, np.float32)
        REF.ref_transpose_f.argtypes = [ctypes.POINTER(ctypes.c_float), i64, i64, i64, i64, i64, i64,
                                        ctypes.POINTER(ctypes.c_float)]
        REF.ref_transpose_f(_f(a), *a.shape, *axes, _f(out))
        assert np.array_equal(out, pp.transpose(a, axes).ravel())
    # pad3d with the forward tool's factor, crop2d back
    f = np.float32(1.41421356237 - 1)
    dims = (i64 * 3)()
    REF.ref_pad3d_f.argtypes = [ctypes.POINTER(ctypes.c_float), i64, i64, i64, ctypes.c_float,
                                ctypes.POINTER(ctypes.c_float), ctypes.POINTER(i64)]
    REF.ref_pad3d_f(_f(a), *a.shape, f, None, dims)
    want = np.empty(tuple(dims), np.float32)
    REF.ref_pad3d_f(_f(a), *a.shape, f, _f(want), dims)
    assert np.array_equal(pp.pad3d(a, f), want)
    crop = np.empty((4, 3, 5), np.float32)
    REF.ref_crop2d_f.argtypes = [ctypes.POINTER(ctypes.c_float), i64, i64, i64, i64, i64, i64,
                                 ctypes.POINTER(ctypes.c_float)]
    REF.ref_crop2d_f(_f(want), *want.shape, 4, 3, 5, _f(crop))
    assert np.array_equal(pp.crop2d(want, (4, 3, 5)), crop)
    # NaN / Inf masking
    b = a.copy()
    b[0, 0, 0], b[1, 2, 3], b[4, 5, 6] = np.nan, np.inf, -np.inf
    out = np.empty_like(b)
    REF.ref_mask_infs_nans_f.argtypes = [ctypes.POINTER(ctypes.c_float), i64, i64, i64,
                                         ctypes.POINTER(ctypes.c_float)]
    REF.ref_mask_infs_nans_f(_f(b), *b.shape, _f(out))
    assert np.array_equal(pp.mask_infs_nans(b), out)


def test_mask_support_vs_reference(REF):
    i64 = ctypes.c_int64
    rng = np.random.default_rng(4)
    projs = rng.random((5, 21, 23)).astype(np.float32) + 1
    theta = np.float32([0.0, 0.4, -1.1, 2.5, 3.0])
    REF.ref_mask_support_f.argtypes = [ctypes.POINTER(ctypes.c_float), i64, i64, i64, i64, i64, i64,
                                       ctypes.POINTER(ctypes.c_float), ctypes.c_float,
                                       ctypes.POINTER(ctypes.c_float)]
    for gamma, dims in [(0.0, (11, 9, 15)), (0.6, (17, 5, 13))]:
        want = np.empty_like(projs)
        REF.ref_mask_support_f(_f(projs), *projs.shape, *dims, _f(theta), ctypes.c_float(gamma), _f(want))
        got = pp.mask_support(projs, dims, theta, gamma)
        assert np.array_equal(got, want)
        assert 0 < (got == 0).sum() < got.size
    with pytest.raises(ValueError):
        pp.mask_support(projs, (11, 9, 15), np.float32([np.pi / 2]), 0.0)


# ---------------------------------------------------------------------------
# GPU: the command-line tools end to end
# ---------------------------------------------------------------------------

def _run(args, cwd):
    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    return subprocess.run([sys.executable, "-m"] + args, cwd=cwd, env=env, capture_output=True, text=True,
                          timeout=600)


_REGULARIZERS = {
    1: "",
    2: '[recon_params.regularizer]\nmethod = "split_bregman"\n'
       '[recon_params.regularizer.split_bregman]\ninner_iters = 2\n',
    3: '[recon_params.regularizer]\nmethod = "qGGMRF"\n[recon_params.regularizer.qGGMRF]\nsigma = 1000.0\n',
}


@pytest.mark.gpu
@pytest.mark.parametrize("method", [1, 2, 3])
def test_recon_tool_end_to_end(L, O, tmp_path, method):
    """TIFF stacks + angle files + TOML -> `python -m lamino_b200.recon` -> TIFF and
    VTI outputs equal to the direct MBIR1/2/3 call in the reference's axis order,
    and to the FP64 oracle's MBIR1/2/3 on the same datasets."""
    T, H, W = 5, 9, 11
    internal = (W, T, H)
    rng = np.random.default_rng(5)
    m = O.synthetic_magnetization(internal, seed=5, sigma=1.0).astype(np.float64)
    plan = O.NufftPlan(internal, exact=True)
    inputs = ""
    for i, gdeg in enumerate((0.0, 30.0)):
        thd = np.sort(rng.uniform(0, 360, 7))
        th = np.float32(np.deg2rad(thd))
        pg = O.PolarGrid(th, 11, 13, np.float32(np.deg2rad(gdeg)))
        proj = (O.forward(m, pg, pg.gamma, plan) + 0.05).astype(np.float32)
        tiffio.write(str(tmp_path / f"p{i}.tif"), proj)
        (tmp_path / f"a{i}.txt").write_text("\n".join(f"{v:.6f}" for v in thd))
        inputs += f'[[input]]\nfilename = "{tmp_path}/p{i}.tif"\nangles = "{tmp_path}/a{i}.txt"\ngamma = {gdeg}\n\n'
    (tmp_path / "c.toml").write_text(inputs + f"""
[output]
filename = "{tmp_path}/out/rec.tiff"
[recon_params]
recon_dims = [{T}, {H}, {W}]
max_iters = 4
""" + _REGULARIZERS[method])
    r = _run(["lamino_b200.recon", str(tmp_path / "c.toml")], tmp_path)
    assert r.returncode == 0, r.stderr
    got = np.stack([tiffio.read(str(tmp_path / "out" / f"rec{i}.tiff"), odd=False) for i in range(3)])
    assert got.shape == (3, T, H, W)
    vt, _ = vti.read_vectors(str(tmp_path / "out" / "rec.vti"))
    assert np.array_equal(np.stack(vt).astype(np.float32), got)
    ds = cfg.parse_input_datasets(cfg.read_toml_file(str(tmp_path / "c.toml")))
    fn = {1: L.MBIR1, 2: L.MBIR2, 3: L.MBIR3}[method]
    want = fn(ds, internal, L.ReconParams(maxIters=4, innerIters=2 if method == 2 else 3))
    want = np.stack([np.transpose(want[i], (1, 2, 0)) for i in range(3)])
    assert rel(got, want) < 1e-5
    # and the FP64 oracle (pinned to the reference's own MBIR drivers) on the
    # datasets the tool read: the reconstruction within 1e-4
    ofn = {1: O.MBIR1, 2: O.MBIR2, 3: O.MBIR3}[method]
    oracle = ofn(ds, internal, O.ReconParams(maxIters=4, innerIters=2 if method == 2 else 3), eps=1e-12)
    oracle = np.stack([np.transpose(oracle[i], (1, 2, 0)) for i in range(3)])
    assert rel(got, oracle) < 1e-4


@pytest.mark.gpu
def test_forward_tool_end_to_end(L, O, tmp_path):
    """`python -m lamino_b200.forward_tool` against the oracle running the same steps
    (permute, pad by sqrt(2) - 1, project on the padded detector, crop)."""
    T, H, W = 5, 9, 11
    rng = np.random.default_rng(6)
    comps = [rng.standard_normal((T, H, W)).astype(np.float32) for _ in range(3)]
    for i, c in enumerate(comps):
        tiffio.write(str(tmp_path / f"m{i}.tif"), c)
    thd = np.sort(rng.uniform(0, 360, 6))
    (tmp_path / "ang.txt").write_text(" ".join(f"{v:.5f}" for v in thd))
    (tmp_path / "f.toml").write_text(f"""
[input]
data_path = "{tmp_path}"
component_1 = "m0.tif"
component_2 = "m1.tif"
component_3 = "m2.tif"
[angles]
filename = "{tmp_path}/ang.txt"
[orientation]
gamma = 20
[output]
filename = "proj.tif"
basedir = "{tmp_path}/out"
dims = [13, 15]
""")
    r = _run(["lamino_b200.forward_tool", str(tmp_path / "f.toml")], tmp_path)
    assert r.returncode == 0, r.stderr
    got = tiffio.read(str(tmp_path / "out" / "proj.tif"), odd=False)
    assert got.shape == (6, 13, 15)
    f = np.float32(1.41421356237 - 1)
    vol = np.stack([O.pad3d(np.transpose(c, (2, 0, 1)), f) for c in comps]).astype(np.float64)
    th = cfg.read_angles_file(str(tmp_path / "ang.txt"))
    nr, nc = 13 + 2 * int(13 * (1.41421356237 - 1) / 2), 15 + 2 * int(15 * (1.41421356237 - 1) / 2)
    pg = O.PolarGrid(th, nr, nc, np.float32(20 * math.pi / 180))
    want = O.crop2d(O.forward(vol, pg, pg.gamma, O.NufftPlan(vol.shape[1:], exact=True)), (6, 13, 15))
    assert rel(got, want) < 1e-5
