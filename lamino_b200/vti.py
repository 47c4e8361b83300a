"""VTK ImageData (.vti) output of a vector volume (include/write_vti.h:37-113):
the x, y, z components as one Float64 3-vector point field, raw appended
binary with a 32-bit byte count, origin at the volume centre, unit spacing."""
from __future__ import annotations

import os
import struct

import numpy as np

__all__ = ["write_vectors", "read_vectors"]


def write_vectors(filename: str, vol3, field_name: str = "magnetization") -> str:
    """Write vol3 = 3 arrays (nz, ny, nx) to <filename with extension .vti>;
    returns the path written."""
    comps = [np.asarray(vol3[i], dtype=np.float64) for i in range(3)]
    if any(c.shape != comps[0].shape or c.ndim != 3 for c in comps):
        raise ValueError("expected three (nz, ny, nx) arrays of one shape")
    nz, ny, nx = comps[0].shape
    data = np.stack([c.ravel() for c in comps], axis=1)  # (npoints, 3), x fastest
    nbytes = data.nbytes
    if nbytes >= 1 << 32:
        raise ValueError("volume too large for a 32-bit appended-data header")
    path = os.path.splitext(filename)[0] + ".vti"
    ox, oy, oz = -0.5 * nx, -0.5 * ny, -0.5 * nz
    head = (
        '<?xml version="1.0"?>\n'
        '<VTKFile type="ImageData" version="0.1" byte_order="LittleEndian">\n'
        f'  <ImageData WholeExtent="0 {nx - 1} 0 {ny - 1} 0 {nz - 1}" '
        f'Origin="{_num(ox)} {_num(oy)} {_num(oz)}" Spacing="1 1 1">\n'
        f'    <Piece Extent="0 {nx - 1} 0 {ny - 1} 0 {nz - 1}">\n'
        f'      <PointData Vectors="{field_name}">\n'
        f'        <DataArray type="Float64" Name="{field_name}" NumberOfComponents="3" '
        'format="appended" offset="0"/>\n'
        '      </PointData>\n'
        '      <CellData></CellData>\n'
        '    </Piece>\n'
        '  </ImageData>\n'
        '  <AppendedData encoding="raw">\n'
        '   _'
    )
    with open(path, "wb") as f:
        f.write(head.encode("ascii"))
        f.write(struct.pack("<I", nbytes))
        f.write(np.ascontiguousarray(data, dtype="<f8").tobytes())
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")
    return path


def _num(v: float) -> str:
    """Shortest text of a float (as the reference's std::format prints it)."""
    return repr(float(v)) if v != int(v) else str(int(v))


def read_vectors(path: str):
    """Read a file written by write_vectors back: (3 arrays (nz, ny, nx), origin)."""
    with open(path, "rb") as f:
        buf = f.read()
    start = buf.index(b"WholeExtent=\"") + len("WholeExtent=\"")
    ext = [int(v) for v in buf[start:buf.index(b"\"", start)].split()]
    nx, ny, nz = ext[1] + 1, ext[3] + 1, ext[5] + 1
    o0 = buf.index(b"Origin=\"") + len("Origin=\"")
    origin = tuple(float(v) for v in buf[o0:buf.index(b"\"", o0)].split())
    p = buf.index(b"<AppendedData encoding=\"raw\">")
    p = buf.index(b"_", p) + 1
    (nbytes,) = struct.unpack("<I", buf[p:p + 4])
    data = np.frombuffer(buf[p + 4:p + 4 + nbytes], dtype="<f8").reshape(-1, 3)
    return [data[:, i].reshape(nz, ny, nx) for i in range(3)], origin
