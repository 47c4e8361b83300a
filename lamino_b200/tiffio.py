"""Multi-page TIFF stacks without libtiff: the reader and writers the reference
uses for projection stacks and reconstructions (include/tiff.h:31-189).

* ``read(filename)`` returns a float32 array (pages, rows, cols).  Like the
  reference it keeps an odd number of rows and columns (include/tiff.h:49-56:
  one row is dropped when the image WIDTH is even and one column when the
  HEIGHT is even — the reference checks the other dimension in each case, and
  this reader does the same so both read the same pixels).  ``odd=False``
  returns every pixel.  Strips may be uncompressed or LZW-compressed (no
  predictor); samples may be IEEE float (32/64 bit) or integers of 8-32 bits,
  either byte order.
* ``write(filename, arr)`` writes a float32 stack, one uncompressed strip per
  page (include/tiff.h:71-103).
* ``write3(name, vol3)`` writes the three components of a vector volume to
  ``<base>0.tiff``, ``<base>1.tiff``, ``<base>2.tiff`` (include/tiff.h:168-182).
* ``write_vectors(filename, vol3)`` writes one stack with 3 float32 samples per
  pixel (x, y, z components), RGB photometric, as include/tiff.h:105-161; the
  reference LZW-compresses it, this writer stores it uncompressed unless
  ``compression="lzw"`` is asked for (the pure-Python encoder is slow on large
  volumes).
"""
from __future__ import annotations

import struct

import numpy as np

__all__ = ["read", "write", "write3", "write_vectors"]

_TYPE_SIZE = {1: 1, 2: 1, 3: 2, 4: 4, 5: 8, 6: 1, 7: 1, 8: 2, 9: 4, 10: 8, 11: 4, 12: 8, 16: 8}
_TYPE_FMT = {1: "B", 3: "H", 4: "I", 6: "b", 8: "h", 9: "i", 11: "f", 12: "d", 16: "Q"}

TAG_WIDTH, TAG_LENGTH, TAG_BITS, TAG_COMPRESSION, TAG_PHOTOMETRIC = 256, 257, 258, 259, 262
TAG_DESCRIPTION, TAG_STRIP_OFFSETS, TAG_ORIENTATION, TAG_SPP = 270, 273, 274, 277
TAG_ROWS_PER_STRIP, TAG_STRIP_BYTES, TAG_PLANAR, TAG_PREDICTOR, TAG_SAMPLE_FORMAT = 278, 279, 284, 317, 339


# ---------------------------------------------------------------------------
# LZW (TIFF 6.0 section 13: MSB-first codes of 9-12 bits, Clear 256, EOI 257,
# the code width grows one code early)
# ---------------------------------------------------------------------------

def _lzw_decode(data: bytes) -> bytes:
    out = bytearray()
    table = [bytes([i]) for i in range(256)] + [b"", b""]
    width, pos, nbits = 9, 0, len(data) * 8
    prev = None
    while pos + width <= nbits:
        byte, bit = divmod(pos, 8)
        chunk = int.from_bytes(data[byte:byte + 3].ljust(3, b"\0"), "big")
        code = (chunk >> (24 - bit - width)) & ((1 << width) - 1)
        pos += width
        if code == 256:
            table = table[:258]
            width, prev = 9, None
            continue
        if code == 257:
            break
        if prev is None:
            entry = table[code]
        elif code < len(table):
            entry = table[code]
            table.append(prev + entry[:1])
        elif code == len(table):
            entry = prev + prev[:1]
            table.append(entry)
        else:
            raise ValueError("corrupt LZW stream")
        out += entry
        prev = entry
        if len(table) + 1 >= (1 << width) and width < 12:
            width += 1
    return bytes(out)


def _lzw_encode(data: bytes) -> bytes:
    codes = [(256, 9)]
    table = {bytes([i]): i for i in range(256)}
    next_code, width = 258, 9
    w = b""
    for c in data:
        wc = w + bytes([c])
        if wc in table:
            w = wc
            continue
        codes.append((table[w], width))
        table[wc] = next_code
        next_code += 1
        if next_code == 4094:  # table full: clear (at the current width) and start over
            codes.append((256, width))
            table = {bytes([i]): i for i in range(256)}
            next_code, width = 258, 9
        elif next_code >= (1 << width):
            width += 1
        w = bytes([c])
    if w:
        codes.append((table[w], width))
        if next_code + 1 >= (1 << width) and width < 12:  # the decoder's entry for this last code
            width += 1
    codes.append((257, width))
    acc, nacc, out = 0, 0, bytearray()
    for code, wd in codes:
        acc = (acc << wd) | code
        nacc += wd
        while nacc >= 8:
            nacc -= 8
            out.append((acc >> nacc) & 0xFF)
        acc &= (1 << nacc) - 1
    if nacc:
        out.append((acc << (8 - nacc)) & 0xFF)
    return bytes(out)


# ---------------------------------------------------------------------------
# reader
# ---------------------------------------------------------------------------

def _ifds(buf: bytes):
    if buf[:2] == b"II":
        bo = "<"
    elif buf[:2] == b"MM":
        bo = ">"
    else:
        raise ValueError("not a TIFF file")
    magic, off = struct.unpack(bo + "HI", buf[2:8])
    if magic != 42:
        raise ValueError("unsupported TIFF variant (BigTIFF or corrupt header)")
    seen = set()
    while off:
        if off in seen or off + 2 > len(buf):
            raise ValueError("corrupt IFD chain")
        seen.add(off)
        (n,) = struct.unpack(bo + "H", buf[off:off + 2])
        tags = {}
        for e in range(n):
            p = off + 2 + 12 * e
            tag, typ, cnt = struct.unpack(bo + "HHI", buf[p:p + 8])
            size = _TYPE_SIZE.get(typ, 1) * cnt
            vp = p + 8 if size <= 4 else struct.unpack(bo + "I", buf[p + 8:p + 12])[0]
            raw = buf[vp:vp + size]
            if typ == 2:
                tags[tag] = raw.rstrip(b"\0").decode("latin-1")
            elif typ in (5, 10):
                v = struct.unpack(bo + ("I" if typ == 5 else "i") * (2 * cnt), raw)
                tags[tag] = [v[2 * i] / v[2 * i + 1] for i in range(cnt)]
            elif typ in _TYPE_FMT:
                tags[tag] = list(struct.unpack(bo + _TYPE_FMT[typ] * cnt, raw))
            else:
                tags[tag] = raw
        yield bo, tags
        (off,) = struct.unpack(bo + "I", buf[off + 2 + 12 * n:off + 6 + 12 * n])


def _page(buf: bytes, bo: str, t: dict) -> np.ndarray:
    w, h = t[TAG_WIDTH][0], t[TAG_LENGTH][0]
    spp = t.get(TAG_SPP, [1])[0]
    bits = t.get(TAG_BITS, [1])[0]
    fmt = t.get(TAG_SAMPLE_FORMAT, [1])[0]
    comp = t.get(TAG_COMPRESSION, [1])[0]
    if t.get(TAG_PLANAR, [1])[0] != 1:
        raise ValueError("planar-separate TIFF pages are not supported")
    if t.get(TAG_PREDICTOR, [1])[0] != 1:
        raise ValueError("TIFF predictors are not supported")
    if TAG_STRIP_OFFSETS not in t:
        raise ValueError("tiled TIFF pages are not supported")
    kind = {1: "u", 2: "i", 3: "f"}.get(fmt)
    if kind is None or bits not in (8, 16, 32, 64) or (kind == "f" and bits < 32):
        raise ValueError(f"unsupported TIFF samples: format {fmt}, {bits} bits")
    dt = np.dtype(f"{bo}{kind}{bits // 8}")
    parts = []
    for o, c in zip(t[TAG_STRIP_OFFSETS], t[TAG_STRIP_BYTES]):
        s = buf[o:o + c]
        if comp == 5:
            s = _lzw_decode(s)
        elif comp != 1:
            raise ValueError(f"unsupported TIFF compression {comp}")
        parts.append(s)
    raw = b"".join(parts)
    need = w * h * spp * dt.itemsize
    if len(raw) < need:
        raise ValueError("TIFF strips shorter than the image")
    a = np.frombuffer(raw[:need], dtype=dt).reshape(h, w, spp) if spp > 1 else \
        np.frombuffer(raw[:need], dtype=dt).reshape(h, w)
    return a.astype(np.float32)


def read(filename: str, odd: bool = True) -> np.ndarray:
    """All pages of a TIFF stack as float32 (pages, rows, cols[, samples])."""
    with open(filename, "rb") as f:
        buf = f.read()
    pages = [_page(buf, bo, t) for bo, t in _ifds(buf)]
    if not pages:
        raise ValueError(f"no images in {filename}")
    if any(p.shape != pages[0].shape for p in pages):
        raise ValueError("TIFF pages differ in size")
    data = np.stack(pages)
    if odd:
        h, w = data.shape[1], data.shape[2]
        nrows = h - 1 if w % 2 == 0 else h
        ncols = w - 1 if h % 2 == 0 else w
        data = np.ascontiguousarray(data[:, :nrows, :ncols])
    return data


# ---------------------------------------------------------------------------
# writers (little-endian, one strip per page)
# ---------------------------------------------------------------------------

def _write_pages(filename: str, pages, spp: int, photometric: int, description: str | None,
                 compression: str):
    comp = {"none": 1, "lzw": 5}[compression]
    out = bytearray(b"II" + struct.pack("<HI", 42, 0))
    next_ptr = 4  # where the offset of the next IFD goes
    for page in pages:
        page = np.ascontiguousarray(page, dtype="<f4")
        h, w = page.shape[0], page.shape[1]
        data = page.tobytes()
        if comp == 5:
            data = _lzw_encode(data)
        if len(out) % 2:
            out.append(0)
        strip_off = len(out)
        out += data
        entries = [  # (tag, type, values or bytes), in ascending tag order
            (TAG_WIDTH, 4, [w]), (TAG_LENGTH, 4, [h]), (TAG_BITS, 3, [32] * spp),
            (TAG_COMPRESSION, 3, [comp]), (TAG_PHOTOMETRIC, 3, [photometric])]
        if description:
            entries.append((TAG_DESCRIPTION, 2, description.encode("latin-1") + b"\0"))
        entries += [(TAG_STRIP_OFFSETS, 4, [strip_off]), (TAG_ORIENTATION, 3, [1]), (TAG_SPP, 3, [spp]),
                    (TAG_ROWS_PER_STRIP, 4, [h]), (TAG_STRIP_BYTES, 4, [len(data)]), (TAG_PLANAR, 3, [1]),
                    (TAG_SAMPLE_FORMAT, 3, [3] * spp)]
        if len(out) % 2:
            out.append(0)
        ifd_off = len(out)
        extra_base = ifd_off + 2 + 12 * len(entries) + 4
        ifd, extra = bytearray(struct.pack("<H", len(entries))), bytearray()
        for tag, typ, vals in entries:
            if isinstance(vals, (bytes, bytearray)):
                payload, cnt = bytes(vals), len(vals)
            else:
                payload, cnt = struct.pack("<" + _TYPE_FMT[typ] * len(vals), *vals), len(vals)
            if len(payload) <= 4:
                ifd += struct.pack("<HHI", tag, typ, cnt) + payload.ljust(4, b"\0")
            else:
                if len(extra) % 2:
                    extra.append(0)
                ifd += struct.pack("<HHII", tag, typ, cnt, extra_base + len(extra))
                extra += payload
        ifd += struct.pack("<I", 0)
        out += ifd + extra
        struct.pack_into("<I", out, next_ptr, ifd_off)
        next_ptr = ifd_off + 2 + 12 * len(entries)
    with open(filename, "wb") as f:
        f.write(out)


def write(filename: str, arr, compression: str = "none") -> None:
    """A float32 stack (pages, rows, cols), minimum-is-black, one strip per page."""
    a = np.asarray(arr, dtype=np.float32)
    if a.ndim == 2:
        a = a[None]
    if a.ndim != 3:
        raise ValueError("expected a (pages, rows, cols) array")
    _write_pages(filename, list(a), 1, 1, None, compression)


def write3(name: str, vol3) -> list:
    """The 3 components of a vector volume as <base>0.tiff, <base>1.tiff, <base>2.tiff
    (a trailing .tif / .tiff of `name` is dropped); returns the file names."""
    base = name[:name.rfind(".tif")] if ".tif" in name else name
    names = []
    for i in range(3):
        fn = f"{base}{i}.tiff"
        write(fn, vol3[i])
        names.append(fn)
    return names


def write_vectors(filename: str, vol3, compression: str = "none") -> None:
    """One stack with the x, y, z components as 3 float32 samples per pixel."""
    v = np.stack([np.asarray(vol3[i], dtype=np.float32) for i in range(3)], axis=-1)
    _write_pages(filename, list(v), 3, 2, "3D vector field: x,y,z components; layout: [slice, row, col]",
                 compression)

