"""A small WKB writer for tests (both byte orders, ISO Z/M and EWKB flags)."""
import struct

import numpy as np


def _hdr(little, base, dims="xy", ewkb=False, srid=None):
    bo = "<" if little else ">"
    code = base
    if ewkb:
        if "z" in dims:
            code |= 0x80000000
        if "m" in dims:
            code |= 0x40000000
        if srid is not None:
            code |= 0x20000000
    else:
        code += {"xy": 0, "xyz": 1000, "xym": 2000, "xyzm": 3000}[dims]
    out = struct.pack("B", 1 if little else 0) + struct.pack(bo + "I", code)
    if ewkb and srid is not None:
        out += struct.pack(bo + "I", srid)
    return out


def _coords(little, pts, dims):
    bo = "<" if little else ">"
    extra = len(dims) - 2
    out = b""
    for x, y in pts:
        out += struct.pack(bo + "dd", float(x), float(y)) + struct.pack(bo + "d" * extra, *([7.0] * extra))
    return out


def point(x, y, little=True, dims="xy", ewkb=False, srid=None):
    return _hdr(little, 1, dims, ewkb, srid) + _coords(little, [(x, y)], dims)


def _polygon_body(rings, little, dims):
    bo = "<" if little else ">"
    out = struct.pack(bo + "I", len(rings))
    for r in rings:
        r = np.asarray(r, float)
        out += struct.pack(bo + "I", len(r)) + _coords(little, r, dims)
    return out


def polygon(rings, little=True, dims="xy", ewkb=False, srid=None):
    return _hdr(little, 3, dims, ewkb, srid) + _polygon_body(rings, little, dims)


def multipolygon(parts, little=True, dims="xy", ewkb=False, srid=None, part_little=None):
    bo = "<" if little else ">"
    out = _hdr(little, 6, dims, ewkb, srid) + struct.pack(bo + "I", len(parts))
    for k, rings in enumerate(parts):
        pl = little if part_little is None else part_little[k]
        out += _hdr(pl, 3, dims, ewkb, None) + _polygon_body(rings, pl, dims)
    return out
