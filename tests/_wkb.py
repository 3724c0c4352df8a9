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


def _rings(rng, max_rings=3, max_pts=12):
    out = []
    for _ in range(int(rng.integers(0, max_rings + 1))):
        m = int(rng.integers(0, max_pts + 1))
        out.append(rng.uniform(-1e3, 1e3, size=(m, 2)))
    return out


def fuzz_values(rng, n):
    """WKB values of every encoding the decoders accept, plus nulls, other
    geometry types, truncations, corrupted bytes and junk (seeded)."""
    vals = []
    for _ in range(n):
        k = int(rng.integers(0, 12))
        little = bool(rng.integers(0, 2))
        dims = ["xy", "xyz", "xym", "xyzm"][int(rng.integers(0, 4))]
        ewkb = bool(rng.integers(0, 2))
        srid = 4326 if ewkb and rng.integers(0, 2) else None
        kw = dict(little=little, dims=dims, ewkb=ewkb, srid=srid)
        if k == 0:
            vals.append(None)
        elif k <= 2:
            vals.append(point(*rng.uniform(-1e3, 1e3, 2), **kw))
        elif k <= 4:
            vals.append(polygon(_rings(rng), **kw))
        elif k <= 6:
            parts = [_rings(rng) for _ in range(int(rng.integers(0, 4)))]
            vals.append(multipolygon(parts, part_little=[bool(rng.integers(0, 2)) for _ in parts], **kw))
        elif k == 7:  # another geometry type, with a body of random bytes
            base = [0, 2, 4, 5, 7, 15, 17][int(rng.integers(0, 7))]
            vals.append(_hdr(little, base, dims, ewkb, srid) + rng.bytes(int(rng.integers(0, 40))))
        elif k == 8:  # a valid value cut short
            v = polygon(_rings(rng, 2, 6), **kw) if rng.integers(0, 2) else point(1.0, 2.0, **kw)
            vals.append(v[:int(rng.integers(1, len(v)))])
        elif k == 9:  # a valid value with one byte changed
            v = bytearray(multipolygon([_rings(rng, 2, 6)], **kw) if rng.integers(0, 2) else polygon(_rings(rng, 2, 6), **kw))
            v[int(rng.integers(0, min(len(v), 24)))] = int(rng.integers(0, 256))
            vals.append(bytes(v))
        elif k == 10:  # junk
            vals.append(rng.bytes(int(rng.integers(0, 48))))
        else:  # zero-length value
            vals.append(b"")
    return vals


def arrow_layout(vals):
    """(bytes uint8, int64 offsets, validity uint8) of a list of bytes/None."""
    lens = np.array([0 if v is None else len(v) for v in vals], dtype=np.int64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    data = np.frombuffer(b"".join(v for v in vals if v is not None), dtype=np.uint8).copy()
    valid = np.array([v is not None for v in vals], dtype=np.uint8)
    return data, off, valid
