"""Generate the golden fixtures under ``tests/golden/`` from the reference's test data.

Run once where a checkout of the reference project is available (read-only),
passing its root directory:

    python tests/golden/make_golden.py <path to the vibeSpatial checkout>

It reads the shapefiles the reference's vendored GeoPandas test-suite uses
(``tests/upstream/geopandas/tests/data/nybb_16a.zip`` and the
``naturalearth_lowres`` / ``naturalearth_cities`` directories) with the small
shapefile/DBF reader below, and writes compact ``.npz`` files holding the
polygon SoA (geom -> parts -> rings -> coords) plus attribute columns.  The
known answers those tests assert are recorded in ``expected.json`` with the
citing file:line.  Nothing at test time reads the reference checkout.

Ring grouping follows the shapefile convention: clockwise rings are shells,
counter-clockwise rings are holes and belong to the smallest shell whose
interior contains the hole's first vertex (decided by exact point location).
"""
from __future__ import annotations

import io
import json
import struct
import sys
import zipfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent / "oracle"))
import oracle as O  # noqa: E402


def _signed_area(xs, ys):
    return 0.5 * float(np.sum(xs[:-1] * ys[1:] - xs[1:] * ys[:-1]))


def read_shp(buf: bytes):
    """Return a list of records; each record is (shape_type, payload)."""
    file_len = struct.unpack(">i", buf[24:28])[0] * 2
    pos = 100
    out = []
    while pos < file_len:
        _, clen = struct.unpack(">2i", buf[pos:pos + 8])
        content = buf[pos + 8: pos + 8 + clen * 2]
        pos += 8 + clen * 2
        stype = struct.unpack("<i", content[:4])[0]
        if stype == 0:
            out.append((0, None))
        elif stype in (1, 11, 21):
            x, y = struct.unpack("<2d", content[4:20])
            out.append((1, (x, y)))
        elif stype in (5, 15, 25):
            nparts, npts = struct.unpack("<2i", content[36:44])
            parts = np.frombuffer(content[44:44 + 4 * nparts], dtype="<i4").astype(np.int64)
            pts = np.frombuffer(content[44 + 4 * nparts: 44 + 4 * nparts + 16 * npts], dtype="<f8").reshape(npts, 2)
            rings = []
            bounds = list(parts) + [npts]
            for a, b in zip(bounds[:-1], bounds[1:]):
                rings.append(np.array(pts[a:b], dtype=np.float64))
            out.append((5, rings))
        else:
            raise ValueError(f"unsupported shape type {stype}")
    return out


def read_dbf(buf: bytes):
    nrec, hlen, rlen = struct.unpack("<xxxxIHH", buf[:12])
    fields = []
    pos = 32
    while buf[pos] != 0x0D:
        name = buf[pos:pos + 11].split(b"\x00")[0].decode("latin1")
        ftype = chr(buf[pos + 11])
        flen = buf[pos + 16]
        fdec = buf[pos + 17]
        fields.append((name, ftype, flen, fdec))
        pos += 32
    cols = {f[0]: [] for f in fields}
    for r in range(nrec):
        rec = buf[hlen + r * rlen: hlen + (r + 1) * rlen]
        off = 1
        for name, ftype, flen, fdec in fields:
            raw = rec[off:off + flen]
            off += flen
            s = raw.decode("utf-8", errors="replace").strip()
            if ftype in "NF":
                if s == "" or set(s) <= {"*"}:
                    v = float("nan")
                elif fdec == 0 and "." not in s and "e" not in s.lower():
                    v = int(s)
                else:
                    v = float(s)
            else:
                v = s
            cols[name].append(v)
    return cols


def group_rings(rings):
    """Shapefile rings -> list of parts, each a list of rings (shell first)."""
    shells, holes = [], []
    for r in rings:
        (shells if _signed_area(r[:, 0], r[:, 1]) < 0 else holes).append(r)
    if not shells:  # counter-clockwise only: treat every ring as a shell
        shells, holes = holes, []
    parts = [[s] for s in shells]
    for h in holes:
        best, best_area = None, None
        for k, s in enumerate(shells):
            polys = O.Polygons(s[:, 0], s[:, 1], [0, len(s)], [0, 1], [0, 1])
            if O.location(h[0, 0], h[0, 1], polys, 0) != O.OUTSIDE:
                a = abs(_signed_area(s[:, 0], s[:, 1]))
                if best is None or a < best_area:
                    best, best_area = k, a
        parts[best if best is not None else 0].append(h)
    return parts


def pack(records):
    """Polygon records -> SoA arrays + geom types (Polygon/MultiPolygon)."""
    xs, ys, ring_off, part_off, geom_off, types = [], [], [0], [0], [0], []
    for stype, rings in records:
        parts = group_rings(rings) if stype == 5 and rings else []
        for part in parts:
            for r in part:
                xs.append(r[:, 0])
                ys.append(r[:, 1])
                ring_off.append(ring_off[-1] + len(r))
            part_off.append(part_off[-1] + len(part))
        geom_off.append(geom_off[-1] + len(parts))
        types.append("MultiPolygon" if len(parts) > 1 else "Polygon")
    return dict(
        x=np.concatenate(xs), y=np.concatenate(ys),
        ring_off=np.asarray(ring_off, np.int32), part_off=np.asarray(part_off, np.int32),
        geom_off=np.asarray(geom_off, np.int32), geom_type=np.asarray(types),
    )


def main(ref_root: str) -> None:
    data = Path(ref_root) / "tests/upstream/geopandas/tests/data"
    # --- NYBB boroughs (all MultiPolygon in GeoPandas) ---
    z = zipfile.ZipFile(data / "nybb_16a.zip")
    names = {Path(n).suffix: n for n in z.namelist()}
    shp = read_shp(z.read(names[".shp"]))
    dbf = read_dbf(z.read(names[".dbf"]))
    nybb = pack(shp)
    nybb["geom_type"] = np.asarray(["MultiPolygon"] * len(shp))  # GDAL promotes the layer type
    for k, v in dbf.items():
        nybb[f"attr_{k}"] = np.asarray(v)
    np.savez_compressed(HERE / "nybb.npz", **nybb)

    # --- Natural Earth countries + cities ---
    ne = data / "naturalearth_lowres"
    world = pack(read_shp((ne / "naturalearth_lowres.shp").read_bytes()))
    for k, v in read_dbf((ne / "naturalearth_lowres.dbf").read_bytes()).items():
        world[f"attr_{k}"] = np.asarray(v)
    nc = data / "naturalearth_cities"
    cities_shp = read_shp((nc / "naturalearth_cities.shp").read_bytes())
    cxy = np.asarray([p for _, p in cities_shp], dtype=np.float64)
    cities = dict(x=cxy[:, 0], y=cxy[:, 1])
    for k, v in read_dbf((nc / "naturalearth_cities.dbf").read_bytes()).items():
        cities[f"attr_{k}"] = np.asarray(v)
    np.savez_compressed(HERE / "naturalearth_lowres.npz", **world)
    np.savez_compressed(HERE / "naturalearth_cities.npz", **cities)

    expected = {
        "nybb_within_left_shape": {
            "value": [21, 8],
            "source": "tests/upstream/geopandas/tools/tests/test_sjoin.py:890-892",
        },
        "nybb_within_left_row1_boro": {
            "value": "Staten Island",
            "source": "tests/upstream/geopandas/tools/tests/test_sjoin.py:893",
        },
        "nybb_inner_intersects_shape": {
            "value": [11, 8],
            "source": "tests/upstream/geopandas/tools/tests/test_sjoin.py:885-887",
        },
        "nybb_left_intersects_shape": {
            "value": [21, 8],
            "source": "tests/upstream/geopandas/tools/tests/test_sjoin.py:866-868",
        },
        "nybb_right_intersects_shape": {
            "value": [12, 8],
            "source": "tests/upstream/geopandas/tools/tests/test_sjoin.py:874-878",
        },
        "cities_countries_inner_intersects_shape": {
            "value": [213, 4],
            "source": "tests/upstream/geopandas/tools/tests/test_sjoin.py:1039-1044",
        },
        "cities_countries_shared_first_letter_shape": {
            "value": [23, 5],
            "source": "tests/upstream/geopandas/tools/tests/test_sjoin.py:513-526",
        },
    }
    (HERE / "expected.json").write_text(json.dumps(expected, indent=2) + "\n")
    for f in ("nybb.npz", "naturalearth_lowres.npz", "naturalearth_cities.npz"):
        print(f, (HERE / f).stat().st_size)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path to the vibeSpatial checkout>")
    main(sys.argv[1])
