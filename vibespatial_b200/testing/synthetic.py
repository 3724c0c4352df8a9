"""Seeded synthetic workloads for the point-by-polygon join.

Each generator returns plain numpy arrays: query points ``px, py`` (float64)
and a polygon SoA (``x, y, ring_off, part_off, geom_off``; a Polygon is a
one-part MultiPolygon).  All randomness comes from
``numpy.random.default_rng(seed)``.  The reference keeps its generators in
src/vibespatial/testing/synthetic.py (star polygons ``_star_polygon`` :241);
these follow the five workload definitions this project is measured on:

* ``star_join``       100k points uniform in [0,1000]^2 x 1k star polygons
                      (radius lognormal(ln 10, 0.5), 8-64 vertices at sorted
                      uniform angles, radial jitter U(0.6, 1.0))
* ``utm_join``        10M points from a 64-component Gaussian mixture
                      (sigma = 2 % of the extent) in a 100 km frame offset by
                      (5e5, 3e6) m x 100k building footprints (rotated
                      rectangle / L / T / U / cross, 4-12 vertices, sides
                      lognormal with median 15 m and sigma 0.5)
* ``batched_jobs``    256 star joins with per-job seeds, points log-uniform in
                      [1k, 2M], polygons log-uniform in [10, 50k]
* ``zipf_join``       50M points x 1M footprints, cluster centres
                      Zipf(s=1.1)-weighted over 1024 sites in [0,1000]^2,
                      footprints scaled to the frame (median side 0.15)
* ``degenerate_join`` 20M points x 200k polygons with 1-5 holes and 2-4 part
                      multipolygons on an integer lattice; 10 % of points on
                      vertices, 10 % on edges (dyadic t), 10 % one ulp off an
                      edge point, the rest uniform
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class PolygonSoA:
    x: np.ndarray
    y: np.ndarray
    ring_off: np.ndarray
    part_off: np.ndarray
    geom_off: np.ndarray
    valid: np.ndarray | None = None

    def __len__(self) -> int:
        return len(self.geom_off) - 1

    @property
    def n_coords(self) -> int:
        return len(self.x)

    def nbytes(self) -> int:
        return int(self.x.nbytes + self.y.nbytes + self.ring_off.nbytes + self.part_off.nbytes + self.geom_off.nbytes)


@dataclass
class Workload:
    name: str
    px: np.ndarray
    py: np.ndarray
    polys: PolygonSoA
    meta: dict = field(default_factory=dict)

    @property
    def n_points(self) -> int:
        return len(self.px)


def _rings_to_soa(ring_sizes: np.ndarray, xs: np.ndarray, ys: np.ndarray, rings_per_part=None, parts_per_geom=None):
    """Closed rings given as flat coordinate arrays -> SoA offsets."""
    nr = len(ring_sizes)
    ring_off = np.zeros(nr + 1, dtype=np.int64)
    np.cumsum(ring_sizes, out=ring_off[1:])
    if rings_per_part is None:
        rings_per_part = np.ones(nr, dtype=np.int64)
    part_off = np.zeros(len(rings_per_part) + 1, dtype=np.int64)
    np.cumsum(rings_per_part, out=part_off[1:])
    if parts_per_geom is None:
        parts_per_geom = np.ones(len(rings_per_part), dtype=np.int64)
    geom_off = np.zeros(len(parts_per_geom) + 1, dtype=np.int64)
    np.cumsum(parts_per_geom, out=geom_off[1:])
    if ring_off[-1] >= 2**31:
        raise ValueError("too many coordinates for int32 offsets")
    return PolygonSoA(xs.astype(np.float64), ys.astype(np.float64), ring_off.astype(np.int32),
                      part_off.astype(np.int32), geom_off.astype(np.int32))


def star_polygons(rng, n: int, lo: float = 0.0, hi: float = 1000.0, median_r: float = 10.0,
                  sigma: float = 0.5, vmin: int = 8, vmax: int = 64) -> PolygonSoA:
    """Star-shaped simple polygons (closed rings, counter-clockwise)."""
    cx = rng.uniform(lo, hi, n)
    cy = rng.uniform(lo, hi, n)
    r = rng.lognormal(np.log(median_r), sigma, n)
    nv = rng.integers(vmin, vmax + 1, n)
    tot = int(nv.sum())
    owner = np.repeat(np.arange(n), nv)
    ang = rng.uniform(0.0, 2 * np.pi, tot)
    # sort angles within each polygon
    order = np.lexsort((ang, owner))
    ang = ang[order]
    jit = rng.uniform(0.6, 1.0, tot)
    vx = cx[owner] + r[owner] * jit * np.cos(ang)
    vy = cy[owner] + r[owner] * jit * np.sin(ang)
    # close each ring: append its first vertex
    starts = np.zeros(n, dtype=np.int64)
    np.cumsum(nv[:-1], out=starts[1:])
    ring_sizes = nv + 1
    out_x = np.empty(tot + n)
    out_y = np.empty(tot + n)
    dst_start = starts + np.arange(n)
    idx = np.arange(tot) + owner  # shift by number of closers before this ring
    out_x[idx] = vx
    out_y[idx] = vy
    close_at = dst_start + nv
    out_x[close_at] = vx[starts]
    out_y[close_at] = vy[starts]
    return _rings_to_soa(ring_sizes, out_x, out_y)


def uniform_points(rng, n: int, lo: float = 0.0, hi: float = 1000.0):
    return rng.uniform(lo, hi, n), rng.uniform(lo, hi, n)


def star_join(seed: int = 0, n_points: int = 100_000, n_polys: int = 1_000) -> Workload:
    rng = np.random.default_rng(seed)
    px, py = uniform_points(rng, n_points)
    polys = star_polygons(rng, n_polys)
    return Workload("star_join", px, py, polys, {"seed": seed, "n_points": n_points, "n_polys": n_polys})


# Footprint templates in unit-side local coordinates (counter-clockwise, not closed).
_TEMPLATES = [
    np.array([[0, 0], [1, 0], [1, 1], [0, 1]], float),                                     # rectangle, 4
    np.array([[0, 0], [1, 0], [1, .4], [.4, .4], [.4, 1], [0, 1]], float),                 # L, 6
    np.array([[0, 0], [1, 0], [1, .35], [.65, .35], [.65, 1], [.35, 1], [.35, .35], [0, .35]], float)[::1],  # T-ish, 8
    np.array([[0, 0], [1, 0], [1, 1], [.7, 1], [.7, .35], [.3, .35], [.3, 1], [0, 1]], float),  # U, 8
    np.array([[.35, 0], [.65, 0], [.65, .35], [1, .35], [1, .65], [.65, .65], [.65, 1], [.35, 1],
              [.35, .65], [0, .65], [0, .35], [.35, .35]], float),                            # cross, 12
]


def _signed_area(t):
    x, y = t[:, 0], t[:, 1]
    return 0.5 * np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y)


def footprints(rng, cx: np.ndarray, cy: np.ndarray, median_side: float, sigma: float = 0.5) -> PolygonSoA:
    """Rotated building footprints centred at (cx, cy)."""
    n = len(cx)
    kind = rng.choice(len(_TEMPLATES), size=n, p=[0.4, 0.25, 0.12, 0.12, 0.11])
    w = rng.lognormal(np.log(median_side), sigma, n)
    h = rng.lognormal(np.log(median_side), sigma, n)
    th = rng.uniform(0, np.pi, n)
    nv = np.array([len(t) for t in _TEMPLATES])[kind]
    order = np.argsort(kind, kind="stable")
    # build per template, then scatter back to row order
    xs = np.empty(int(nv.sum()) + n)
    ys = np.empty_like(xs)
    ring_sizes = nv + 1
    starts = np.zeros(n, dtype=np.int64)
    np.cumsum(ring_sizes[:-1], out=starts[1:])
    c, s = np.cos(th), np.sin(th)
    for k, t in enumerate(_TEMPLATES):
        assert _signed_area(t) > 0
        rows = order[kind[order] == k]
        if len(rows) == 0:
            continue
        lx = (t[None, :, 0] - 0.5) * w[rows, None]
        ly = (t[None, :, 1] - 0.5) * h[rows, None]
        gx = cx[rows, None] + lx * c[rows, None] - ly * s[rows, None]
        gy = cy[rows, None] + lx * s[rows, None] + ly * c[rows, None]
        gx = np.concatenate([gx, gx[:, :1]], axis=1)
        gy = np.concatenate([gy, gy[:, :1]], axis=1)
        dst = starts[rows, None] + np.arange(len(t) + 1)[None, :]
        xs[dst] = gx
        ys[dst] = gy
    return _rings_to_soa(ring_sizes, xs, ys)


def _gmm(rng, n, centers, weights, sigma, lo, hi):
    comp = rng.choice(len(centers), size=n, p=weights)
    x = centers[comp, 0] + rng.normal(0, sigma, n)
    y = centers[comp, 1] + rng.normal(0, sigma, n)
    np.clip(x, lo[0], hi[0], out=x)
    np.clip(y, lo[1], hi[1], out=y)
    return x, y


def utm_join(seed: int = 1, n_points: int = 10_000_000, n_polys: int = 100_000) -> Workload:
    rng = np.random.default_rng(seed)
    ox, oy, ext = 5.0e5, 3.0e6, 1.0e5
    lo, hi = (ox, oy), (ox + ext, oy + ext)
    centers = np.stack([rng.uniform(ox, ox + ext, 64), rng.uniform(oy, oy + ext, 64)], axis=1)
    weights = np.full(64, 1 / 64)
    sigma = 0.02 * ext
    px, py = _gmm(rng, n_points, centers, weights, sigma, lo, hi)
    fx, fy = _gmm(rng, n_polys, centers, weights, sigma, lo, hi)
    polys = footprints(rng, fx, fy, 15.0, 0.5)
    return Workload("utm_join", px, py, polys,
                    {"seed": seed, "n_points": n_points, "n_polys": n_polys, "frame": [ox, oy, ox + ext, oy + ext],
                     "gmm_components": 64, "sigma_m": sigma, "side_median_m": 15.0, "side_sigma": 0.5})


def zipf_join(seed: int = 3, n_points: int = 50_000_000, n_polys: int = 1_000_000, sites: int = 1024,
              s: float = 1.1) -> Workload:
    rng = np.random.default_rng(seed)
    ext = 1000.0
    centers = np.stack([rng.uniform(0, ext, sites), rng.uniform(0, ext, sites)], axis=1)
    w = 1.0 / np.arange(1, sites + 1) ** s
    w /= w.sum()
    sigma = 0.02 * ext
    px, py = _gmm(rng, n_points, centers, w, sigma, (0, 0), (ext, ext))
    fx, fy = _gmm(rng, n_polys, centers, w, sigma, (0, 0), (ext, ext))
    polys = footprints(rng, fx, fy, 15.0 * ext / 1.0e5, 0.5)
    return Workload("zipf_join", px, py, polys,
                    {"seed": seed, "n_points": n_points, "n_polys": n_polys, "sites": sites, "zipf_s": s,
                     "sigma": sigma, "side_median": 15.0 * ext / 1.0e5})


def batched_jobs(seed: int = 2, n_jobs: int = 256, pts_range=(1_000, 2_000_000), poly_range=(10, 50_000)):
    """List of independent star joins with per-job seeds (log-uniform sizes)."""
    rng = np.random.default_rng(seed)
    npts = np.exp(rng.uniform(np.log(pts_range[0]), np.log(pts_range[1]), n_jobs)).astype(np.int64)
    npol = np.exp(rng.uniform(np.log(poly_range[0]), np.log(poly_range[1]), n_jobs)).astype(np.int64)
    return [star_join(seed=seed * 100_003 + j + 1, n_points=int(npts[j]), n_polys=int(npol[j])) for j in range(n_jobs)]


def _lattice_star(rng, cx, cy, r, nv):
    """Integer-lattice star ring (closed, counter-clockwise, simple)."""
    # keep a minimum angular gap so rounding cannot fold the ring
    ang = (np.arange(nv) + rng.uniform(0.1, 0.9, nv)) * (2 * np.pi / nv)
    jit = rng.uniform(0.75, 1.0, nv)
    x = np.round(cx + r * jit * np.cos(ang))
    y = np.round(cy + r * jit * np.sin(ang))
    keep = np.ones(nv, bool)
    keep[1:] = (x[1:] != x[:-1]) | (y[1:] != y[:-1])
    x, y = x[keep], y[keep]
    return np.append(x, x[0]), np.append(y, y[0])


def degenerate_join(seed: int = 5, n_points: int = 20_000_000, n_polys: int = 200_000,
                    extent: float = 16384.0) -> Workload:
    """Holes, multipolygons and points exactly on / one ulp off the boundary."""
    rng = np.random.default_rng(seed)
    ring_sizes, xs, ys, rings_per_part, parts_per_geom = [], [], [], [], []
    edges_a, edges_b, verts = [], [], []
    multi = rng.random(n_polys) < 0.3
    for g in range(n_polys):
        nparts = int(rng.integers(2, 5)) if multi[g] else 1
        base_x = rng.uniform(64, extent - 192)
        base_y = rng.uniform(64, extent - 192)
        r = float(rng.integers(24, 48))
        for k in range(nparts):
            # parts spaced 2.5 r apart along x: disjoint
            cx = np.round(base_x + k * 2.5 * r)
            cy = np.round(base_y)
            ox, oy = _lattice_star(rng, cx, cy, r, int(rng.integers(8, 17)))
            rings = [(ox, oy)]
            nh = int(rng.integers(1, 6)) if not multi[g] or k == 0 else 0
            # holes: small lattice squares on a 3x3 grid strictly inside the 0.5 r disk
            slots = rng.permutation(9)[:nh]
            hs = max(2.0, np.floor(r * 0.12))
            for sl in slots:
                hx = cx + (sl % 3 - 1) * np.floor(r * 0.28)
                hy = cy + (sl // 3 - 1) * np.floor(r * 0.28)
                # clockwise square
                hxs = np.array([hx - hs, hx - hs, hx + hs, hx + hs, hx - hs])
                hys = np.array([hy - hs, hy + hs, hy + hs, hy - hs, hy - hs])
                rings.append((hxs, hys))
            for rx, ry in rings:
                ring_sizes.append(len(rx))
                xs.append(rx)
                ys.append(ry)
                verts.append(np.stack([rx[:-1], ry[:-1]], 1))
                edges_a.append(np.stack([rx[:-1], ry[:-1]], 1))
                edges_b.append(np.stack([rx[1:], ry[1:]], 1))
            rings_per_part.append(len(rings))
        parts_per_geom.append(nparts)
    polys = _rings_to_soa(np.asarray(ring_sizes), np.concatenate(xs), np.concatenate(ys),
                          np.asarray(rings_per_part), np.asarray(parts_per_geom))
    verts = np.concatenate(verts)
    ea = np.concatenate(edges_a)
    eb = np.concatenate(edges_b)
    n_v = n_points // 10
    n_e = n_points // 10
    n_u = n_points // 10
    n_r = n_points - n_v - n_e - n_u
    px = np.empty(n_points)
    py = np.empty(n_points)
    rx, ry = uniform_points(rng, n_r, 0.0, extent)
    px[:n_r], py[:n_r] = rx, ry
    vi = rng.integers(0, len(verts), n_v)
    px[n_r:n_r + n_v] = verts[vi, 0]
    py[n_r:n_r + n_v] = verts[vi, 1]
    # on-edge: a + t (b - a), t = k / 2^10 -- exact for lattice vertices < 2^15
    ei = rng.integers(0, len(ea), n_e + n_u)
    t = rng.integers(1, 1024, n_e + n_u) / 1024.0
    ex = ea[ei, 0] + t * (eb[ei, 0] - ea[ei, 0])
    ey = ea[ei, 1] + t * (eb[ei, 1] - ea[ei, 1])
    o = n_r + n_v
    px[o:o + n_e], py[o:o + n_e] = ex[:n_e], ey[:n_e]
    # one ulp off an edge point, in x or y, up or down
    ux, uy = ex[n_e:].copy(), ey[n_e:].copy()
    axis = rng.integers(0, 2, n_u)
    sign = np.where(rng.integers(0, 2, n_u) == 1, np.inf, -np.inf)
    ux = np.where(axis == 0, np.nextafter(ux, sign), ux)
    uy = np.where(axis == 1, np.nextafter(uy, sign), uy)
    px[o + n_e:], py[o + n_e:] = ux, uy
    perm = rng.permutation(n_points)
    return Workload("degenerate_join", px[perm], py[perm], polys,
                    {"seed": seed, "n_points": n_points, "n_polys": n_polys, "extent": extent,
                     "frac_vertex": 0.1, "frac_edge": 0.1, "frac_ulp": 0.1})


WORKLOADS = {
    "star": star_join,
    "utm": utm_join,
    "zipf": zipf_join,
    "degenerate": degenerate_join,
}


def wkb_points(x: np.ndarray, y: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Little-endian 2D WKB Points (21 bytes each), vectorised: (bytes uint8, offsets int64)."""
    n = len(x)
    rec = np.empty((n, 21), dtype=np.uint8)
    rec[:, 0] = 1
    rec[:, 1:5] = np.frombuffer(np.uint32(1).tobytes(), np.uint8)
    rec[:, 5:13] = np.ascontiguousarray(x, dtype="<f8").view(np.uint8).reshape(n, 8)
    rec[:, 13:21] = np.ascontiguousarray(y, dtype="<f8").view(np.uint8).reshape(n, 8)
    return rec.reshape(-1), np.arange(n + 1, dtype=np.int64) * 21


def wkb_polygons(p: PolygonSoA) -> tuple[np.ndarray, np.ndarray]:
    """Little-endian 2D WKB of single-part polygons (MultiPolygon rows become MultiPolygons), vectorised."""
    geom_off = np.asarray(p.geom_off, np.int64)
    part_off = np.asarray(p.part_off, np.int64)
    ring_off = np.asarray(p.ring_off, np.int64)
    n = len(geom_off) - 1
    nparts = np.diff(geom_off)
    multi = nparts != 1
    rings_per_part = np.diff(part_off)
    pts_per_ring = np.diff(ring_off)
    # bytes: row header 5 (+4 part count for multi); per part header 5 (multi only) + 4 ring count;
    # per ring 4 + 16 * points
    ring_bytes = 4 + 16 * pts_per_ring
    part_bytes = 4 + np.add.reduceat(ring_bytes, part_off[:-1]) if len(ring_bytes) else np.zeros(0, np.int64)
    part_bytes = np.where(rings_per_part > 0, part_bytes, 4)
    part_row = np.repeat(np.arange(n), nparts)
    part_hdr = np.where(multi[part_row], 5, 0)
    row_bytes = 5 + 4 * multi + np.bincount(part_row, weights=part_bytes + part_hdr, minlength=n).astype(np.int64)
    offsets = np.concatenate([[0], np.cumsum(row_bytes)])
    out = np.zeros(offsets[-1], dtype=np.uint8)
    u32 = lambda v: np.frombuffer(np.asarray(v, "<u4").tobytes(), np.uint8).reshape(-1, 4)  # noqa: E731

    def put_u32(pos, vals):
        b = u32(vals)
        for k in range(4):
            out[pos + k] = b[:, k]

    out[offsets[:-1]] = 1
    put_u32(offsets[:-1] + 1, np.where(multi, 6, 3))
    put_u32(offsets[:-1][multi] + 5, nparts[multi])
    # part starts
    part_start_in_row = np.zeros(len(part_row), np.int64)
    if len(part_row):
        cum = np.cumsum(part_bytes + part_hdr) - (part_bytes + part_hdr)
        part_start_in_row = cum - cum[geom_off[part_row]] if len(cum) else cum
    part_pos = offsets[:-1][part_row] + 5 + 4 * multi[part_row] + part_start_in_row
    mp = multi[part_row]
    out[part_pos[mp]] = 1
    put_u32(part_pos[mp] + 1, np.full(mp.sum(), 3))
    ring_count_pos = part_pos + part_hdr
    put_u32(ring_count_pos, rings_per_part)
    # rings
    ring_part = np.repeat(np.arange(len(rings_per_part)), rings_per_part)
    cum_r = np.cumsum(ring_bytes) - ring_bytes
    ring_start_in_part = cum_r - cum_r[part_off[ring_part]] if len(cum_r) else cum_r
    ring_pos = ring_count_pos[ring_part] + 4 + ring_start_in_part
    put_u32(ring_pos, pts_per_ring)
    coord_ring = np.repeat(np.arange(len(pts_per_ring)), pts_per_ring)
    k = np.arange(len(p.x)) - ring_off[coord_ring]
    cpos = ring_pos[coord_ring] + 4 + 16 * k
    xb = np.ascontiguousarray(p.x, "<f8").view(np.uint8).reshape(-1, 8)
    yb = np.ascontiguousarray(p.y, "<f8").view(np.uint8).reshape(-1, 8)
    for b in range(8):
        out[cpos + b] = xb[:, b]
        out[cpos + 8 + b] = yb[:, b]
    return out, offsets
