/* CPU WKB decoder: TEST INFRASTRUCTURE ONLY (the checker for the device
 * decoder and the CPU leg of the WKB ingest benchmark; never linked by the
 * product).
 *
 * Restates the reference's staged WKB decode for the families the join
 * consumes (src/vibespatial/io/wkb.py): the header scan of _scan_wkb_value
 * (wkb.py:3755-3781: byte-order flag 0/1, EWKB Z/M/SRID flag bits, ISO
 * type + 1000 * dims) and the payload walks of _decode_polygon_wkb_payload
 * (wkb.py:3954-3980) and _decode_multipolygon_wkb_payload (wkb.py:4043),
 * with every read bounds-checked against the value's bytes.  Output is the
 * columnar layout the device decoder writes: per-row tags (-1 null, 0 Point,
 * 2 Polygon, 5 MultiPolygon) and point coordinates (NaN for non-points), and
 * one MultiPolygon-form SoA over all rows (geom_off -> part_off -> ring_off
 * -> x, y).  Empty polygons and empty parts own no part entry; Z and M
 * ordinates are dropped; rows of other types count as unsupported and rows
 * whose reads overrun count as malformed, both decoding to null rows.
 *
 * Two passes, each parallel over rows (OpenMP): counts per row, a serial
 * exclusive scan, then the fill of offsets and coordinates. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

enum { TAG_NULL = -1, TAG_POINT = 0, TAG_POLYGON = 2, TAG_MULTIPOLYGON = 5 };
enum { ROW_OK = 0, ROW_UNSUPPORTED = 1, ROW_MALFORMED = 2 };

typedef struct {
    const uint8_t* p;
    const uint8_t* end;
    int ok;
} cur_t;

static uint32_t rd_u32(cur_t* c, int little) {
    if (c->end - c->p < 4) {
        c->ok = 0;
        return 0;
    }
    const uint8_t* b = c->p;
    c->p += 4;
    return little ? ((uint32_t)b[0] | (uint32_t)b[1] << 8 | (uint32_t)b[2] << 16 | (uint32_t)b[3] << 24)
                  : ((uint32_t)b[3] | (uint32_t)b[2] << 8 | (uint32_t)b[1] << 16 | (uint32_t)b[0] << 24);
}

static void skip(cur_t* c, uint64_t n) {
    if ((uint64_t)(c->end - c->p) < n) {
        c->ok = 0;
        c->p = c->end;
        return;
    }
    c->p += n;
}

static double rd_f64(const uint8_t* p, int little) {
    uint8_t b[8];
    for (int k = 0; k < 8; ++k) b[k] = p[little ? k : 7 - k];
    double v;
    memcpy(&v, b, 8);  /* host is little-endian */
    return v;
}

typedef struct {
    int little;
    uint32_t base;
    int dims;
} hdr_t;

static hdr_t rd_header(cur_t* c) {
    hdr_t h = {1, 0, 2};
    uint8_t bo = 0;
    if (c->end - c->p < 1) c->ok = 0;
    else bo = *c->p++;
    if (bo > 1) c->ok = 0;
    h.little = bo == 1;
    uint32_t t = rd_u32(c, h.little);
    int z = (t & 0x80000000u) != 0, m = (t & 0x40000000u) != 0;
    if (t & 0x20000000u) skip(c, 4); /* EWKB SRID */
    t &= 0x0fffffffu;
    uint32_t iso = t / 1000u;
    t %= 1000u;
    if (iso == 1 || iso == 3) z = 1;
    if (iso == 2 || iso == 3) m = 1;
    if (iso > 3) c->ok = 0;
    h.base = t;
    h.dims = 2 + z + m;
    return h;
}

typedef struct {
    int8_t tag;
    int status;
    uint32_t parts, rings;
    uint64_t coords;
    double px, py;
} row_t;

static void polygon_counts(cur_t* c, const hdr_t* h, uint32_t* rings, uint64_t* coords) {
    uint32_t nr = rd_u32(c, h->little);
    for (uint32_t r = 0; r < nr && c->ok; ++r) {
        uint32_t np = rd_u32(c, h->little);
        skip(c, (uint64_t)np * 8u * (uint64_t)h->dims);
        *coords += np;
    }
    *rings += nr;
}

static row_t parse_row(const uint8_t* data, const int64_t* off, const uint8_t* valid, int64_t i) {
    row_t r = {TAG_NULL, ROW_OK, 0, 0, 0, NAN, NAN};
    if (valid && !valid[i]) return r;
    if (off[i + 1] <= off[i]) return r;
    cur_t c = {data + off[i], data + off[i + 1], 1};
    hdr_t h = rd_header(&c);
    if (!c.ok) {
        r.status = ROW_MALFORMED;
        return r;
    }
    if (h.base == 1) {
        if (c.end - c.p < 8 * h.dims) {
            r.status = ROW_MALFORMED;
            return r;
        }
        r.tag = TAG_POINT;
        r.px = rd_f64(c.p, h.little);
        r.py = rd_f64(c.p + 8, h.little);
        return r;
    }
    if (h.base == 3) {
        r.tag = TAG_POLYGON;
        uint32_t rings = 0;
        polygon_counts(&c, &h, &rings, &r.coords);
        r.parts = rings > 0;
        r.rings = rings;
    } else if (h.base == 6) {
        r.tag = TAG_MULTIPOLYGON;
        uint32_t np = rd_u32(&c, h.little);
        for (uint32_t k = 0; k < np && c.ok; ++k) {
            hdr_t ph = rd_header(&c);
            if (!c.ok) break;
            if (ph.base != 3) {
                c.ok = 0;
                break;
            }
            uint32_t rings = 0;
            polygon_counts(&c, &ph, &rings, &r.coords);
            r.parts += rings > 0;
            r.rings += rings;
        }
    } else {
        r.status = ROW_UNSUPPORTED;
        return r;
    }
    if (!c.ok) {
        r.status = ROW_MALFORMED;
        r.tag = TAG_NULL;
        r.parts = r.rings = 0;
        r.coords = 0;
    }
    return r;
}

/* sizes[10]: rows, points, polygons, multipolygons, nulls, unsupported,
 * malformed, parts, rings, coords.  counts (3 * n int64, caller-owned) keeps
 * the per-row part / ring / coordinate counts for orc_wkb_fill. */
void orc_wkb_count(const uint8_t* data, const int64_t* off, const uint8_t* valid, int64_t n, int8_t* tags,
                   double* px, double* py, int64_t* counts, int64_t* sizes, int threads) {
    int64_t pts = 0, pol = 0, mpol = 0, nul = 0, uns = 0, mal = 0, parts = 0, rings = 0, coords = 0;
    if (threads <= 0) threads = 1;
#pragma omp parallel for num_threads(threads) schedule(static) \
    reduction(+ : pts, pol, mpol, nul, uns, mal, parts, rings, coords)
    for (int64_t i = 0; i < n; ++i) {
        row_t r = parse_row(data, off, valid, i);
        tags[i] = r.tag;
        px[i] = r.px;
        py[i] = r.py;
        counts[3 * i] = r.parts;
        counts[3 * i + 1] = r.rings;
        counts[3 * i + 2] = (int64_t)r.coords;
        pts += r.tag == TAG_POINT;
        pol += r.tag == TAG_POLYGON;
        mpol += r.tag == TAG_MULTIPOLYGON;
        nul += r.tag == TAG_NULL && r.status == ROW_OK;
        uns += r.status == ROW_UNSUPPORTED;
        mal += r.status == ROW_MALFORMED;
        parts += r.parts;
        rings += r.rings;
        coords += (int64_t)r.coords;
    }
    sizes[0] = n;
    sizes[1] = pts;
    sizes[2] = pol;
    sizes[3] = mpol;
    sizes[4] = nul;
    sizes[5] = uns;
    sizes[6] = mal;
    sizes[7] = parts;
    sizes[8] = rings;
    sizes[9] = coords;
}

/* Fills geom_off (n + 1), part_off (parts + 1), ring_off (rings + 1), x, y
 * (coords) from the counts of orc_wkb_count (turned into start offsets here). */
void orc_wkb_fill(const uint8_t* data, const int64_t* off, int64_t n, const int8_t* tags, int64_t* counts,
                  int32_t* geom_off, int32_t* part_off, int32_t* ring_off, double* x, double* y, int threads) {
    int64_t s[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            int64_t v = counts[3 * i + k];
            counts[3 * i + k] = s[k];
            s[k] += v;
        }
    geom_off[n] = (int32_t)s[0];
    part_off[s[0]] = (int32_t)s[1];
    ring_off[s[1]] = (int32_t)s[2];
    if (threads <= 0) threads = 1;
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        int64_t part = counts[3 * i], ring = counts[3 * i + 1], coord = counts[3 * i + 2];
        geom_off[i] = (int32_t)part;
        if (tags[i] != TAG_POLYGON && tags[i] != TAG_MULTIPOLYGON) continue;
        cur_t c = {data + off[i], data + off[i + 1], 1};
        hdr_t h = rd_header(&c);
        uint32_t np = 1;
        if (tags[i] == TAG_MULTIPOLYGON) np = rd_u32(&c, h.little);
        for (uint32_t k = 0; k < np; ++k) {
            hdr_t ph = h;
            if (tags[i] == TAG_MULTIPOLYGON) ph = rd_header(&c);
            uint32_t nr = rd_u32(&c, ph.little);
            if (nr == 0) continue;
            part_off[part++] = (int32_t)ring;
            for (uint32_t r = 0; r < nr; ++r) {
                uint32_t cnt = rd_u32(&c, ph.little);
                ring_off[ring++] = (int32_t)coord;
                for (uint32_t q = 0; q < cnt; ++q) {
                    x[coord] = rd_f64(c.p, ph.little);
                    y[coord] = rd_f64(c.p + 8, ph.little);
                    ++coord;
                    c.p += 8 * ph.dims;
                }
            }
        }
    }
}
