/*
 * Exact CPU oracle for the point-by-polygon spatial join.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against; it is loaded by the test-suite, by the smoke check and
 * by the CPU-baseline leg of the benchmark.  The product (libvsjoin.so) never
 * links or calls it.
 *
 * What it restates (reference files, paths inside the vibeSpatial project):
 *   - ring classification, 0 outside / 1 boundary / 2 interior:
 *       src/vibespatial/cuda/device_functions/point_in_ring.py:148-188
 *   - polygon / multipolygon location with hole toggling and part order:
 *       src/vibespatial/predicates/point_relations_kernels.py:37-96
 *   - orientation predicate (made exact here, see orc_orient2d):
 *       src/vibespatial/cuda/device_functions/orient2d.py:37-85
 *   - location -> predicate mapping:
 *       src/vibespatial/predicates/point_relations.py:100-130
 *   - null / empty rows never match: src/vibespatial/api/tools/sjoin.py:502-544
 *
 * Exactness: orc_orient2d computes the sign of
 *     (ax-cx)(by-cy) - (ay-cy)(bx-cx)
 * exactly for finite doubles (barring underflow of partial products below
 * 2^-969), by splitting every difference into an exact two-term expansion and
 * summing the sixteen exact partial products with expansion arithmetic
 * (Shewchuk, "Adaptive Precision Floating-Point Arithmetic and Fast Robust
 * Geometric Predicates", DCG 1997, sections 2.4-2.6).  The reference's own
 * device function rounds ax-cx before its error-free stage, so the oracle is
 * the exact-real-arithmetic truth that GEOS approximates with double-double.
 *
 * Build: see oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OUTSIDE 0
#define ORC_BOUNDARY 1
#define ORC_INTERIOR 2

/* ------------------------------------------------------------------ */
/* Error-free transformations                                          */
/* ------------------------------------------------------------------ */
static inline void two_sum(double a, double b, double *x, double *y) {
    double s = a + b;
    double bv = s - a;
    double av = s - bv;
    double br = b - bv;
    double ar = a - av;
    *x = s;
    *y = ar + br;
}

static inline void two_diff(double a, double b, double *x, double *y) {
    double s = a - b;
    double bv = a - s;
    double av = s + bv;
    double br = bv - b;
    double ar = a - av;
    *x = s;
    *y = ar + br;
}

static inline void two_product(double a, double b, double *x, double *y) {
    double p = a * b;
    *x = p;
    *y = fma(a, b, -p);
}

/* h := e + b, zero-eliminating, e nonoverlapping with increasing magnitude. */
static int grow_expansion_zeroelim(int elen, const double *e, double b, double *h) {
    double q = b, hh;
    int hindex = 0;
    for (int i = 0; i < elen; ++i) {
        two_sum(q, e[i], &q, &hh);
        if (hh != 0.0) h[hindex++] = hh;
    }
    if (q != 0.0 || hindex == 0) h[hindex++] = q;
    return hindex;
}

/* Exact sign of orient2d(a, b, c) = (ax-cx)(by-cy) - (ay-cy)(bx-cx). */
int orc_orient2d(double ax, double ay, double bx, double by, double cx, double cy) {
    double acx, acxt, bcx, bcxt, acy, acyt, bcy, bcyt;
    two_diff(ax, cx, &acx, &acxt);
    two_diff(bx, cx, &bcx, &bcxt);
    two_diff(ay, cy, &acy, &acyt);
    two_diff(by, cy, &bcy, &bcyt);
    /* det = (acx + acxt)(bcy + bcyt) - (acy + acyt)(bcx + bcxt) */
    const double lp[4][2] = {{acx, bcy}, {acx, bcyt}, {acxt, bcy}, {acxt, bcyt}};
    const double rp[4][2] = {{acy, bcx}, {acy, bcxt}, {acyt, bcx}, {acyt, bcxt}};
    double e[40], f[40];
    int elen = 0;
    double *cur = e, *nxt = f;
    for (int k = 0; k < 4; ++k) {
        double p, q;
        two_product(lp[k][0], lp[k][1], &p, &q);
        elen = grow_expansion_zeroelim(elen, cur, q, nxt); { double *t = cur; cur = nxt; nxt = t; }
        elen = grow_expansion_zeroelim(elen, cur, p, nxt); { double *t = cur; cur = nxt; nxt = t; }
        two_product(rp[k][0], rp[k][1], &p, &q);
        elen = grow_expansion_zeroelim(elen, cur, -q, nxt); { double *t = cur; cur = nxt; nxt = t; }
        elen = grow_expansion_zeroelim(elen, cur, -p, nxt); { double *t = cur; cur = nxt; nxt = t; }
    }
    const double top = cur[elen - 1];
    return (top > 0.0) - (top < 0.0);
}

/* ------------------------------------------------------------------ */
/* Ring / polygon location (follows point_in_ring.py:148-188 and        */
/* point_relations_kernels.py:63-96)                                    */
/* ------------------------------------------------------------------ */
int orc_ring_classify(double px, double py, const double *x, const double *y,
                      int64_t start, int64_t end) {
    int inside = 0;
    if (end - start < 2) return ORC_OUTSIDE;
    for (int64_t i = start, j = end - 1; i < end; j = i++) {
        const double ax = x[j], ay = y[j], bx = x[i], by = y[i];
        const int crosses = (ay > py) != (by > py);
        const double minx = fmin(ax, bx), maxx = fmax(ax, bx);
        const int on_bbox = py >= fmin(ay, by) && py <= fmax(ay, by) && px >= minx && px <= maxx;
        if (!crosses && !on_bbox) continue;
        if (crosses && px < minx) { inside = !inside; continue; }
        if (crosses && px > maxx) continue;
        const int o = orc_orient2d(ax, ay, bx, by, px, py);
        if (on_bbox && o == 0) return ORC_BOUNDARY;
        if (crosses && ((o > 0) == (by > ay))) inside = !inside;
    }
    return inside ? ORC_INTERIOR : ORC_OUTSIDE;
}

/* Location of (px,py) in geometry g of a polygon/multipolygon SoA where a
 * Polygon is a one-part MultiPolygon: geom_off -> parts, part_off -> rings,
 * ring_off -> coordinates. */
int orc_geometry_location(double px, double py, const double *x, const double *y,
                          const int32_t *ring_off, const int32_t *part_off,
                          const int32_t *geom_off, int64_t g) {
    for (int32_t part = geom_off[g]; part < geom_off[g + 1]; ++part) {
        int inside = 0;
        for (int32_t ring = part_off[part]; ring < part_off[part + 1]; ++ring) {
            const int k = orc_ring_classify(px, py, x, y, ring_off[ring], ring_off[ring + 1]);
            if (k == ORC_BOUNDARY) return ORC_BOUNDARY;
            if (k == ORC_INTERIOR) inside = !inside;
        }
        if (inside) return ORC_INTERIOR;
    }
    return ORC_OUTSIDE;
}

/* Element-wise location: row i of points against row i of polygons.
 * Rows where either side is null/empty get 255 (the host maps it to False). */
void orc_locate_aligned(const double *px, const double *py, const uint8_t *pvalid, int64_t n,
                        const double *x, const double *y, const int32_t *ring_off,
                        const int32_t *part_off, const int32_t *geom_off, const uint8_t *gvalid,
                        uint8_t *out, int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 4096)
#endif
    for (int64_t i = 0; i < n; ++i) {
        if ((pvalid && !pvalid[i]) || (gvalid && !gvalid[i]) || isnan(px[i]) || isnan(py[i])) {
            out[i] = 255;
            continue;
        }
        out[i] = (uint8_t)orc_geometry_location(px[i], py[i], x, y, ring_off, part_off, geom_off, i);
    }
}

/* ------------------------------------------------------------------ */
/* Join: uniform grid over geometry bounds, exact refine, sorted pairs. */
/* ------------------------------------------------------------------ */
typedef struct {
    int64_t n;
    int32_t *left;
    int32_t *right;
} orc_pairs;

typedef struct { int32_t *l, *r; int64_t n, cap; } vec2;

static void vec2_push(vec2 *v, int32_t l, int32_t r) {
    if (v->n == v->cap) {
        v->cap = v->cap ? v->cap * 2 : 1024;
        v->l = (int32_t *)realloc(v->l, (size_t)v->cap * sizeof(int32_t));
        v->r = (int32_t *)realloc(v->r, (size_t)v->cap * sizeof(int32_t));
    }
    v->l[v->n] = l;
    v->r[v->n] = r;
    v->n++;
}

static int cmp_pair(const void *a, const void *b) {
    const int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

/* Bounds of every geometry; invalid or coordinate-less geometries get an
 * inverted box that contains nothing. */
void orc_geometry_bounds(const double *x, const double *y, const int32_t *ring_off,
                         const int32_t *part_off, const int32_t *geom_off, const uint8_t *gvalid,
                         int64_t ngeoms, double *bounds /* ngeoms x 4 */) {
    for (int64_t g = 0; g < ngeoms; ++g) {
        double b0 = INFINITY, b1 = INFINITY, b2 = -INFINITY, b3 = -INFINITY;
        if (!gvalid || gvalid[g]) {
            const int32_t p0 = geom_off[g], p1 = geom_off[g + 1];
            if (p1 > p0) {
                const int64_t c0 = ring_off[part_off[p0]], c1 = ring_off[part_off[p1]];
                for (int64_t c = c0; c < c1; ++c) {
                    b0 = fmin(b0, x[c]); b1 = fmin(b1, y[c]);
                    b2 = fmax(b2, x[c]); b3 = fmax(b3, y[c]);
                }
            }
        }
        bounds[4 * g + 0] = b0; bounds[4 * g + 1] = b1;
        bounds[4 * g + 2] = b2; bounds[4 * g + 3] = b3;
    }
}

/* accept_mask: bit k set => location k passes the predicate
 * (within = 1<<2, intersects = (1<<1)|(1<<2), touches = 1<<1).
 * accept_mask == 0 => bounding-box candidates only (predicate=None). */
orc_pairs *orc_join(const double *px, const double *py, const uint8_t *pvalid, int64_t npts,
                    const double *x, const double *y, const int32_t *ring_off,
                    const int32_t *part_off, const int32_t *geom_off, const uint8_t *gvalid,
                    int64_t ngeoms, int accept_mask, int nthreads) {
    orc_pairs *res = (orc_pairs *)calloc(1, sizeof(orc_pairs));
    double *bounds = (double *)malloc((size_t)(ngeoms > 0 ? ngeoms : 1) * 4 * sizeof(double));
    orc_geometry_bounds(x, y, ring_off, part_off, geom_off, gvalid, ngeoms, bounds);
    double tx0 = INFINITY, ty0 = INFINITY, tx1 = -INFINITY, ty1 = -INFINITY;
    int64_t nvalid = 0;
    for (int64_t g = 0; g < ngeoms; ++g) {
        if (!(bounds[4 * g] <= bounds[4 * g + 2])) continue;
        nvalid++;
        tx0 = fmin(tx0, bounds[4 * g]); ty0 = fmin(ty0, bounds[4 * g + 1]);
        tx1 = fmax(tx1, bounds[4 * g + 2]); ty1 = fmax(ty1, bounds[4 * g + 3]);
    }
    if (nvalid == 0 || npts == 0) { free(bounds); return res; }
    int64_t side = (int64_t)sqrt((double)nvalid) + 1;
    if (side > 2048) side = 2048;
    const double w = (tx1 - tx0) > 0 ? (tx1 - tx0) : 1.0, h = (ty1 - ty0) > 0 ? (ty1 - ty0) : 1.0;
    const double sx = side / w, sy = side / h;
    const int64_t ncell = side * side;
    int64_t *cnt = (int64_t *)calloc((size_t)ncell + 1, sizeof(int64_t));
#define CELLX(v) ({ int64_t _c = (int64_t)floor(((v) - tx0) * sx); _c < 0 ? 0 : (_c >= side ? side - 1 : _c); })
#define CELLY(v) ({ int64_t _c = (int64_t)floor(((v) - ty0) * sy); _c < 0 ? 0 : (_c >= side ? side - 1 : _c); })
    for (int64_t g = 0; g < ngeoms; ++g) {
        if (!(bounds[4 * g] <= bounds[4 * g + 2])) continue;
        const int64_t cx0 = CELLX(bounds[4 * g]), cx1 = CELLX(bounds[4 * g + 2]);
        const int64_t cy0 = CELLY(bounds[4 * g + 1]), cy1 = CELLY(bounds[4 * g + 3]);
        for (int64_t cy = cy0; cy <= cy1; ++cy)
            for (int64_t cx = cx0; cx <= cx1; ++cx) cnt[cy * side + cx + 1]++;
    }
    for (int64_t c = 0; c < ncell; ++c) cnt[c + 1] += cnt[c];
    int64_t total = cnt[ncell];
    int32_t *items = (int32_t *)malloc((size_t)(total > 0 ? total : 1) * sizeof(int32_t));
    int64_t *fill = (int64_t *)malloc((size_t)ncell * sizeof(int64_t));
    memcpy(fill, cnt, (size_t)ncell * sizeof(int64_t));
    for (int64_t g = 0; g < ngeoms; ++g) {
        if (!(bounds[4 * g] <= bounds[4 * g + 2])) continue;
        const int64_t cx0 = CELLX(bounds[4 * g]), cx1 = CELLX(bounds[4 * g + 2]);
        const int64_t cy0 = CELLY(bounds[4 * g + 1]), cy1 = CELLY(bounds[4 * g + 3]);
        for (int64_t cy = cy0; cy <= cy1; ++cy)
            for (int64_t cx = cx0; cx <= cx1; ++cx) items[fill[cy * side + cx]++] = (int32_t)g;
    }
    free(fill);

    int nt = 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
    nt = omp_get_max_threads();
#endif
    vec2 *per = (vec2 *)calloc((size_t)nt, sizeof(vec2));
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        vec2 *v = &per[tid];
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 2048)
#endif
        for (int64_t i = 0; i < npts; ++i) {
            if (pvalid && !pvalid[i]) continue;
            const double qx = px[i], qy = py[i];
            if (!(qx >= tx0 && qx <= tx1 && qy >= ty0 && qy <= ty1)) continue; /* also drops NaN */
            const int64_t c = CELLY(qy) * side + CELLX(qx);
            for (int64_t k = cnt[c]; k < cnt[c + 1]; ++k) {
                const int32_t g = items[k];
                const double *b = &bounds[4 * g];
                if (!(qx >= b[0] && qx <= b[2] && qy >= b[1] && qy <= b[3])) continue;
                if (accept_mask == 0) { vec2_push(v, (int32_t)i, g); continue; }
                const int loc = orc_geometry_location(qx, qy, x, y, ring_off, part_off, geom_off, g);
                if (accept_mask & (1 << loc)) vec2_push(v, (int32_t)i, g);
            }
        }
    }
#undef CELLX
#undef CELLY
    int64_t n = 0;
    for (int t = 0; t < nt; ++t) n += per[t].n;
    int64_t *packed = (int64_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int64_t));
    int64_t o = 0;
    for (int t = 0; t < nt; ++t) {
        for (int64_t k = 0; k < per[t].n; ++k)
            packed[o++] = ((int64_t)per[t].l[k] << 32) | (int64_t)(uint32_t)per[t].r[k];
        free(per[t].l);
        free(per[t].r);
    }
    free(per);
    qsort(packed, (size_t)n, sizeof(int64_t), cmp_pair);
    res->n = n;
    res->left = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    res->right = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    for (int64_t k = 0; k < n; ++k) {
        res->left[k] = (int32_t)(packed[k] >> 32);
        res->right[k] = (int32_t)(packed[k] & 0xffffffff);
    }
    free(packed);
    free(items);
    free(cnt);
    free(bounds);
    return res;
}

int64_t orc_pairs_count(const orc_pairs *p) { return p ? p->n : 0; }

void orc_pairs_copy(const orc_pairs *p, int32_t *left, int32_t *right) {
    if (!p || p->n == 0) return;
    memcpy(left, p->left, (size_t)p->n * sizeof(int32_t));
    memcpy(right, p->right, (size_t)p->n * sizeof(int32_t));
}

void orc_pairs_free(orc_pairs *p) {
    if (!p) return;
    free(p->left);
    free(p->right);
    free(p);
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
