/*
 * CPU oracle of the distance joins (dwithin, nearest with all ties).
 *
 * TEST INFRASTRUCTURE ONLY: the checker of the device distance joins, loaded
 * by the test-suite; the product never links or calls it.
 *
 * What it restates (reference files, paths inside the vibeSpatial project):
 *   - dwithin = distance(point, polygon) <= threshold per pair:
 *       src/vibespatial/spatial/nearest.py:2855 (_dwithin_refine_gpu), with
 *       the distance of src/vibespatial/spatial/point_distance_kernels.py:238-310
 *       (0 inside, else the minimum point-segment distance over the rings)
 *   - nearest with all ties and max_distance: sjoin_nearest
 *       (src/vibespatial/api/tools/sjoin.py) -> src/vibespatial/spatial/nearest.py
 * The point-segment distance is the comp.graphics.algorithms FAQ method
 * (the one GEOS's Distance::pointToSegment uses); dwithin applies the
 * envelope short-circuit first.  Location is the exact orc_geometry_location.
 * Compiled with -ffp-contract=off, every operation rounds on its own, the
 * same arithmetic as the device code.
 *
 * Candidates come from a uniform grid over the polygon boxes (the square of
 * the search radius around the point, the radius growing for nearest); the
 * exact test decides every candidate.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int orc_geometry_location(double px, double py, const double *x, const double *y, const int32_t *ring_off,
                          const int32_t *part_off, const int32_t *geom_off, int64_t g);
void orc_geometry_bounds(const double *x, const double *y, const int32_t *ring_off, const int32_t *part_off,
                         const int32_t *geom_off, const uint8_t *gvalid, int64_t ngeoms, double *bounds);

typedef struct {
    int64_t n;
    int32_t *left;
    int32_t *right;
    double *dist;
} orc_dpairs;

static double pp_dist(double px, double py, double ax, double ay) {
    const double dx = px - ax, dy = py - ay;
    return sqrt(dx * dx + dy * dy);
}

double orc_point_segment_distance(double px, double py, double ax, double ay, double bx, double by) {
    if (ax == bx && ay == by) return pp_dist(px, py, ax, ay);
    const double ux = bx - ax, uy = by - ay;
    const double len2 = ux * ux + uy * uy;
    const double r = ((px - ax) * ux + (py - ay) * uy) / len2;
    if (r <= 0.0) return pp_dist(px, py, ax, ay);
    if (r >= 1.0) return pp_dist(px, py, bx, by);
    const double s = ((ay - py) * ux - (ax - px) * uy) / len2;
    return fabs(s) * sqrt(len2);
}

double orc_envelope_distance(const double *b, double px, double py) {
    double dx = 0.0, dy = 0.0;
    if (px < b[0]) dx = b[0] - px;
    else if (px > b[2]) dx = px - b[2];
    if (py < b[1]) dy = b[1] - py;
    else if (py > b[3]) dy = py - b[3];
    if (dx == 0.0) return dy;
    if (dy == 0.0) return dx;
    return sqrt(dx * dx + dy * dy);
}

double orc_point_polygon_distance(double px, double py, const double *x, const double *y, const int32_t *ring_off,
                                  const int32_t *part_off, const int32_t *geom_off, int64_t g) {
    if (orc_geometry_location(px, py, x, y, ring_off, part_off, geom_off, g) != 0) return 0.0;
    double best = INFINITY;
    for (int32_t ring = part_off[geom_off[g]]; ring < part_off[geom_off[g + 1]]; ++ring) {
        const int32_t c0 = ring_off[ring], c1 = ring_off[ring + 1];
        for (int32_t c = c0 + 1; c < c1; ++c) {
            const double d = orc_point_segment_distance(px, py, x[c - 1], y[c - 1], x[c], y[c]);
            if (d < best) best = d;
        }
    }
    return best;
}

typedef struct {
    int32_t *l, *r;
    double *d;
    int64_t n, cap;
} dvec;

static void dvec_push(dvec *v, int32_t l, int32_t r, double d) {
    if (v->n == v->cap) {
        v->cap = v->cap ? v->cap * 2 : 1024;
        v->l = (int32_t *)realloc(v->l, (size_t)v->cap * sizeof(int32_t));
        v->r = (int32_t *)realloc(v->r, (size_t)v->cap * sizeof(int32_t));
        v->d = (double *)realloc(v->d, (size_t)v->cap * sizeof(double));
    }
    v->l[v->n] = l;
    v->r[v->n] = r;
    v->d[v->n] = d;
    v->n++;
}

/* Pairs come out of each point's loop in polygon order and points are
 * visited in order by each thread's static chunk, so concatenating the
 * per-thread vectors in thread order yields (left, right)-sorted pairs. */
static orc_dpairs *gather(dvec *per, int nt) {
    orc_dpairs *res = (orc_dpairs *)calloc(1, sizeof(orc_dpairs));
    int64_t n = 0;
    for (int t = 0; t < nt; ++t) n += per[t].n;
    res->n = n;
    res->left = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    res->right = (int32_t *)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
    res->dist = (double *)malloc((size_t)(n > 0 ? n : 1) * sizeof(double));
    int64_t o = 0;
    for (int t = 0; t < nt; ++t) {
        if (per[t].n) {
            memcpy(res->left + o, per[t].l, (size_t)per[t].n * sizeof(int32_t));
            memcpy(res->right + o, per[t].r, (size_t)per[t].n * sizeof(int32_t));
            memcpy(res->dist + o, per[t].d, (size_t)per[t].n * sizeof(double));
            o += per[t].n;
        }
        free(per[t].l);
        free(per[t].r);
        free(per[t].d);
    }
    free(per);
    return res;
}

static int begin_threads(int nthreads) {
    int nt = 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
    nt = omp_get_max_threads();
#endif
    (void)nthreads;
    return nt;
}

/* A uniform grid over the valid polygon boxes: cell -> polygons whose box
 * overlaps it (CSR).  Coordinates outside the frame clamp to the border cells,
 * so a query square overlapping a polygon's box always shares a cell with it. */
typedef struct {
    double x0, y0, sx, sy, cw, ch;
    int64_t side;
    int64_t *start;
    int32_t *items;
    int64_t nvalid;
} grid_t;

static int64_t cell_of(double v, double lo, double s, int64_t side) {
    const double c = floor((v - lo) * s);
    if (!(c >= 0.0)) return 0; /* also NaN and -inf */
    if (c >= (double)side) return side - 1;
    return (int64_t)c;
}

static void grid_build(grid_t *gr, const double *bounds, int64_t ngeoms) {
    double tx0 = INFINITY, ty0 = INFINITY, tx1 = -INFINITY, ty1 = -INFINITY;
    int64_t nvalid = 0;
    for (int64_t g = 0; g < ngeoms; ++g) {
        const double *b = &bounds[4 * g];
        if (!(b[0] <= b[2])) continue;
        nvalid++;
        tx0 = fmin(tx0, b[0]); ty0 = fmin(ty0, b[1]);
        tx1 = fmax(tx1, b[2]); ty1 = fmax(ty1, b[3]);
    }
    gr->nvalid = nvalid;
    int64_t side = (int64_t)sqrt((double)(nvalid > 0 ? nvalid : 1)) + 1;
    if (side > 2048) side = 2048;
    const double w = (tx1 - tx0) > 0 ? (tx1 - tx0) : 1.0, h = (ty1 - ty0) > 0 ? (ty1 - ty0) : 1.0;
    gr->x0 = nvalid ? tx0 : 0.0;
    gr->y0 = nvalid ? ty0 : 0.0;
    gr->side = side;
    gr->sx = side / w;
    gr->sy = side / h;
    gr->cw = w / side;
    gr->ch = h / side;
    const int64_t ncell = side * side;
    gr->start = (int64_t *)calloc((size_t)ncell + 1, sizeof(int64_t));
    for (int pass = 0; pass < 2; ++pass) {
        int64_t *fill = NULL;
        if (pass == 1) {
            for (int64_t c = 0; c < ncell; ++c) gr->start[c + 1] += gr->start[c];
            gr->items = (int32_t *)malloc((size_t)(gr->start[ncell] > 0 ? gr->start[ncell] : 1) * sizeof(int32_t));
            fill = (int64_t *)malloc((size_t)ncell * sizeof(int64_t));
            memcpy(fill, gr->start, (size_t)ncell * sizeof(int64_t));
        }
        for (int64_t g = 0; g < ngeoms; ++g) {
            const double *b = &bounds[4 * g];
            if (!(b[0] <= b[2])) continue;
            const int64_t cx0 = cell_of(b[0], gr->x0, gr->sx, side), cx1 = cell_of(b[2], gr->x0, gr->sx, side);
            const int64_t cy0 = cell_of(b[1], gr->y0, gr->sy, side), cy1 = cell_of(b[3], gr->y0, gr->sy, side);
            for (int64_t cy = cy0; cy <= cy1; ++cy)
                for (int64_t cx = cx0; cx <= cx1; ++cx) {
                    if (pass == 0) gr->start[cy * side + cx + 1]++;
                    else gr->items[fill[cy * side + cx]++] = (int32_t)g;
                }
        }
        free(fill);
    }
}

static void grid_free(grid_t *gr) {
    free(gr->start);
    free(gr->items);
}

/* Cells overlapped by the square of half-width r around (x, y), widened by a
 * relative margin (a polygon whose computed distance is within r is found). */
static void grid_cover(const grid_t *gr, double x, double y, double r, int64_t *c) {
    const double q = r + r * 0x1p-30 + 0x1p-1000;
    c[0] = cell_of(x - q, gr->x0, gr->sx, gr->side);
    c[1] = cell_of(x + q, gr->x0, gr->sx, gr->side);
    c[2] = cell_of(y - q, gr->y0, gr->sy, gr->side);
    c[3] = cell_of(y + q, gr->y0, gr->sy, gr->side);
}

static int cmp_i32(const void *a, const void *b) {
    const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* d: d_pt[point] if d_pt, else d_geom[polygon] if d_geom, else d_scalar. */
orc_dpairs *orc_dwithin_join(const double *px, const double *py, const uint8_t *pvalid, int64_t npts, const double *x,
                             const double *y, const int32_t *ring_off, const int32_t *part_off,
                             const int32_t *geom_off, const uint8_t *gvalid, int64_t ngeoms, const double *d_pt,
                             const double *d_geom, double d_scalar, int nthreads) {
    double *bounds = (double *)malloc((size_t)(ngeoms > 0 ? ngeoms : 1) * 4 * sizeof(double));
    orc_geometry_bounds(x, y, ring_off, part_off, geom_off, gvalid, ngeoms, bounds);
    grid_t gr;
    grid_build(&gr, bounds, ngeoms);
    double dmax = d_scalar;
    if (d_geom) {
        dmax = -INFINITY;
        for (int64_t g = 0; g < ngeoms; ++g)
            if (d_geom[g] == d_geom[g] && d_geom[g] > dmax) dmax = d_geom[g];
    }
    const int nt = begin_threads(nthreads);
    dvec *per = (dvec *)calloc((size_t)nt, sizeof(dvec));
    int64_t *stamp = (int64_t *)malloc((size_t)nt * (size_t)(ngeoms > 0 ? ngeoms : 1) * sizeof(int64_t));
    for (int64_t k = 0; k < (int64_t)nt * (ngeoms > 0 ? ngeoms : 1); ++k) stamp[k] = -1;
    int32_t *cand = (int32_t *)malloc((size_t)nt * (size_t)(ngeoms > 0 ? ngeoms : 1) * sizeof(int32_t));
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < npts; ++i) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        if (gr.nvalid == 0 || (pvalid && !pvalid[i]) || isnan(px[i]) || isnan(py[i])) continue;
        const double q = d_pt ? d_pt[i] : dmax;
        if (!(q >= 0.0)) continue;
        int64_t *st = stamp + (size_t)tid * (size_t)ngeoms;
        int32_t *cd = cand + (size_t)tid * (size_t)ngeoms;
        int64_t nc = 0, c[4];
        grid_cover(&gr, px[i], py[i], q, c);
        for (int64_t cy = c[2]; cy <= c[3]; ++cy)
            for (int64_t cx = c[0]; cx <= c[1]; ++cx)
                for (int64_t k = gr.start[cy * gr.side + cx]; k < gr.start[cy * gr.side + cx + 1]; ++k) {
                    const int32_t g = gr.items[k];
                    if (st[g] == i) continue;
                    st[g] = i;
                    cd[nc++] = g;
                }
        qsort(cd, (size_t)nc, sizeof(int32_t), cmp_i32);
        for (int64_t k = 0; k < nc; ++k) {
            const int32_t g = cd[k];
            const double *b = &bounds[4 * g];
            const double d = d_pt ? d_pt[i] : (d_geom ? d_geom[g] : d_scalar);
            if (!(d >= 0.0)) continue;
            if (orc_envelope_distance(b, px[i], py[i]) > d) continue;
            const double dist = orc_point_polygon_distance(px[i], py[i], x, y, ring_off, part_off, geom_off, g);
            if (dist <= d) dvec_push(&per[tid], (int32_t)i, g, dist);
        }
    }
    free(cand);
    free(stamp);
    grid_free(&gr);
    free(bounds);
    return gather(per, nt);
}

/* Every polygon at each point's minimum distance, if that minimum is finite
 * and <= max_distance.  Grid search over a growing square: the minimum over
 * the polygons registered in the cells within r is final once it is <= r
 * (or once the square covers the whole grid). */
orc_dpairs *orc_nearest_join(const double *px, const double *py, const uint8_t *pvalid, int64_t npts, const double *x,
                             const double *y, const int32_t *ring_off, const int32_t *part_off,
                             const int32_t *geom_off, const uint8_t *gvalid, int64_t ngeoms, double max_distance,
                             int nthreads) {
    double *bounds = (double *)malloc((size_t)(ngeoms > 0 ? ngeoms : 1) * 4 * sizeof(double));
    orc_geometry_bounds(x, y, ring_off, part_off, geom_off, gvalid, ngeoms, bounds);
    grid_t gr;
    grid_build(&gr, bounds, ngeoms);
    const int nt = begin_threads(nthreads);
    dvec *per = (dvec *)calloc((size_t)nt, sizeof(dvec));
    const size_t m = (size_t)(ngeoms > 0 ? ngeoms : 1);
    int64_t *stamp = (int64_t *)malloc((size_t)nt * m * sizeof(int64_t));
    for (size_t k = 0; k < (size_t)nt * m; ++k) stamp[k] = -1;
    double *dist = (double *)malloc((size_t)nt * m * sizeof(double));
    int32_t *cand = (int32_t *)malloc((size_t)nt * m * sizeof(int32_t));
    const double r0 = fmax(gr.cw, gr.ch);
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < npts; ++i) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        if (gr.nvalid == 0 || (pvalid && !pvalid[i]) || isnan(px[i]) || isnan(py[i])) continue;
        int64_t *st = stamp + (size_t)tid * m;
        double *dg = dist + (size_t)tid * m;
        int32_t *cd = cand + (size_t)tid * m;
        int64_t nc = 0;
        double best = INFINITY;
        /* polygons are added as the square grows; each keeps its distance */
        for (double r = r0;; r *= 2.0) {
            int64_t c[4];
            grid_cover(&gr, px[i], py[i], r, c);
            for (int64_t cy = c[2]; cy <= c[3]; ++cy)
                for (int64_t cx = c[0]; cx <= c[1]; ++cx)
                    for (int64_t k = gr.start[cy * gr.side + cx]; k < gr.start[cy * gr.side + cx + 1]; ++k) {
                        const int32_t g = gr.items[k];
                        if (st[g] == i) continue;
                        st[g] = i;
                        cd[nc++] = g;
                        dg[g] = orc_point_polygon_distance(px[i], py[i], x, y, ring_off, part_off, geom_off, g);
                        if (dg[g] < best) best = dg[g];
                    }
            const int all = c[0] == 0 && c[2] == 0 && c[1] == gr.side - 1 && c[3] == gr.side - 1;
            if (best <= r || all || !(r < INFINITY)) break;
        }
        if (!(best < INFINITY) || !(best <= max_distance)) continue;
        qsort(cd, (size_t)nc, sizeof(int32_t), cmp_i32);
        for (int64_t k = 0; k < nc; ++k)
            if (dg[cd[k]] == best) dvec_push(&per[tid], (int32_t)i, cd[k], best);
    }
    free(cand);
    free(dist);
    free(stamp);
    grid_free(&gr);
    free(bounds);
    return gather(per, nt);
}

int64_t orc_dpairs_count(const orc_dpairs *p) { return p ? p->n : 0; }

void orc_dpairs_copy(const orc_dpairs *p, int32_t *left, int32_t *right, double *dist) {
    if (!p || p->n == 0) return;
    memcpy(left, p->left, (size_t)p->n * sizeof(int32_t));
    memcpy(right, p->right, (size_t)p->n * sizeof(int32_t));
    memcpy(dist, p->dist, (size_t)p->n * sizeof(double));
}

void orc_dpairs_free(orc_dpairs *p) {
    if (!p) return;
    free(p->left);
    free(p->right);
    free(p->dist);
    free(p);
}

/* Row-wise: point i against polygon i (NaN for null / NaN / empty rows). */
void orc_distance_aligned(const double *px, const double *py, const uint8_t *pvalid, int64_t n, const double *x,
                          const double *y, const int32_t *ring_off, const int32_t *part_off, const int32_t *geom_off,
                          const uint8_t *gvalid, double *dist, double *env) {
    double b[4];
    for (int64_t i = 0; i < n; ++i) {
        dist[i] = NAN;
        env[i] = NAN;
        if ((pvalid && !pvalid[i]) || (gvalid && !gvalid[i]) || isnan(px[i]) || isnan(py[i])) continue;
        const int32_t r0 = part_off[geom_off[i]], r1 = part_off[geom_off[i + 1]];
        const int32_t c0 = ring_off[r0], c1 = ring_off[r1];
        if (c1 <= c0) continue;
        b[0] = INFINITY; b[1] = INFINITY; b[2] = -INFINITY; b[3] = -INFINITY;
        for (int32_t c = c0; c < c1; ++c) {
            b[0] = fmin(b[0], x[c]); b[1] = fmin(b[1], y[c]);
            b[2] = fmax(b[2], x[c]); b[3] = fmax(b[3], y[c]);
        }
        env[i] = orc_envelope_distance(b, px[i], py[i]);
        dist[i] = orc_point_polygon_distance(px[i], py[i], x, y, ring_off, part_off, geom_off, i);
    }
}

/* Every point at each polygon's minimum distance (pairs sorted by polygon
 * row, then point row), if that minimum is finite and <= max_distance: the
 * sjoin_nearest query with the polygons as the matched side.  Brute force
 * over the points with the envelope lower bound (small test sizes). */
orc_dpairs *orc_nearest_polygons_join(const double *px, const double *py, const uint8_t *pvalid, int64_t npts,
                                      const double *x, const double *y, const int32_t *ring_off,
                                      const int32_t *part_off, const int32_t *geom_off, const uint8_t *gvalid,
                                      int64_t ngeoms, double max_distance, int nthreads) {
    double *bounds = (double *)malloc((size_t)(ngeoms > 0 ? ngeoms : 1) * 4 * sizeof(double));
    orc_geometry_bounds(x, y, ring_off, part_off, geom_off, gvalid, ngeoms, bounds);
    const int nt = begin_threads(nthreads);
    dvec *per = (dvec *)calloc((size_t)nt, sizeof(dvec));
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t g = 0; g < ngeoms; ++g) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        const double *b = &bounds[4 * g];
        if (!(b[0] <= b[2])) continue;
        /* the minimum, then (a second pass) every point at exactly it */
        double best = INFINITY;
        for (int64_t i = 0; i < npts; ++i) {
            if ((pvalid && !pvalid[i]) || isnan(px[i]) || isnan(py[i])) continue;
            if (orc_envelope_distance(b, px[i], py[i]) > best * (1.0 + 0x1p-40)) continue;
            const double d = orc_point_polygon_distance(px[i], py[i], x, y, ring_off, part_off, geom_off, g);
            if (d < best) best = d;
        }
        if (!(best < INFINITY) || !(best <= max_distance)) continue;
        for (int64_t i = 0; i < npts; ++i) {
            if ((pvalid && !pvalid[i]) || isnan(px[i]) || isnan(py[i])) continue;
            if (orc_envelope_distance(b, px[i], py[i]) > best * (1.0 + 0x1p-40)) continue;
            if (orc_point_polygon_distance(px[i], py[i], x, y, ring_off, part_off, geom_off, g) == best)
                dvec_push(&per[tid], (int32_t)g, (int32_t)i, best);
        }
    }
    free(bounds);
    return gather(per, nt);
}
