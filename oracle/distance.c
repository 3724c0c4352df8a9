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
 * Brute force over all polygons per point (small test sizes only).
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

/* d: d_pt[point] if d_pt, else d_geom[polygon] if d_geom, else d_scalar. */
orc_dpairs *orc_dwithin_join(const double *px, const double *py, const uint8_t *pvalid, int64_t npts, const double *x,
                             const double *y, const int32_t *ring_off, const int32_t *part_off,
                             const int32_t *geom_off, const uint8_t *gvalid, int64_t ngeoms, const double *d_pt,
                             const double *d_geom, double d_scalar, int nthreads) {
    double *bounds = (double *)malloc((size_t)(ngeoms > 0 ? ngeoms : 1) * 4 * sizeof(double));
    orc_geometry_bounds(x, y, ring_off, part_off, geom_off, gvalid, ngeoms, bounds);
    const int nt = begin_threads(nthreads);
    dvec *per = (dvec *)calloc((size_t)nt, sizeof(dvec));
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < npts; ++i) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        if ((pvalid && !pvalid[i]) || isnan(px[i]) || isnan(py[i])) continue;
        for (int64_t g = 0; g < ngeoms; ++g) {
            const double *b = &bounds[4 * g];
            if (!(b[0] <= b[2])) continue; /* null or empty polygon */
            const double d = d_pt ? d_pt[i] : (d_geom ? d_geom[g] : d_scalar);
            if (!(d >= 0.0)) continue;
            if (orc_envelope_distance(b, px[i], py[i]) > d) continue;
            const double dist = orc_point_polygon_distance(px[i], py[i], x, y, ring_off, part_off, geom_off, g);
            if (dist <= d) dvec_push(&per[tid], (int32_t)i, (int32_t)g, dist);
        }
    }
    free(bounds);
    return gather(per, nt);
}

/* Every polygon at each point's minimum distance, if that minimum is finite
 * and <= max_distance. */
orc_dpairs *orc_nearest_join(const double *px, const double *py, const uint8_t *pvalid, int64_t npts, const double *x,
                             const double *y, const int32_t *ring_off, const int32_t *part_off,
                             const int32_t *geom_off, const uint8_t *gvalid, int64_t ngeoms, double max_distance,
                             int nthreads) {
    double *bounds = (double *)malloc((size_t)(ngeoms > 0 ? ngeoms : 1) * 4 * sizeof(double));
    orc_geometry_bounds(x, y, ring_off, part_off, geom_off, gvalid, ngeoms, bounds);
    const int nt = begin_threads(nthreads);
    dvec *per = (dvec *)calloc((size_t)nt, sizeof(dvec));
    double *dist = (double *)malloc((size_t)nt * (size_t)(ngeoms > 0 ? ngeoms : 1) * sizeof(double));
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < npts; ++i) {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        if ((pvalid && !pvalid[i]) || isnan(px[i]) || isnan(py[i])) continue;
        double *dg = dist + (size_t)tid * (size_t)ngeoms;
        double best = INFINITY;
        for (int64_t g = 0; g < ngeoms; ++g) {
            const double *b = &bounds[4 * g];
            dg[g] = INFINITY;
            if (!(b[0] <= b[2])) continue;
            /* the envelope bounds the distance from below (a relative margin
             * covers the rounding of both) */
            if (orc_envelope_distance(b, px[i], py[i]) > best * (1.0 + 0x1p-40)) continue;
            dg[g] = orc_point_polygon_distance(px[i], py[i], x, y, ring_off, part_off, geom_off, g);
            if (dg[g] < best) best = dg[g];
        }
        if (!(best < INFINITY) || !(best <= max_distance)) continue;
        for (int64_t g = 0; g < ngeoms; ++g)
            if (dg[g] == best) dvec_push(&per[tid], (int32_t)i, (int32_t)g, best);
    }
    free(dist);
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
