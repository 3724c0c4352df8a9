// Exact point-in-polygon location on the device.
//
// Location codes follow the reference: 0 outside, 1 boundary, 2 interior
// (src/vibespatial/predicates/point_relations_kernels.py:37-96).  The ring
// walk keeps the reference's crossing rule, the half-open (ay > py) != (by > py)
// test plus the closed-bbox boundary check
// (src/vibespatial/cuda/device_functions/point_in_ring.py:148-188), but the
// orientation sign is decided exactly: a Shewchuk stage-A filter on rounded
// differences, then an exact expansion sum over the split differences
// (Shewchuk 1997, sections 2.4-2.6).  The reference's vs_orient2d
// (src/vibespatial/cuda/device_functions/orient2d.py:37-85) rounds ax-cx before
// its error-free stage; this one does not.
//
// Every floating-point step that the exactness argument depends on uses the
// explicit round-to-nearest intrinsics so that nvcc cannot contract it into
// an FMA.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ringbins.cuh"

namespace vs {

enum : int { LOC_OUTSIDE = 0, LOC_BOUNDARY = 1, LOC_INTERIOR = 2 };

__device__ __forceinline__ void two_sum(double a, double b, double& x, double& y) {
    x = __dadd_rn(a, b);
    const double bv = __dsub_rn(x, a);
    const double av = __dsub_rn(x, bv);
    const double br = __dsub_rn(b, bv);
    const double ar = __dsub_rn(a, av);
    y = __dadd_rn(ar, br);
}

__device__ __forceinline__ void two_diff(double a, double b, double& x, double& y) {
    x = __dsub_rn(a, b);
    const double bv = __dsub_rn(a, x);
    const double av = __dadd_rn(x, bv);
    const double br = __dsub_rn(bv, b);
    const double ar = __dsub_rn(a, av);
    y = __dadd_rn(ar, br);
}

__device__ __forceinline__ void two_product(double a, double b, double& x, double& y) {
    x = __dmul_rn(a, b);
    y = __fma_rn(a, b, -x);
}

// h := e + b with zero elimination; e is nonoverlapping, increasing magnitude.
__device__ __forceinline__ int grow_expansion(int elen, const double* e, double b, double* h) {
    double q = b, hh;
    int n = 0;
    for (int i = 0; i < elen; ++i) {
        two_sum(q, e[i], q, hh);
        if (hh != 0.0) h[n++] = hh;
    }
    if (q != 0.0 || n == 0) h[n++] = q;
    return n;
}

// Exact sign of (ax-cx)(by-cy) - (ay-cy)(bx-cx): sixteen exact partial
// products summed as a nonoverlapping expansion; the sign is the sign of the
// largest component.  Kept out of line: it runs only when the filter fails.
static __device__ __noinline__ int orient2d_exact(double ax, double ay, double bx, double by,
                                           double cx, double cy) {
    double acx, acxt, bcx, bcxt, acy, acyt, bcy, bcyt;
    two_diff(ax, cx, acx, acxt);
    two_diff(bx, cx, bcx, bcxt);
    two_diff(ay, cy, acy, acyt);
    two_diff(by, cy, bcy, bcyt);
    if (acxt == 0.0 && bcxt == 0.0 && acyt == 0.0 && bcyt == 0.0) {
        // The differences are exact (lattice or nearby inputs), so the
        // determinant is acx*bcy - acy*bcx = (p1 + q1) - (p2 + q2) with two
        // exact products.  Its expansion x3 + x2 + x1 + x0 (Shewchuk's
        // two-two-diff: nonoverlapping, x3 the largest, zeros possible)
        // takes the sign of its largest nonzero component.  Same sign as the
        // general sum below, in registers.
        double p1, q1, p2, q2;
        two_product(acx, bcy, p1, q1);
        two_product(acy, bcx, p2, q2);
        double i0, j0, z0, x0, x1, x2, x3;
        two_diff(q1, q2, i0, x0);
        two_sum(p1, i0, j0, z0);
        two_diff(z0, p2, i0, x1);
        two_sum(j0, i0, x3, x2);
        const double top = x3 != 0.0 ? x3 : (x2 != 0.0 ? x2 : (x1 != 0.0 ? x1 : x0));
        return (top > 0.0) - (top < 0.0);
    }
    const double la[4] = {acx, acx, acxt, acxt};
    const double lb[4] = {bcy, bcyt, bcy, bcyt};
    const double ra[4] = {acy, acy, acyt, acyt};
    const double rb[4] = {bcx, bcxt, bcx, bcxt};
    double e[34], f[34];
    double* cur = e;
    double* nxt = f;
    int n = 0;
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
        // a pair of products with a zero factor each adds nothing: skipping it
        // leaves the expansion (and so the sign) unchanged.  When the four
        // differences are exact (their tails are zero, as for lattice or
        // nearby inputs) only k = 0 remains.
        if ((la[k] == 0.0 || lb[k] == 0.0) && (ra[k] == 0.0 || rb[k] == 0.0)) continue;
        double p, q, t[4];
        two_product(la[k], lb[k], p, q);
        t[0] = q;
        t[1] = p;
        two_product(ra[k], rb[k], p, q);
        t[2] = -q;
        t[3] = -p;
#pragma unroll 1
        for (int m = 0; m < 4; ++m) {
            n = grow_expansion(n, cur, t[m], nxt);
            double* s = cur;
            cur = nxt;
            nxt = s;
        }
    }
    if (n == 0) return 0;
    const double top = cur[n - 1];
    return (top > 0.0) - (top < 0.0);
}

// Shewchuk's stage-A bound (3 + 16 eps) eps with eps = 2^-53.
constexpr double kCcwErrBoundA = 3.3306690738754716e-16;

// Exact orientation sign; counts calls that needed the exact stage.
__device__ __forceinline__ int orient2d(double ax, double ay, double bx, double by,
                                        double cx, double cy, unsigned& n_exact) {
    const double acx = __dsub_rn(ax, cx), bcx = __dsub_rn(bx, cx);
    const double acy = __dsub_rn(ay, cy), bcy = __dsub_rn(by, cy);
    const double l = __dmul_rn(acx, bcy), r = __dmul_rn(acy, bcx);
    const double det = __dsub_rn(l, r);
    const double bound = __dmul_rn(kCcwErrBoundA, __dadd_rn(fabs(l), fabs(r)));
    if (det > bound) return 1;
    if (-det > bound) return -1;
    ++n_exact;
    return orient2d_exact(ax, ay, bx, by, cx, cy);
}

// One edge (a -> b) of the crossing-number walk, decided exactly.  Returns
// true if the point lies on the edge (boundary); otherwise toggles `inside`
// when the +x ray from the point crosses the edge.  Same decision sequence as
// the reference's vs_ring_point_classify loop body.
__device__ __forceinline__ bool edge_step_exact(double ax, double ay, double bx, double by, double px, double py,
                                                bool& inside, unsigned& n_exact) {
    const bool crosses = (ay > py) != (by > py);
    const double minx = fmin(ax, bx), maxx = fmax(ax, bx);
    const bool on_bbox = py >= fmin(ay, by) && py <= fmax(ay, by) && px >= minx && px <= maxx;
    if (!crosses && !on_bbox) return false;
    if (crosses && px < minx) {
        inside = !inside;
        return false;
    }
    if (crosses && px > maxx) return false;
    const int o = orient2d(ax, ay, bx, by, px, py, n_exact);
    if (on_bbox && o == 0) return true;
    if (crosses && ((o > 0) == (by > ay))) inside = !inside;
    return false;
}

// ---------------------------------------------------------------------------
// Filtered variants for the hot join kernels: identical decisions, but an
// orientation the stage-A filter cannot certify makes the whole pair
// UNDECIDED instead of calling the exact stage in line.  The join defers such
// pairs to a separate exact pass, which keeps the out-of-line call (and the
// register spills around it) out of the hot loops.
// ---------------------------------------------------------------------------
enum : int { LOC_UNDECIDED = -1 };

// +1 / -1 when the stage-A filter certifies the sign, 0 when it cannot.
__device__ __forceinline__ int orient2d_filter(double ax, double ay, double bx, double by, double cx, double cy) {
    const double acx = __dsub_rn(ax, cx), bcx = __dsub_rn(bx, cx);
    const double acy = __dsub_rn(ay, cy), bcy = __dsub_rn(by, cy);
    const double l = __dmul_rn(acx, bcy), r = __dmul_rn(acy, bcx);
    const double det = __dsub_rn(l, r);
    const double bound = __dmul_rn(kCcwErrBoundA, __dadd_rn(fabs(l), fabs(r)));
    return det > bound ? 1 : (-det > bound ? -1 : 0);
}

// 0: decided, not on the edge; 1: on the edge (boundary); 2: undecided.
__device__ __forceinline__ int edge_step_filtered(double ax, double ay, double bx, double by, double px, double py,
                                                  bool& inside) {
    const bool crosses = (ay > py) != (by > py);
    const double minx = fmin(ax, bx), maxx = fmax(ax, bx);
    const bool on_bbox = py >= fmin(ay, by) && py <= fmax(ay, by) && px >= minx && px <= maxx;
    if (!crosses && !on_bbox) return 0;
    if (crosses && px < minx) {
        inside = !inside;
        return 0;
    }
    if (crosses && px > maxx) return 0;
    const int o = orient2d_filter(ax, ay, bx, by, px, py);
    if (o == 0) return 2;
    if (crosses && ((o > 0) == (by > ay))) inside = !inside;
    return 0;
}

// Walk only the edges of the point's y-bin when the ring has bins; `Step`
// decides one edge (a -> b) and returns 0 to go on, or a nonzero code that
// ends the walk and is returned.
template <class Step>
__device__ __forceinline__ int ring_walk(double py, const double2* __restrict__ xy, int start, int end, int ring,
                                         const RingIndex& ri, bool& inside, Step step) {
    const int rb = ri.ring_bin ? ri.ring_bin[ring] : -1;
    if (rb >= 0) {
        const RingBins& b = ri.bins[rb];
        const int k = ring_bin_of(py, b.y0, b.scale);
        const uint32_t e1 = b.off[k + 1];
        int last = -2;  // an edge that continues the previous one reuses its end vertex
        double2 lb = make_double2(0.0, 0.0);
        for (uint32_t e = b.off[k]; e < e1; ++e) {
            const int i = start + ri.edges[e];
            const int ia = i == start ? end - 1 : i - 1;
            const double2 A = ia == last ? lb : xy[ia], B = xy[i];
            const int r = step(A, B, inside);
            if (r) return r;
            last = i;
            lb = B;
        }
        return 0;
    }
    double2 a = xy[end - 1];
    for (int i = start; i < end; ++i) {
        const double2 b = xy[i];
        const int r = step(a, b, inside);
        if (r) return r;
        a = b;
    }
    return 0;
}

__device__ __forceinline__ int ring_location_filtered(double px, double py, const double2* __restrict__ xy, int start,
                                                      int end, int ring, const RingIndex& ri) {
    if (end - start < 2) return LOC_OUTSIDE;
    bool inside = false;
    // step codes: 1 on the edge, 2 undecided by the filter
    const int r = ring_walk(py, xy, start, end, ring, ri, inside, [&](const double2& A, const double2& B, bool& in) {
        return edge_step_filtered(A.x, A.y, B.x, B.y, px, py, in);
    });
    if (r == 1) return LOC_BOUNDARY;
    if (r == 2) return LOC_UNDECIDED;
    return inside ? LOC_INTERIOR : LOC_OUTSIDE;
}

__device__ __forceinline__ int geometry_location_filtered(double px, double py, const double2* __restrict__ xy,
                                                          const int32_t* __restrict__ ring_off,
                                                          const int32_t* __restrict__ part_off,
                                                          const int32_t* __restrict__ geom_off, int g,
                                                          const RingIndex& ri) {
    const int p0 = geom_off[g], p1 = geom_off[g + 1];
    for (int part = p0; part < p1; ++part) {
        bool inside = false;
        const int r0 = part_off[part], r1 = part_off[part + 1];
        for (int ring = r0; ring < r1; ++ring) {
            const int k = ring_location_filtered(px, py, xy, ring_off[ring], ring_off[ring + 1], ring, ri);
            if (k == LOC_BOUNDARY || k == LOC_UNDECIDED) return k;
            if (k == LOC_INTERIOR) inside = !inside;
        }
        if (inside) return LOC_INTERIOR;
    }
    return LOC_OUTSIDE;
}

// Ring walk over interleaved vertices xy[start, end); the edge (end-1 -> start)
// closes the ring exactly as in the reference's (i, j = i - 1) loop.
__device__ __forceinline__ int ring_location(double px, double py, const double2* __restrict__ xy,
                                             int start, int end, int ring, const RingIndex& ri, unsigned& n_exact) {
    if (end - start < 2) return LOC_OUTSIDE;
    bool inside = false;
    const int r = ring_walk(py, xy, start, end, ring, ri, inside, [&](const double2& A, const double2& B, bool& in) {
        return edge_step_exact(A.x, A.y, B.x, B.y, px, py, in, n_exact) ? 1 : 0;
    });
    if (r) return LOC_BOUNDARY;
    return inside ? LOC_INTERIOR : LOC_OUTSIDE;
}

// Same walk over separate x[] / y[] arrays (caller-layout inputs).
__device__ __forceinline__ int ring_location_soa(double px, double py, const double* __restrict__ x,
                                                 const double* __restrict__ y, int start, int end,
                                                 unsigned& n_exact) {
    if (end - start < 2) return LOC_OUTSIDE;
    bool inside = false;
    double ax = x[end - 1], ay = y[end - 1];
    for (int i = start; i < end; ++i) {
        const double bx = x[i], by = y[i];
        if (edge_step_exact(ax, ay, bx, by, px, py, inside, n_exact)) return LOC_BOUNDARY;
        ax = bx;
        ay = by;
    }
    return inside ? LOC_INTERIOR : LOC_OUTSIDE;
}

// Location of a point in polygonal geometry g (a Polygon is a one-part
// MultiPolygon): geom_off -> parts, part_off -> rings, ring_off -> vertices.
__device__ __forceinline__ int geometry_location(double px, double py, const double2* __restrict__ xy,
                                                 const int32_t* __restrict__ ring_off,
                                                 const int32_t* __restrict__ part_off,
                                                 const int32_t* __restrict__ geom_off, int g,
                                                 const RingIndex& ri, unsigned& n_exact) {
    const int p0 = geom_off[g], p1 = geom_off[g + 1];
    for (int part = p0; part < p1; ++part) {
        bool inside = false;
        const int r0 = part_off[part], r1 = part_off[part + 1];
        for (int ring = r0; ring < r1; ++ring) {
            const int k = ring_location(px, py, xy, ring_off[ring], ring_off[ring + 1], ring, ri, n_exact);
            if (k == LOC_BOUNDARY) return LOC_BOUNDARY;
            if (k == LOC_INTERIOR) inside = !inside;
        }
        if (inside) return LOC_INTERIOR;
    }
    return LOC_OUTSIDE;
}

__device__ __forceinline__ int geometry_location_soa(double px, double py, const double* __restrict__ x,
                                                     const double* __restrict__ y,
                                                     const int32_t* __restrict__ ring_off,
                                                     const int32_t* __restrict__ part_off,
                                                     const int32_t* __restrict__ geom_off, int g,
                                                     unsigned& n_exact) {
    const int p0 = geom_off[g], p1 = geom_off[g + 1];
    for (int part = p0; part < p1; ++part) {
        bool inside = false;
        const int r0 = part_off[part], r1 = part_off[part + 1];
        for (int ring = r0; ring < r1; ++ring) {
            const int k = ring_location_soa(px, py, x, y, ring_off[ring], ring_off[ring + 1], n_exact);
            if (k == LOC_BOUNDARY) return LOC_BOUNDARY;
            if (k == LOC_INTERIOR) inside = !inside;
        }
        if (inside) return LOC_INTERIOR;
    }
    return LOC_OUTSIDE;
}

}  // namespace vs
