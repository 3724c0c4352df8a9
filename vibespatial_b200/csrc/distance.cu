// Distance joins of points against the polygon index: dwithin
// (sjoin(predicate='dwithin'), sindex.query(..., predicate='dwithin')) and
// nearest (sjoin_nearest).
//
// Reference behaviour replaced (src/vibespatial/...):
//   spatial/query.py:663-810         dwithin: bbox candidates with the query
//       bounds expanded by the distance, then _dwithin_refine_gpu
//       (spatial/nearest.py:2855): a distance per candidate pair
//       (spatial/point_distance_kernels.py:238-310), then distance <= threshold
//   api/tools/sjoin.py sjoin_nearest -> spatial/nearest.py (query_nearest with
//       all ties, max_distance, distances)
//
// Distance arithmetic.  distance(point, polygon) is 0 when the point is
// inside or on the polygon (exact location, exact.cuh); otherwise it is the
// minimum over every ring segment of the point-segment distance of the
// comp.graphics.algorithms FAQ, the method GEOS's Distance::pointToSegment
// uses:
//   A == B            -> |p - A|
//   r = ((p - A).(B - A)) / |B - A|^2;  r <= 0 -> |p - A|;  r >= 1 -> |p - B|
//   otherwise         -> |s| * sqrt(|B - A|^2),
//                        s = ((A.y - p.y)(B.x - A.x) - (A.x - p.x)(B.y - A.y)) / |B - A|^2
// with |u| = sqrt(u.x^2 + u.y^2).  dwithin first applies the envelope
// short-circuit (envelope distance > d -> false), then distance <= d.  Every
// operation is rounded on its own (__dmul_rn, __dadd_rn, ...: no FMA
// contraction), so an IEEE host evaluating the same expressions without
// contraction gets the same bits.
//
// Candidates come from the packed Hilbert R-tree, walked by warp packets as
// in the plain join (join.cu) with every point's box inflated by its search
// radius (rounded outward, plus a relative 2^-30 margin, so no polygon within
// the radius can be missed); the exact test above decides every candidate.
//
// Nearest (all ties), two walks.  The first finds each point's minimum: a
// greedy descent per point (at every level the child box nearest to the
// point, then the nearest item box) gives an upper bound; the walk then
// visits, nearest first, only what lies within each point's current minimum
// (capped by max_distance) -- a polygon nearer than the minimum is always
// inside that box -- and the packet's box shrinks as the minima drop.  The
// second walk emits every polygon at exactly the minimum.
// Candidates whose envelope is certainly farther than the bound are skipped
// before the exact distance.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "emit.cuh"
#include "exact.cuh"
#include "hilbert.cuh"
#include "index.cuh"
#include "join.cuh"
#include "primitives.cuh"
#include "vs_common.cuh"

namespace vs {
namespace {

constexpr int kDistThreads = 256;
constexpr int kDistWarps = kDistThreads / 32;
constexpr int kDistStack = 112;
constexpr int kDistMaxStaged = 273;
constexpr int64_t kDistGrab = 32;

enum : int { kDwithin = 0, kNearestMin = 1, kNearestEmit = 2 };

__device__ __forceinline__ double point_point_distance(double px, double py, double ax, double ay) {
    const double dx = __dsub_rn(px, ax), dy = __dsub_rn(py, ay);
    return __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
}

__device__ __forceinline__ double point_segment_distance(double px, double py, double ax, double ay, double bx,
                                                         double by) {
    if (ax == bx && ay == by) return point_point_distance(px, py, ax, ay);
    const double ux = __dsub_rn(bx, ax), uy = __dsub_rn(by, ay);
    const double len2 = __dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy));
    const double r = __ddiv_rn(__dadd_rn(__dmul_rn(__dsub_rn(px, ax), ux), __dmul_rn(__dsub_rn(py, ay), uy)), len2);
    if (r <= 0.0) return point_point_distance(px, py, ax, ay);
    if (r >= 1.0) return point_point_distance(px, py, bx, by);
    const double s =
        __ddiv_rn(__dsub_rn(__dmul_rn(__dsub_rn(ay, py), ux), __dmul_rn(__dsub_rn(ax, px), uy)), len2);
    return __dmul_rn(fabs(s), __dsqrt_rn(len2));
}

// Distance between the point and a polygon envelope (GEOS Envelope::distance
// with the point's degenerate envelope).
__device__ __forceinline__ double envelope_distance(const vs_box& b, double px, double py) {
    double dx = 0.0, dy = 0.0;
    if (px < b.minx) dx = __dsub_rn(b.minx, px);
    else if (px > b.maxx) dx = __dsub_rn(px, b.maxx);
    if (py < b.miny) dy = __dsub_rn(b.miny, py);
    else if (py > b.maxy) dy = __dsub_rn(py, b.maxy);
    if (dx == 0.0) return dy;
    if (dy == 0.0) return dx;
    return __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
}

// Minimum segment distance over all rings of slot g; stops early once a
// segment is within `stop` (the minimum's comparison with `stop` is then
// already decided).
__device__ double facet_distance(double px, double py, const double2* __restrict__ xy,
                                 const int32_t* __restrict__ ring_off, const int32_t* __restrict__ part_off,
                                 const int32_t* __restrict__ geom_off, int g, double stop) {
    double best = INFINITY;
    const int r0 = part_off[geom_off[g]], r1 = part_off[geom_off[g + 1]];
    for (int ring = r0; ring < r1; ++ring) {
        const int c0 = ring_off[ring], c1 = ring_off[ring + 1];
        if (c1 - c0 < 2) continue;
        double2 a = xy[c0];
        for (int c = c0 + 1; c < c1; ++c) {
            const double2 b = xy[c];
            const double d = point_segment_distance(px, py, a.x, a.y, b.x, b.y);
            best = d < best ? d : best;
            if (best <= stop) return best;
            a = b;
        }
    }
    return best;
}

struct DistArgs {
    const double* px;
    const double* py;
    const uint32_t* order;   // sorted position -> point row
    const uint32_t* list;    // positions to visit (nullable: every position below *n_list)
    const uint32_t* n_list;
    const vs_box* nodes;
    int64_t level_off[kMaxLevels];
    int64_t level_size[kMaxLevels];
    int levels;
    int stage_level;
    int staged;
    const int32_t* item_geom;
    const int32_t* geom_off;
    const int32_t* part_off;
    const int32_t* ring_off;
    const double2* xy;
    RingIndex rings;
    const double* dist_pt;    // dwithin: per point row (nullable)
    const double* dist_geom;  // dwithin: per polygon row (nullable)
    double dist_scalar;       // dwithin: the distance, or the largest per-polygon one
    double radius;            // nearest, min pass: the search radius of this pass
    double* best;             // nearest: per point row minimum distance
    PairSink sink;
    unsigned long long* counters;
    unsigned long long* work;
};

// Search radius rounded outward with a relative margin: a polygon whose
// computed distance is within q has its envelope within inflate(q).
__device__ __forceinline__ double inflate(double q) {
    return __dadd_ru(__dadd_ru(q, __dmul_ru(q, 0x1p-30)), 0x1p-1000);
}

__device__ __forceinline__ vs_box load_node(const DistArgs& a, const vs_box* s_nodes, int64_t stage_base, int cl,
                                            int64_t c) {
    return cl >= a.stage_level ? s_nodes[a.level_off[cl] - stage_base + c] : a.nodes[a.level_off[cl] + c];
}

// Squared distance from (x, y) to a box (plain rounding: only steers the
// greedy descent and the walk's order).
__device__ __forceinline__ double box_dist2(const vs_box& b, double x, double y) {
    const double dx = fmax(fmax(b.minx - x, x - b.maxx), 0.0);
    const double dy = fmax(fmax(b.miny - y, y - b.maxy), 0.0);
    return dx * dx + dy * dy;
}

// Descent key of the greedy bound: the box distance, plus the distance to
// the box centre so that of several boxes containing the point the one
// centred nearest to it wins.
__device__ __forceinline__ double descent_key(const vs_box& b, double x, double y) {
    const double cx = 0.5 * (b.minx + b.maxx) - x, cy = 0.5 * (b.miny + b.maxy) - y;
    return box_dist2(b, x, y) + cx * cx + cy * cy;
}

// Exact point-polygon distance of slot g (0 inside or on the boundary).  Out
// of line: the nearest walks call it from two places, and one shared copy of
// the exact location keeps them smaller (measured: the min walk stalls on
// instruction fetch, and 118.7 -> 91.6 ms on Zipf 50M x 1M).
__device__ __noinline__ double polygon_distance(const DistArgs& a, double x, double y, int g, unsigned& n_exact) {
    const int loc = geometry_location(x, y, a.xy, a.ring_off, a.part_off, a.geom_off, g, a.rings, n_exact);
    return loc != LOC_OUTSIDE ? 0.0 : facet_distance(x, y, a.xy, a.ring_off, a.part_off, a.geom_off, g, -1.0);
}

// Warp-packet R-tree walk of the distance joins.
//   kDwithin      per lane radius d (per point / per polygon / scalar); emits
//                 the pairs within it
//   kNearestMin   per lane minimum distance: each lane's greedy descent
//                 (level by level the child box nearest to its point, ties
//                 broken by the box centre, then the nearest item box) gives
//                 it an upper bound; the walk then
//                 visits, nearest to the packet's centroid first, what lies
//                 within each lane's current minimum (capped by max_distance
//                 in a.radius), the packet's box shrinking as the minima
//                 drop; writes best[row]
//   kNearestEmit  radius best[row]; emits every polygon at exactly that distance
// A dwithin candidate that passed the envelope test, queued for the exact test.
struct DwPair {
    double x, y, d;
    int32_t row, slot;
};

template <int kMode>
__global__ void __launch_bounds__(kDistThreads) dist_join_kernel(const DistArgs a) {
    constexpr int kQ = kMode != kNearestMin ? 64 : 1;
    extern __shared__ vs_box s_nodes[];
    __shared__ int2 s_buf[kDistWarps][kWarpBuf];
    __shared__ unsigned s_cnt[kDistWarps];
    __shared__ int s_stack[kDistWarps][kDistStack];
    __shared__ vs_box s_items[kDistWarps][kFanout];
    __shared__ DwPair s_dq[kDistWarps][kQ];
    const int64_t stage_base = a.level_off[a.stage_level];
    for (int k = threadIdx.x; k < a.staged; k += blockDim.x) s_nodes[k] = a.nodes[stage_base + k];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_cnt[warp] = 0;
    __syncthreads();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    // dwithin and the tie walk: candidates that passed the envelope test queue
    // up here and are decided 32 at a time, one per lane, so the exact tests
    // run with every lane busy whichever lanes' boxes the candidates fell in
    // (d is the radius, or the lane's minimum for the tie walk)
    DwPair* dq = s_dq[warp];
    int nq = 0;  // warp-uniform
    unsigned n_exact_q = 0;
    auto drain = [&](int cnt) {
        bool want = false;
        int32_t prow = 0, pgeom = 0;
        if (lane < cnt) {
            const DwPair e = dq[lane];
            if (kMode == kDwithin)
                want = geometry_location(e.x, e.y, a.xy, a.ring_off, a.part_off, a.geom_off, e.slot, a.rings,
                                         n_exact_q) != LOC_OUTSIDE ||
                       facet_distance(e.x, e.y, a.xy, a.ring_off, a.part_off, a.geom_off, e.slot, e.d) <= e.d;
            else
                want = polygon_distance(a, e.x, e.y, e.slot, n_exact_q) == e.d;
            prow = e.row;
            pgeom = a.item_geom[e.slot];
        }
        wemit_sync(out, a.sink, want, prow, pgeom);
    };
    const unsigned lt = (1u << lane) - 1u;
    const int top = a.levels - 1;
    const int64_t n = (int64_t)*a.n_list;
    unsigned long long n_cand = 0;
    unsigned n_exact = 0;
    for (;;) {
        const int64_t b0 = warp_grab(a.work, kDistGrab);
        if (b0 >= n) break;
        const int64_t i = b0 + lane;
        bool active = i < n;
        double x = 0.0, y = 0.0, q = 0.0;
        int32_t row = -1;
        if (active) {
            const uint32_t pos = a.list ? a.list[i] : (uint32_t)i;
            row = (int32_t)a.order[pos];
            x = a.px[row];
            y = a.py[row];
            if (kMode == kDwithin) q = a.dist_pt ? a.dist_pt[row] : a.dist_scalar;
            else if (kMode == kNearestMin) q = a.radius;  // the cap (max_distance or INFINITY)
            else q = a.best[row];
            // a negative or NaN radius matches nothing; nearest emits only finite minima
            active = q >= 0.0 && (kMode != kNearestEmit || q < INFINITY);
        }
        double my_best = INFINITY;  // nearest, min pass
        double cx = 0.0, cy = 0.0;  // nearest, min pass: the packet's centroid
        if (kMode == kNearestMin && __any_sync(0xffffffffu, active)) {
            // the packet's centroid orders the walk below
            double sx = active ? x : 0.0, sy = active ? y : 0.0;
            int cnt = active ? 1 : 0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                sx += __shfl_xor_sync(0xffffffffu, sx, o);
                sy += __shfl_xor_sync(0xffffffffu, sy, o);
                cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            }
            cx = sx / cnt;
            cy = sy / cnt;
            // every lane descends on its own: at each level the child box nearest to
            // its point, then the exact distance to the nearest item box of the
            // leaf block reached -- an upper bound of the lane's minimum
            if (active) {
                int64_t node = 0;
                bool ok = true;
                for (int cl = top - 1; cl >= 1 && ok; --cl) {
                    const int64_t first = node * kFanout;
                    const int64_t last = first + kFanout < a.level_size[cl] ? first + kFanout : a.level_size[cl];
                    double bd = INFINITY;
                    int64_t bc = -1;
                    for (int64_t c = first; c < last; ++c) {
                        const vs_box b = load_node(a, s_nodes, stage_base, cl, c);
                        if (!(b.minx <= b.maxx)) continue;
                        const double d = descent_key(b, x, y);
                        if (d < bd) {
                            bd = d;
                            bc = c;
                        }
                    }
                    ok = bc >= 0;
                    node = bc;
                }
                if (ok) {
                    const int64_t first = top == 0 ? 0 : node * kFanout;
                    const int64_t last = top == 0 ? 1 : (first + kFanout < a.level_size[0] ? first + kFanout
                                                                                          : a.level_size[0]);
                    double bd = INFINITY;
                    int64_t bi = -1;
                    for (int64_t c = first; c < last; ++c) {
                        const vs_box b = a.nodes[a.level_off[0] + c];
                        if (!(b.minx <= b.maxx)) continue;
                        const double d = descent_key(b, x, y);
                        if (d < bd) {
                            bd = d;
                            bi = c;
                        }
                    }
                    if (bi >= 0) my_best = polygon_distance(a, x, y, (int)bi, n_exact);
                }
            }
        }
        // per lane search box and the packet's union box
        double lx0, lx1, ly0, ly1, x0, x1, y0, y1;
        auto boxes = [&]() {
            const double r = kMode == kNearestMin ? fmin(my_best, q) : q;
            const double qi = active ? inflate(r) : 0.0;
            lx0 = active ? __dsub_rd(x, qi) : INFINITY;
            lx1 = active ? __dadd_ru(x, qi) : -INFINITY;
            ly0 = active ? __dsub_rd(y, qi) : INFINITY;
            ly1 = active ? __dadd_ru(y, qi) : -INFINITY;
            x0 = lx0, x1 = lx1, y0 = ly0, y1 = ly1;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                x0 = fmin(x0, __shfl_xor_sync(0xffffffffu, x0, o));
                x1 = fmax(x1, __shfl_xor_sync(0xffffffffu, x1, o));
                y0 = fmin(y0, __shfl_xor_sync(0xffffffffu, y0, o));
                y1 = fmax(y1, __shfl_xor_sync(0xffffffffu, y1, o));
            }
        };
        boxes();
        int sp = 0;
        if (__any_sync(0xffffffffu, active)) {
            if (lane == 0) s_stack[warp][0] = top;
            sp = 1;
        }
        __syncwarp();
        while (sp > 0) {
            --sp;
            const int e = s_stack[warp][sp];
            __syncwarp();
            const int cl = e & 15;
            const int64_t c = (int64_t)(e >> 4) * kFanout + (lane & 15);
            // the root level has one node; below it 16 children per node
            const bool root = cl == top;
            const bool in_range = root ? lane == 0 : (lane < kFanout && c < a.level_size[cl]);
            const int64_t cc = root ? 0 : c;
            vs_box b{INFINITY, INFINITY, -INFINITY, -INFINITY};
            if (in_range) b = load_node(a, s_nodes, stage_base, cl, cc);
            const bool hit = in_range && b.minx <= x1 && b.maxx >= x0 && b.miny <= y1 && b.maxy >= y0;
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (cl > 0) {
                // push the hit nodes' children blocks: node cc of level cl owns block cc of level cl - 1
                int rank = __popc(m & lt);
                if (kMode == kNearestMin) {
                    // nearest to the packet's centroid on top of the stack: the first
                    // leaves reached shrink the minima, and the boxes with them
                    const double key = hit ? box_dist2(b, cx, cy) : INFINITY;
                    int closer = 0;
#pragma unroll
                    for (int j = 0; j < kFanout; ++j) {
                        const double kj = __shfl_sync(0xffffffffu, key, j);
                        closer += ((m >> j) & 1u) && (kj < key || (kj == key && j < lane)) ? 1 : 0;
                    }
                    rank = __popc(m) - 1 - closer;
                }
                if (hit) {
                    const int pos = sp + rank;
                    if (pos < kDistStack) s_stack[warp][pos] = (int)(cc << 4) | (cl - 1);
                }
                int add = __popc(m);
                if (sp + add > kDistStack) {
                    if (lane == 0) atomicOr(&a.counters[4], 1ull);
                    add = kDistStack - sp;
                }
                sp += add;
                __syncwarp();
            } else {
                if (lane < kFanout) s_items[warp][lane] = b;
                __syncwarp();
                unsigned mm = m;
                const int64_t slot0 = root ? 0 : (int64_t)(e >> 4) * kFanout;
                while (mm) {
                    const int j = __ffs(mm) - 1;
                    mm &= mm - 1;
                    const vs_box ib = s_items[warp][j];
                    const int slot = (int)(slot0 + j);
                    bool queue = false;
                    double qd = 0.0;
                    if (active && ib.minx <= lx1 && ib.maxx >= lx0 && ib.miny <= ly1 && ib.maxy >= ly0) {
                        ++n_cand;
                        if (kMode == kDwithin) {
                            qd = a.dist_geom ? a.dist_geom[a.item_geom[slot]] : q;
                            queue = qd >= 0.0 && !(envelope_distance(ib, x, y) > qd);
                        } else {
                            // a polygon whose envelope is farther than the bound (with a
                            // margin above the rounding of both distances) can neither
                            // lower the minimum nor tie it
                            const double bound = kMode == kNearestMin ? my_best : q;
                            // (a minimum of 0 cannot drop further: the min walk skips the rest)
                            if ((kMode != kNearestMin || my_best > 0.0) &&
                                !(envelope_distance(ib, x, y) > bound * (1.0 + 0x1p-40))) {
                                if (kMode == kNearestMin) {
                                    const double d = polygon_distance(a, x, y, slot, n_exact);
                                    my_best = d < my_best ? d : my_best;
                                } else {
                                    queue = true;
                                    qd = q;
                                }
                            }
                        }
                    }
                    if (kMode != kNearestMin) {
                        const unsigned qm = __ballot_sync(0xffffffffu, queue);
                        if (queue) dq[nq + __popc(qm & lt)] = DwPair{x, y, qd, row, slot};
                        nq += __popc(qm);
                        __syncwarp();
                        if (nq >= 32) {
                            drain(32);
                            __syncwarp();
                            if (lane < nq - 32) dq[lane] = dq[32 + lane];
                            nq -= 32;
                            __syncwarp();
                        }
                    }
                }
                __syncwarp();
                if (kMode == kNearestMin) boxes();  // the minima only shrink: so does the packet's box
            }
        }
        if (kMode == kNearestMin && active) a.best[row] = my_best <= q ? my_best : INFINITY;
        if (kMode != kNearestMin) wflush(out, a.sink, false);
    }
    if (kMode != kNearestMin && nq > 0) {
        drain(nq);
        __syncwarp();
    }
    if (kMode != kNearestMin) wflush(out, a.sink, true);
    add_counter(a.counters, 5, n_cand);
    add_counter(a.counters, 1, n_exact + n_exact_q);
}

// Element-wise: row i of the points against row i of the polygons (SoA
// inputs).  dist = the point-polygon distance, env = the envelope distance
// (GEOS's dwithin short-circuit); NaN for null / NaN points, null polygons
// and polygons without vertices.
__global__ void distance_aligned_kernel(vs_points pts, vs_polygons polys, double* __restrict__ dist,
                                        double* __restrict__ env, unsigned long long* counters) {
    unsigned n_exact = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < pts.n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool pv = pts.d_valid == nullptr || pts.d_valid[i];
        const bool gv = polys.d_valid == nullptr || polys.d_valid[i];
        const double x = pts.d_x[i], y = pts.d_y[i];
        double d = NAN, e = NAN;
        if (pv && gv && !isnan(x) && !isnan(y)) {
            const int g = (int)i;
            const int r0 = polys.d_part_off[polys.d_geom_off[g]], r1 = polys.d_part_off[polys.d_geom_off[g + 1]];
            const int c0 = polys.d_ring_off[r0], c1 = polys.d_ring_off[r1];
            if (c1 > c0) {
                vs_box b{INFINITY, INFINITY, -INFINITY, -INFINITY};
                for (int c = c0; c < c1; ++c) {
                    b.minx = fmin(b.minx, polys.d_x[c]);
                    b.miny = fmin(b.miny, polys.d_y[c]);
                    b.maxx = fmax(b.maxx, polys.d_x[c]);
                    b.maxy = fmax(b.maxy, polys.d_y[c]);
                }
                e = envelope_distance(b, x, y);
                const int loc = geometry_location_soa(x, y, polys.d_x, polys.d_y, polys.d_ring_off, polys.d_part_off,
                                                      polys.d_geom_off, g, n_exact);
                if (loc != LOC_OUTSIDE) {
                    d = 0.0;
                } else {
                    d = INFINITY;
                    for (int ring = r0; ring < r1; ++ring) {
                        const int a0 = polys.d_ring_off[ring], a1 = polys.d_ring_off[ring + 1];
                        for (int c = a0 + 1; c < a1; ++c) {
                            const double s = point_segment_distance(x, y, polys.d_x[c - 1], polys.d_y[c - 1],
                                                                    polys.d_x[c], polys.d_y[c]);
                            d = s < d ? s : d;
                        }
                    }
                }
            }
        }
        dist[i] = d;
        if (env) env[i] = e;
    }
    if (n_exact) atomicAdd(&counters[1], (unsigned long long)n_exact);
}

__global__ void gather_pair_distance_kernel(const int32_t* __restrict__ left, int64_t n,
                                            const double* __restrict__ best, double* __restrict__ out) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = best[left[i]];
}

// Largest non-NaN value (as an order-preserving integer; all inputs >= 0 or
// negative values that never match).
__global__ void max_distance_kernel(const double* __restrict__ d, int64_t n, unsigned long long* __restrict__ out) {
    long long m = dbl_to_ordered(-INFINITY);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = d[i];
        if (v == v) {
            const long long k = dbl_to_ordered(v);
            m = k > m ? k : m;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const long long t = __shfl_xor_sync(0xffffffffu, m, o);
        m = t > m ? t : m;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<long long*>(out), m);
}

DistArgs dist_args(vs_context* ctx, const vs_index* idx, const vs_points* pts, const QueryOrder& q, size_t* smem) {
    DistArgs a{};
    a.px = pts->d_x;
    a.py = pts->d_y;
    a.order = q.order.p;
    a.nodes = idx->nodes;
    for (int l = 0; l < kMaxLevels; ++l) {
        a.level_off[l] = idx->level_off[l];
        a.level_size[l] = idx->level_size[l];
    }
    a.levels = idx->levels;
    int sl = idx->levels - 1;
    int64_t staged = idx->level_size[sl];
    while (sl > 0 && staged + idx->level_size[sl - 1] <= kDistMaxStaged) {
        --sl;
        staged += idx->level_size[sl];
    }
    a.stage_level = sl;
    a.staged = (int)staged;
    a.item_geom = idx->item_geom;
    a.geom_off = idx->geom_off;
    a.part_off = idx->part_off;
    a.ring_off = idx->ring_off;
    a.xy = idx->xy;
    a.rings = idx->ring_index();
    a.counters = ctx->d_counters;
    a.work = &ctx->d_counters[kWorkCounter];
    *smem = (size_t)a.staged * sizeof(vs_box);
    return a;
}

template <int kMode>
int launch_dist(vs_context* ctx, const DistArgs& a, size_t smem, int64_t n_items) {
    cudaStream_t s = ctx->stream;
    VS_CUDA_TRY(cudaMemsetAsync(&ctx->d_counters[kWorkCounter], 0, sizeof(unsigned long long), s));
    auto* kernel = dist_join_kernel<kMode>;
    VS_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kernel<<<resident_grid(kernel, n_items > 0 ? n_items : 1, kDistThreads, smem), kDistThreads, smem, s>>>(a);
    VS_LAUNCHED(kMode == kDwithin ? "dist_join<dwithin>" : kMode == kNearestMin ? "dist_join<nearest_min>"
                                                                                : "dist_join<nearest_emit>",
                s);
    return VS_OK;
}

int check_join_args(vs_context* ctx, const vs_index* idx, const vs_points* pts, int32_t* d_left, int32_t* d_right,
                    int64_t capacity, int64_t* n_pairs) {
    if (!ctx || !idx || !n_pairs) {
        set_error("ctx/index/n_pairs is NULL");
        return VS_E_ARG;
    }
    *n_pairs = 0;
    VS_TRY(check_points(pts));
    if (capacity < 0 || (capacity > 0 && (!d_left || !d_right))) {
        set_error("invalid pair buffers (capacity %lld)", (long long)capacity);
        return VS_E_ARG;
    }
    if (idx->device != ctx->device) {
        set_error("index lives on device %d, context on device %d", idx->device, ctx->device);
        return VS_E_ARG;
    }
    if (pts->n > 0x7fffffffLL) {
        set_error("%lld points: more than the 32-bit rows address", (long long)pts->n);
        return VS_E_ARG;
    }
    return VS_OK;
}

// Counters after the passes: pair count, flags, capacity, stats.
int finish_join(vs_context* ctx, const vs_index* idx, const vs_points* pts, uint32_t flags, int32_t* d_left,
                int32_t* d_right, int64_t capacity, int64_t* n_pairs, vs_join_stats* stats, EventPair& ev,
                long long launches0) {
    cudaStream_t s = ctx->stream;
    cudaEventRecord(ev.b, s);
    VS_CUDA_TRY(cudaMemcpyAsync(ctx->h_counter, ctx->d_counters, 8 * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    const unsigned long long* c = ctx->h_counter;
    const int64_t n = (int64_t)c[0];
    *n_pairs = n;
    if (stats) {
        stats->exact_fallbacks = (int64_t)c[1];
        stats->candidates = (int64_t)c[5];
        stats->kernel_ms = ev.ms();
        stats->kernel_launches = g_launches - launches0;
    }
    if (c[4] != 0) {
        set_error("device-side consistency check failed (flags 0x%llx)", (unsigned long long)c[4]);
        return VS_E_STATE;
    }
    if (n > capacity) {
        set_error("pair buffer holds %lld pairs, %lld required", (long long)capacity, (long long)n);
        return VS_E_CAPACITY;
    }
    if ((flags & VS_JOIN_SORT) && n > 1) {
        EventPair es;
        cudaEventRecord(es.a, s);
        VS_TRY(sort_pairs(ctx, d_left, d_right, n, (uint64_t)pts->n, (uint64_t)idx->n_geoms));
        cudaEventRecord(es.b, s);
        VS_CUDA_TRY(cudaStreamSynchronize(s));
        if (stats) {
            stats->sort_ms = es.ms();
            stats->kernel_launches = g_launches - launches0;
        }
    }
    return VS_OK;
}

// ---------------------------------------------------------- reverse nearest
// Nearest points of every polygon (all ties).  The tree is an index over the
// points, each point a one-vertex polygon, so a level-0 box is the point
// itself; the queries are the polygons, in the Hilbert order of their
// envelope centres.  Same two walks as the point queries: a greedy bound, a
// nearest-first walk that keeps each lane's minimum, then the ties.

struct PolyArgs {
    const double* x;  // query polygons, original rows
    const double* y;
    const int32_t* ring_off;
    const int32_t* part_off;
    const int32_t* geom_off;
    const vs_box* qbox;         // envelopes (inverted for null / empty rows)
    const uint32_t* order;      // query rows, valid ones first
    const uint32_t* n_valid;
    const vs_box* nodes;        // the point index
    int64_t level_off[kMaxLevels];
    int64_t level_size[kMaxLevels];
    int levels;
    int stage_level;
    int staged;
    const int32_t* item_geom;   // slot -> point row
    double cap;                 // max_distance (INFINITY: unbounded)
    double* best;               // per query row
    PairSink sink;
    unsigned long long* counters;
    unsigned long long* work;
};

// Distance from a point to query polygon g (SoA, original row): 0 inside or
// on it, else the smallest point-segment distance over its rings.
__device__ double point_polygon_soa(const PolyArgs& a, double px, double py, int g, unsigned& n_exact) {
    if (geometry_location_soa(px, py, a.x, a.y, a.ring_off, a.part_off, a.geom_off, g, n_exact) != LOC_OUTSIDE)
        return 0.0;
    double best = INFINITY;
    const int r0 = a.part_off[a.geom_off[g]], r1 = a.part_off[a.geom_off[g + 1]];
    for (int ring = r0; ring < r1; ++ring) {
        const int c0 = a.ring_off[ring], c1 = a.ring_off[ring + 1];
        for (int c = c0 + 1; c < c1; ++c) {
            const double d = point_segment_distance(px, py, a.x[c - 1], a.y[c - 1], a.x[c], a.y[c]);
            best = d < best ? d : best;
        }
    }
    return best;
}

__device__ __forceinline__ vs_box load_pnode(const PolyArgs& a, const vs_box* s_nodes, int64_t stage_base, int cl,
                                             int64_t c) {
    return cl >= a.stage_level ? s_nodes[a.level_off[cl] - stage_base + c] : a.nodes[a.level_off[cl] + c];
}

// Query polygons: envelope, Hilbert key of its centre in the point frame
// (clamped; null / empty rows get the all-ones key and are counted out).
__global__ void poly_query_key_kernel(vs_polygons q, const double* __restrict__ frame, vs_box* __restrict__ qbox,
                                      uint32_t* __restrict__ keys, uint32_t* __restrict__ order,
                                      uint32_t* __restrict__ n_valid) {
    const double f0 = frame[0], f1 = frame[1], f2 = frame[2], f3 = frame[3];
    const double sx = f2 > f0 ? 4294967295.0 / (f2 - f0) : 0.0;
    const double sy = f3 > f1 ? 4294967295.0 / (f3 - f1) : 0.0;
    uint32_t cnt = 0;
    for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < q.n_geoms; g += (int64_t)gridDim.x * blockDim.x) {
        vs_box b{INFINITY, INFINITY, -INFINITY, -INFINITY};
        if (q.d_valid == nullptr || q.d_valid[g]) {
            const int c0 = q.d_ring_off[q.d_part_off[q.d_geom_off[g]]];
            const int c1 = q.d_ring_off[q.d_part_off[q.d_geom_off[g + 1]]];
            for (int c = c0; c < c1; ++c) {
                b.minx = fmin(b.minx, q.d_x[c]);
                b.miny = fmin(b.miny, q.d_y[c]);
                b.maxx = fmax(b.maxx, q.d_x[c]);
                b.maxy = fmax(b.maxy, q.d_y[c]);
            }
        }
        qbox[g] = b;
        const bool ok = b.minx <= b.maxx && b.miny <= b.maxy;
        uint32_t k = 0xffffffffu;
        if (ok) {
            const double cx = fmin(fmax(0.5 * (b.minx + b.maxx), f0), f2);
            const double cy = fmin(fmax(0.5 * (b.miny + b.maxy), f1), f3);
            k = (uint32_t)hilbert_key(quantize(cx, f0, sx), quantize(cy, f1, sy), 16);
            if (k == 0xffffffffu) k = 0xfffffffeu;
        }
        keys[g] = k;
        order[g] = (uint32_t)g;
        cnt += ok ? 1u : 0u;
    }
    cnt = (uint32_t)warp_sum(cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(n_valid, cnt);
}

template <bool kEmit>
__global__ void __launch_bounds__(kDistThreads) poly_nearest_kernel(const PolyArgs a) {
    constexpr int kQ = kEmit ? 64 : 1;
    extern __shared__ vs_box s_nodes[];
    __shared__ int2 s_buf[kDistWarps][kWarpBuf];
    __shared__ unsigned s_cnt[kDistWarps];
    __shared__ int s_stack[kDistWarps][kDistStack];
    __shared__ vs_box s_items[kDistWarps][kFanout];
    __shared__ DwPair s_dq[kDistWarps][kQ];
    const int64_t stage_base = a.level_off[a.stage_level];
    for (int k = threadIdx.x; k < a.staged; k += blockDim.x) s_nodes[k] = a.nodes[stage_base + k];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_cnt[warp] = 0;
    __syncthreads();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    const unsigned lt = (1u << lane) - 1u;
    const int top = a.levels - 1;
    const int64_t n = (int64_t)*a.n_valid;
    unsigned long long n_cand = 0;
    unsigned n_exact = 0;
    // tie walk: candidate points queue up here (point, the polygon's minimum,
    // polygon row, point slot) and are decided 32 at a time, one per lane
    DwPair* dq = s_dq[warp];
    int nq = 0;  // warp-uniform
    auto drain = [&](int cnt) {
        bool want = false;
        int32_t prow = 0, ppt = 0;
        if (lane < cnt) {
            const DwPair e = dq[lane];
            want = point_polygon_soa(a, e.x, e.y, e.row, n_exact) == e.d;
            prow = e.row;
            ppt = a.item_geom[e.slot];
        }
        wemit_sync(out, a.sink, want, prow, ppt);
    };
    for (;;) {
        const int64_t b0 = warp_grab(a.work, kDistGrab);
        if (b0 >= n) break;
        const int64_t i = b0 + lane;
        bool active = i < n;
        int32_t row = -1;
        vs_box qb{INFINITY, INFINITY, -INFINITY, -INFINITY};
        double q = 0.0;
        if (active) {
            row = (int32_t)a.order[i];
            qb = a.qbox[row];
            q = kEmit ? a.best[row] : a.cap;
            active = q >= 0.0 && (!kEmit || q < INFINITY);
        }
        const double mx = 0.5 * (qb.minx + qb.maxx), my = 0.5 * (qb.miny + qb.maxy);
        double my_best = INFINITY;
        double sx = active ? mx : 0.0, sy = active ? my : 0.0;
        int cnt = active ? 1 : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        }
        const double cx = cnt ? sx / cnt : 0.0, cy = cnt ? sy / cnt : 0.0;
        if (!kEmit && active) {
            // greedy descent towards the envelope centre, then the nearest point of the block
            int64_t node = 0;
            bool ok = true;
            for (int cl = top - 1; cl >= 1 && ok; --cl) {
                const int64_t first = node * kFanout;
                const int64_t last = first + kFanout < a.level_size[cl] ? first + kFanout : a.level_size[cl];
                double bd = INFINITY;
                int64_t bc = -1;
                for (int64_t c = first; c < last; ++c) {
                    const vs_box b = load_pnode(a, s_nodes, stage_base, cl, c);
                    if (!(b.minx <= b.maxx)) continue;
                    const double d = descent_key(b, mx, my);
                    if (d < bd) {
                        bd = d;
                        bc = c;
                    }
                }
                ok = bc >= 0;
                node = bc;
            }
            if (ok) {
                const int64_t first = top == 0 ? 0 : node * kFanout;
                const int64_t last = top == 0 ? 1 : (first + kFanout < a.level_size[0] ? first + kFanout
                                                                                      : a.level_size[0]);
                double bd = INFINITY;
                int64_t bi = -1;
                for (int64_t c = first; c < last; ++c) {
                    const vs_box b = a.nodes[a.level_off[0] + c];
                    if (!(b.minx <= b.maxx)) continue;
                    const double d = box_dist2(qb, b.minx, b.miny);
                    if (d < bd) {
                        bd = d;
                        bi = c;
                    }
                }
                if (bi >= 0) {
                    const vs_box b = a.nodes[a.level_off[0] + bi];
                    my_best = point_polygon_soa(a, b.minx, b.miny, row, n_exact);
                }
            }
        }
        double lx0, lx1, ly0, ly1, x0, x1, y0, y1;
        auto boxes = [&]() {
            const double r = kEmit ? q : fmin(my_best, q);
            const double qi = active ? inflate(r) : 0.0;
            lx0 = active ? __dsub_rd(qb.minx, qi) : INFINITY;
            lx1 = active ? __dadd_ru(qb.maxx, qi) : -INFINITY;
            ly0 = active ? __dsub_rd(qb.miny, qi) : INFINITY;
            ly1 = active ? __dadd_ru(qb.maxy, qi) : -INFINITY;
            x0 = lx0, x1 = lx1, y0 = ly0, y1 = ly1;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                x0 = fmin(x0, __shfl_xor_sync(0xffffffffu, x0, o));
                x1 = fmax(x1, __shfl_xor_sync(0xffffffffu, x1, o));
                y0 = fmin(y0, __shfl_xor_sync(0xffffffffu, y0, o));
                y1 = fmax(y1, __shfl_xor_sync(0xffffffffu, y1, o));
            }
        };
        boxes();
        int sp = 0;
        if (__any_sync(0xffffffffu, active)) {
            if (lane == 0) s_stack[warp][0] = top;
            sp = 1;
        }
        __syncwarp();
        while (sp > 0) {
            --sp;
            const int e = s_stack[warp][sp];
            __syncwarp();
            const int cl = e & 15;
            const int64_t c = (int64_t)(e >> 4) * kFanout + (lane & 15);
            const bool root = cl == top;
            const bool in_range = root ? lane == 0 : (lane < kFanout && c < a.level_size[cl]);
            const int64_t cc = root ? 0 : c;
            vs_box b{INFINITY, INFINITY, -INFINITY, -INFINITY};
            if (in_range) b = load_pnode(a, s_nodes, stage_base, cl, cc);
            const bool hit = in_range && b.minx <= x1 && b.maxx >= x0 && b.miny <= y1 && b.maxy >= y0;
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (cl > 0) {
                int rank = __popc(m & lt);
                if (!kEmit) {
                    // nearest to the packet's centre on top of the stack
                    const double key = hit ? box_dist2(b, cx, cy) : INFINITY;
                    int closer = 0;
#pragma unroll
                    for (int j = 0; j < kFanout; ++j) {
                        const double kj = __shfl_sync(0xffffffffu, key, j);
                        closer += ((m >> j) & 1u) && (kj < key || (kj == key && j < lane)) ? 1 : 0;
                    }
                    rank = __popc(m) - 1 - closer;
                }
                if (hit) {
                    const int pos = sp + rank;
                    if (pos < kDistStack) s_stack[warp][pos] = (int)(cc << 4) | (cl - 1);
                }
                int add = __popc(m);
                if (sp + add > kDistStack) {
                    if (lane == 0) atomicOr(&a.counters[4], 1ull);
                    add = kDistStack - sp;
                }
                sp += add;
                __syncwarp();
            } else {
                if (lane < kFanout) s_items[warp][lane] = b;
                __syncwarp();
                unsigned mm = m;
                const int64_t slot0 = root ? 0 : (int64_t)(e >> 4) * kFanout;
                while (mm) {
                    const int j = __ffs(mm) - 1;
                    mm &= mm - 1;
                    const vs_box ib = s_items[warp][j];  // a point: (x, y, x, y)
                    const int slot = (int)(slot0 + j);
                    bool queue = false;
                    if (active && ib.minx <= lx1 && ib.maxx >= lx0 && ib.miny <= ly1 && ib.maxy >= ly0) {
                        ++n_cand;
                        const double bound = kEmit ? q : my_best;
                        // (a minimum of 0 cannot drop further: the min walk skips the rest)
                        if ((kEmit || my_best > 0.0) &&
                            !(envelope_distance(qb, ib.minx, ib.miny) > bound * (1.0 + 0x1p-40))) {
                            if (kEmit) {
                                queue = true;
                            } else {
                                const double d = point_polygon_soa(a, ib.minx, ib.miny, row, n_exact);
                                my_best = d < my_best ? d : my_best;
                            }
                        }
                    }
                    if (kEmit) {
                        const unsigned qm = __ballot_sync(0xffffffffu, queue);
                        if (queue) dq[nq + __popc(qm & lt)] = DwPair{ib.minx, ib.miny, q, row, slot};
                        nq += __popc(qm);
                        __syncwarp();
                        if (nq >= 32) {
                            drain(32);
                            __syncwarp();
                            if (lane < nq - 32) dq[lane] = dq[32 + lane];
                            nq -= 32;
                            __syncwarp();
                        }
                    }
                }
                __syncwarp();
                if (!kEmit) boxes();
            }
        }
        if (!kEmit && active) a.best[row] = my_best <= q ? my_best : INFINITY;
        if (kEmit) wflush(out, a.sink, false);
    }
    if (kEmit && nq > 0) {
        drain(nq);
        __syncwarp();
    }
    if (kEmit) wflush(out, a.sink, true);
    add_counter(a.counters, 5, n_cand);
    add_counter(a.counters, 1, n_exact);
}

}  // namespace
}  // namespace vs

using namespace vs;

extern "C" {

int vs_join_dwithin(vs_context* ctx, const vs_index* idx, const vs_points* pts, const double* d_point_distance,
                    const double* d_geom_distance, double distance, uint32_t flags, int32_t* d_left,
                    int32_t* d_right, int64_t capacity, int64_t* n_pairs, vs_join_stats* stats) {
    if (stats) memset(stats, 0, sizeof(*stats));
    VS_TRY(check_join_args(ctx, idx, pts, d_left, d_right, capacity, n_pairs));
    if (d_point_distance && d_geom_distance) {
        set_error("give per-point or per-polygon distances, not both");
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    if (pts->n == 0 || idx->n_geoms == 0 || !(idx->h_frame[0] <= idx->h_frame[2])) return VS_OK;
    cudaStream_t s = ctx->stream;
    const long long launches0 = g_launches;
    if (d_geom_distance) {
        // the candidate search uses the largest per-polygon distance
        const unsigned long long init = (unsigned long long)host_dbl_to_ordered(-INFINITY);
        VS_CUDA_TRY(cudaMemcpyAsync(&ctx->d_counters[9], &init, sizeof(init), cudaMemcpyHostToDevice, s));
        max_distance_kernel<<<resident_grid(max_distance_kernel, idx->n_geoms, 256), 256, 0, s>>>(
            d_geom_distance, idx->n_geoms, &ctx->d_counters[9]);
        VS_LAUNCHED("max_distance", s);
        unsigned long long m = 0;
        VS_CUDA_TRY(cudaMemcpyAsync(&m, &ctx->d_counters[9], sizeof(m), cudaMemcpyDeviceToHost, s));
        VS_CUDA_TRY(cudaStreamSynchronize(s));
        long long k = (long long)m;
        k = k >= 0 ? k : (k ^ 0x7fffffffffffffffLL);
        memcpy(&distance, &k, sizeof(distance));
    }
    EventPair ev;
    VS_CUDA_TRY(cudaMemsetAsync(ctx->d_counters, 0, kDevCounters * sizeof(unsigned long long), s));
    cudaEventRecord(ev.a, s);
    QueryOrder q;
    VS_TRY(prepare_queries(ctx, idx, pts, q, true));
    size_t smem = 0;
    DistArgs a = dist_args(ctx, idx, pts, q, &smem);
    a.n_list = q.n_valid.p;
    a.dist_pt = d_point_distance;
    a.dist_geom = d_geom_distance;
    a.dist_scalar = distance;
    a.sink = PairSink{d_left, d_right, (unsigned long long)(capacity > 0 ? capacity : 0), &ctx->d_counters[0]};
    VS_TRY(launch_dist<kDwithin>(ctx, a, smem, pts->n));
    return finish_join(ctx, idx, pts, flags, d_left, d_right, capacity, n_pairs, stats, ev, launches0);
}

int vs_join_nearest(vs_context* ctx, const vs_index* idx, const vs_points* pts, double max_distance, uint32_t flags,
                    int32_t* d_left, int32_t* d_right, double* d_distance, int64_t capacity, int64_t* n_pairs,
                    vs_join_stats* stats) {
    if (stats) memset(stats, 0, sizeof(*stats));
    VS_TRY(check_join_args(ctx, idx, pts, d_left, d_right, capacity, n_pairs));
    if (max_distance != max_distance) {
        set_error("max_distance is NaN");
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    if (pts->n == 0 || idx->n_geoms == 0 || !(idx->h_frame[0] <= idx->h_frame[2])) return VS_OK;
    if (max_distance < 0.0) return VS_OK;
    cudaStream_t s = ctx->stream;
    const long long launches0 = g_launches;
    EventPair ev;
    VS_CUDA_TRY(cudaMemsetAsync(ctx->d_counters, 0, kDevCounters * sizeof(unsigned long long), s));
    cudaEventRecord(ev.a, s);
    QueryOrder q;
    VS_TRY(prepare_queries(ctx, idx, pts, q, true));
    Scratch<double> best;
    VS_TRY(best.alloc((size_t)pts->n, s));
    size_t smem = 0;
    DistArgs a = dist_args(ctx, idx, pts, q, &smem);
    a.n_list = q.n_valid.p;
    a.best = best.p;
    a.radius = max_distance;  // the search cap
    a.sink = PairSink{d_left, d_right, (unsigned long long)(capacity > 0 ? capacity : 0), &ctx->d_counters[0]};
    // each point's minimum distance, then every polygon at exactly that distance
    VS_TRY(launch_dist<kNearestMin>(ctx, a, smem, pts->n));
    VS_TRY(launch_dist<kNearestEmit>(ctx, a, smem, pts->n));
    const int st = finish_join(ctx, idx, pts, flags, d_left, d_right, capacity, n_pairs, stats, ev, launches0);
    if (st != VS_OK) return st;
    if (d_distance && *n_pairs > 0) {
        gather_pair_distance_kernel<<<resident_grid(gather_pair_distance_kernel, *n_pairs, 256), 256, 0, s>>>(
            d_left, *n_pairs, best.p, d_distance);
        VS_LAUNCHED("gather_pair_distance", s);
        VS_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return VS_OK;
}

int vs_distance_aligned(vs_context* ctx, const vs_points* pts, const vs_polygons* polys, double* d_distance,
                        double* d_envelope_distance) {
    if (!ctx || !polys || !d_distance) {
        set_error("ctx/polys/distance is NULL");
        return VS_E_ARG;
    }
    VS_TRY(check_points(pts));
    if (polys->n_geoms != pts->n) {
        set_error("aligned rows: %lld points, %d polygons", (long long)pts->n, polys->n_geoms);
        return VS_E_ARG;
    }
    if (pts->n > 0x7fffffffLL) {
        set_error("%lld rows: more than the 32-bit rows address", (long long)pts->n);
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    if (pts->n == 0) return VS_OK;
    cudaStream_t s = ctx->stream;
    distance_aligned_kernel<<<resident_grid(distance_aligned_kernel, pts->n, 256), 256, 0, s>>>(
        *pts, *polys, d_distance, d_envelope_distance, ctx->d_counters);
    VS_LAUNCHED("distance_aligned", s);
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    return VS_OK;
}

int vs_join_nearest_polygons(vs_context* ctx, const vs_index* point_index, const vs_polygons* queries,
                              double max_distance, uint32_t flags, int32_t* d_left, int32_t* d_right,
                              double* d_distance, int64_t capacity, int64_t* n_pairs, vs_join_stats* stats) {
    if (stats) memset(stats, 0, sizeof(*stats));
    if (!ctx || !point_index || !n_pairs) {
        set_error("ctx/index/n_pairs is NULL");
        return VS_E_ARG;
    }
    *n_pairs = 0;
    VS_TRY(check_polygons(queries));
    if (capacity < 0 || (capacity > 0 && (!d_left || !d_right))) {
        set_error("invalid pair buffers (capacity %lld)", (long long)capacity);
        return VS_E_ARG;
    }
    if (point_index->device != ctx->device) {
        set_error("index lives on device %d, context on device %d", point_index->device, ctx->device);
        return VS_E_ARG;
    }
    if (max_distance != max_distance) {
        set_error("max_distance is NaN");
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    const int64_t nq = queries->n_geoms;
    if (nq == 0 || point_index->n_geoms == 0 || !(point_index->h_frame[0] <= point_index->h_frame[2]) ||
        max_distance < 0.0)
        return VS_OK;
    cudaStream_t s = ctx->stream;
    const long long launches0 = g_launches;
    EventPair ev;
    VS_CUDA_TRY(cudaMemsetAsync(ctx->d_counters, 0, kDevCounters * sizeof(unsigned long long), s));
    cudaEventRecord(ev.a, s);
    Scratch<vs_box> qbox;
    Scratch<uint32_t> keys, order, n_valid;
    Scratch<double> best;
    VS_TRY(qbox.alloc((size_t)nq, s));
    VS_TRY(keys.alloc((size_t)nq, s));
    VS_TRY(order.alloc((size_t)nq, s));
    VS_TRY(n_valid.alloc(1, s));
    VS_TRY(best.alloc((size_t)nq, s));
    VS_CUDA_TRY(cudaMemsetAsync(n_valid.p, 0, sizeof(uint32_t), s));
    poly_query_key_kernel<<<resident_grid(poly_query_key_kernel, nq, 256), 256, 0, s>>>(
        *queries, point_index->frame, qbox.p, keys.p, order.p, n_valid.p);
    VS_LAUNCHED("poly_query_key", s);
    VS_TRY(radix_sort_u32_u32(keys.p, order.p, nq, 32, s, 0));
    PolyArgs a{};
    a.x = queries->d_x;
    a.y = queries->d_y;
    a.ring_off = queries->d_ring_off;
    a.part_off = queries->d_part_off;
    a.geom_off = queries->d_geom_off;
    a.qbox = qbox.p;
    a.order = order.p;
    a.n_valid = n_valid.p;
    a.nodes = point_index->nodes;
    for (int l = 0; l < kMaxLevels; ++l) {
        a.level_off[l] = point_index->level_off[l];
        a.level_size[l] = point_index->level_size[l];
    }
    a.levels = point_index->levels;
    int sl = point_index->levels - 1;
    int64_t staged = point_index->level_size[sl];
    while (sl > 0 && staged + point_index->level_size[sl - 1] <= kDistMaxStaged) {
        --sl;
        staged += point_index->level_size[sl];
    }
    a.stage_level = sl;
    a.staged = (int)staged;
    a.item_geom = point_index->item_geom;
    a.cap = max_distance;
    a.best = best.p;
    a.sink = PairSink{d_left, d_right, (unsigned long long)(capacity > 0 ? capacity : 0), &ctx->d_counters[0]};
    a.counters = ctx->d_counters;
    a.work = &ctx->d_counters[kWorkCounter];
    const size_t smem = (size_t)a.staged * sizeof(vs_box);
    // each polygon's minimum distance, then every point at exactly that distance
    VS_CUDA_TRY(cudaMemsetAsync(a.work, 0, sizeof(unsigned long long), s));
    VS_CUDA_TRY(cudaFuncSetAttribute(poly_nearest_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    poly_nearest_kernel<false><<<resident_grid(poly_nearest_kernel<false>, nq, kDistThreads, smem), kDistThreads,
                                 smem, s>>>(a);
    VS_LAUNCHED("poly_nearest<min>", s);
    VS_CUDA_TRY(cudaMemsetAsync(a.work, 0, sizeof(unsigned long long), s));
    VS_CUDA_TRY(cudaFuncSetAttribute(poly_nearest_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    poly_nearest_kernel<true><<<resident_grid(poly_nearest_kernel<true>, nq, kDistThreads, smem), kDistThreads,
                                smem, s>>>(a);
    VS_LAUNCHED("poly_nearest<emit>", s);
    vs_points qp{};
    qp.n = nq;  // the pair sort keys left rows by the query count
    const int st = finish_join(ctx, point_index, &qp, flags, d_left, d_right, capacity, n_pairs, stats, ev, launches0);
    if (st != VS_OK) return st;
    if (d_distance && *n_pairs > 0) {
        gather_pair_distance_kernel<<<resident_grid(gather_pair_distance_kernel, *n_pairs, 256), 256, 0, s>>>(
            d_left, *n_pairs, best.p, d_distance);
        VS_LAUNCHED("gather_pair_distance", s);
        VS_CUDA_TRY(cudaStreamSynchronize(s));
    }
    return VS_OK;
}

}  // extern "C"
