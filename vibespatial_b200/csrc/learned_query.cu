// Learned + split-precision join: the query passes over the learned cell
// index (built in learned.cu), for one index or a batch of them.
//
// Three passes over the points (a counting sort keyed by the learned index's
// own positions, so no general sort is needed):
//   map      input order: the point's job (batch) -> level-L cell key ->
//            occupancy bit -> root table -> leaf model -> binary search inside
//            the leaf's error window -> cell index (or none); the per-cell
//            counts are incremented, and every matched point is appended to
//            a striped staging region as one 16-byte CellPoint: its FP32
//            offsets from the cell's anchor, its row and its cell
//   place    after an exclusive scan of the counts, every staged CellPoint is
//            copied to its cell's next free position (per-cell cursors), so
//            the points end up grouped by cell
//   refine   a warp takes 32 consecutive grouped points, which share a
//            candidate list except at cell boundaries, so the lanes read each
//            entry record together (broadcast); each candidate is box-filtered
//            in FP32 against the entry's box relative to the same anchor
//            (rounded outward); survivors are queued per warp and refined 32
//            at a time with the FP32 crossing test on slot-relative
//            coordinates; a pair with an edge whose FP32 decision lies within
//            the rounding-error bound is deferred to the exact pass, which
//            walks it on the FP64 coordinates (Shewchuk's stage-A filter, then
//            the exact expansion).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "emit.cuh"
#include "exact.cuh"
#include "hilbert.cuh"
#include "index.cuh"
#include "join.cuh"
#include "learned.cuh"
#include "primitives.cuh"
#include "rmi.cuh"
#include "tma.cuh"

namespace vs {
namespace {

constexpr int kThreads = 256;

// The map pass appends matched points to kStripes regions of the staging
// array, region s taking the packets p with p % kStripes == s, so each
// region's append counter sees 1/kStripes of the atomics and a region never
// holds more than 32 * ceil(packets / kStripes) points.
constexpr int kStripes = 2048;

// A (point, candidate) pair that passed the FP32 box filter, queued for the
// ring walk: the point relative to the slot origin, the tolerance of every
// FP32 coordinate difference, and what the walk and the emission need.
struct __align__(16) QueuedPair {
    float qx, qy;
    float t;
    int32_t row;
    int32_t slot;
    int32_t job;
    int32_t pad0, pad1;
};
constexpr int kQueue = 64;  // >= 31 left over + 32 appended in one step

struct LqArgs {
    LearnedQuery q;
    LearnedJob single;  // the one job of a single join (kernel parameter space)
    CellPoint* staged;
    uint32_t* stripe_count;
    int64_t stripe_cap;
    uint32_t* cell_count;
    CellPoint* grouped;
    const uint32_t* n_grouped;
    PairSink sink;
    DeferSink defer;
    unsigned long long* counters;
    unsigned long long* work;  // refine work queue (grouped points handed out)
    int64_t grab;              // grouped points a refine warp takes per grab (multiple of 32)
    bool no_stage;             // entry records read from global memory (no bulk-copy staging)
    bool no_interior;          // every box candidate is ring-walked (no interior-box shortcut)
};

// Streaming (evict-first) accesses for the read-once streams of the passes:
// the query points, the staged cell points and the grouped cell points.  They
// leave L2 to what is re-read: the index (cell keys, occupancy bitmap, leaves,
// records, vertices) and the half-written sectors of the place pass.
__device__ __forceinline__ CellPoint load_stream(const CellPoint* p) {
    const float4 v = __ldcs(reinterpret_cast<const float4*>(p));
    return CellPoint{v.x, v.y, __float_as_int(v.z), __float_as_uint(v.w)};
}

__device__ __forceinline__ void store_stream(CellPoint* p, const CellPoint& c) {
    __stcs(reinterpret_cast<float4*>(p), make_float4(c.qx, c.qy, __int_as_float(c.row), __uint_as_float(c.gcell)));
}

// Job descriptor of a batch query (global memory) or of a single join (the
// kernel parameters: uniform reads, no extra registers).
template <bool kMulti>
__device__ __forceinline__ const LearnedJob& job_desc(const LqArgs& a, int job) {
    if constexpr (kMulti) return a.q.jobs[job];
    else return a.single;
}

// Job of query point pi (its index in the query's point arrays).
template <bool kMulti>
__device__ __forceinline__ int point_job(const LearnedQuery& q, int64_t pi) {
    if (!kMulti || q.n_jobs <= 1) return 0;
    int lo = 0, hi = q.n_jobs;  // last job with job_start[job] <= pi
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (q.job_start[mid] <= pi) lo = mid;
        else hi = mid;
    }
    return lo;
}

// ------------------------------------------------------- split refine ---
// One edge in FP32 on tile-relative coordinates.  Returns false when some
// decision the exact walk needs lies within the rounding-error bound `t`
// (the caller then defers the pair to the exact pass); otherwise applies the
// same decision the exact walk would (the point cannot be on this edge).
__device__ __forceinline__ bool edge_step_fp32(float ax, float ay, float bx, float by, float px, float py, float t,
                                               bool& inside) {
    const float A2 = __fsub_rn(ay, py), B2 = __fsub_rn(by, py);
    if (fabsf(A2) <= t || fabsf(B2) <= t) return false;
    const bool sA = A2 > 0.f, sB = B2 > 0.f;
    if (sA == sB) return true;  // py strictly outside the edge's y-range
    const float A1 = __fsub_rn(ax, px), B1 = __fsub_rn(bx, px);
    if (A1 > t && B1 > t) {  // edge strictly right of the point: the +x ray crosses it
        inside = !inside;
        return true;
    }
    if (A1 < -t && B1 < -t) return true;  // strictly left
    const float l = __fmul_rn(A1, B2), r = __fmul_rn(A2, B1);
    const float det = __fsub_rn(l, r);
    const float m = fmaxf(fmaxf(fabsf(A1), fabsf(A2)), fmaxf(fabsf(B1), fabsf(B2)));
    const float e = __fmaf_ru(m, 6.0e-8f, t);
    const float S = __fadd_ru(__fadd_ru(fabsf(A1), fabsf(A2)), __fadd_ru(fabsf(B1), fabsf(B2)));
    float bound = __fmaf_ru(3.6e-7f, __fadd_ru(fabsf(l), fabsf(r)), __fmaf_ru(S, e, __fmul_ru(2.0f, __fmul_ru(e, e))));
    bound = __fmaf_ru(bound, 1.01f, 1e-30f);
    if (det > bound) {
        if (sB) inside = !inside;  // o > 0 and, since the edge crosses, by > ay <=> sB
        return true;
    }
    if (det < -bound) {
        if (!sB) inside = !inside;
        return true;
    }
    return false;
}

// The point's FP64 coordinates in the query arrays (X, Y at pi): read only to
// pick a ring's y-bin.
struct PointRef {
    const double* X;
    const double* Y;
    int64_t pi;
};

// One edge of the split ring walk in FP32.  0: decided, go on; 2: the FP32
// bound is inconclusive, the pair goes to the exact pass (counted in n64).
// Re-deciding such an edge in line in FP64 (the point's FP64 coordinates read
// by row, the FP64 vertices, the stage-A filter) sent one lane on a long
// detour while the others waited, and its registers made the 48-register
// build spill; deferring the pair made the Zipf join 2% and the 256-job batch
// 5% faster.
__device__ __forceinline__ int split_edge(float qx, float qy, float t, float2 a, float2 b, bool& inside,
                                          unsigned& n32, unsigned& n64) {
    if (edge_step_fp32(a.x, a.y, b.x, b.y, qx, qy, t, inside)) {
        ++n32;
        return 0;
    }
    ++n64;
    return 2;
}

// Split-precision location of a point in one ring, every edge.
__device__ __forceinline__ int ring_location_split(float qx, float qy, float t, const float2* __restrict__ xy32,
                                                   int start, int end, unsigned& n32, unsigned& n64) {
    if (end - start < 2) return LOC_OUTSIDE;
    bool inside = false;
    float2 a = xy32[end - 1];
    float2 b = xy32[start];
    // an edge's start offset in y is the previous edge's end offset: carried
    float dA = __fsub_rn(a.y, qy);
    for (int i = start; i < end; ++i) {
        // the next vertex's load is in flight while this edge is decided
        const float2 nb = xy32[i + 1 < end ? i + 1 : i];
        const float dB = __fsub_rn(b.y, qy);
        if (fabsf(dA) > t && fabsf(dB) > t && (dA > 0.f) == (dB > 0.f)) {
            ++n32;  // both ends strictly on one side of the point's y: the edge changes nothing
        } else {
            if (split_edge(qx, qy, t, a, b, inside, n32, n64)) return LOC_UNDECIDED;
        }
        a = b;
        dA = dB;
        b = nb;
    }
    return inside ? LOC_INTERIOR : LOC_OUTSIDE;
}

// The same for a ring with y-bins: only the edges of the point's bin, in ring
// order; an edge that continues the previous one reuses its end vertex.  The
// bin is chosen from the point's FP64 y (bins are defined on FP64 y).
__device__ __forceinline__ int ring_location_split_binned(float qx, float qy, float t,
                                                          const float2* __restrict__ xy32, int start, int end,
                                                          const RingBins& bins, const uint16_t* __restrict__ edges,
                                                          const PointRef& P, unsigned& n32, unsigned& n64) {
    bool inside = false;
    const int k = ring_bin_of(P.Y[P.pi], bins.y0, bins.scale);
    const uint32_t e1 = bins.off[k + 1];
    int last = -2;
    float2 lb = make_float2(0.f, 0.f);
    for (uint32_t e = bins.off[k]; e < e1; ++e) {
        const int i = start + edges[e];
        const int ia = i == start ? end - 1 : i - 1;
        const float2 a = ia == last ? lb : xy32[ia];
        const float2 b = xy32[i];
        if (split_edge(qx, qy, t, a, b, inside, n32, n64)) return LOC_UNDECIDED;
        last = i;
        lb = b;
    }
    return inside ? LOC_INTERIOR : LOC_OUTSIDE;
}

// kBins: the index has y-binned rings (kernels without bins carry no binned
// walk, which keeps their registers for the common short rings).
template <bool kBins>
__device__ __forceinline__ int geometry_location_split(float qx, float qy, float t, const LearnedJob& J, int g,
                                                       const PointRef& P, unsigned& n32, unsigned& n64) {
    const int p0 = J.geom_off[g], p1 = J.geom_off[g + 1];
    for (int part = p0; part < p1; ++part) {
        bool inside = false;
        const int r0 = J.part_off[part], r1 = J.part_off[part + 1];
        // the only ring of a polygon is walked binned from fewer vertices than a ring beside holes or parts
        const int bin_min = (p1 - p0 == 1 && r1 - r0 == 1) ? kSplitBinMinSingleRing : kSplitBinMinVertices;
        for (int ring = r0; ring < r1; ++ring) {
            // A ring whose box lies strictly beyond the point (by more than t) neither holds it nor crosses its
            // +x ray an odd number of times: the walk of it would change nothing.
            const float4 box = J.ring_box32[ring];
            if (__fadd_ru(qx, t) < box.x || __fsub_rd(qx, t) > box.z || __fadd_ru(qy, t) < box.y ||
                __fsub_rd(qy, t) > box.w)
                continue;
            const int c0 = J.ring_off[ring], c1 = J.ring_off[ring + 1];
            // the FP32 walk is cheap per edge, so bins pay off only on longer rings than for the FP64 walk
            const int rb = (kBins && J.rings.ring_bin && c1 - c0 >= bin_min) ? J.rings.ring_bin[ring] : -1;
            const int k = rb >= 0 ? ring_location_split_binned(qx, qy, t, J.xy32, c0, c1, J.rings.bins[rb],
                                                               J.rings.edges, P, n32, n64)
                                  : ring_location_split(qx, qy, t, J.xy32, c0, c1, n32, n64);
            if (k == LOC_BOUNDARY || k == LOC_UNDECIDED) return k;
            if (k == LOC_INTERIOR) inside = !inside;
        }
        if (inside) return LOC_INTERIOR;
    }
    return LOC_OUTSIDE;
}

// ---------------------------------------------------------------- map ---
// Exact lookup of grid cell (gx, gy) (32-bit grid coordinates) in job J's
// learned index: level-L cell key -> occupancy bit -> root table -> leaf
// model -> binary search inside the leaf's error window.  Returns the cell's
// index, or -1 when no stored cell matches (no polygon box overlaps it).
// kBsearch (an ablation): the model is skipped and the search covers every
// stored key.
template <bool kBsearch>
__device__ __forceinline__ int learned_lookup(const LearnedJob& J, uint32_t gx, uint32_t gy, const uint16_t* lut,
                                              unsigned long long& n_wide) {
    const uint32_t cell = hilbert_key_lut(gx, gy, J.L, lut);
    const uint32_t ob = cell >> J.occ_shift;
    // the occupancy word and the root-table entry depend only on the key:
    // both loads are issued before either is tested
    const uint32_t occ_word = J.occ[ob >> 5];
    const uint32_t leaf_id = kBsearch ? 0u : (uint32_t)J.root_table[cell >> J.root_shift];
    if (!((occ_word >> (ob & 31)) & 1u)) return -1;
    // search [l0, h0) with 32-bit indices (a cell count fits in 31 bits)
    int l0 = 0, h0 = (int)J.n_cells;
    if constexpr (!kBsearch) {
        const RmiLeaf lf = J.leaves[leaf_id];
        if (lf.lo > lf.hi) return -1;  // no stored key routes to this leaf
        const long long pred = rmi_predict(make_double2(lf.a, lf.b), cell);
        long long w0 = pred + lf.lo, w1 = pred + lf.hi + 1;
        w0 = w0 < 0 ? 0 : w0;
        w1 = w1 > J.n_cells ? J.n_cells : w1;
        if (w1 <= w0) return -1;  // the window lies outside the stored keys
        l0 = (int)w0;
        h0 = (int)w1;
        if (h0 - l0 > 256) ++n_wide;
    }
    const int h1 = h0;
    while (l0 < h0) {
        const int mid = (int)(((uint32_t)l0 + (uint32_t)h0) >> 1);
        if (J.cell_keys[mid] < cell) l0 = mid + 1;
        else h0 = mid;
    }
    return (l0 < h1 && J.cell_keys[l0] == cell) ? l0 : -1;
}

// Job of every lane's point: lane 0 binary-searches the packet's first point,
// the lanes step forward over the (contiguous) job ranges from there.
template <bool kMulti>
__device__ __forceinline__ int packet_job(const LearnedQuery& q, int64_t b0, int64_t i, int lane) {
    if (!kMulti || q.n_jobs <= 1) return 0;
    int j = 0;
    if (lane == 0) j = point_job<kMulti>(q, b0);
    j = __shfl_sync(0xffffffffu, j, 0);
    if (i < q.n)
        while (j + 1 < q.n_jobs && i >= q.job_start[j + 1]) ++j;
    return j;
}

// One point of the map pass: its batch-wide cell (-1: none) and its FP32
// offsets from the cell's anchor (|offset| <= half a cell).
template <bool kMulti, bool kBsearch>
__device__ __forceinline__ int map_point(const LqArgs& a, int64_t i, int job, const uint16_t* lut,
                                         unsigned long long& n_wide, float& qx, float& qy) {
    const LearnedQuery& q = a.q;
    if (i >= q.n) return -1;
    const LearnedJob& J = job_desc<kMulti>(a, job);
    const double x = __ldcs(q.px + i), y = __ldcs(q.py + i);
    if (!((q.pvalid == nullptr || q.pvalid[i]) && J.n_cells > 0 && x >= J.lox && x <= J.hix && y >= J.loy &&
          y <= J.hiy))
        return -1;
    const uint32_t gx = quantize(x, J.lox, J.sx), gy = quantize(y, J.loy, J.sy);
    const int c = learned_lookup<kBsearch>(J, gx, gy, lut, n_wide);
    if (c < 0) return -1;
    const int sh = 32 - J.L;
    qx = __double2float_rn(__dsub_rn(x, cell_anchor(J.lox, J.cwx, gx >> sh)));
    qy = __double2float_rn(__dsub_rn(y, cell_anchor(J.loy, J.cwy, gy >> sh)));
    return (int)(J.cell_base + (uint32_t)c);
}

// Count a packet's matched points and append them to the packet's stripe
// region.  Whole warp, converged.
__device__ __forceinline__ void map_emit(const LqArgs& a, int64_t b0, int lane, int gc, float qx, float qy) {
    if (gc >= 0) atomicAdd(&a.cell_count[gc], 1u);
    const unsigned mm = __ballot_sync(0xffffffffu, gc >= 0);
    if (!mm) return;
    const int64_t stripe = (b0 >> 5) % kStripes;
    uint32_t sb = 0;
    if (lane == 0) sb = atomicAdd(&a.stripe_count[stripe], (uint32_t)__popc(mm));
    sb = __shfl_sync(0xffffffffu, sb, 0);
    if (gc >= 0) {
        CellPoint p;
        p.qx = qx;
        p.qy = qy;
        p.row = (int32_t)(b0 + lane + a.q.row_base);
        p.gcell = (uint32_t)gc;
        store_stream(&a.staged[stripe * a.stripe_cap + sb + __popc(mm & ((1u << lane) - 1u))], p);
    }
}

// Pass 1 (map), points in input order: each point's cell, the per-cell
// counts, and the matched points appended to the staging regions as
// CellPoints.  A warp takes kPackets packets of 32 points per iteration and
// runs their lookups together, so that many independent chains of dependent
// index loads (occupancy bit, root table, leaf, binary search) are in flight.
template <bool kMulti, bool kBsearch, int kPackets>
__global__ void __launch_bounds__(kThreads, kPackets == 1 ? 8 : 6) learned_map_kernel(const LqArgs a) {
    __shared__ uint16_t s_lut[kHilbertLutSize];
    hilbert_lut_init(s_lut);
    __syncthreads();
    const LearnedQuery& q = a.q;
    unsigned long long n_wide = 0;
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    // Warp-uniform loop: the whole warp reaches the ballots and shuffles together.
    for (int64_t b0 = gw * 32 * kPackets; b0 < q.n; b0 += nw * 32 * kPackets) {
        int gc[kPackets];
        float qx[kPackets], qy[kPackets];
#pragma unroll
        for (int u = 0; u < kPackets; ++u) {
            const int64_t bu = b0 + 32 * u;
            const int job = packet_job<kMulti>(q, bu < q.n ? bu : b0, bu + lane, lane);
            qx[u] = qy[u] = 0.f;
            gc[u] = map_point<kMulti, kBsearch>(a, bu + lane, job, s_lut, n_wide, qx[u], qy[u]);
        }
#pragma unroll
        for (int u = 0; u < kPackets; ++u) map_emit(a, b0 + 32 * u, lane, gc[u], qx[u], qy[u]);
    }
    add_counter(a.counters, 6, n_wide);
}

// -------------------------------------------------------------- place ---
// Pass 2 (place): after the exclusive scan of the counts (cell_count[c] is
// then the first position of cell c), every staged point takes the next
// position of its cell (warp-aggregated cursor increments) and is copied
// there.  Records of one cell placed close together in time fill whole
// 32-byte sectors in L2 before they are written back.  A block walks whole
// stripe regions; a warp keeps kPlaceUnroll groups of 32 records in flight
// (loads, then cursor increments, then stores).
#ifndef VS_PLACE_UNROLL
#define VS_PLACE_UNROLL 4
#endif
constexpr int kPlaceUnroll = VS_PLACE_UNROLL;

__global__ void __launch_bounds__(kThreads) learned_place_kernel(const LqArgs a) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    constexpr uint32_t kStep = 32u * kPlaceUnroll;
    for (int stripe = blockIdx.x; stripe < kStripes; stripe += gridDim.x) {
        const uint32_t cnt = a.stripe_count[stripe];
        const CellPoint* src = a.staged + (int64_t)stripe * a.stripe_cap;
        // warp-uniform loop: every lane runs the same iterations
        for (uint32_t k0 = (uint32_t)warp * kStep; k0 < cnt; k0 += (kThreads / 32) * kStep) {
            CellPoint p[kPlaceUnroll];
            int gc[kPlaceUnroll];
#pragma unroll
            for (int u = 0; u < kPlaceUnroll; ++u) {
                const uint32_t k = k0 + u * 32 + lane;
                gc[u] = -1;
                if (k < cnt) {
                    p[u] = load_stream(src + k);
                    gc[u] = (int)p[u].gcell;
                }
            }
            unsigned peers[kPlaceUnroll];
            uint32_t base[kPlaceUnroll];
#pragma unroll
            for (int u = 0; u < kPlaceUnroll; ++u) {
                peers[u] = __match_any_sync(0xffffffffu, gc[u]);
                base[u] = 0;
                if (gc[u] >= 0 && lane == __ffs(peers[u]) - 1)
                    base[u] = atomicAdd(&a.cell_count[gc[u]], (uint32_t)__popc(peers[u]));
            }
#pragma unroll
            for (int u = 0; u < kPlaceUnroll; ++u) {
                const uint32_t b = __shfl_sync(0xffffffffu, base[u], __ffs(peers[u]) - 1);
                if (gc[u] >= 0) a.grouped[b + __popc(peers[u] & lt)] = p[u];
            }
        }
    }
}

// ------------------------------------------------------------- refine ---
#ifndef VS_JOIN_MIN_BLOCKS
#define VS_JOIN_MIN_BLOCKS 5  // the bbox kernel's register cap (blocks per SM)
#endif
constexpr int64_t kJoinGrab = 32;  // default grouped points per work-queue grab (multiple of 32)

// A grouped point's candidate range and conversion-error bound.  The bound
// dq covers |q - (p - anchor)|: the FP64 subtraction (2^-53 relative) and the
// FP32 rounding (2^-24 relative, or the subnormal spacing).
struct GroupedLane {
    CellPoint p;
    uint32_t lo, len;
    int job;
    float dq;
};

template <bool kMulti>
__device__ __forceinline__ GroupedLane load_grouped(const LqArgs& a, int64_t j, int64_t e0) {
    GroupedLane g;
    g.p = CellPoint{0.f, 0.f, 0, 0u};
    g.lo = g.len = 0;
    g.job = 0;
    if (j < e0) {
        g.p = load_stream(a.grouped + j);
        g.job = point_job<kMulti>(a.q, (int64_t)g.p.row - a.q.row_base);
        const LearnedJob& J = job_desc<kMulti>(a, g.job);
        const uint32_t c = g.p.gcell - J.cell_base;
        g.lo = J.cell_start[c];
        g.len = J.cell_start[c + 1] - g.lo;
    }
    g.dq = __fmaf_ru(fmaxf(fabsf(g.p.qx), fabsf(g.p.qy)), 6.1e-8f, 1e-37f);
    return g;
}

// FP32 box filter of one candidate (the box is rounded outward and the point
// widened by its error bound: never rejects a point of the polygon's box).
__device__ __forceinline__ bool box_filter_fp32(const float4& bx, float qx, float qy, float dq) {
    return !(__fadd_ru(qx, dq) < bx.x || __fsub_rd(qx, dq) > bx.z || __fadd_ru(qy, dq) < bx.y ||
             __fsub_rd(qy, dq) > bx.w);
}

__device__ __forceinline__ unsigned warp_max_u32(unsigned v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned t = __shfl_xor_sync(0xffffffffu, v, o);
        v = t > v ? t : v;
    }
    return v;
}

// Box candidates only (predicate BBOX): a warp takes 32 consecutive grouped
// points and walks their candidate lists; the FP32 filter's survivors are
// decided exactly on the FP64 box with the point's FP64 coordinates.
template <bool kMulti>
__global__ void __launch_bounds__(kThreads, VS_JOIN_MIN_BLOCKS) learned_bbox_kernel(const LqArgs a) {
    __shared__ int2 s_buf[kThreads / 32][kWarpBuf];
    __shared__ unsigned s_cnt[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_cnt[warp] = 0;
    __syncwarp();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    const int64_t n = (int64_t)*a.n_grouped;
    unsigned long long n_cand = 0;
    for (;;) {
        const int64_t b0 = warp_grab(a.work, a.grab);
        if (b0 >= n) break;
        const int64_t e0 = b0 + a.grab < n ? b0 + a.grab : n;
        for (int64_t base = b0; base < e0; base += 32) {
            const GroupedLane g = load_grouped<kMulti>(a, base + lane, e0);
            const uint32_t maxlen = warp_max_u32(g.len);
            const LearnedJob& J = job_desc<kMulti>(a, g.job);
            const int64_t pi = (int64_t)g.p.row - a.q.row_base;
            for (uint32_t k = 0; k < maxlen; ++k) {
                bool want = false;
                int32_t right = 0;
                if (k < g.len) {
                    const EntryRecord r = J.recs[g.lo + k];
                    if (box_filter_fp32(r.box, g.p.qx, g.p.qy, g.dq)) {
                        const int32_t slot = entry_slot(r);
                        const vs_box bb = J.boxes[slot];
                        const double x = a.q.px[pi], y = a.q.py[pi];
                        if (x >= bb.minx && x <= bb.maxx && y >= bb.miny && y <= bb.maxy) {
                            ++n_cand;
                            want = true;
                            right = J.item_geom[slot];
                        }
                    }
                }
                wemit_sync(out, a.sink, want, g.p.row, right);
            }
            wflush(out, a.sink, false);
        }
    }
    wflush(out, a.sink, true);
    add_counter(a.counters, 5, n_cand);
}

// Ring walks of up to 32 queued pairs, one per lane.
// kF64 (an ablation): the walk is the plain method's FP64 filtered walk on
// the point's FP64 coordinates, with no FP32 edge stage.
template <bool kMulti, bool kBins, bool kF64>
__device__ __forceinline__ void refine_queued(const LqArgs& a, const WarpOut& out, const QueuedPair* qp, int nq,
                                              int lane, unsigned& n32, unsigned& n64) {
    bool want = false;
    int32_t row = 0, right = 0;
    if (lane < nq) {
        const QueuedPair jb = qp[lane];
        const LearnedJob& J = job_desc<kMulti>(a, jb.job);
        row = jb.row;
        const PointRef P{a.q.px, a.q.py, (int64_t)jb.row - a.q.row_base};
        int loc;
        if constexpr (kF64) {
            loc = geometry_location_filtered(P.X[P.pi], P.Y[P.pi], J.xy, J.ring_off, J.part_off, J.geom_off, jb.slot,
                                             J.rings);
        } else {
            const int2 cr = J.c01[jb.slot];
            loc = cr.x >= 0 ? ring_location_split(jb.qx, jb.qy, jb.t, J.xy32, cr.x, cr.y, n32, n64)
                            : geometry_location_split<kBins>(jb.qx, jb.qy, jb.t, J, jb.slot, P, n32, n64);
        }
        if (loc == LOC_UNDECIDED) {
            defer(a.defer, jb.row, jb.slot);  // a batch's exact pass finds the job from the row
        } else if ((a.q.accept_mask >> loc) & 1) {
            want = true;
            right = J.item_geom[jb.slot];
        }
    }
    wemit_sync(out, a.sink, want, row, right);
}

// Pass 3 with a location test: the warp walks its grouped points' candidate
// lists, and every (point, candidate) pair that passes the FP32 box filter is
// appended to a warp-local queue in shared memory, converted to the slot's
// frame (q + off) with its error tolerance.  Each time 32 pairs are queued,
// every lane refines one of them, so the ring walks, which dominate, run
// with all lanes busy instead of only the lanes whose point lies in the
// current candidate's box.  Neighbouring queue entries mostly share a
// polygon, so vertex reads stay broadcasts.
// Entry records a warp stages in shared memory for one packet of 32 grouped
// points: the lanes' cells ascend, so their candidate lists lie in one
// contiguous run of the job's records, from the first lane's first record to
// the last lane's last; a run of at most kStageRecs records arrives by one
// bulk copy (TMA), and longer runs are read from global memory.
constexpr int kStageRecs = 64;

// kMinBlocks: resident blocks per SM the registers are capped for (4: 64
// registers, no spills; 5: 48 registers, more warps, a few spills).
template <bool kMulti, bool kBins, bool kF64, int kMinBlocks>
__global__ void __launch_bounds__(kThreads, kMinBlocks) learned_refine_kernel(const LqArgs a) {
    __shared__ int2 s_buf[kThreads / 32][kWarpBuf];
    __shared__ unsigned s_cnt[kThreads / 32];
    __shared__ QueuedPair s_q[kThreads / 32][kQueue];
    __shared__ __align__(128) EntryRecord s_recs[kThreads / 32][kStageRecs];
    __shared__ uint64_t s_bar[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_cnt[warp] = 0;
        mbar_init(&s_bar[warp]);
    }
    __syncwarp();
    uint32_t phase = 0;
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    QueuedPair* qp = s_q[warp];
    const EntryRecord* st = s_recs[warp];
    const unsigned lt = (1u << lane) - 1u;
    const int64_t n = (int64_t)*a.n_grouped;
    unsigned long long n_cand = 0;
    unsigned n32 = 0, n64 = 0;
    int nq = 0;  // warp-uniform queue length
    for (;;) {
        const int64_t b0 = warp_grab(a.work, a.grab);
        if (b0 >= n) break;
        const int64_t e0 = b0 + a.grab < n ? b0 + a.grab : n;
        for (int64_t base = b0; base < e0; base += 32) {
            const GroupedLane g = load_grouped<kMulti>(a, base + lane, e0);
            const uint32_t maxlen = warp_max_u32(g.len);
            const EntryRecord* recs = job_desc<kMulti>(a, g.job).recs;
            // stage the packet's run of records (warp-uniform decision)
            const unsigned has = __ballot_sync(0xffffffffu, g.len > 0);
            const int first = has ? __ffs(has) - 1 : 0, last = has ? 31 - __clz(has) : 0;
            const uint32_t run_lo = __shfl_sync(0xffffffffu, g.lo, first);
            const uint32_t run_hi = __shfl_sync(0xffffffffu, g.lo + g.len, last);
            const int job0 = __shfl_sync(0xffffffffu, g.job, first);  // every lane takes part in the shuffle
            const bool one_job = !kMulti || __all_sync(0xffffffffu, g.len == 0 || g.job == job0);
            const bool staged = !a.no_stage && has != 0 && one_job && run_hi - run_lo <= (uint32_t)kStageRecs;
            if (staged) {
                __syncwarp();  // every lane is done with the buffer's previous run
                if (lane == 0) bulk_load(s_recs[warp], recs + run_lo, (run_hi - run_lo) * (uint32_t)sizeof(EntryRecord),
                                         &s_bar[warp]);
                if (!__all_sync(0xffffffffu, mbar_wait_bounded(&s_bar[warp], phase))) {
                    // record the timeout, give the copy one more bounded wait, stop this warp
                    if (lane == 0) atomicOr(&a.counters[4], 2ull);
                    mbar_wait_bounded(&s_bar[warp], phase);
                    return;
                }
                phase ^= 1u;
            }
            const float4* ib32 = job_desc<kMulti>(a, g.job).ib32;
            for (uint32_t k = 0; k < maxlen; ++k) {
                bool inbox = false;
                EntryRecord r;
                if (k < g.len) {
                    const uint32_t si = g.lo + k - run_lo;  // unsigned: below the run wraps to a large index
                    r = (staged && si < run_hi - run_lo) ? st[si] : recs[g.lo + k];
                    inbox = box_filter_fp32(r.box, g.p.qx, g.p.qy, g.dq);
                }
                // the point in the slot's frame; its error against the real p -
                // origin is at most dq + |off error| (in r.err with the vertex
                // error) + the rounding of this addition (es)
                float sx = 0.f, sy = 0.f, t = 0.f;
                bool walk = false, direct = false;
                if (inbox) {
                    ++n_cand;
                    sx = __fadd_rn(g.p.qx, r.offx);
                    sy = __fadd_rn(g.p.qy, r.offy);
                    const float es = __fmaf_ru(fmaxf(fabsf(sx), fabsf(sy)), 6.1e-8f, 1e-37f);
                    t = __fmul_ru(__fadd_ru(__fadd_ru(r.err, g.dq), es), 1.0001f);
                    walk = true;
                    if (!a.no_interior && entry_has_interior(r)) {
                        // strictly inside the slot's interior box, whatever the
                        // rounding: interior, no ring walk
                        const float4 ib = ib32[entry_slot(r)];
                        if (__fsub_rd(sx, t) > ib.x && __fadd_ru(sx, t) < ib.z && __fsub_rd(sy, t) > ib.y &&
                            __fadd_ru(sy, t) < ib.w) {
                            walk = false;
                            direct = (a.q.accept_mask >> LOC_INTERIOR) & 1;
                        }
                    }
                }
                wemit_sync(out, a.sink, direct, g.p.row,
                           direct ? job_desc<kMulti>(a, g.job).item_geom[entry_slot(r)] : 0);
                const unsigned m = __ballot_sync(0xffffffffu, walk);
                if (walk) {
                    // the queue entry as two 16-byte stores
                    float4* e = reinterpret_cast<float4*>(&qp[nq + __popc(m & lt)]);
                    e[0] = make_float4(sx, sy, t, __int_as_float(g.p.row));
                    e[1] = make_float4(__int_as_float(entry_slot(r)), __int_as_float(g.job), 0.f, 0.f);
                }
                nq += __popc(m);
                __syncwarp();
                if (nq >= 32) {
                    refine_queued<kMulti, kBins, kF64>(a, out, qp, 32, lane, n32, n64);
                    __syncwarp();
                    if (lane < nq - 32) qp[lane] = qp[32 + lane];
                    nq -= 32;
                    __syncwarp();
                }
            }
            wflush(out, a.sink, false);
        }
    }
    if (nq > 0) refine_queued<kMulti, kBins, kF64>(a, out, qp, nq, lane, n32, n64);
    wflush(out, a.sink, true);
    add_counter(a.counters, 5, n_cand);
    add_counter(a.counters, 2, n32);
    add_counter(a.counters, 3, n64);
}

int64_t stripe_cap_for(int64_t n) {
    const int64_t packets = (n + 31) / 32;
    return 32 * ((packets + kStripes - 1) / kStripes);
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

size_t learned_scratch_bytes(int64_t n, int64_t n_cells) {
    const int64_t cap = stripe_cap_for(n);
    return align256(sizeof(CellPoint) * (size_t)(kStripes * cap)) + align256(sizeof(uint32_t) * kStripes) +
           align256(sizeof(uint32_t) * (size_t)(n_cells > 0 ? n_cells : 1)) +
           align256(sizeof(CellPoint) * (size_t)(n > 0 ? n : 1)) + align256(sizeof(uint32_t));
}

void learned_scratch_carve(void* base, int64_t n, int64_t n_cells, LearnedScratch& sc) {
    char* p = (char*)base;
    sc.stripe_cap = stripe_cap_for(n);
    sc.staged = p;
    p += align256(sizeof(CellPoint) * (size_t)(kStripes * sc.stripe_cap));
    sc.stripe_count = (uint32_t*)p;
    p += align256(sizeof(uint32_t) * kStripes);
    sc.cell_count = (uint32_t*)p;
    p += align256(sizeof(uint32_t) * (size_t)(n_cells > 0 ? n_cells : 1));
    sc.grouped = p;
    p += align256(sizeof(CellPoint) * (size_t)(n > 0 ? n : 1));
    sc.n_grouped = (uint32_t*)p;
}

namespace {

// The refine variant for the launch shape: 5 or more blocks per SM asked for
// take the 48-register build, 4 (or the default) the 64-register one, 1 to 3
// the 80-register one.
template <bool kMulti, bool kBins>
const void* pick_refine(uint32_t flags, int blocks_per_sm) {
    if (flags & kLearnedFp64Walk) return (const void*)learned_refine_kernel<kMulti, kBins, true, 4>;
    if (blocks_per_sm >= 5) return (const void*)learned_refine_kernel<kMulti, kBins, false, 5>;
    if (blocks_per_sm >= 1 && blocks_per_sm <= 3) return (const void*)learned_refine_kernel<kMulti, kBins, false, 3>;
    return (const void*)learned_refine_kernel<kMulti, kBins, false, 4>;
}

// Grid of a persistent kernel: blocks_per_sm per SM when given (capped at the
// occupancy limit), else every block that fits; never more than the work needs.
int persistent_grid(const void* kernel, int64_t n, int blocks_per_sm) {
    int dev = 0, sms = 1, fit = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, kernel, kThreads, 0);
    fit = fit > 0 ? fit : 1;
    const int per = blocks_per_sm > 0 && blocks_per_sm < fit ? blocks_per_sm : fit;
    const int64_t need = (n + kThreads - 1) / kThreads;
    const int64_t g = (int64_t)per * sms;
    return (int)(need < 1 ? 1 : (need < g ? need : g));
}

template <bool kMulti>
int launch_passes(cudaStream_t s, vs_context* ctx, const LqArgs& a) {
    const int64_t n = a.q.n;
    const LearnedShape& sh = a.q.shape;
    const int map_grid = grid_for(n, kThreads, sh.map_blocks_per_sm > 0 ? sh.map_blocks_per_sm : 8);
    const bool two = sh.map_packets == 2;
    if (sh.flags & kLearnedBsearch) {
        if (two) learned_map_kernel<kMulti, true, 2><<<map_grid, kThreads, 0, s>>>(a);
        else learned_map_kernel<kMulti, true, 1><<<map_grid, kThreads, 0, s>>>(a);
    } else {
        if (two) learned_map_kernel<kMulti, false, 2><<<map_grid, kThreads, 0, s>>>(a);
        else learned_map_kernel<kMulti, false, 1><<<map_grid, kThreads, 0, s>>>(a);
    }
    VS_LAUNCHED("learned_map", s);
    VS_TRY(exclusive_scan_u32(a.cell_count, a.cell_count, a.q.n_cells, (uint32_t*)a.n_grouped, s));
    if (ctx) phase_mark(ctx, 1);
    learned_place_kernel<<<kStripes, kThreads, 0, s>>>(a);
    VS_LAUNCHED("learned_place", s);
    if (ctx) phase_mark(ctx, 2);
    if (a.q.accept_mask) {
        const void* kernel = a.q.has_ring_bins ? pick_refine<kMulti, true>(sh.flags, sh.refine_blocks_per_sm)
                                               : pick_refine<kMulti, false>(sh.flags, sh.refine_blocks_per_sm);
        const int grid = persistent_grid(kernel, n, sh.refine_blocks_per_sm);
        void* args[] = {(void*)&a};
        VS_CUDA_TRY(cudaLaunchKernel(kernel, dim3(grid), dim3(kThreads), args, 0, s));
        VS_LAUNCHED("learned_refine", s);
    } else {
        const void* kernel = (const void*)learned_bbox_kernel<kMulti>;
        const int grid = persistent_grid(kernel, n, sh.refine_blocks_per_sm);
        void* args[] = {(void*)&a};
        VS_CUDA_TRY(cudaLaunchKernel(kernel, dim3(grid), dim3(kThreads), args, 0, s));
        VS_LAUNCHED("learned_bbox", s);
    }
    return VS_OK;
}

}  // namespace

int enqueue_learned(cudaStream_t s, vs_context* ctx, const LearnedQuery& q, const LearnedJob* single,
                    const LearnedScratch& sc, const PairSink& sink, const DeferSink& defer,
                    unsigned long long* counters, unsigned long long* work) {
    LqArgs a{};
    a.q = q;
    if (single) a.single = *single;
    a.staged = (CellPoint*)sc.staged;
    a.stripe_count = sc.stripe_count;
    a.stripe_cap = sc.stripe_cap;
    a.cell_count = sc.cell_count;
    a.grouped = (CellPoint*)sc.grouped;
    a.n_grouped = sc.n_grouped;
    a.sink = sink;
    a.defer = defer;
    a.counters = counters;
    a.work = work;
    a.grab = q.shape.grab > 0 ? (int64_t)((q.shape.grab + 31) / 32 * 32) : kJoinGrab;
    a.no_stage = (q.shape.flags & kLearnedNoStage) != 0;
    a.no_interior = (q.shape.flags & kLearnedNoInterior) != 0;
    VS_CUDA_TRY(cudaMemsetAsync(sc.cell_count, 0, (size_t)(q.n_cells > 0 ? q.n_cells : 1) * sizeof(uint32_t), s));
    VS_CUDA_TRY(cudaMemsetAsync(sc.stripe_count, 0, (size_t)kStripes * sizeof(uint32_t), s));
    if (q.n_jobs > 1) return launch_passes<true>(s, ctx, a);
    return launch_passes<false>(s, ctx, a);
}

int launch_learned_join(vs_context* ctx, const vs_index* idx, const vs_points* pts, int accept_mask, int32_t* d_left,
                        int32_t* d_right, int64_t capacity, const DeferSink& dsink, int64_t row_base,
                        const LearnedShape& shape) {
    const LearnedIndex& li = idx->learned;
    cudaStream_t s = ctx->stream;
    Scratch<char> buf;
    VS_TRY(buf.alloc(learned_scratch_bytes(pts->n, li.n_cells), s));
    LearnedScratch sc;
    learned_scratch_carve(buf.p, pts->n, li.n_cells, sc);
    LearnedQuery q{};
    q.px = pts->d_x;
    q.py = pts->d_y;
    q.pvalid = pts->d_valid;
    q.n = pts->n;
    q.jobs = li.desc;
    q.n_jobs = 1;
    q.job_start = nullptr;
    q.n_cells = li.n_cells;
    q.accept_mask = accept_mask;
    q.has_ring_bins = idx->n_split_binned_rings > 0;
    q.row_base = row_base;
    q.shape = shape;
    const PairSink sink{d_left, d_right, (unsigned long long)(capacity > 0 ? capacity : 0), &ctx->d_counters[0]};
    return enqueue_learned(s, ctx, q, &li.h_desc, sc, sink, dsink, ctx->d_counters, &ctx->d_counters[kWorkCounter]);
}

}  // namespace vs
