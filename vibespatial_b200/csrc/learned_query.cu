// Learned + split-precision join: the query passes over the learned cell
// index (built in learned.cu), for one index or a batch of them.
//
// Three passes over the points (a counting sort keyed by the learned index's
// own positions, so no general sort is needed):
//   map      input order: the point's job (batch) -> level-L cell key ->
//            occupancy bit -> root table -> leaf model -> binary search inside
//            the leaf's error window -> cell index (or none); warp-aggregated
//            atomics on the per-cell counts return each point's rank within
//            its cell, and the matched points are appended to striped staging
//            regions
//   scatter  after an exclusive scan of the counts, every staged point writes
//            one aligned 32-byte record at start[cell] + rank, carrying its
//            cell's candidate range
//   refine   a warp takes 32 consecutive records, which share a candidate
//            list except at cell boundaries, so the lanes read each polygon's
//            data together (broadcast); each candidate is box-filtered in
//            FP32 (rounded outward); survivors are queued per warp and
//            refined 32 at a time with the FP32 crossing test on
//            tile-relative coordinates; only edges whose FP32 decision lies
//            within the rounding-error bound are re-decided in FP64, and a
//            pair the FP64 filter cannot certify is deferred to the exact pass.
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

namespace vs {
namespace {

constexpr int kThreads = 256;

// A matched query point as the map pass leaves it: coordinates, row, its
// job's cell index, its rank among the cell's points, and the job.
struct __align__(32) StagedPoint {
    double x, y;
    int32_t row;
    int32_t cell;
    uint32_t rank;
    int32_t job;
};

// The map pass appends matched points to kStripes regions of the staging
// array, region s taking the packets p with p % kStripes == s, so each
// region's append counter sees 1/kStripes of the atomics and a region never
// holds more than 32 * ceil(packets / kStripes) points.
constexpr int kStripes = 2048;

// A query point in cell order, with its cell's candidate range
// [lo, lo + len) of its job's per-entry records.  A full 32-byte sector, so
// the scatter writes whole sectors.
struct __align__(32) GroupedPoint {
    double x, y;
    int32_t row;
    uint32_t lo;
    uint32_t len;
    int32_t job;
};

// A (point, candidate) pair that passed the FP32 box filter, queued for the
// ring walk.
struct __align__(16) QueuedPair {
    double x, y;
    int32_t row;
    uint32_t rec;  // index into the job's per-entry records
    int32_t job;
    int32_t pad;
};
constexpr int kQueue = 64;  // >= 31 left over + 32 appended in one step

struct LqArgs {
    LearnedQuery q;
    LearnedJob single;  // the one job of a single join (kernel parameter space)
    StagedPoint* staged;
    uint32_t* stripe_count;
    int64_t stripe_cap;
    uint32_t* cell_count;
    GroupedPoint* grouped;
    const uint32_t* n_grouped;
    PairSink sink;
    DeferSink defer;
    unsigned long long* counters;
    unsigned long long* work;  // refine work queue (grouped points handed out)
};

// Job descriptor of a batch query (global memory) or of a single join (the
// kernel parameters: uniform reads, no extra registers).
template <bool kMulti>
__device__ __forceinline__ const LearnedJob& job_desc(const LqArgs& a, int job) {
    if constexpr (kMulti) return a.q.jobs[job];
    else return a.single;
}

// ------------------------------------------------------- split refine ---
// One edge in FP32 on tile-relative coordinates.  Returns false when some
// decision the exact walk needs lies within the rounding-error bound `t`
// (the caller then re-decides the edge in FP64); otherwise applies the same
// decision the exact walk would (the point cannot be on this edge).
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

// One edge (vertex ia -> vertex ib) of the split ring walk: FP32 first, the
// FP64 filter when the FP32 bound is inconclusive.  0: go on, 1: on the
// edge, 2: undecided by the FP64 filter too.
__device__ __forceinline__ int split_edge(double px, double py, float qx, float qy, float t, float2 a, float2 b,
                                          const double2* __restrict__ xy, int ia, int ib, bool& inside,
                                          unsigned& n32, unsigned& n64) {
    if (edge_step_fp32(a.x, a.y, b.x, b.y, qx, qy, t, inside)) {
        ++n32;
        return 0;
    }
    ++n64;
    const double2 A = xy[ia], B = xy[ib];
    return edge_step_filtered(A.x, A.y, B.x, B.y, px, py, inside);
}

// Split-precision location of a point in one ring, every edge.
__device__ __forceinline__ int ring_location_split(double px, double py, float qx, float qy, float t,
                                                   const float2* __restrict__ xy32, const double2* __restrict__ xy,
                                                   int start, int end, unsigned& n32, unsigned& n64) {
    if (end - start < 2) return LOC_OUTSIDE;
    bool inside = false;
    float2 a = xy32[end - 1];
    int ia = end - 1;
    for (int i = start; i < end; ++i) {
        const float2 b = xy32[i];
        const int r = split_edge(px, py, qx, qy, t, a, b, xy, ia, i, inside, n32, n64);
        if (r == 1) return LOC_BOUNDARY;
        if (r == 2) return LOC_UNDECIDED;
        a = b;
        ia = i;
    }
    return inside ? LOC_INTERIOR : LOC_OUTSIDE;
}

// The same for a ring with y-bins: only the edges of the point's bin, in ring
// order; an edge that continues the previous one reuses its end vertex.
__device__ __forceinline__ int ring_location_split_binned(double px, double py, float qx, float qy, float t,
                                                          const float2* __restrict__ xy32,
                                                          const double2* __restrict__ xy, int start, int end,
                                                          const RingBins& bins, const uint16_t* __restrict__ edges,
                                                          unsigned& n32, unsigned& n64) {
    bool inside = false;
    const int k = ring_bin_of(py, bins.y0, bins.scale);
    const uint32_t e1 = bins.off[k + 1];
    int last = -2;
    float2 lb = make_float2(0.f, 0.f);
    for (uint32_t e = bins.off[k]; e < e1; ++e) {
        const int i = start + edges[e];
        const int ia = i == start ? end - 1 : i - 1;
        const float2 a = ia == last ? lb : xy32[ia];
        const float2 b = xy32[i];
        const int r = split_edge(px, py, qx, qy, t, a, b, xy, ia, i, inside, n32, n64);
        if (r == 1) return LOC_BOUNDARY;
        if (r == 2) return LOC_UNDECIDED;
        last = i;
        lb = b;
    }
    return inside ? LOC_INTERIOR : LOC_OUTSIDE;
}

// kBins: the index has y-binned rings (kernels without bins carry no binned
// walk, which keeps their registers for the common short rings).
template <bool kBins>
__device__ __forceinline__ int geometry_location_split(double px, double py, float qx, float qy, float t,
                                                       const LearnedJob& J, int g, unsigned& n32, unsigned& n64) {
    const int p0 = J.geom_off[g], p1 = J.geom_off[g + 1];
    for (int part = p0; part < p1; ++part) {
        bool inside = false;
        const int r0 = J.part_off[part], r1 = J.part_off[part + 1];
        for (int ring = r0; ring < r1; ++ring) {
            const int c0 = J.ring_off[ring], c1 = J.ring_off[ring + 1];
            // the FP32 walk is cheap per edge, so bins pay off only on longer rings than for the FP64 walk
            const int rb = (kBins && J.rings.ring_bin && c1 - c0 >= kSplitBinMinVertices) ? J.rings.ring_bin[ring] : -1;
            const int k = rb >= 0
                              ? ring_location_split_binned(px, py, qx, qy, t, J.xy32, J.xy, c0, c1, J.rings.bins[rb],
                                                           J.rings.edges, n32, n64)
                              : ring_location_split(px, py, qx, qy, t, J.xy32, J.xy, c0, c1, n32, n64);
            if (k == LOC_BOUNDARY || k == LOC_UNDECIDED) return k;
            if (k == LOC_INTERIOR) inside = !inside;
        }
        if (inside) return LOC_INTERIOR;
    }
    return LOC_OUTSIDE;
}

// ---------------------------------------------------------------- map ---
// Exact lookup of a point's cell in job J's learned index: level-L cell key ->
// occupancy bit -> root table -> leaf model -> binary search inside the
// leaf's error window.  Returns the cell's index, or -1 when no stored cell
// matches (no polygon box overlaps the point's cell).
__device__ __forceinline__ int learned_lookup(const LearnedJob& J, double x, double y, const uint16_t* lut,
                                              unsigned long long& n_wide) {
    const uint32_t cell = hilbert_key_lut(quantize(x, J.lox, J.sx), quantize(y, J.loy, J.sy), J.L, lut);
    const uint32_t ob = cell >> J.occ_shift;
    if (!((J.occ[ob >> 5] >> (ob & 31)) & 1u)) return -1;
    const RmiLeaf lf = J.leaves[J.root_table[cell >> J.root_shift]];
    if (lf.lo > lf.hi) return -1;  // no stored key routes to this leaf
    const long long pred = rmi_predict(make_double2(lf.a, lf.b), cell);
    long long l0 = pred + lf.lo, h0 = pred + lf.hi + 1;  // search [l0, h0)
    l0 = l0 < 0 ? 0 : l0;
    h0 = h0 > J.n_cells ? J.n_cells : h0;
    if (h0 - l0 > 256) ++n_wide;
    const long long h1 = h0;
    while (l0 < h0) {
        const long long mid = (l0 + h0) >> 1;
        if (J.cell_keys[mid] < cell) l0 = mid + 1;
        else h0 = mid;
    }
    return (l0 < h1 && J.cell_keys[l0] == cell) ? (int)l0 : -1;
}

// Job of every lane's point: lane 0 binary-searches the packet's first point,
// the lanes step forward over the (contiguous) job ranges from there.
template <bool kMulti>
__device__ __forceinline__ int packet_job(const LearnedQuery& q, int64_t b0, int64_t i, int lane) {
    if (!kMulti || q.n_jobs <= 1) return 0;
    int j = 0;
    if (lane == 0) {
        int lo = 0, hi = q.n_jobs;  // last job with job_start[job] <= b0
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (q.job_start[mid] <= b0) lo = mid;
            else hi = mid;
        }
        j = lo;
    }
    j = __shfl_sync(0xffffffffu, j, 0);
    if (i < q.n)
        while (j + 1 < q.n_jobs && i >= q.job_start[j + 1]) ++j;
    return j;
}

// Pass 1 (map), points in input order: each point's cell and its rank among
// the cell's points (warp-aggregated atomics on the per-cell counts); the
// matched points are appended to the staging regions.
template <bool kMulti>
__global__ void __launch_bounds__(kThreads, 8) learned_map_kernel(const LqArgs a) {
    __shared__ uint16_t s_lut[kHilbertLutSize];
    hilbert_lut_init(s_lut);
    __syncthreads();
    const LearnedQuery& q = a.q;
    unsigned long long n_wide = 0;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    // Warp-uniform loop: the whole warp reaches the match and shuffle together.
    for (int64_t b0 = gw * 32; b0 < q.n; b0 += nw * 32) {
        const int64_t i = b0 + lane;
        const int job = packet_job<kMulti>(q, b0, i, lane);
        int c = -1, gc = -1;
        double x = 0.0, y = 0.0;
        if (i < q.n) {
            const LearnedJob& J = job_desc<kMulti>(a, job);
            x = q.px[i];
            y = q.py[i];
            if ((q.pvalid == nullptr || q.pvalid[i]) && J.n_cells > 0 && x >= J.lox && x <= J.hix && y >= J.loy &&
                y <= J.hiy)
                c = learned_lookup(J, x, y, s_lut, n_wide);
            if (c >= 0) gc = (int)(J.cell_base + (uint32_t)c);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, gc);
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (gc >= 0 && lane == leader) base = atomicAdd(&a.cell_count[gc], (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        // append the matched points of this packet to its stripe region
        const unsigned mm = __ballot_sync(0xffffffffu, gc >= 0);
        if (mm) {
            const int64_t stripe = (b0 >> 5) % kStripes;
            uint32_t sb = 0;
            if (lane == 0) sb = atomicAdd(&a.stripe_count[stripe], (uint32_t)__popc(mm));
            sb = __shfl_sync(0xffffffffu, sb, 0);
            if (gc >= 0) {
                StagedPoint p;
                p.x = x;
                p.y = y;
                p.row = (int32_t)(i + q.row_base);
                p.cell = c;
                p.rank = base + __popc(peers & lt);
                p.job = job;
                a.staged[stripe * a.stripe_cap + sb + __popc(mm & lt)] = p;
            }
        }
    }
    add_counter(a.counters, 6, n_wide);
}

// ------------------------------------------------------------ scatter ---
// Pass 2 (scatter): after the exclusive scan of the counts, every staged
// point writes one aligned 32-byte record at start[cell] + rank, carrying its
// cell's candidate range.  A block walks whole stripe regions (coalesced
// reads, every lane busy); each thread keeps kScatterUnroll records in flight.
#ifndef VS_SCATTER_UNROLL
#define VS_SCATTER_UNROLL 4
#endif
constexpr int kScatterUnroll = VS_SCATTER_UNROLL;

#ifndef VS_SCATTER_MIN_BLOCKS
#define VS_SCATTER_MIN_BLOCKS 1
#endif
template <bool kMulti>
__global__ void __launch_bounds__(kThreads, VS_SCATTER_MIN_BLOCKS) learned_scatter_kernel(const LqArgs a) {
    for (int stripe = blockIdx.x; stripe < kStripes; stripe += gridDim.x) {
        const uint32_t cnt = a.stripe_count[stripe];
        const StagedPoint* src = a.staged + (int64_t)stripe * a.stripe_cap;
        for (uint32_t k0 = threadIdx.x; k0 < cnt; k0 += blockDim.x * kScatterUnroll) {
            StagedPoint p[kScatterUnroll];
#pragma unroll
            for (int u = 0; u < kScatterUnroll; ++u) {
                const uint32_t k = k0 + u * blockDim.x;
                if (k < cnt) p[u] = src[k];
            }
            GroupedPoint g[kScatterUnroll];
            uint32_t pos[kScatterUnroll];
#pragma unroll
            for (int u = 0; u < kScatterUnroll; ++u) {
                const uint32_t k = k0 + u * blockDim.x;
                if (k < cnt) {
                    const LearnedJob& J = job_desc<kMulti>(a, p[u].job);
                    const int c = p[u].cell;
                    g[u].x = p[u].x;
                    g[u].y = p[u].y;
                    g[u].row = p[u].row;
                    g[u].lo = J.cell_start[c];
                    g[u].len = J.cell_start[c + 1] - g[u].lo;
                    g[u].job = p[u].job;
                    pos[u] = a.cell_count[J.cell_base + (uint32_t)c] + p[u].rank;
                }
            }
#pragma unroll
            for (int u = 0; u < kScatterUnroll; ++u)
                if (k0 + u * blockDim.x < cnt) a.grouped[pos[u]] = g[u];
        }
    }
}

// ------------------------------------------------------------- refine ---
#ifndef VS_JOIN_MIN_BLOCKS
#define VS_JOIN_MIN_BLOCKS 5
#endif
#ifndef VS_JOIN_GRAB
#define VS_JOIN_GRAB 32
#endif
constexpr int64_t kJoinGrab = VS_JOIN_GRAB;  // grouped points per work-queue grab (multiple of 32)

// FP32 box filter of one candidate record (rounded outward: never rejects a
// point of the box).
__device__ __forceinline__ bool box_filter_fp32(const SlotRecord* rp, double x, double y) {
    const double2 o = *reinterpret_cast<const double2*>(&rp->ox);
    const float4 bx = rp->box;
    const float qx = __double2float_rn(x - o.x), qy = __double2float_rn(y - o.y);
    const float dp = __fmaf_ru(fmaxf(fabsf(qx), fabsf(qy)), 6.1e-8f, 1e-37f);
    return !(__fadd_ru(qx, dp) < bx.x || __fsub_rd(qx, dp) > bx.z || __fadd_ru(qy, dp) < bx.y ||
             __fsub_rd(qy, dp) > bx.w);
}

// Box candidates only (predicate BBOX): a warp takes 32 consecutive grouped
// points and walks their candidate lists; the FP32 filter's survivors are
// decided exactly on the FP64 box.
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
        const int64_t b0 = warp_grab(a.work, kJoinGrab);
        if (b0 >= n) break;
        const int64_t e0 = b0 + kJoinGrab < n ? b0 + kJoinGrab : n;
        for (int64_t base = b0; base < e0; base += 32) {
            const int64_t j = base + lane;
            GroupedPoint g{0.0, 0.0, 0, 0, 0, 0};
            if (j < e0) g = a.grouped[j];
            uint32_t maxlen = g.len;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const uint32_t t = __shfl_xor_sync(0xffffffffu, maxlen, o);
                maxlen = t > maxlen ? t : maxlen;
            }
            for (uint32_t k = 0; k < maxlen; ++k) {
                bool want = false;
                int32_t right = 0;
                if (k < g.len) {
                    const LearnedJob& J = job_desc<kMulti>(a, g.job);
                    const SlotRecord* rp = J.recs + g.lo + k;
                    if (box_filter_fp32(rp, g.x, g.y)) {
                        const int slot = rp->slot;
                        const vs_box bb = J.boxes[slot];
                        if (g.x >= bb.minx && g.x <= bb.maxx && g.y >= bb.miny && g.y <= bb.maxy) {
                            ++n_cand;
                            want = true;
                            right = J.item_geom[slot];
                        }
                    }
                }
                wemit_sync(out, a.sink, want, g.row, right);
            }
            wflush(out, a.sink, false);
        }
    }
    wflush(out, a.sink, true);
    add_counter(a.counters, 5, n_cand);
}

// Ring walks of up to 32 queued pairs, one per lane.
template <bool kMulti, bool kBins>
__device__ __forceinline__ void refine_queued(const LqArgs& a, const WarpOut& out, const QueuedPair* qp, int nq,
                                              int lane, unsigned& n32, unsigned& n64) {
    bool want = false;
    int32_t row = 0, right = 0;
    if (lane < nq) {
        const QueuedPair jb = qp[lane];
        const LearnedJob& J = job_desc<kMulti>(a, jb.job);
        row = jb.row;
        const SlotRecord r = J.recs[jb.rec];
        const float qx = __double2float_rn(jb.x - r.ox), qy = __double2float_rn(jb.y - r.oy);
        const float dp = __fmaf_ru(fmaxf(fabsf(qx), fabsf(qy)), 6.1e-8f, 1e-37f);
        const float t = __fmul_ru(__fadd_ru(r.err, dp), 1.0001f);
        const int loc = r.c0 >= 0 ? ring_location_split(jb.x, jb.y, qx, qy, t, J.xy32, J.xy, r.c0, r.c1, n32, n64)
                                  : geometry_location_split<kBins>(jb.x, jb.y, qx, qy, t, J, r.slot, n32, n64);
        if (loc == LOC_UNDECIDED) {
            defer(a.defer, jb.row, r.slot);  // a batch's exact pass finds the job from the row
        } else if ((a.q.accept_mask >> loc) & 1) {
            want = true;
            right = J.item_geom[r.slot];
        }
    }
    wemit_sync(out, a.sink, want, row, right);
}

// Pass 3 with a location test: the warp walks its grouped points' candidate
// lists, and every (point, candidate) pair that passes the FP32 box filter is
// appended to a warp-local queue in shared memory.  Each time 32 pairs are
// queued, every lane refines one of them, so the ring walks, which dominate,
// run with all lanes busy instead of only the lanes whose point lies in the
// current candidate's box.  Neighbouring queue entries mostly share a
// polygon, so vertex reads stay broadcasts.
template <bool kMulti, bool kBins>
__global__ void __launch_bounds__(kThreads, VS_JOIN_MIN_BLOCKS) learned_refine_kernel(const LqArgs a) {
    __shared__ int2 s_buf[kThreads / 32][kWarpBuf];
    __shared__ unsigned s_cnt[kThreads / 32];
    __shared__ QueuedPair s_q[kThreads / 32][kQueue];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_cnt[warp] = 0;
    __syncwarp();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    QueuedPair* qp = s_q[warp];
    const unsigned lt = (1u << lane) - 1u;
    const int64_t n = (int64_t)*a.n_grouped;
    unsigned long long n_cand = 0;
    unsigned n32 = 0, n64 = 0;
    int nq = 0;  // warp-uniform queue length
    for (;;) {
        const int64_t b0 = warp_grab(a.work, kJoinGrab);
        if (b0 >= n) break;
        const int64_t e0 = b0 + kJoinGrab < n ? b0 + kJoinGrab : n;
        for (int64_t base = b0; base < e0; base += 32) {
            const int64_t j = base + lane;
            GroupedPoint g{0.0, 0.0, 0, 0, 0, 0};
            if (j < e0) g = a.grouped[j];
            uint32_t maxlen = g.len;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const uint32_t t = __shfl_xor_sync(0xffffffffu, maxlen, o);
                maxlen = t > maxlen ? t : maxlen;
            }
            const SlotRecord* recs = job_desc<kMulti>(a, g.job).recs;
            for (uint32_t k = 0; k < maxlen; ++k) {
                const bool inbox = k < g.len && box_filter_fp32(recs + g.lo + k, g.x, g.y);
                const unsigned m = __ballot_sync(0xffffffffu, inbox);
                if (inbox) {
                    QueuedPair& e = qp[nq + __popc(m & lt)];
                    e.x = g.x;
                    e.y = g.y;
                    e.row = g.row;
                    e.rec = g.lo + k;
                    e.job = g.job;
                    ++n_cand;
                }
                nq += __popc(m);
                __syncwarp();
                if (nq >= 32) {
                    refine_queued<kMulti, kBins>(a, out, qp, 32, lane, n32, n64);
                    __syncwarp();
                    if (lane < nq - 32) qp[lane] = qp[32 + lane];
                    nq -= 32;
                    __syncwarp();
                }
            }
            wflush(out, a.sink, false);
        }
    }
    if (nq > 0) refine_queued<kMulti, kBins>(a, out, qp, nq, lane, n32, n64);
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
    return align256(sizeof(StagedPoint) * (size_t)(kStripes * cap)) + align256(sizeof(uint32_t) * kStripes) +
           align256(sizeof(uint32_t) * (size_t)(n_cells > 0 ? n_cells : 1)) +
           align256(sizeof(GroupedPoint) * (size_t)(n > 0 ? n : 1)) + align256(sizeof(uint32_t));
}

void learned_scratch_carve(void* base, int64_t n, int64_t n_cells, LearnedScratch& sc) {
    char* p = (char*)base;
    sc.stripe_cap = stripe_cap_for(n);
    sc.staged = p;
    p += align256(sizeof(StagedPoint) * (size_t)(kStripes * sc.stripe_cap));
    sc.stripe_count = (uint32_t*)p;
    p += align256(sizeof(uint32_t) * kStripes);
    sc.cell_count = (uint32_t*)p;
    p += align256(sizeof(uint32_t) * (size_t)(n_cells > 0 ? n_cells : 1));
    sc.grouped = p;
    p += align256(sizeof(GroupedPoint) * (size_t)(n > 0 ? n : 1));
    sc.n_grouped = (uint32_t*)p;
}

namespace {

#ifndef VS_LEARNED_BLOCKS_PER_SM
#define VS_LEARNED_BLOCKS_PER_SM 8  // map blocks per SM (0: one resident wave)
#endif

template <bool kMulti>
int launch_passes(cudaStream_t s, vs_context* ctx, const LqArgs& a) {
    const int64_t n = a.q.n;
    const int map_grid = VS_LEARNED_BLOCKS_PER_SM > 0 ? grid_for(n, kThreads, VS_LEARNED_BLOCKS_PER_SM)
                                                      : resident_grid(learned_map_kernel<kMulti>, n, kThreads);
    learned_map_kernel<kMulti><<<map_grid, kThreads, 0, s>>>(a);
    VS_LAUNCHED("learned_map", s);
    VS_TRY(exclusive_scan_u32(a.cell_count, a.cell_count, a.q.n_cells, (uint32_t*)a.n_grouped, s));
    if (ctx) phase_mark(ctx, 1);
    learned_scatter_kernel<kMulti><<<kStripes, kThreads, 0, s>>>(a);
    VS_LAUNCHED("learned_scatter", s);
    if (ctx) phase_mark(ctx, 2);
    if (a.q.accept_mask) {
        auto* kernel = a.q.has_ring_bins ? learned_refine_kernel<kMulti, true> : learned_refine_kernel<kMulti, false>;
        kernel<<<resident_grid(kernel, n, kThreads), kThreads, 0, s>>>(a);
        VS_LAUNCHED("learned_refine", s);
    } else {
        learned_bbox_kernel<kMulti><<<resident_grid(learned_bbox_kernel<kMulti>, n, kThreads), kThreads, 0, s>>>(a);
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
    a.staged = (StagedPoint*)sc.staged;
    a.stripe_count = sc.stripe_count;
    a.stripe_cap = sc.stripe_cap;
    a.cell_count = sc.cell_count;
    a.grouped = (GroupedPoint*)sc.grouped;
    a.n_grouped = sc.n_grouped;
    a.sink = sink;
    a.defer = defer;
    a.counters = counters;
    a.work = work;
    VS_CUDA_TRY(cudaMemsetAsync(sc.cell_count, 0, (size_t)(q.n_cells > 0 ? q.n_cells : 1) * sizeof(uint32_t), s));
    VS_CUDA_TRY(cudaMemsetAsync(sc.stripe_count, 0, (size_t)kStripes * sizeof(uint32_t), s));
    if (q.n_jobs > 1) return launch_passes<true>(s, ctx, a);
    return launch_passes<false>(s, ctx, a);
    return VS_OK;
}

int launch_learned_join(vs_context* ctx, const vs_index* idx, const vs_points* pts, int accept_mask, int32_t* d_left,
                        int32_t* d_right, int64_t capacity, const DeferSink& dsink, int64_t row_base) {
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
    const PairSink sink{d_left, d_right, (unsigned long long)(capacity > 0 ? capacity : 0), &ctx->d_counters[0]};
    return enqueue_learned(s, ctx, q, &li.h_desc, sc, sink, dsink, ctx->d_counters, &ctx->d_counters[kWorkCounter]);
}

}  // namespace vs
