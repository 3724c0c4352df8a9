// Point x polygon join on the packed Hilbert R-tree (the plain method),
// element-wise location, and pair sorting.
//
// Reference behaviour replaced (src/vibespatial/...):
//   spatial/spatial_index_device.py:228-1035   candidates: Morton range +
//       serial per-query scan, count pass -> exclusive_sum -> host fence on
//       the total -> scatter pass
//   spatial/query_utils.py:578-868             refine: one thread per
//       candidate pair, then boolean-mask compaction d_left[keep]
//
// Query points are first keyed (level-16 Hilbert key in the polygon frame;
// points outside the frame, null or NaN get the sentinel key and are never
// visited) and radix-sorted, so the 32 lanes of a warp hold spatially
// coherent points.  Each warp then walks the R-tree once for its packet of
// points: lanes 0-15 load the 16 children of the current node (coalesced,
// upper levels from shared memory), test them against the packet's bounding
// box and push the hits on a warp-shared stack in shared memory.  At the leaf
// level every lane tests its own point against the hit item boxes and refines
// each hit immediately (stage-A filtered orientation; a pair the filter cannot
// certify is deferred to the exact pass); accepted pairs go through a
// warp-private buffer.  No candidate array, no count pass, no host fence, no
// block-wide barrier inside the loop.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "emit.cuh"
#include "exact.cuh"
#include "hilbert.cuh"
#include "index.cuh"
#include "join.cuh"
#include "primitives.cuh"
#include "tma.cuh"

namespace vs {
namespace {

constexpr int kJoinThreads = 256;
constexpr int kWarps = kJoinThreads / 32;
constexpr int kStack = 112;            // > (fanout-1) * (max levels-2) + 1
constexpr int kMaxStagedBoxes = 273;   // 1 + 16 + 256 FP64 boxes (~8.5 KB)

struct RtreeArgs {
    const double* px;
    const double* py;
    const uint8_t* pvalid;
    int64_t n;
    const uint32_t* order;     // sorted position -> point row
    const uint32_t* n_sorted;  // points with a valid key (a prefix of order)
    const vs_box* nodes;
    int64_t level_off[kMaxLevels];
    int64_t level_size[kMaxLevels];
    int levels;
    int stage_level;  // levels >= stage_level live in shared memory
    int staged;       // number of staged boxes
    const int32_t* item_geom;
    const int32_t* geom_off;
    const int32_t* part_off;
    const int32_t* ring_off;
    const double2* xy;
    int accept_mask;  // bit k: location k accepted; 0 = box candidates only
    PairSink sink;
    DeferSink defer;
    unsigned long long* counters;
    unsigned long long* work;  // traversal work queue (sorted points handed out)
    RingIndex rings;           // y-bins of the long rings
    int64_t row_base;          // added to emitted / deferred rows (chunked joins)
};

#ifndef VS_RTREE_GRAB
#define VS_RTREE_GRAB 64
#endif
constexpr int64_t kRtreeGrab = VS_RTREE_GRAB;  // sorted points per work-queue grab (multiple of 32)

__device__ __forceinline__ bool box_has(const vs_box& b, double x, double y) {
    return x >= b.minx && x <= b.maxx && y >= b.miny && y <= b.maxy;
}

__device__ __forceinline__ bool box_overlaps(const vs_box& b, double x0, double y0, double x1, double y1) {
    return b.minx <= x1 && b.maxx >= x0 && b.miny <= y1 && b.maxy >= y0;
}

// clamp: points outside the frame are keyed at the nearest frame position
// and kept (distance joins); otherwise they get the sentinel key.
__global__ void point_sort_key_kernel(vs_points p, const double* __restrict__ frame, uint32_t* __restrict__ keys,
                                      uint32_t* __restrict__ idx, uint32_t* __restrict__ n_valid, bool clamp) {
    __shared__ uint16_t s_lut[kHilbertLutSize];
    hilbert_lut_init(s_lut);
    __syncthreads();
    const double f0 = frame[0], f1 = frame[1], f2 = frame[2], f3 = frame[3];
    const double sx = f2 > f0 ? 4294967295.0 / (f2 - f0) : 0.0;
    const double sy = f3 > f1 ? 4294967295.0 / (f3 - f1) : 0.0;
    uint32_t cnt = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.n; i += (int64_t)gridDim.x * blockDim.x) {
        double x = p.d_x[i], y = p.d_y[i];
        if (clamp && x == x && y == y) {
            x = fmin(fmax(x, f0), f2);
            y = fmin(fmax(y, f1), f3);
        }
        const bool ok = (p.d_valid == nullptr || p.d_valid[i]) && x >= f0 && x <= f2 && y >= f1 && y <= f3;
        uint32_t k = 0xffffffffu;
        if (ok) {
            // The sort orders the top 24 bits only: keep valid keys out of the
            // sentinel's top-24 group, so every valid point sorts before it.
            k = hilbert_key_lut(quantize(x, f0, sx), quantize(y, f1, sy), 16, s_lut);
            if (k > 0xfffffeffu) k = 0xfffffeffu;
        }
        keys[i] = k;
        idx[i] = (uint32_t)i;
        cnt += ok ? 1u : 0u;
    }
    // one atomic per block
    cnt = (uint32_t)warp_sum(cnt);
    __shared__ uint32_t wsum[32];
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += wsum[w];
        if (t) atomicAdd(n_valid, t);
    }
}

// kBulk: leaf blocks (up to 16 FP64 boxes, 512 B) arrive by one bulk copy
// (TMA, cp.async.bulk) into the warp's item buffer instead of lane loads
// (VS_JOIN_BULK_LEAVES).
// kBins: the index has y-binned rings (kernels without bins carry no binned
// walk, which keeps their registers for the plain one).
template <bool kBulk, bool kBins>
__global__ void __launch_bounds__(kJoinThreads) join_rtree_packet_kernel(const RtreeArgs a) {
    const RingIndex rings = kBins ? a.rings : RingIndex{};
    extern __shared__ vs_box s_nodes[];
    __shared__ int2 s_buf[kWarps][kWarpBuf];
    __shared__ unsigned s_cnt[kWarps];
    __shared__ int s_stack[kWarps][kStack];
    __shared__ vs_box s_items[kWarps][kFanout];
    __shared__ uint64_t s_bar[kWarps];
    const int64_t stage_base = a.level_off[a.stage_level];
    for (int k = threadIdx.x; k < a.staged; k += blockDim.x) s_nodes[k] = a.nodes[stage_base + k];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_cnt[warp] = 0;
        mbar_init(&s_bar[warp]);
    }
    uint32_t phase = 0;
    __syncthreads();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    const unsigned lt = (1u << lane) - 1u;
    const int top = a.levels - 1;
    const int64_t n = (int64_t)*a.n_sorted;
    unsigned long long n_cand = 0;
    for (;;) {
        const int64_t b0 = warp_grab(a.work, kRtreeGrab);
        if (b0 >= n) break;
        const int64_t e0 = b0 + kRtreeGrab < n ? b0 + kRtreeGrab : n;
        for (int64_t base = b0; base < e0; base += 32) {
            const int64_t i = base + lane;
            const bool active = i < e0;
            double x = 0.0, y = 0.0;
            int32_t row = -1;
            int32_t grow = -1;  // the row reported for the point
            if (active) {
                row = (int32_t)a.order[i];
                x = a.px[row];
                y = a.py[row];
                grow = (int32_t)(row + a.row_base);
            }
            double x0 = active ? x : INFINITY, x1 = active ? x : -INFINITY;
            double y0 = active ? y : INFINITY, y1 = active ? y : -INFINITY;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                x0 = fmin(x0, __shfl_xor_sync(0xffffffffu, x0, o));
                x1 = fmax(x1, __shfl_xor_sync(0xffffffffu, x1, o));
                y0 = fmin(y0, __shfl_xor_sync(0xffffffffu, y0, o));
                y1 = fmax(y1, __shfl_xor_sync(0xffffffffu, y1, o));
            }
            int sp = 0;
            const vs_box root = s_nodes[a.level_off[top] - stage_base];
            if (box_overlaps(root, x0, y0, x1, y1)) {
                if (top == 0) {
                    // a single polygon: the root is the item
                    bool want = false;
                    if (active && box_has(root, x, y)) {
                        ++n_cand;
                        const int loc = a.accept_mask ? geometry_location_filtered(x, y, a.xy, a.ring_off, a.part_off,
                                                                                   a.geom_off, 0, rings) : 0;
                        if (loc == LOC_UNDECIDED) defer(a.defer, grow, 0);
                        else want = !a.accept_mask || ((a.accept_mask >> loc) & 1);
                    }
                    wemit_sync(out, a.sink, want, grow, a.item_geom[0]);
                } else {
                    if (lane == 0) s_stack[warp][0] = top;  // node 0 of the top level
                    sp = 1;
                }
            }
            __syncwarp();
            while (sp > 0) {
                --sp;
                const int e = s_stack[warp][sp];
                __syncwarp();
                const int cl = (e & 15) - 1;
                const int64_t c = (int64_t)(e >> 4) * kFanout + (lane & 15);
                const bool in_range = lane < kFanout && c < a.level_size[cl];
                vs_box b{INFINITY, INFINITY, -INFINITY, -INFINITY};
                const bool bulk = kBulk && cl == 0 && cl < a.stage_level;  // warp-uniform
                if (bulk) {
                    // The leaf block (up to 16 boxes, 32 B each, 512-B aligned) arrives in the
                    // warp's item buffer by one bulk copy; the lanes then read their box from it.
                    const int64_t first = (int64_t)(e >> 4) * kFanout;
                    const int64_t left = a.level_size[0] - first;
                    const uint32_t bytes = (uint32_t)((left < kFanout ? left : kFanout) * sizeof(vs_box));
                    if (lane == 0) bulk_load(s_items[warp], a.nodes + first, bytes, &s_bar[warp]);
                    const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&s_bar[warp], phase));
                    if (!ok) {
                        // record the timeout, give the copy one more bounded wait, stop this warp
                        if (lane == 0) atomicOr(&a.counters[4], 2ull);
                        mbar_wait_bounded(&s_bar[warp], phase);
                        return;
                    }
                    phase ^= 1u;
                    if (in_range) b = s_items[warp][lane];
                } else if (in_range) {
                    b = cl >= a.stage_level ? s_nodes[a.level_off[cl] - stage_base + c] : a.nodes[a.level_off[cl] + c];
                }
                const bool hit = in_range && box_overlaps(b, x0, y0, x1, y1);
                const unsigned m = __ballot_sync(0xffffffffu, hit);
                if (cl > 0) {
                    if (hit) {
                        const int pos = sp + __popc(m & lt);
                        if (pos < kStack) s_stack[warp][pos] = (int)(c << 4) | cl;
                    }
                    int add = __popc(m);
                    if (sp + add > kStack) {
                        if (lane == 0) atomicOr(&a.counters[4], 1ull);  // cannot happen for < 2^31 items
                        add = kStack - sp;
                    }
                    sp += add;
                    __syncwarp();
                } else {
                    if (!bulk && lane < kFanout) s_items[warp][lane] = b;
                    __syncwarp();
                    unsigned mm = m;
                    const int64_t slot0 = (int64_t)(e >> 4) * kFanout;
                    while (mm) {
                        const int j = __ffs(mm) - 1;
                        mm &= mm - 1;
                        const vs_box ib = s_items[warp][j];
                        const int slot = (int)(slot0 + j);
                        bool want = false;
                        if (active && box_has(ib, x, y)) {
                            ++n_cand;
                            int loc = 0;
                            if (a.accept_mask)
                                loc = geometry_location_filtered(x, y, a.xy, a.ring_off, a.part_off, a.geom_off, slot,
                                                                 rings);
                            if (loc == LOC_UNDECIDED) defer(a.defer, grow, slot);
                            else want = !a.accept_mask || ((a.accept_mask >> loc) & 1);
                        }
                        wemit_sync(out, a.sink, want, grow, a.item_geom[slot]);
                    }
                    __syncwarp();
                }
            }
            wflush(out, a.sink, false);
        }
    }
    wflush(out, a.sink, true);
    add_counter(a.counters, 5, n_cand);
}

// Every point against every polygon box, one thread per point in input order
// (small joins and cross-checks).
__global__ void __launch_bounds__(kJoinThreads) join_brute_kernel(const RtreeArgs a) {
    __shared__ int2 s_buf[kWarps][kWarpBuf];
    __shared__ unsigned s_cnt[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_cnt[warp] = 0;
    __syncwarp();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    const int64_t M = a.level_size[0];
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned long long n_cand = 0;
    for (int64_t base = gw * 32; base < a.n; base += nw * 32) {
        const int64_t i = base + lane;
        const bool act = i < a.n && (a.pvalid == nullptr || a.pvalid[i]);
        const double x = act ? a.px[i] : 0.0, y = act ? a.py[i] : 0.0;
        for (int64_t c = 0; c < M; ++c) {  // the same trip count in every lane
            bool want = false;
            if (act && box_has(a.nodes[c], x, y)) {
                ++n_cand;
                int loc = 0;
                if (a.accept_mask)
                    loc = geometry_location_filtered(x, y, a.xy, a.ring_off, a.part_off, a.geom_off, (int)c, a.rings);
                if (loc == LOC_UNDECIDED) defer(a.defer, (int32_t)(i + a.row_base), (int32_t)c);
                else want = !a.accept_mask || ((a.accept_mask >> loc) & 1);
            }
            wemit_sync(out, a.sink, want, (int32_t)(i + a.row_base), a.item_geom[c]);
        }
        wflush(out, a.sink, false);
    }
    wflush(out, a.sink, true);
    add_counter(a.counters, 5, n_cand);
}

// Exact pass over the deferred (point row, polygon slot) pairs: the full
// location with the exact orientation stage.
struct ResolveArgs {
    const double* px;
    const double* py;
    const int32_t* item_geom;
    const int32_t* geom_off;
    const int32_t* part_off;
    const int32_t* ring_off;
    const double2* xy;
    int accept_mask;
    const int2* pairs;
    unsigned long long capacity;
    const unsigned long long* count;
    PairSink sink;
    unsigned long long* counters;
    RingIndex rings;
    int64_t row_base;  // deferred rows are chunk rows + row_base
};

__global__ void __launch_bounds__(kJoinThreads) resolve_deferred_kernel(const ResolveArgs a) {
    __shared__ int2 s_buf[kWarps][kWarpBuf];
    __shared__ unsigned s_cnt[kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_cnt[warp] = 0;
    __syncwarp();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    const unsigned long long cnt = *a.count;
    const int64_t n = (int64_t)(cnt < a.capacity ? cnt : a.capacity);
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned n_exact = 0;
    for (int64_t base = gw * 32; base < n; base += nw * 32) {
        const int64_t k = base + lane;
        bool want = false;
        int2 pr = make_int2(0, 0);
        if (k < n) {
            pr = a.pairs[k];
            const double x = a.px[pr.x - a.row_base], y = a.py[pr.x - a.row_base];
            const int loc = geometry_location(x, y, a.xy, a.ring_off, a.part_off, a.geom_off, pr.y, a.rings, n_exact);
            want = (a.accept_mask >> loc) & 1;
        }
        wemit_sync(out, a.sink, want, pr.x, want ? a.item_geom[pr.y] : 0);
        wflush(out, a.sink, false);
    }
    wflush(out, a.sink, true);
    add_counter(a.counters, 1, n_exact);
}

__global__ void locate_aligned_kernel(vs_points pts, vs_polygons polys, uint8_t* __restrict__ out,
                                      unsigned long long* counters) {
    unsigned n_exact = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < pts.n; i += (int64_t)gridDim.x * blockDim.x) {
        const bool pv = pts.d_valid == nullptr || pts.d_valid[i];
        const bool gv = polys.d_valid == nullptr || polys.d_valid[i];
        const double x = pts.d_x[i], y = pts.d_y[i];
        if (!pv || !gv || isnan(x) || isnan(y)) {
            out[i] = 255;
            continue;
        }
        out[i] = (uint8_t)geometry_location_soa(x, y, polys.d_x, polys.d_y, polys.d_ring_off, polys.d_part_off,
                                                polys.d_geom_off, (int)i, n_exact);
    }
    if (n_exact) atomicAdd(&counters[1], (unsigned long long)n_exact);
}

__global__ void pack_pairs_kernel(const int32_t* __restrict__ l, const int32_t* __restrict__ r, int64_t n, int rbits,
                                  uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        keys[k] = ((uint64_t)(uint32_t)l[k] << rbits) | (uint64_t)(uint32_t)r[k];
        vals[k] = 0;
    }
}

__global__ void unpack_pairs_kernel(const uint64_t* __restrict__ keys, int64_t n, int rbits, int32_t* __restrict__ l,
                                    int32_t* __restrict__ r) {
    const uint64_t rmask = rbits >= 64 ? ~0ull : ((1ull << rbits) - 1);
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        l[k] = (int32_t)(keys[k] >> rbits);
        r[k] = (int32_t)(keys[k] & rmask);
    }
}

int bits_for(uint64_t v) {
    int b = 1;
    while (b < 63 && (1ull << b) <= v) ++b;
    return b;
}

}  // namespace

int accept_mask_for(int predicate, int* mask) {
    switch (predicate) {
        case VS_PRED_BBOX: *mask = 0; return VS_OK;
        case VS_PRED_INTERSECTS: *mask = (1 << LOC_BOUNDARY) | (1 << LOC_INTERIOR); return VS_OK;
        case VS_PRED_WITHIN: *mask = 1 << LOC_INTERIOR; return VS_OK;
        case VS_PRED_COVERED_BY: *mask = (1 << LOC_BOUNDARY) | (1 << LOC_INTERIOR); return VS_OK;
        case VS_PRED_TOUCHES: *mask = 1 << LOC_BOUNDARY; return VS_OK;
        default: set_error("unknown predicate code %d", predicate); return VS_E_ARG;
    }
}

int prepare_queries(vs_context* ctx, const vs_index* idx, const vs_points* pts, QueryOrder& q, bool clamp) {
    cudaStream_t s = ctx->stream;
    const int64_t n = pts->n;
    VS_TRY(q.keys.alloc((size_t)n, s));
    VS_TRY(q.order.alloc((size_t)n, s));
    VS_TRY(q.n_valid.alloc(1, s));
    VS_CUDA_TRY(cudaMemsetAsync(q.n_valid.p, 0, sizeof(uint32_t), s));
    point_sort_key_kernel<<<resident_grid(point_sort_key_kernel, n, 256), 256, 0, s>>>(*pts, idx->frame, q.keys.p, q.order.p, q.n_valid.p,
                                                                                   clamp);
    VS_LAUNCHED("point_sort_key", s);
    // Sorting by the top 24 key bits (a level-12 Hilbert cell) already makes
    // a warp's 32 points spatially coherent; the low byte is left unsorted.
    VS_TRY(radix_sort_u32_u32(q.keys.p, q.order.p, n, 32, s, 8));
    return VS_OK;
}

int launch_rtree_join(vs_context* ctx, const vs_index* idx, const vs_points* pts, int accept_mask, bool brute,
                      bool bulk_leaves, int32_t* d_left, int32_t* d_right, int64_t capacity, const DeferSink& dsink,
                      int64_t row_base) {
    RtreeArgs a{};
    a.px = pts->d_x;
    a.py = pts->d_y;
    a.pvalid = pts->d_valid;
    a.n = pts->n;
    a.nodes = idx->nodes;
    for (int l = 0; l < kMaxLevels; ++l) {
        a.level_off[l] = idx->level_off[l];
        a.level_size[l] = idx->level_size[l];
    }
    a.levels = idx->levels;
    // Stage the top levels whose boxes fit the shared-memory budget.
    int sl = idx->levels - 1;
    int64_t staged = idx->level_size[sl];
    while (sl > 0 && staged + idx->level_size[sl - 1] <= kMaxStagedBoxes) {
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
    a.accept_mask = accept_mask;
    a.sink = PairSink{d_left, d_right, (unsigned long long)(capacity > 0 ? capacity : 0), &ctx->d_counters[0]};
    a.defer = dsink;
    a.counters = ctx->d_counters;
    a.rings = idx->ring_index();
    a.row_base = row_base;
    if (brute) {
        phase_mark(ctx, 1);
        phase_mark(ctx, 2);
        join_brute_kernel<<<resident_grid(join_brute_kernel, pts->n, kJoinThreads), kJoinThreads, 0, ctx->stream>>>(a);
        VS_LAUNCHED("join_brute", ctx->stream);
        return VS_OK;
    }
    QueryOrder q;
    VS_TRY(prepare_queries(ctx, idx, pts, q));
    phase_mark(ctx, 1);
    phase_mark(ctx, 2);
    a.order = q.order.p;
    a.n_sorted = q.n_valid.p;
    a.work = &ctx->d_counters[kWorkCounter];
    const size_t smem = (size_t)a.staged * sizeof(vs_box);
    const bool bins = idx->ring_bin != nullptr;
    auto* kernel = bulk_leaves ? (bins ? join_rtree_packet_kernel<true, true> : join_rtree_packet_kernel<true, false>)
                               : (bins ? join_rtree_packet_kernel<false, true> : join_rtree_packet_kernel<false, false>);
    VS_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kernel<<<resident_grid(kernel, pts->n, kJoinThreads, smem), kJoinThreads, smem, ctx->stream>>>(a);
    VS_LAUNCHED("join_rtree_packet", ctx->stream);
    return VS_OK;
}

int launch_resolve_deferred(vs_context* ctx, const vs_index* idx, const vs_points* pts, int accept_mask,
                            int32_t* d_left, int32_t* d_right, int64_t capacity, const DeferSink& dsink,
                            int64_t row_base) {
    ResolveArgs a{};
    a.px = pts->d_x;
    a.py = pts->d_y;
    a.item_geom = idx->item_geom;
    a.geom_off = idx->geom_off;
    a.part_off = idx->part_off;
    a.ring_off = idx->ring_off;
    a.xy = idx->xy;
    a.accept_mask = accept_mask;
    a.pairs = dsink.buf;
    a.capacity = dsink.capacity;
    a.count = dsink.counter;
    a.sink = PairSink{d_left, d_right, (unsigned long long)(capacity > 0 ? capacity : 0), &ctx->d_counters[0]};
    a.counters = ctx->d_counters;
    a.rings = idx->ring_index();
    a.row_base = row_base;
    resolve_deferred_kernel<<<resident_grid(resolve_deferred_kernel, (int64_t)1 << 30, kJoinThreads), kJoinThreads, 0,
                              ctx->stream>>>(a);
    VS_LAUNCHED("resolve_deferred", ctx->stream);
    return VS_OK;
}

int launch_locate_aligned(vs_context* ctx, const vs_points* pts, const vs_polygons* polys, uint8_t* d_out) {
    if (pts->n == 0) return VS_OK;
    locate_aligned_kernel<<<resident_grid(locate_aligned_kernel, pts->n, 256), 256, 0, ctx->stream>>>(*pts, *polys, d_out, ctx->d_counters);
    VS_LAUNCHED("locate_aligned", ctx->stream);
    return VS_OK;
}

int sort_pairs(vs_context* ctx, int32_t* d_left, int32_t* d_right, int64_t n, uint64_t max_left,
               uint64_t max_right) {
    if (n <= 1) return VS_OK;
    const int rbits = bits_for(max_right);
    const int lbits = bits_for(max_left);
    if (rbits + lbits > 64) {
        set_error("pair key does not fit 64 bits");
        return VS_E_ARG;
    }
    cudaStream_t s = ctx->stream;
    Scratch<uint64_t> keys;
    Scratch<uint32_t> vals;
    VS_TRY(keys.alloc((size_t)n, s));
    VS_TRY(vals.alloc((size_t)n, s));
    pack_pairs_kernel<<<grid_for(n, 256), 256, 0, s>>>(d_left, d_right, n, rbits, keys.p, vals.p);
    VS_LAUNCHED("pack_pairs", s);
    VS_TRY(radix_sort_u64_u32(keys.p, vals.p, n, rbits + lbits, s));
    unpack_pairs_kernel<<<grid_for(n, 256), 256, 0, s>>>(keys.p, n, rbits, d_left, d_right);
    VS_LAUNCHED("unpack_pairs", s);
    return VS_OK;
}

}  // namespace vs
