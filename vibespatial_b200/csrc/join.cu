// Point x polygon join on the packed Hilbert R-tree (the plain method),
// element-wise location, and pair sorting.
//
// Reference behaviour replaced (src/vibespatial/...):
//   spatial/spatial_index_device.py:228-1035   candidates: Morton range +
//       serial per-query scan, count pass -> exclusive_sum -> host fence on
//       the total -> scatter pass
//   spatial/query_utils.py:578-868             refine: one thread per
//       candidate pair, then boolean-mask compaction d_left[keep]
// Here one kernel does both: each thread descends the R-tree for one point
// (upper levels staged in shared memory), refines every leaf hit immediately
// with the exact location, and appends accepted pairs to a shared-memory
// buffer that is flushed to HBM with one global atomic per block iteration.
// There is no candidate array, no count pass and no host fence inside the
// join; the only read-back is the final pair count.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "exact.cuh"
#include "index.cuh"
#include "join.cuh"
#include "primitives.cuh"

namespace vs {
namespace {

constexpr int kJoinThreads = 256;
constexpr int kOutBuf = 1024;     // pairs buffered per block iteration
constexpr int kStack = 112;       // (fanout-1) * (max levels-2) + 1 < 112
constexpr int kMaxStagedBoxes = 1365;  // 1 + 16 + 256 + 1092: ~43 KB of FP64 boxes

struct RtreeArgs {
    const double* px;
    const double* py;
    const uint8_t* pvalid;
    int64_t n;
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
    int32_t* out_left;
    int32_t* out_right;
    unsigned long long capacity;
    unsigned long long* counters;
};

__device__ __forceinline__ bool box_has(const vs_box& b, double x, double y) {
    return x >= b.minx && x <= b.maxx && y >= b.miny && y <= b.maxy;
}

struct BlockOut {
    int2* buf;
    unsigned* cnt;
};

__device__ __forceinline__ void emit(const BlockOut& o, int32_t l, int32_t r, unsigned long long capacity,
                                     int32_t* out_left, int32_t* out_right, unsigned long long* counters) {
    const unsigned pos = atomicAdd(o.cnt, 1u);
    if (pos < (unsigned)kOutBuf) {
        o.buf[pos] = make_int2(l, r);
    } else {
        const unsigned long long gp = atomicAdd(&counters[0], 1ull);
        if (gp < capacity) {
            out_left[gp] = l;
            out_right[gp] = r;
        }
    }
}

// Flush the block buffer; every thread of the block must call it.
__device__ __forceinline__ void flush(const BlockOut& o, unsigned long long* s_base, unsigned* s_n,
                                      unsigned long long capacity, int32_t* out_left, int32_t* out_right,
                                      unsigned long long* counters) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned c = *o.cnt < (unsigned)kOutBuf ? *o.cnt : (unsigned)kOutBuf;
        *s_n = c;
        *s_base = c ? atomicAdd(&counters[0], (unsigned long long)c) : 0ull;
        *o.cnt = 0;
    }
    __syncthreads();
    const unsigned c = *s_n;
    const unsigned long long b = *s_base;
    for (unsigned k = threadIdx.x; k < c; k += blockDim.x) {
        const unsigned long long gp = b + k;
        if (gp < capacity) {
            const int2 v = o.buf[k];
            out_left[gp] = v.x;
            out_right[gp] = v.y;
        }
    }
    __syncthreads();
}

__device__ __forceinline__ void add_stats(unsigned long long* counters, unsigned long long cand, unsigned nexact) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cand += __shfl_xor_sync(0xffffffffu, cand, o);
        nexact += __shfl_xor_sync(0xffffffffu, nexact, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (cand) atomicAdd(&counters[5], cand);
        if (nexact) atomicAdd(&counters[1], (unsigned long long)nexact);
    }
}

__global__ void __launch_bounds__(kJoinThreads) join_rtree_kernel(const RtreeArgs a) {
    extern __shared__ vs_box s_nodes[];
    __shared__ int2 s_buf[kOutBuf];
    __shared__ unsigned s_cnt, s_n;
    __shared__ unsigned long long s_base;
    const int64_t stage_base = a.level_off[a.stage_level];
    for (int k = threadIdx.x; k < a.staged; k += blockDim.x) s_nodes[k] = a.nodes[stage_base + k];
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    const BlockOut out{s_buf, &s_cnt};
    const int top = a.levels - 1;
    unsigned long long n_cand = 0;
    unsigned n_exact = 0;
    int stack[kStack];

    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < a.n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        if (i < a.n && (a.pvalid == nullptr || a.pvalid[i])) {
            const double x = a.px[i], y = a.py[i];
            int sp = 0;
            const vs_box root = s_nodes[a.level_off[top] - stage_base];
            if (box_has(root, x, y)) {
                if (top == 0) {
                    // single polygon: the root is the item
                    ++n_cand;
                    const int loc = a.accept_mask ? geometry_location(x, y, a.xy, a.ring_off, a.part_off,
                                                                      a.geom_off, 0, n_exact)
                                                  : 0;
                    if (!a.accept_mask || ((a.accept_mask >> loc) & 1))
                        emit(out, (int32_t)i, a.item_geom[0], a.capacity, a.out_left, a.out_right, a.counters);
                } else {
                    stack[sp++] = top;  // node 0 of the top level
                }
            }
            while (sp > 0) {
                const int e = stack[--sp];
                const int lvl = e & 15;
                const int64_t node = (int64_t)(e >> 4);
                const int cl = lvl - 1;
                const int64_t c0 = node * kFanout;
                const int64_t cend = c0 + kFanout < a.level_size[cl] ? c0 + kFanout : a.level_size[cl];
                const vs_box* cb = cl >= a.stage_level ? s_nodes + (a.level_off[cl] - stage_base)
                                                       : a.nodes + a.level_off[cl];
                for (int64_t c = c0; c < cend; ++c) {
                    const vs_box b = cb[c];
                    if (!box_has(b, x, y)) continue;
                    if (cl == 0) {
                        ++n_cand;
                        const int slot = (int)c;
                        int loc = 0;
                        if (a.accept_mask)
                            loc = geometry_location(x, y, a.xy, a.ring_off, a.part_off, a.geom_off, slot, n_exact);
                        if (!a.accept_mask || ((a.accept_mask >> loc) & 1))
                            emit(out, (int32_t)i, a.item_geom[slot], a.capacity, a.out_left, a.out_right,
                                 a.counters);
                    } else if (sp < kStack) {
                        stack[sp++] = (int)(c << 4) | cl;
                    } else {
                        atomicOr(&a.counters[4], 1ull);  // stack overflow: result incomplete
                    }
                }
            }
        }
        flush(out, &s_base, &s_n, a.capacity, a.out_left, a.out_right, a.counters);
    }
    add_stats(a.counters, n_cand, n_exact);
}

// Every point against every polygon box (small joins and cross-checks).
__global__ void __launch_bounds__(kJoinThreads) join_brute_kernel(const RtreeArgs a) {
    __shared__ int2 s_buf[kOutBuf];
    __shared__ unsigned s_cnt, s_n;
    __shared__ unsigned long long s_base;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    const BlockOut out{s_buf, &s_cnt};
    const int64_t M = a.level_size[0];
    unsigned long long n_cand = 0;
    unsigned n_exact = 0;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < a.n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        if (i < a.n && (a.pvalid == nullptr || a.pvalid[i])) {
            const double x = a.px[i], y = a.py[i];
            for (int64_t c = 0; c < M; ++c) {
                if (!box_has(a.nodes[c], x, y)) continue;
                ++n_cand;
                int loc = 0;
                if (a.accept_mask)
                    loc = geometry_location(x, y, a.xy, a.ring_off, a.part_off, a.geom_off, (int)c, n_exact);
                if (!a.accept_mask || ((a.accept_mask >> loc) & 1))
                    emit(out, (int32_t)i, a.item_geom[c], a.capacity, a.out_left, a.out_right, a.counters);
            }
        }
        flush(out, &s_base, &s_n, a.capacity, a.out_left, a.out_right, a.counters);
    }
    add_stats(a.counters, n_cand, n_exact);
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

int launch_rtree_join(vs_context* ctx, const vs_index* idx, const vs_points* pts, int accept_mask, bool brute,
                      int32_t* d_left, int32_t* d_right, int64_t capacity) {
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
    a.out_left = d_left;
    a.out_right = d_right;
    a.capacity = (unsigned long long)(capacity > 0 ? capacity : 0);
    a.counters = ctx->d_counters;
    const int grid = grid_for(pts->n, kJoinThreads, 8);
    if (brute) {
        join_brute_kernel<<<grid, kJoinThreads, 0, ctx->stream>>>(a);
    } else {
        const size_t smem = (size_t)a.staged * sizeof(vs_box);
        join_rtree_kernel<<<grid, kJoinThreads, smem, ctx->stream>>>(a);
    }
    VS_CUDA_TRY(cudaGetLastError());
    return VS_OK;
}

int launch_locate_aligned(vs_context* ctx, const vs_points* pts, const vs_polygons* polys, uint8_t* d_out) {
    if (pts->n == 0) return VS_OK;
    locate_aligned_kernel<<<grid_for(pts->n, 256, 16), 256, 0, ctx->stream>>>(*pts, *polys, d_out, ctx->d_counters);
    VS_CUDA_TRY(cudaGetLastError());
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
    VS_CUDA_TRY(cudaGetLastError());
    VS_TRY(radix_sort_u64_u32(keys.p, vals.p, n, rbits + lbits, s));
    unpack_pairs_kernel<<<grid_for(n, 256), 256, 0, s>>>(keys.p, n, rbits, d_left, d_right);
    VS_CUDA_TRY(cudaGetLastError());
    return VS_OK;
}

}  // namespace vs
