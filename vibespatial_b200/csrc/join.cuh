// Host-side launchers shared by the C-ABI translation unit.
#pragma once
#include <stdint.h>

#include "emit.cuh"
#include "index.cuh"
#include "primitives.cuh"
#include "vs_common.cuh"

namespace vs {
// Query points keyed by their level-16 Hilbert key in the polygon frame and
// radix-sorted; order[0, *n_valid) are the points that can match.
struct QueryOrder {
    Scratch<uint32_t> keys, order, n_valid;
};
// clamp: keep points outside the polygon frame (keyed at the frame's edge),
// as distance joins need them; otherwise they are left out.
int prepare_queries(vs_context* ctx, const vs_index* idx, const vs_points* pts, QueryOrder& q, bool clamp = false);
int accept_mask_for(int predicate, int* mask);
// row_base is added to every emitted or deferred point row (a chunk of a
// larger point array); the exact pass subtracts it to read the chunk's points.
int launch_rtree_join(vs_context* ctx, const vs_index* idx, const vs_points* pts, int accept_mask, bool brute,
                      bool bulk_leaves, int32_t* d_left, int32_t* d_right, int64_t capacity, const DeferSink& dsink,
                      int64_t row_base = 0);
int launch_learned_join(vs_context* ctx, const vs_index* idx, const vs_points* pts, int accept_mask,
                        int32_t* d_left, int32_t* d_right, int64_t capacity, const DeferSink& dsink,
                        int64_t row_base = 0, const LearnedShape& shape = LearnedShape{});
// Exact pass over the pairs the filtered kernels deferred (count read on device).
int launch_resolve_deferred(vs_context* ctx, const vs_index* idx, const vs_points* pts, int accept_mask,
                            int32_t* d_left, int32_t* d_right, int64_t capacity, const DeferSink& dsink,
                            int64_t row_base = 0);
// Grow the context's deferred-pair buffer to at least `want` pairs.
int ensure_defer_capacity(vs_context* ctx, unsigned long long want);
// Release the context's vs_join_host pipeline (streams, events, buffers).
void free_host_pipe(vs_context* ctx);
int launch_locate_aligned(vs_context* ctx, const vs_points* pts, const vs_polygons* polys, uint8_t* d_out);
int sort_pairs(vs_context* ctx, int32_t* d_left, int32_t* d_right, int64_t n, uint64_t max_left,
               uint64_t max_right);
int build_rtree(vs_context* ctx, const vs_polygons* P, vs_index* idx);
// y-bins for rings of at least min_vertices vertices (0: the default, < 0: none).
int build_ring_bins(vs_context* ctx, vs_index* idx, int min_vertices);
void free_index_memory(vs_index* idx);
int hilbert_point_keys(const double* x, const double* y, int64_t n, double minx, double miny, double maxx,
                       double maxy, uint64_t* keys, cudaStream_t s);
}  // namespace vs
