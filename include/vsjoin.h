/*
 * vsjoin: B200-native point-by-polygon spatial join, C-ABI.
 *
 * Every pointer argument named d_* is a DEVICE pointer on the context's
 * device; h_* are host pointers.  Polygonal inputs use the GeoArrow-style
 * MultiPolygon SoA that the reference's OwnedGeometryArray uses for its
 * polygon/multipolygon families (src/vibespatial/geometry/buffers.py:140-249):
 * geom_off (row -> part), part_off (part -> ring), ring_off (ring -> coord),
 * x[] and y[] coordinates.  A Polygon row is a MultiPolygon row with one part.
 *
 * Status codes: every entry point returns VS_OK or one of the VS_E_* codes
 * and leaves a message in vs_last_error() (thread-local).  This mirrors the
 * reference's error classes: ValueError for bad arguments (VS_E_ARG),
 * CandidateRelationCapacityError for an undersized pair buffer
 * (VS_E_CAPACITY, src/vibespatial/spatial/query_types.py:41-93) and
 * RuntimeError for driver failures (VS_E_CUDA,
 * src/vibespatial/cuda/_runtime.py:95-108).
 */
#ifndef VSJOIN_H
#define VSJOIN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VSJOIN_ABI_VERSION 2

enum vs_status {
    VS_OK = 0,
    VS_E_ARG = 1,      /* invalid argument */
    VS_E_OOM = 2,      /* device allocation failed */
    VS_E_CAPACITY = 3, /* pair buffer too small; *n_pairs holds the required size */
    VS_E_CUDA = 4,     /* CUDA runtime error */
    VS_E_TIMEOUT = 5,  /* a bounded device wait gave up */
    VS_E_STATE = 6     /* inconsistent handle / device-side consistency check failed */
};

/* Predicates, stated with the POINT as the query (left) side and the polygon
 * as the tree (right) side.  Location -> predicate mapping follows
 * src/vibespatial/predicates/point_relations.py:100-130 (point_on_left):
 *   WITHIN      interior                 (sjoin predicate='within')
 *   INTERSECTS  interior or boundary     (predicate='intersects')
 *   COVERED_BY  interior or boundary
 *   TOUCHES     boundary
 *   BBOX        bounding-box candidates only (predicate=None)
 * Polygon-on-the-left predicates (contains, covers, contains_properly) are the
 * mirror images: the host swaps sides (src/vibespatial/api/tools/sjoin.py:1049-1082). */
enum vs_predicate {
    VS_PRED_BBOX = 0,
    VS_PRED_INTERSECTS = 1,
    VS_PRED_WITHIN = 2,
    VS_PRED_COVERED_BY = 3,
    VS_PRED_TOUCHES = 4
};

/* Query methods. */
enum vs_method {
    VS_METHOD_RTREE = 0,   /* plain: packed Hilbert R-tree traversal, FP64 filter, exact refine */
    VS_METHOD_LEARNED = 1, /* learned cell index + FP32 tile-relative filter, exact fallback;
                              an index built without it answers with the R-tree */
    VS_METHOD_BRUTE = 2    /* every point against every polygon box (small joins, testing) */
};

/* Join flags. */
#define VS_JOIN_SORT 1u        /* return pairs sorted by (left, right) */
#define VS_JOIN_BULK_LEAVES 2u /* R-tree method: load leaf blocks with bulk copies (TMA, cp.async.bulk) into
                                  shared memory instead of lane loads (same pairs; measured ~2% slower) */
/* Ablations of the learned method (same pairs; for measuring what each choice buys): */
#define VS_JOIN_LEARNED_BSEARCH 4u   /* cell lookup by binary search over every cell key instead of the RMI */
#define VS_JOIN_LEARNED_FP64_WALK 8u /* ring walks in FP64 (the plain method's filter) instead of FP32 first */
#define VS_JOIN_LEARNED_NO_STAGE 16u /* candidate records read by the lanes from global memory instead of one
                                        bulk copy (TMA) per 32-point packet into shared memory */
#define VS_JOIN_LEARNED_NO_INTERIOR 32u /* every box candidate ring-walked: no interior-box shortcut */

typedef struct vs_context vs_context;
typedef struct vs_index vs_index;

typedef struct vs_polygons {
    const double* d_x;
    const double* d_y;
    const int32_t* d_ring_off; /* n_rings + 1 */
    const int32_t* d_part_off; /* n_parts + 1 */
    const int32_t* d_geom_off; /* n_geoms + 1 */
    const uint8_t* d_valid;    /* n_geoms, nullable: 0 = null row (never matches) */
    int64_t n_coords;
    int32_t n_rings;
    int32_t n_parts;
    int32_t n_geoms;
} vs_polygons;

typedef struct vs_points {
    const double* d_x;
    const double* d_y;
    const uint8_t* d_valid; /* nullable: 0 = null row; NaN coordinates = empty point */
    int64_t n;
} vs_points;

typedef struct vs_index_options {
    int32_t method_mask; /* bit 0: R-tree (always built), bit 1: learned cell index */
    int32_t cell_level;  /* learned index grid level (0 = choose automatically) */
    int32_t rmi_leaves;  /* learned index leaf models (0 = 4096, or one per 64 cell keys above 256k keys;
                            at most 65535) */
    int32_t rmi_train_steps; /* 0 = default */
    int32_t ring_bin_min_vertices; /* rings with at least this many vertices get 8 y-bins of edges, so a
                                      point's ring walk visits only the edges of its bin (0 = 16, < 0 = none) */
} vs_index_options;

typedef struct vs_join_stats {
    int64_t candidates;       /* point/polygon pairs that passed the box filter */
    int64_t exact_fallbacks;  /* orientation signs that needed the exact expansion stage */
    int64_t fp32_edges;       /* edges decided by the FP32 tile-relative filter */
    int64_t fp64_edges;       /* edges the FP32 bound left inconclusive: their pairs go to the FP64 / exact
                                 pass (the R-tree method: 0) */
    int64_t rmi_fallbacks;    /* learned-index lookups whose error window exceeded 256 cells (binary search) */
    float kernel_ms;          /* device time of the join kernels */
    float sort_ms;            /* device time of the optional pair sort */
    int64_t kernel_launches;  /* kernels the call enqueued (a graph replay: the kernels in the graph) */
    float phase_ms[4];        /* device time per phase: [0] locate (learned: cell lookup; R-tree: point
                                 keys + sort), [1] group (learned: points scattered by cell), [2] refine
                                 (traversal / candidate loop with the filtered tests), [3] exact pass */
} vs_join_stats;

typedef struct vs_index_info {
    int32_t n_geoms;
    int32_t fanout;
    int32_t levels;
    int32_t cell_level;
    int64_t n_cells;          /* non-empty learned-index cells */
    int64_t n_cell_entries;   /* (cell, polygon) entries */
    int64_t device_bytes;     /* bytes owned by the index */
    float build_ms;
    float rmi_train_ms;
    float rmi_mean_window;    /* mean learned-index search window (entries) */
    int32_t rmi_max_window;
    int64_t n_binned_rings;   /* rings with y-bins */
    int64_t n_bin_edges;      /* (bin, edge) entries */
    int32_t rmi_leaves;       /* learned-index leaf models (0 without the learned part) */
} vs_index_info;

/* ---------------------------------------------------------------------- */

/* ABI version (VSJOIN_ABI_VERSION). */
int vs_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char* vs_last_error(void);

/* Kernels the library has launched from the calling thread so far; the
 * difference across calls counts their launches (benchmark diagnostics; no
 * counterpart in the reference). */
long long vs_thread_kernel_launches(void);

/* A context = one device + one stream + a scratch arena.  `stream` is a
 * cudaStream_t (NULL: the context creates its own non-blocking stream; pass
 * cudaStreamLegacy to run on the legacy default stream).  Not thread-safe: callers
 * serialise use of one context.  Replaces the reference's per-process runtime
 * (src/vibespatial/cuda/_runtime.py:1821-1852, launches on CuPy's stream). */
int vs_context_create(int device, void* stream, vs_context** out);
int vs_context_destroy(vs_context* ctx);
int vs_context_synchronize(vs_context* ctx);

/* Build the spatial index of a polygon/multipolygon array (the tree side).
 * Replaces build_flat_spatial_index (src/vibespatial/spatial/indexing.py:1357)
 * and its Morton-key + CCCL sort_pairs steps (:1265-1322).  The index copies
 * what it needs; the input buffers may be freed after the call returns. */
int vs_index_build(vs_context* ctx, const vs_polygons* polys, const vs_index_options* opts,
                   vs_index** out);
int vs_index_info_get(const vs_index* index, vs_index_info* info);
int vs_index_free(vs_index* index);

/* Join points (query side) against the index (tree side).  Replaces
 * query_spatial_index (src/vibespatial/spatial/query.py:247) for point
 * queries: candidate generation (spatial_index_device_query,
 * src/vibespatial/spatial/spatial_index_device.py:228) + exact refine
 * (_filter_predicate_pairs_owned, src/vibespatial/spatial/query_utils.py:578).
 * Writes (left = point row, right = polygon row) int32 pairs to d_left /
 * d_right (capacity entries each).  If more pairs exist than `capacity`,
 * returns VS_E_CAPACITY with *n_pairs = the required size and the buffers
 * partially written.  Blocks until the pairs are resident. */
int vs_join(vs_context* ctx, const vs_index* index, const vs_points* pts, int32_t predicate,
            int32_t method, uint32_t flags, int32_t* d_left, int32_t* d_right, int64_t capacity,
            int64_t* n_pairs, vs_join_stats* stats);

/* Pairs within a distance: (point row, polygon row) with
 * distance(point, polygon) <= d.  Replaces the reference's dwithin query
 * (query_spatial_index with predicate 'dwithin', src/vibespatial/spatial/query.py:663-810:
 * expanded-bounds candidates + _dwithin_refine_gpu, spatial/nearest.py:2855).
 * distance(point, polygon) is 0 when the point is inside or on the polygon
 * (exact location) and otherwise the smallest point-segment distance over all
 * rings (comp.graphics.algorithms FAQ method, each operation rounded
 * separately); a pair whose envelope distance exceeds d is rejected first.
 * d is d_point_distance[point row] (device, n points), or
 * d_geom_distance[polygon row] (device, polygon rows), or `distance` when
 * both are NULL; negative or NaN distances match nothing.  Pairs, capacity,
 * VS_JOIN_SORT and the VS_E_CAPACITY contract as for vs_join. */
int vs_join_dwithin(vs_context* ctx, const vs_index* index, const vs_points* pts,
                    const double* d_point_distance, const double* d_geom_distance, double distance,
                    uint32_t flags, int32_t* d_left, int32_t* d_right, int64_t capacity,
                    int64_t* n_pairs, vs_join_stats* stats);

/* Nearest polygons of every point, all ties: for each valid point, every
 * polygon at its minimum distance (same distance as vs_join_dwithin), if that
 * minimum is <= max_distance (INFINITY: unbounded; negative: no pairs).
 * Replaces sjoin_nearest's query (src/vibespatial/api/tools/sjoin.py
 * sjoin_nearest -> query_nearest, src/vibespatial/spatial/nearest.py).
 * d_distance (device, capacity entries, nullable) receives each pair's
 * distance.  Pairs, capacity, VS_JOIN_SORT and VS_E_CAPACITY as for vs_join. */
int vs_join_nearest(vs_context* ctx, const vs_index* index, const vs_points* pts, double max_distance,
                    uint32_t flags, int32_t* d_left, int32_t* d_right, double* d_distance,
                    int64_t capacity, int64_t* n_pairs, vs_join_stats* stats);

/* Nearest points of every polygon, all ties (sjoin_nearest with the polygons
 * as the matched side): for each valid query polygon, every point at its
 * minimum distance (the same point-polygon distance as vs_join_nearest), if
 * that minimum is <= max_distance.  point_index is an index over the points
 * built by vs_index_build with each point as a polygon of one ring of one
 * vertex (geom_off = part_off = ring_off = 0, 1, ..., n; null or NaN points
 * get no box).  Pairs: d_left = query polygon row, d_right = point row;
 * d_distance (nullable) the pair distances.  Capacity, VS_JOIN_SORT and
 * VS_E_CAPACITY as for vs_join.  Replaces the reference's sjoin_nearest query
 * with the polygon frame as the query side (src/vibespatial/api/tools/sjoin.py:1398,
 * src/vibespatial/spatial/nearest.py). */
int vs_join_nearest_polygons(vs_context* ctx, const vs_index* point_index, const vs_polygons* queries,
                             double max_distance, uint32_t flags, int32_t* d_left, int32_t* d_right,
                             double* d_distance, int64_t capacity, int64_t* n_pairs, vs_join_stats* stats);

/* Element-wise distance of aligned rows: row i of the points against row i
 * of the polygons (polys->n_geoms == pts->n).  d_distance[i] = the same
 * point-polygon distance as vs_join_dwithin, d_envelope_distance[i]
 * (nullable) = the distance to the polygon's envelope; both NaN for null or
 * NaN points, null polygons and polygons without vertices.  Replaces the
 * element-wise distance / dwithin of point x polygon rows
 * (src/vibespatial/spatial/point_distance_kernels.py:238-310 via
 * GeometryArray.distance / dwithin); dwithin(i) = !(envelope > d) && distance <= d. */
int vs_distance_aligned(vs_context* ctx, const vs_points* pts, const vs_polygons* polys, double* d_distance,
                        double* d_envelope_distance);

/* Join export: the row indexers of a relation join.  Replaces the
 * reference's export (_adjust_join_indexers, src/vibespatial/api/_native_results.py:395-470)
 * and its shared-attribute filter (src/vibespatial/api/tools/sjoin.py:826-888).
 * Pairs (n_pairs, sorted by (left, right), as the joins return them) are
 * first filtered by d_left_code[left] == d_right_code[right] when codes are
 * given (int64 per row, equal values equal codes, < 0 = missing, never
 * equal).  Output rows (int64, -1 = no row on that side):
 *   VS_HOW_INNER  the kept pairs
 *   VS_HOW_LEFT   every left row in order: its pairs, or (row, -1)
 *   VS_HOW_RIGHT  every right row in order: its pairs (by left row), or (-1, row)
 *   VS_HOW_OUTER  as LEFT, then (-1, row) for every right row without a pair
 * d_out_src (nullable) receives each output row's input pair position (-1
 * for an added row).  *n_out = the number of rows; VS_E_CAPACITY (buffers
 * untouched) when it exceeds capacity.  Pairs naming rows outside
 * [0, n_left) x [0, n_right) give VS_E_ARG before anything is written.
 * Up to 2^31 - 1 pairs and rows a side. */
enum { VS_HOW_INNER = 0, VS_HOW_LEFT = 1, VS_HOW_RIGHT = 2, VS_HOW_OUTER = 3 };
int vs_join_export(vs_context* ctx, const int32_t* d_left, const int32_t* d_right, int64_t n_pairs,
                   int64_t n_left, int64_t n_right, int32_t how, const int64_t* d_left_code,
                   const int64_t* d_right_code, int64_t* d_out_left, int64_t* d_out_right,
                   int64_t* d_out_src, int64_t capacity, int64_t* n_out);

/* vs_join on HOST buffers: h_x / h_y / h_valid (n points; pinned memory lets
 * the copies run asynchronously) in, (left, right) pairs into h_left /
 * h_right (capacity entries each) out.  The points are streamed in chunks
 * so host-to-device copies, the join and device-to-host copies of the pairs
 * overlap.  Same predicates, methods, VS_JOIN_SORT, VS_E_CAPACITY contract
 * and stats as vs_join (stats->kernel_ms: the whole pipeline).  Replaces the
 * reference's move_to H2D + device join + pair D2H round trip
 * (src/vibespatial/spatial/query.py:124, query_spatial_index :247). */
int vs_join_host(vs_context* ctx, const vs_index* index, const double* h_x, const double* h_y,
                 const uint8_t* h_valid, int64_t n, int32_t predicate, int32_t method, uint32_t flags,
                 int32_t* h_left, int32_t* h_right, int64_t capacity, int64_t* n_pairs,
                 vs_join_stats* stats);

/* Element-wise location of point row i in polygon row i (aligned arrays):
 * d_out[i] = 0 outside / 1 boundary / 2 interior / 255 null-or-empty.
 * Replaces the point-region fast path of GeometryArray.within/contains
 * (src/vibespatial/predicates/binary.py:1469-1692). */
int vs_locate_aligned(vs_context* ctx, const vs_points* pts, const vs_polygons* polys,
                      uint8_t* d_out);

/* Sort int32 pairs in place by (left, right) with the in-house radix sort.
 * Mirrors the lexsort the reference applies to host-path pairs
 * (src/vibespatial/api/tools/sjoin.py:1079-1082). */
int vs_sort_pairs(vs_context* ctx, int32_t* d_left, int32_t* d_right, int64_t n);

/* Sort (u64 key, u32 value) pairs in place by key (in-house LSD radix sort;
 * replaces CCCL sort_pairs, src/vibespatial/cuda/cccl_primitives.py:1054). */
int vs_radix_sort_pairs(vs_context* ctx, uint64_t* d_keys, uint32_t* d_vals, int64_t n,
                        int32_t key_bits);

/* 64-bit Hilbert keys of (x, y) on the 2^32 grid spanning the given frame
 * (replaces morton_keys_from_bounds, src/vibespatial/spatial/indexing_kernels.py:20-49). */
int vs_hilbert_keys(vs_context* ctx, const double* d_x, const double* d_y, int64_t n,
                    double minx, double miny, double maxx, double maxy, uint64_t* d_keys);

/* ---------------------------------------------------------------------- */
/* Batched joins: many independent point x polygon joins of uneven sizes run
 * as one persistent launch, replayed from a CUDA graph.  The reference runs
 * such work as one query_spatial_index call per job
 * (src/vibespatial/spatial/query.py:247), each with its own launches and host
 * fences (count_scatter_total, src/vibespatial/cuda/_runtime.py:2015-2038);
 * here the whole batch is key -> sort -> traversal -> exact pass on the
 * device with no host round trip, and the pair sizes are checked after the
 * graph.  Job j joins points [h_job_start[j], h_job_start[j+1]) of `pts`
 * against indexes[j]; a pair is (left = row in `pts`, right = polygon row of
 * job j's index).  Pairs come back unordered.  The plan borrows `pts` and
 * the indexes for its lifetime. */
typedef struct vs_batch_plan vs_batch_plan;

typedef struct vs_batch_options {
    int32_t blocks_per_sm;    /* R-tree: join kernel blocks per SM, 1..8 (0 = 4) */
    int32_t packets_per_grab; /* R-tree: 32-point packets a warp takes per work-counter grab (0 = 4) */
    int32_t sort_levels;      /* R-tree: Hilbert levels the points of a job are sorted by (0 = 8) */
    int32_t method;           /* VS_METHOD_RTREE (0) or VS_METHOD_LEARNED: every index with polygons
                                 must then have its learned part (VS_E_ARG otherwise) */
    int32_t learned_map_blocks_per_sm;    /* learned: map pass blocks per SM (0 = 8) */
    int32_t learned_refine_blocks_per_sm; /* learned: refine pass blocks per SM: 1-3 run the 80-register build,
                                             4 (and 0, the default: as many as fit) the 64-register one, 5-8 the
                                             48-register one */
    int32_t learned_grab;     /* learned: grouped points a refine warp takes per grab (0 = 32; rounded up to 32s) */
    uint32_t learned_flags;   /* learned: VS_JOIN_LEARNED_BSEARCH | _FP64_WALK | _NO_STAGE | _NO_INTERIOR (ablations) */
    int32_t learned_map_packets; /* learned: 32-point packets a map warp looks up together, 1 or 2 (0 = 1) */
} vs_batch_options;

/* At most 4096 jobs and 2^31-1 points in total. */
int vs_batch_plan_create(vs_context* ctx, const vs_index* const* indexes, int32_t n_jobs,
                         const vs_points* pts, const int64_t* h_job_start,
                         const vs_batch_options* opts, vs_batch_plan** out);

/* One batched join.  use_graph != 0 replays a CUDA graph captured on the
 * first call (and again whenever predicate or the pair buffers change);
 * 0 launches the same kernels directly.  VS_E_CAPACITY: *n_pairs holds the
 * required size.  stats->kernel_ms is the device time of the batch. */
int vs_batch_run(vs_batch_plan* plan, int32_t predicate, int32_t* d_left, int32_t* d_right,
                 int64_t capacity, int32_t use_graph, int64_t* n_pairs, vs_join_stats* stats);

int vs_batch_plan_free(vs_batch_plan* plan);

/* ---------------------------------------------------------------------- */
/* WKB decode on the device (GeoParquet / GeoArrow WKB columns -> the
 * columnar layout of the join's inputs).  Replaces the reference's Arrow WKB
 * decode (decode_wkb_arrow_array_owned, src/vibespatial/io/wkb.py:5224) for
 * Point, Polygon and MultiPolygon rows, either byte order, ISO or EWKB (Z, M
 * and SRID are accepted; Z and M are dropped).  Two calls: the plan writes
 * the per-row outputs and sizes the rest (rows of other types count as
 * unsupported, truncated or invalid bytes as malformed, and decode to null
 * rows), the caller allocates the part / ring / coordinate buffers, and the
 * decode fills them. */
typedef struct vs_wkb_plan vs_wkb_plan;

typedef struct vs_wkb_sizes {
    int64_t n_rows;
    int64_t n_points, n_polygons, n_multipolygons, n_null;
    int64_t n_unsupported, n_malformed;
    int64_t n_parts, n_rings, n_coords;
} vs_wkb_sizes;

/* Output buffers (device).  Per row, written by vs_wkb_plan_create: tags
 * (int8: -1 null, 0 Point, 2 Polygon, 5 MultiPolygon), px/py (the Point
 * coordinates, NaN otherwise) and geom_off (n_rows + 1).  Written by
 * vs_wkb_plan_decode: part_off (n_parts + 1), ring_off (n_rings + 1), x/y
 * (n_coords). */
typedef struct vs_wkb_out {
    int8_t* d_tags;
    double* d_px;
    double* d_py;
    int32_t* d_geom_off;
    int32_t* d_part_off;
    int32_t* d_ring_off;
    double* d_x;
    double* d_y;
} vs_wkb_out;

/* d_offsets: n + 1 int64 byte offsets into d_wkb (Arrow binary layout);
 * d_valid nullable.  `rows` gives the per-row outputs (its other fields are
 * ignored); the plan borrows the inputs and the row outputs until it is
 * freed.  Returns after one host synchronisation (the sizes). */
int vs_wkb_plan_create(vs_context* ctx, const uint8_t* d_wkb, const int64_t* d_offsets,
                       const uint8_t* d_valid, int64_t n, const vs_wkb_out* rows,
                       vs_wkb_plan** plan, vs_wkb_sizes* sizes);
/* Fills out->d_part_off, d_ring_off, d_x, d_y (the row fields are ignored);
 * returns when the outputs are complete. */
int vs_wkb_plan_decode(vs_wkb_plan* plan, const vs_wkb_out* out);
int vs_wkb_plan_free(vs_wkb_plan* plan);

/* ---------------------------------------------------------------------- */
/* Row reductions of a join's pairs on the device (the relation flow of the
 * index without exported pairs).  Replace the reference's native relation
 * reductions: sindex.query_left_match_count_expression,
 * query_left_semijoin / query_left_antijoin / query_right_semijoin
 * (src/vibespatial/api/sindex.py:1592-1760), query_aggregate's size and sum
 * (:505) and query_pair_aggregate's shared counts (:973, host path
 * :1257-1270).  Rows outside their range: VS_E_ARG.  Each call returns when
 * its outputs are complete. */

/* d_counts[r] (int64, n_rows of them) = pairs whose row is r, counting only
 * the pairs whose d_mask byte is non-zero when d_mask is given. */
int vs_row_counts(vs_context* ctx, const int32_t* d_rows, const uint8_t* d_mask, int64_t n_pairs, int64_t n_rows,
                  int64_t* d_counts);

/* d_sums[r] = sum of d_values[d_cols[k]] over the pairs k with d_rows[k] == r,
 * added in pair order (so equal to numpy's bincount(rows, weights=...)); the
 * rows must ascend (VS_E_ARG otherwise), as a join's sorted pairs do. */
int vs_row_sums(vs_context* ctx, const int32_t* d_rows, const int32_t* d_cols, int64_t n_pairs, int64_t n_rows,
                const double* d_values, int64_t n_values, double* d_sums);

/* The rows r in ascending order whose d_counts[r] > 0 (matched != 0: a
 * semijoin) or == 0 (matched == 0: an antijoin), into d_out (n_rows
 * capacity); their number in *n_out. */
int vs_select_rows(vs_context* ctx, const int64_t* d_counts, int64_t n_rows, int32_t matched, int32_t* d_out,
                   int64_t* n_out);

/* d_flags[k] = 1 when pair k of relation a is also a pair of relation b, else
 * 0.  b's pairs must be sorted by (left, right) (VS_E_ARG otherwise), as a
 * join's sorted output is; left rows lie in [0, n_left_rows). */
int vs_pairs_member(vs_context* ctx, const int32_t* d_a_left, const int32_t* d_a_right, int64_t n_a,
                    const int32_t* d_b_left, const int32_t* d_b_right, int64_t n_b, int64_t n_left_rows,
                    uint8_t* d_flags);

/* Brute-force point x polygon join that allocates no device memory, for
 * callers that cannot allocate (a host that owns all device memory in a
 * fixed arena, a process on a hard memory budget).  No counterpart in the
 * reference: it has no allocation-free join.  Inputs and the pair buffers are
 * the caller's; the kernels' only scratch (one box per polygon and a pair
 * counter) is a fixed 2 MiB device array inside the library, held by every
 * GPU that loads it.  At most 65,536 polygon rows (larger inputs: VS_E_ARG).
 * Runs on `stream` (a cudaStream_t, NULL = legacy default) of the current
 * device and blocks the calling thread until the pair count is back on the
 * host.  The first call on a device resolves the array's address
 * (cudaGetSymbolAddress) and keeps it for the life of the process: make that
 * first call before any stream capture, with the device's primary context
 * current, and make no call after cudaDeviceReset.  Calls that overlap on the
 * GPU share the array and race: serialise them.  Pairs come back unordered;
 * VS_E_CAPACITY reports the required size in *n_pairs. */
int vs_join_brute_noalloc(const vs_points* pts, const vs_polygons* polys, int32_t predicate,
                          int32_t* d_left, int32_t* d_right, int64_t capacity, int64_t* n_pairs,
                          void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VSJOIN_H */
