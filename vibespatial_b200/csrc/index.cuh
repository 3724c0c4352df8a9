// Device-resident spatial index of the polygon (tree) side.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "ringbins.cuh"
#include "vs_common.cuh"

namespace vs {

constexpr int kFanout = 16;      // children per R-tree node
constexpr int kMaxLevels = 16;   // 16^15 > 2^31 items

// Learned cell index (the headline query path): the frame is cut into a
// 2^L x 2^L grid, every polygon box is registered in the cells it overlaps,
// and the non-empty cells are stored as a sorted array of Hilbert cell keys
// with a CSR list of polygon slots.  A two-stage RMI (FP32 MLP root 1->32->32->1
// + linear leaves) predicts a key's position in that array, and a per-leaf
// error window bounds the search, so every lookup is exact.
constexpr int kRmiHidden = 32;

// Everything the learned join needs about one (cell, polygon) entry of the
// learned index, in two 16-byte words.  Coordinates are FP32 offsets from
// the cell's anchor (its centre, cell_anchor below):
//   box       the polygon's box relative to the anchor, rounded outward
//   off       fl32(anchor - slot origin): a query point q relative to the
//             anchor is q + off relative to the slot origin, the frame of
//             the slot's FP32 vertices (xy32)
//   err       bound on |FP32 vertex - (vertex - origin)| of the slot plus
//             |off - (anchor - origin)|
//   slot      the polygon's slot (its original row is item_geom[slot]) in
//             the low 31 bits; bit 31 set when the slot has an interior box
// The learned index stores one record per entry, in cell order, so a
// candidate is one 32-byte read.
struct __align__(16) EntryRecord {
    float4 box;
    float offx, offy;
    float err;
    int32_t slot;
};
constexpr uint32_t kEntryInteriorBit = 0x80000000u;
__host__ __device__ __forceinline__ int32_t entry_slot(const EntryRecord& r) {
    return (int32_t)((uint32_t)r.slot & ~kEntryInteriorBit);
}
__host__ __device__ __forceinline__ bool entry_has_interior(const EntryRecord& r) {
    return ((uint32_t)r.slot & kEntryInteriorBit) != 0;
}

// A query point matched to a cell: FP32 offsets from the cell's anchor, its
// row, and its batch-wide cell number.  The map pass stages these, the place
// pass permutes them into cell order, and the refine pass reads them.
struct __align__(16) CellPoint {
    float qx, qy;
    int32_t row;
    uint32_t gcell;
};

// Leaf of the RMI: position = floor(a + b * key), error window [lo, hi].
struct __align__(16) RmiLeaf {
    double a, b;
    int32_t lo, hi;
    int32_t pad0, pad1;
};

struct RmiModel {
    // root MLP weights (FP32): h1 = relu(w1 * x + b1); h2 = relu(W2 h1 + b2); y = w3 . h2 + b3
    float w1[kRmiHidden], b1[kRmiHidden];
    float w2[kRmiHidden * kRmiHidden], b2[kRmiHidden];
    float w3[kRmiHidden], b3;
    // input normalisation: x = (key - key_lo) * key_scale   (double)
    double key_lo, key_scale;
    int32_t n_leaves;
    int32_t n_keys;
};

// One learned index as the query kernels see it (device memory, or
// the kernel parameters for a single join).  A batch of
// joins passes an array of these; job j's cells are numbered from
// cell_base in the batch-wide cell numbering.
struct LearnedJob {
    // frame and quantisation scales, computed on the device exactly as the
    // build computed them
    double lox, loy, hix, hiy, sx, sy;
    double cwx, cwy;     // level-L cell width per axis (cell_anchor)
    int32_t L;
    int32_t occ_shift;   // cell key >> occ_shift = occupancy bit
    int32_t root_shift;  // cell key >> root_shift = root-table index
    uint32_t cell_base;
    int64_t n_cells;
    const uint32_t* occ;
    const uint16_t* root_table;
    const RmiLeaf* leaves;
    const uint32_t* cell_keys;
    const uint32_t* cell_start;
    const EntryRecord* recs;  // [n_entries] per-entry records, cell order
    const int2* c01;          // [n_geoms] coordinate range of a single-ring slot, (-1, -1) otherwise
    const float4* ring_box32; // [n_rings] box of each ring's FP32 vertices (minx, miny, maxx, maxy)
    const float4* ib32;       // [n_geoms] interior box of each slot, relative to its origin (empty: none)
    const float2* xy32;
    const double2* xy;
    const int32_t* item_geom;
    const int32_t* geom_off;
    const int32_t* part_off;
    const int32_t* ring_off;
    const vs_box* boxes;     // FP64 slot boxes (R-tree level 0)
    RingIndex rings;         // y-bins of the index's long rings
};

// Launch shape of the learned pipeline (every field 0 = the default), and the
// ablation switches that replace one of its choices by the plain method.
struct LearnedShape {
    int32_t map_blocks_per_sm;     // map pass blocks per SM (0 = 8)
    int32_t refine_blocks_per_sm;  // refine pass blocks per SM (0 = as many as fit)
    int32_t grab;                  // grouped points a refine warp takes per work grab (0 = 32; multiple of 32)
    uint32_t flags;                // kLearnedBsearch | kLearnedFp64Walk | kLearnedNoStage | kLearnedNoInterior
    int32_t map_packets;           // 32-point packets a map warp looks up together (1 or 2; 0 = 1)
};
constexpr uint32_t kLearnedBsearch = 1u;   // cell lookup by binary search over all cell keys (no RMI)
constexpr uint32_t kLearnedFp64Walk = 2u;  // ring walks in FP64 (no FP32 edge stage)
constexpr uint32_t kLearnedNoStage = 4u;   // entry records read from global memory (no bulk-copy staging)
constexpr uint32_t kLearnedNoInterior = 8u;  // every box candidate is ring-walked (no interior-box shortcut)

// Centre of level-L grid cell c on one axis: lo + (c + 0.5) * cell width,
// one fused multiply-add, so the index build (from a cell's key) and the
// query (from a point's quantised coordinates) compute the same bits.
__device__ __forceinline__ double cell_anchor(double lo, double cw, uint32_t c) {
    return __fma_rn((double)c + 0.5, cw, lo);
}

struct LearnedIndex {
    int32_t level = 0;               // grid level L (cells of frame / 2^L per axis)
    int32_t occ_level = 0;           // occupancy bitmap level (<= L)
    int64_t n_cells = 0;             // non-empty cells
    int64_t n_entries = 0;           // (cell, polygon) registrations
    uint32_t* cell_keys = nullptr;   // [n_cells] sorted level-L Hilbert keys
    uint32_t* cell_start = nullptr;  // [n_cells + 1] CSR offsets into entries
    uint32_t* entries = nullptr;     // [n_entries] polygon slots (Hilbert order)
    uint32_t* occ = nullptr;         // occupancy bitmap of level occ_level
    // RMI: root MLP + per-leaf linear model and error window.  The root's
    // input is the cell's level-R ancestor key (R = root_level <= L), a
    // finite domain of 4^R values, so the trained MLP is tabulated over that
    // whole domain once (root_table[ancestor] = leaf).  Routing at build and
    // query time reads the same table, which is what makes the per-leaf
    // error windows exact bounds for every stored key.
    RmiModel* model = nullptr;       // device
    int32_t root_level = 0;
    uint16_t* root_table = nullptr;  // [4^root_level] leaf of each ancestor cell
    double2* leaf_ab = nullptr;      // [n_leaves] position = a + b * key
    int2* leaf_err = nullptr;        // [n_leaves] inclusive error window (lo, hi)
    RmiLeaf* leaves = nullptr;       // [n_leaves] the two above packed for queries
    int32_t n_leaves = 0;
    EntryRecord* recs = nullptr;     // [n_entries] record of each entry, cell order
    int2* c01 = nullptr;             // [n_geoms] single-ring coordinate range per slot
    float4* ring_box32 = nullptr;    // [n_rings] box of each ring's FP32 vertices (everything if one is NaN)
    float4* ib32 = nullptr;          // [n_geoms] interior box per slot (csrc/learned.cu interior_box_kernel)
    LearnedJob* desc = nullptr;      // device: this index as the query kernels see it
    LearnedJob h_desc{};             // host copy of *desc
    // FP32 tile-relative copies used by the split-precision filter
    double2* origin = nullptr;       // [n_geoms] slot origin (box centre, FP64)
    float* err32 = nullptr;          // [n_geoms] bound on |vertex rounding error| of the slot
    float2* xy32 = nullptr;          // [n_coords] vertices relative to their slot origin (nearest)
    float rmi_train_ms = 0.f;
    float rmi_final_loss = 0.f;
    float mean_window = 0.f;
    int32_t max_window = 0;
};

}  // namespace vs

struct vs_index {
    int device = 0;
    int32_t n_geoms = 0, n_parts = 0, n_rings = 0;
    int64_t n_coords = 0;
    int32_t levels = 0;
    int64_t level_off[vs::kMaxLevels] = {};
    int64_t level_size[vs::kMaxLevels] = {};
    vs_box* nodes = nullptr;      // all levels, level 0 = polygon boxes in Hilbert order
    int32_t* item_geom = nullptr; // slot -> original polygon row
    // polygon data re-laid out in slot (Hilbert) order, vertices interleaved
    int32_t* geom_off = nullptr;
    int32_t* part_off = nullptr;
    int32_t* ring_off = nullptr;
    double2* xy = nullptr;
    double* frame = nullptr;      // device [4]: minx, miny, maxx, maxy of valid boxes
    // y-bins of the rings with many vertices (ringbins.cuh)
    int32_t* ring_bin = nullptr;        // [n_rings] -1 or index into ring_bins
    vs::RingBins* ring_bins = nullptr;  // [n_binned_rings]
    uint16_t* bin_edges = nullptr;      // [n_bin_edges]
    int64_t n_binned_rings = 0, n_bin_edges = 0;
    int64_t n_split_binned_rings = 0;   // binned rings the split walk takes binned (kSplitBinMin*)
    vs::RingIndex ring_index() const {
        vs::RingIndex ri;
        ri.ring_bin = ring_bin;
        ri.bins = ring_bins;
        ri.edges = bin_edges;
        return ri;
    }
    double h_frame[4] = {0, 0, 0, 0};
    bool has_learned = false;
    vs::LearnedIndex learned;
    int64_t device_bytes = 0;
    float build_ms = 0.f;
};

namespace vs {
int build_learned_index(vs_context* ctx, vs_index* idx, const vs_index_options* opts);
void free_learned_index(vs_index* idx);
}  // namespace vs
