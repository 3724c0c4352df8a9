// Per-ring y-bins: a ring with many vertices has its y-extent cut into
// kRingBins equal bins, each listing the ring's edges whose closed y-range
// meets the bin.  An edge whose closed y-range does not contain the point's
// y neither crosses the point's +x ray nor holds the point, so walking only
// the edges of the point's bin gives the same location as walking them all,
// with the same first boundary / undecided edge (the bin keeps the ring's
// edge order).  Plays the part of the reference's per-part y-bin edge index
// (predicates/point_location_index.py:103, point_location_index_kernels.py:49-155).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace vs {

constexpr int kRingBins = 8;
constexpr int kRingBinMinVertices = 16;  // default: rings with at least this many vertices are binned
// The FP32 split walk is cheap per edge, so it uses a ring's bins only from
// these lengths on.  Measured: the only ring of a polygon (16-64-vertex
// stars) was faster binned from 16 vertices (256-job batch 17.4 -> 16.8 ms);
// a ring of a polygon with holes or several parts was slower binned at 16-17
// vertices (degenerate refine 8.8 -> 9.2 ms) and faster from 20.
constexpr int kSplitBinMinVertices = 20;    // a ring of a polygon with holes or several parts
constexpr int kSplitBinMinSingleRing = 16;  // the only ring of a polygon

struct __align__(16) RingBins {
    double y0;     // the ring's minimum y
    double scale;  // kRingBins / (maximum y - minimum y)
    uint32_t off[kRingBins + 1];  // bin k's edges are edges[off[k] .. off[k+1])
    uint32_t pad[3];
};

// Read-only view of an index's ring bins; ring_bin == nullptr means none.
struct RingIndex {
    const int32_t* ring_bin = nullptr;  // [n_rings] index into bins, -1: walk every edge
    const RingBins* bins = nullptr;
    const uint16_t* edges = nullptr;    // edge e of a ring joins vertex e-1 (the last for e == 0) to vertex e
};

// Bin of y.  Monotone in y (rounded subtraction and multiplication by a
// positive constant are monotone), so an edge listed in bins
// [bin(min y), bin(max y)] is in the bin of every y it spans.  Build and
// query both call this on the device.
__device__ __forceinline__ int ring_bin_of(double y, double y0, double scale) {
    const double t = __dmul_rn(__dsub_rn(y, y0), scale);
    if (!(t >= 0.0)) return 0;  // below the ring, or NaN
    if (t >= (double)kRingBins) return kRingBins - 1;
    return (int)t;
}

}  // namespace vs
