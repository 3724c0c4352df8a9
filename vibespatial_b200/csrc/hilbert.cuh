// 64-bit Hilbert keys on a 2^32 x 2^32 grid.
//
// The reference orders its flat index by a 32-bit Morton code of bbox centres
// (16 bits per axis, src/vibespatial/spatial/indexing_kernels.py:20-49).  Here
// keys are Hilbert indices with 32 bits per axis: the curve visits the four
// quadrants of every cell in the U-order fixed by the rotation state, so
// consecutive keys are spatially adjacent (no Morton "jumps"), which keeps the
// packed R-tree's node boxes small.  Written from the standard quadrant
// recursion (rotate/reflect per level), MSB first.
#pragma once
#include <stdint.h>

namespace vs {

// Hilbert index of cell (x, y) after `levels` refinements (1..32) of the
// 2^32 grid, i.e. the top 2*levels bits of the full key.  x, y are full
// 32-bit grid coordinates.
__host__ __device__ __forceinline__ uint64_t hilbert_key(uint32_t x, uint32_t y, int levels = 32) {
    uint64_t d = 0;
    for (int lv = 31; lv >= 32 - levels; --lv) {
        const uint32_t rx = (x >> lv) & 1u;
        const uint32_t ry = (y >> lv) & 1u;
        d = (d << 2) | (uint64_t)((3u * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) {
                x = ~x;
                y = ~y;
            }
            const uint32_t t = x;
            x = y;
            y = t;
        }
    }
    return d;
}

// Quantise a coordinate to the 2^32 grid spanning [lo, lo + span] with scale
// = (2^32 - 1) / span; values outside clamp to the border cells.
__host__ __device__ __forceinline__ uint32_t quantize(double v, double lo, double scale) {
    double q = (v - lo) * scale;
    if (!(q > 0.0)) return 0u;  // also NaN
    if (q >= 4294967295.0) return 0xffffffffu;
    return (uint32_t)q;
}

}  // namespace vs
