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

// Table-driven form of the same curve, four levels per step.  The walk above
// only ever swaps x/y and/or complements both, so after any prefix the
// remaining bits are read through one of four transforms (state = swap |
// complement << 1).  Entry [state][4 bits of x][4 bits of y] holds the 8 key
// bits of those four levels and the next state (bits 8-9).  Each block builds
// the 1024 entries in shared memory from the per-level rule.
constexpr int kHilbertLutSize = 1024;

__device__ __forceinline__ void hilbert_lut_init(uint16_t* lut) {
    for (int e = threadIdx.x; e < kHilbertLutSize; e += blockDim.x) {
        uint32_t sw = (uint32_t)(e >> 8) & 1u, inv = (uint32_t)(e >> 9) & 1u;
        const uint32_t bx = (uint32_t)(e >> 4) & 15u, by = (uint32_t)e & 15u;
        uint32_t d = 0;
        for (int lv = 3; lv >= 0; --lv) {
            const uint32_t x0 = (bx >> lv) & 1u, y0 = (by >> lv) & 1u;
            const uint32_t rx = (sw ? y0 : x0) ^ inv, ry = (sw ? x0 : y0) ^ inv;
            d = (d << 2) | ((3u * rx) ^ ry);
            if (ry == 0) {
                if (rx == 1) inv ^= 1u;
                sw ^= 1u;
            }
        }
        lut[e] = (uint16_t)(d | ((sw | (inv << 1)) << 8));
    }
}

// Top 2*levels bits of the Hilbert key (levels <= 16), equal to
// hilbert_key(x, y, levels).
__device__ __forceinline__ uint32_t hilbert_key_lut(uint32_t x, uint32_t y, int levels, const uint16_t* lut) {
    const int chunks = (levels + 3) >> 2;
    uint32_t d = 0, state = 0;
    for (int c = 0; c < chunks; ++c) {
        const int sh = 28 - 4 * c;
        const uint32_t e = lut[(state << 8) | (((x >> sh) & 15u) << 4) | ((y >> sh) & 15u)];
        d = (d << 8) | (e & 255u);
        state = e >> 8;
    }
    return d >> (2 * (4 * chunks - levels));
}

// Inverse of hilbert_key at `levels` levels: the cell (cx, cy) of the
// level-`levels` grid (so hilbert_key(cx << (32 - levels), cy << (32 - levels),
// levels) == key).  The walk reads the key's base-4 digits MSB first under the
// same swap / complement state as the table above: digit d = (3 rx) ^ ry gives
// rx = d >> 1 and ry = (d ^ rx) & 1 in the transformed frame.
__host__ __device__ __forceinline__ void hilbert_cell(uint32_t key, int levels, uint32_t& cx, uint32_t& cy) {
    uint32_t sw = 0, inv = 0, x = 0, y = 0;
    for (int lv = levels - 1; lv >= 0; --lv) {
        const uint32_t d = (key >> (2 * lv)) & 3u;
        const uint32_t rx = d >> 1, ry = (d ^ rx) & 1u;
        const uint32_t a = rx ^ inv, b = ry ^ inv;
        x = (x << 1) | (sw ? b : a);
        y = (y << 1) | (sw ? a : b);
        if (ry == 0) {
            if (rx == 1) inv ^= 1u;
            sw ^= 1u;
        }
    }
    cx = x;
    cy = y;
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
