// Learned cell index: build, RMI training, and the learned + split-precision join.
//
// Build (after the packed R-tree, reusing its Hilbert slot order and frame):
//   1. every polygon box is registered in the level-L grid cells it overlaps
//      (cell key = level-L Hilbert key, the top 2L bits of a point's key)
//   2. (cell key, slot) pairs are radix-sorted; unique keys + CSR offsets
//      give the sorted build-side array the RMI indexes
//   3. an occupancy bitmap at a coarser level lets empty regions skip lookups
//   4. the RMI (FP32 MLP 1->32->32->1 root + linear leaves) is trained on the
//      sorted cell keys with hand-written forward/backward and Adam kernels;
//      the root's input is the cell's level-R ancestor (R <= 10), so the
//      trained MLP is tabulated over all 4^R ancestors; every stored key is
//      routed through that table to fit the leaves and to measure each
//      leaf's inclusive error window
//   5. FP32 copies of every polygon relative to its own origin (box centre),
//      with a per-polygon bound on the rounding error, for the split filter
//
// The query passes over this index live in learned_query.cu.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <cmath>
#include <vector>

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
constexpr int kRmiP = kRmiHidden + kRmiHidden + kRmiHidden * kRmiHidden + kRmiHidden + kRmiHidden + 1;  // 1153
constexpr int kOffW1 = 0, kOffB1 = 32, kOffW2 = 64, kOffB2 = 64 + 1024, kOffW3 = 64 + 1024 + 32,
              kOffB3 = 64 + 1024 + 64;
constexpr int kTrainBlocks = 64;

__device__ __forceinline__ void frame_q(const double* fr, double& lox, double& loy, double& sx, double& sy) {
    lox = fr[0];
    loy = fr[1];
    sx = fr[2] > fr[0] ? 4294967295.0 / (fr[2] - fr[0]) : 0.0;
    sy = fr[3] > fr[1] ? 4294967295.0 / (fr[3] - fr[1]) : 0.0;
}

// ---------------------------------------------------------------- build ---
__global__ void box_side_kernel(const vs_box* __restrict__ box, int64_t M, double* __restrict__ acc) {
    double s = 0.0, c = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x) {
        const vs_box b = box[i];
        if (b.minx <= b.maxx) {
            s += fmax(b.maxx - b.minx, b.maxy - b.miny);
            c += 1.0;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0 && c > 0) {
        atomicAdd(&acc[0], s);
        atomicAdd(&acc[1], c);
    }
}

__device__ __forceinline__ bool cell_range(const vs_box& b, const double* fr, int L, uint32_t& cx0, uint32_t& cx1,
                                           uint32_t& cy0, uint32_t& cy1) {
    if (!(b.minx <= b.maxx)) return false;
    double lox, loy, sx, sy;
    frame_q(fr, lox, loy, sx, sy);
    const int sh = 32 - L;
    cx0 = quantize(b.minx, lox, sx) >> sh;
    cx1 = quantize(b.maxx, lox, sx) >> sh;
    cy0 = quantize(b.miny, loy, sy) >> sh;
    cy1 = quantize(b.maxy, loy, sy) >> sh;
    return true;
}

__global__ void cell_count_kernel(const vs_box* __restrict__ box, int64_t M, const double* __restrict__ fr, int L,
                                  uint32_t* __restrict__ cnt, unsigned long long* __restrict__ total) {
    unsigned long long t = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t x0, x1, y0, y1;
        uint64_t c = 0;
        if (cell_range(box[i], fr, L, x0, x1, y0, y1)) c = (uint64_t)(x1 - x0 + 1) * (uint64_t)(y1 - y0 + 1);
        cnt[i] = c > 0xffffffffull ? 0xffffffffu : (uint32_t)c;
        t += c;
    }
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0 && t) atomicAdd(total, t);
}

__global__ void cell_emit_kernel(const vs_box* __restrict__ box, int64_t M, const double* __restrict__ fr, int L,
                                 const uint32_t* __restrict__ off, uint32_t* __restrict__ keys,
                                 uint32_t* __restrict__ vals) {
    const int sh = 32 - L;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t x0, x1, y0, y1;
        if (!cell_range(box[i], fr, L, x0, x1, y0, y1)) continue;
        uint32_t o = off[i];
        for (uint32_t cy = y0; cy <= y1; ++cy)
            for (uint32_t cx = x0; cx <= x1; ++cx) {
                keys[o] = (uint32_t)hilbert_key(cx << sh, cy << sh, L);
                vals[o] = (uint32_t)i;
                ++o;
            }
    }
}

__global__ void cell_flag_kernel(const uint32_t* __restrict__ keys, int64_t E, uint32_t* __restrict__ flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// Sum over the distinct cells of (entries in the cell)^2, from the sorted
// keys: each cell's first entry measures its run.  Divided by the entry
// count it is the mean list length seen from an entry (its own cell's count).
__global__ void cell_run_sq_kernel(const uint32_t* __restrict__ keys, int64_t E, unsigned long long* __restrict__ acc) {
    unsigned long long t = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        if (i > 0 && keys[i] == keys[i - 1]) continue;
        int64_t j = i + 1;
        while (j < E && keys[j] == keys[i]) ++j;
        t += (unsigned long long)(j - i) * (unsigned long long)(j - i);
    }
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0 && t) atomicAdd(acc, t);
}

__global__ void cell_compact_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ id, int64_t E,
                                    uint32_t* __restrict__ cell_keys, uint32_t* __restrict__ cell_start) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        if (i == 0 || keys[i] != keys[i - 1]) {
            cell_keys[id[i]] = keys[i];
            cell_start[id[i]] = (uint32_t)i;
        }
    }
}

__global__ void occ_kernel(const uint32_t* __restrict__ cell_keys, int64_t n, int shift, uint32_t* __restrict__ occ) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t b = cell_keys[i] >> shift;
        atomicOr(&occ[b >> 5], 1u << (b & 31));
    }
}

// One warp per slot: origin, outward-rounded FP32 box, FP32 vertices and the
// slot's rounding-error bound.
__global__ void split_copy_kernel(const vs_box* __restrict__ box, int64_t M, const int32_t* __restrict__ geom_off,
                                  const int32_t* __restrict__ part_off, const int32_t* __restrict__ ring_off,
                                  const double2* __restrict__ xy, double2* __restrict__ origin,
                                  float* __restrict__ err32, float2* __restrict__ xy32) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const double u64 = 1.1102230246251565e-16;  // 2^-53
    for (int64_t s = warp; s < M; s += nw) {
        const vs_box b = box[s];
        const bool ok = b.minx <= b.maxx;
        const double ox = ok ? 0.5 * b.minx + 0.5 * b.maxx : 0.0;
        const double oy = ok ? 0.5 * b.miny + 0.5 * b.maxy : 0.0;
        const int32_t c0 = ring_off[part_off[geom_off[s]]], c1 = ring_off[part_off[geom_off[s + 1]]];
        double emax = 0.0;
        for (int32_t c = c0 + lane; c < c1; c += 32) {
            const double2 v = xy[c];
            const double dx = v.x - ox, dy = v.y - oy;
            const float fx = __double2float_rn(dx), fy = __double2float_rn(dy);
            xy32[c] = make_float2(fx, fy);
            const double ex = fabs((double)fx - dx) + fabs(dx) * u64;
            const double ey = fabs((double)fy - dy) + fabs(dy) * u64;
            emax = fmax(emax, fmax(ex, ey));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
        if (lane == 0) {
            origin[s] = make_double2(ox, oy);
            err32[s] = __double2float_ru(emax * (1.0 + 1e-6));
        }
    }
}

// Box of every ring's FP32 (slot-relative) vertices, a warp per ring.  A
// ring with a NaN vertex gets the whole plane, so no walk ever skips it.
__global__ void ring_box_kernel(const int32_t* __restrict__ ring_off, int64_t n_rings,
                                const float2* __restrict__ xy32, float4* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r = warp; r < n_rings; r += nw) {
        const int32_t c0 = ring_off[r], c1 = ring_off[r + 1];
        float mnx = INFINITY, mny = INFINITY, mxx = -INFINITY, mxy = -INFINITY;
        bool nan = false;
        for (int32_t c = c0 + lane; c < c1; c += 32) {
            const float2 v = xy32[c];
            nan |= isnan(v.x) || isnan(v.y);
            mnx = fminf(mnx, v.x);
            mny = fminf(mny, v.y);
            mxx = fmaxf(mxx, v.x);
            mxy = fmaxf(mxy, v.y);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
            mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
            mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
            mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
        }
        nan = __any_sync(0xffffffffu, nan);
        if (lane == 0)
            out[r] = nan ? make_float4(-INFINITY, -INFINITY, INFINITY, INFINITY) : make_float4(mnx, mny, mxx, mxy);
    }
}

// Smallest s >= 0 for which the box [-s a, s a] x [-s b, s b] (a = 1 / ia,
// b = 1 / ib) touches the segment (x0, y0) -> (x1, y1): the minimum over the
// segment of max(|x| ia, |y| ib).  That function of the segment parameter is
// convex and piecewise linear, so its minimum lies at an end or where |x| ia
// and |y| ib are 0 or equal; all of these are evaluated.
__device__ __forceinline__ double box_reach(double x0, double y0, double x1, double y1, double ia, double ib) {
    const double dx = x1 - x0, dy = y1 - y0;
    auto f = [&](double t) {
        t = fmin(fmax(t, 0.0), 1.0);
        return fmax(fabs(x0 + t * dx) * ia, fabs(y0 + t * dy) * ib);
    };
    double m = fmin(f(0.0), f(1.0));
    if (dx != 0.0) m = fmin(m, f(-x0 / dx));
    if (dy != 0.0) m = fmin(m, f(-y0 / dy));
    const double p = dx * ia - dy * ib, q = dx * ia + dy * ib;
    if (p != 0.0) m = fmin(m, f((y0 * ib - x0 * ia) / p));
    if (q != 0.0) m = fmin(m, f(-(y0 * ib + x0 * ia) / q));
    return m;
}

// Interior box of every slot, a warp per slot: an axis-aligned box around the
// slot origin (its box centre) with the slot box's proportions that touches
// no edge of any ring, kept only when the origin itself is strictly interior
// (decided exactly).  Such a box lies in the face of the origin, so every
// point strictly inside it is interior.  Its half sizes are 0.999 of the
// largest such box (the margin dwarfs the FP64 rounding of the vertex
// offsets, and boxes below 1e-9 of the coordinates' magnitude are dropped);
// stored in FP32 relative to the origin, rounded inward.  Slots without one
// get an empty box.
__global__ void interior_box_kernel(const vs_box* __restrict__ boxes, int64_t M, const int32_t* __restrict__ geom_off,
                                    const int32_t* __restrict__ part_off, const int32_t* __restrict__ ring_off,
                                    const double2* __restrict__ xy, RingIndex ri, const double2* __restrict__ origin,
                                    float4* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = warp; s < M; s += nw) {
        const vs_box b = boxes[s];
        const double2 o = origin[s];
        const double ha = 0.5 * (b.maxx - b.minx), hb = 0.5 * (b.maxy - b.miny);
        bool ok = b.minx <= b.maxx && b.miny <= b.maxy && ha > 0.0 && hb > 0.0;
        int loc = LOC_OUTSIDE;
        if (ok && lane == 0) {
            unsigned n_exact = 0;
            loc = geometry_location(o.x, o.y, xy, ring_off, part_off, geom_off, (int)s, ri, n_exact);
        }
        ok = ok && __shfl_sync(0xffffffffu, loc, 0) == LOC_INTERIOR;
        double reach = INFINITY;
        bool nan = false;
        if (ok) {
            const double ia = 1.0 / ha, ib = 1.0 / hb;
            const int p0 = geom_off[s], p1 = geom_off[s + 1];
            for (int ring = part_off[p0]; ring < part_off[p1]; ++ring) {  // warp-uniform
                const int c0 = ring_off[ring], c1 = ring_off[ring + 1];
                for (int i = c0 + lane; i < c1; i += 32) {
                    const double2 v0 = xy[i == c0 ? c1 - 1 : i - 1], v1 = xy[i];
                    nan |= isnan(v0.x) || isnan(v0.y) || isnan(v1.x) || isnan(v1.y);
                    reach = fmin(reach, box_reach(v0.x - o.x, v0.y - o.y, v1.x - o.x, v1.y - o.y, ia, ib));
                }
            }
        }
#pragma unroll
        for (int k = 16; k > 0; k >>= 1) reach = fmin(reach, __shfl_xor_sync(0xffffffffu, reach, k));
        nan = __any_sync(0xffffffffu, nan);
        if (lane == 0) {
            const double hx = 0.999 * reach * ha, hy = 0.999 * reach * hb;
            const double floor_abs = 1e-9 * fmax(fabs(o.x), fabs(o.y));
            const bool keep = ok && !nan && reach > 0.0 && reach < INFINITY && hx > floor_abs && hy > floor_abs;
            out[s] = keep ? make_float4(__double2float_ru(-hx), __double2float_ru(-hy), __double2float_rd(hx),
                                        __double2float_rd(hy))
                          : make_float4(INFINITY, INFINITY, -INFINITY, -INFINITY);
        }
    }
}

// Coordinate range of every single-ring slot: such polygons take the short
// ring walk (c0 >= 0) unless the split walk uses the ring's y-bins (from
// kSplitBinMinSingleRing vertices).  n_extra counts the rings this walks
// binned below kSplitBinMinVertices, which the index's count of rings for
// the binned walk does not hold yet.
__global__ void slot_c01_kernel(int64_t M, const int32_t* __restrict__ geom_off, const int32_t* __restrict__ part_off,
                                const int32_t* __restrict__ ring_off, const int32_t* __restrict__ ring_bin,
                                int2* __restrict__ out, unsigned* __restrict__ n_extra) {
    unsigned extra = 0;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M; s += (int64_t)gridDim.x * blockDim.x) {
        int2 r = make_int2(-1, -1);
        const int32_t p0 = geom_off[s], p1 = geom_off[s + 1];
        if (p1 - p0 == 1 && part_off[p0 + 1] - part_off[p0] == 1) {
            const int ring = part_off[p0];
            const int c0 = ring_off[ring], c1 = ring_off[ring + 1];
            if (ring_bin == nullptr || ring_bin[ring] < 0 || c1 - c0 < kSplitBinMinSingleRing) r = make_int2(c0, c1);
            else if (c1 - c0 < kSplitBinMinVertices) ++extra;
        }
        out[s] = r;
    }
    if (extra) atomicAdd(n_extra, extra);
}

// One record per (cell, polygon) entry, in cell order, relative to the cell's
// anchor.  The cell comes from the entry's sorted key (Hilbert decode); a
// decode that does not re-encode to the key sets *bad (the build then fails).
__global__ void entry_recs_kernel(int64_t E, const uint32_t* __restrict__ keys, const uint32_t* __restrict__ entries,
                                  const LearnedJob* __restrict__ d, const vs_box* __restrict__ boxes,
                                  const double2* __restrict__ origin, const float* __restrict__ err32,
                                  const float4* __restrict__ ib32, EntryRecord* __restrict__ out,
                                  unsigned* __restrict__ bad) {
    const double u64 = 1.1102230246251565e-16;  // 2^-53
    const int L = d->L, sh = 32 - L;
    const double lox = d->lox, loy = d->loy, cwx = d->cwx, cwy = d->cwy;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t key = keys[e];
        uint32_t cx, cy;
        hilbert_cell(key, L, cx, cy);
        if ((uint32_t)hilbert_key(cx << sh, cy << sh, L) != key) atomicOr(bad, 1u);
        const double ax = cell_anchor(lox, cwx, cx), ay = cell_anchor(loy, cwy, cy);
        const int32_t slot = (int32_t)entries[e];
        const vs_box b = boxes[slot];
        const double2 o = origin[slot];
        EntryRecord r;
        if (b.minx <= b.maxx && b.miny <= b.maxy) {
            // each FP64 difference is within u64 |v| of the real one; widen by that, then round outward
            const double a = b.minx - ax, c = b.miny - ay, f = b.maxx - ax, g = b.maxy - ay;
            r.box = make_float4(__double2float_rd(a - fabs(a) * u64), __double2float_rd(c - fabs(c) * u64),
                                __double2float_ru(f + fabs(f) * u64), __double2float_ru(g + fabs(g) * u64));
        } else {
            r.box = make_float4(INFINITY, INFINITY, -INFINITY, -INFINITY);
        }
        const double dx = ax - o.x, dy = ay - o.y;
        r.offx = __double2float_rn(dx);
        r.offy = __double2float_rn(dy);
        const double ex = fabs((double)r.offx - dx) + fabs(dx) * u64;
        const double ey = fabs((double)r.offy - dy) + fabs(dy) * u64;
        r.err = __double2float_ru(((double)err32[slot] + fmax(ex, ey)) * (1.0 + 1e-6));
        const float4 ib = ib32[slot];
        r.slot = (int32_t)((uint32_t)slot | (ib.x < ib.z ? kEntryInteriorBit : 0u));
        out[e] = r;
    }
}

__global__ void pack_leaves_kernel(int nl, const double2* __restrict__ ab, const int2* __restrict__ err,
                                   RmiLeaf* __restrict__ out) {
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nl; l += gridDim.x * blockDim.x) {
        RmiLeaf f;
        f.a = ab[l].x;
        f.b = ab[l].y;
        f.lo = err[l].x;
        f.hi = err[l].y;
        f.pad0 = f.pad1 = 0;
        out[l] = f;
    }
}

// ------------------------------------------------------------ RMI train ---
// Training pairs: x = normalised ancestor key of stored cell i, t = i / n.
__global__ void rmi_samples_kernel(const uint32_t* __restrict__ keys, int64_t n, int S, int anc_shift, double key_lo,
                                   double key_scale, float* __restrict__ xs, float* __restrict__ ts) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < S; s += gridDim.x * blockDim.x) {
        const int64_t i = (int64_t)((double)s * (double)n / (double)S);
        xs[s] = __double2float_rn(((double)(keys[i] >> anc_shift) - key_lo) * key_scale);
        ts[s] = (float)((double)i / (double)n);
    }
}

// Full-batch gradient of the mean squared error over S samples.  A warp takes
// one sample at a time with lane j owning hidden unit j; each block sums its
// warps' gradients in shared memory and writes one partial row.
__global__ void __launch_bounds__(kThreads) rmi_grad_kernel(const float* __restrict__ P, const float* __restrict__ xs,
                                                            const float* __restrict__ ts, int S,
                                                            float* __restrict__ partial, float* __restrict__ loss) {
    __shared__ float g[kRmiP];
    for (int i = threadIdx.x; i < kRmiP; i += blockDim.x) g[i] = 0.f;
    __syncthreads();
    const int j = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const float w1 = P[kOffW1 + j], b1 = P[kOffB1 + j], b2 = P[kOffB2 + j], w3 = P[kOffW3 + j], b3 = P[kOffB3];
    float row[kRmiHidden], col[kRmiHidden], grow[kRmiHidden];
#pragma unroll
    for (int k = 0; k < kRmiHidden; ++k) {
        row[k] = P[kOffW2 + j * kRmiHidden + k];
        col[k] = P[kOffW2 + k * kRmiHidden + j];
        grow[k] = 0.f;
    }
    float gw1 = 0.f, gb1 = 0.f, gb2 = 0.f, gw3 = 0.f, gb3 = 0.f, l2 = 0.f;
    const float inv = 1.0f / (float)S;
    for (int s = warp; s < S; s += nwarps) {
        const float x = xs[s], t = ts[s];
        const float z1 = fmaf(w1, x, b1);
        const float h1 = fmaxf(z1, 0.f);
        float z2 = b2;
#pragma unroll
        for (int k = 0; k < kRmiHidden; ++k) z2 = fmaf(row[k], __shfl_sync(0xffffffffu, h1, k), z2);
        const float h2 = fmaxf(z2, 0.f);
        float y = w3 * h2;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) y += __shfl_xor_sync(0xffffffffu, y, o);
        y += b3;
        const float err = y - t;
        const float gy = 2.f * err * inv;
        l2 += err * err * inv;
        gw3 += gy * h2;
        gb3 += gy;
        const float d2 = z2 > 0.f ? gy * w3 : 0.f;
        gb2 += d2;
#pragma unroll
        for (int k = 0; k < kRmiHidden; ++k) grow[k] = fmaf(d2, __shfl_sync(0xffffffffu, h1, k), grow[k]);
        float dh1 = 0.f;
#pragma unroll
        for (int i = 0; i < kRmiHidden; ++i) dh1 = fmaf(__shfl_sync(0xffffffffu, d2, i), col[i], dh1);
        const float d1 = z1 > 0.f ? dh1 : 0.f;
        gw1 += d1 * x;
        gb1 += d1;
    }
    atomicAdd(&g[kOffW1 + j], gw1);
    atomicAdd(&g[kOffB1 + j], gb1);
    atomicAdd(&g[kOffB2 + j], gb2);
    atomicAdd(&g[kOffW3 + j], gw3);
#pragma unroll
    for (int k = 0; k < kRmiHidden; ++k) atomicAdd(&g[kOffW2 + j * kRmiHidden + k], grow[k]);
    if (j == 0) {
        atomicAdd(&g[kOffB3], gb3);
        atomicAdd(loss, l2);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kRmiP; i += blockDim.x) partial[(int64_t)blockIdx.x * kRmiP + i] = g[i];
}

__global__ void rmi_adam_kernel(float* __restrict__ P, float* __restrict__ m1, float* __restrict__ m2,
                                const float* __restrict__ partial, int G, int step, float lr) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kRmiP) return;
    float g = 0.f;
    for (int b = 0; b < G; ++b) g += partial[(int64_t)b * kRmiP + p];
    const float b1 = 0.9f, b2 = 0.999f;
    const float m = b1 * m1[p] + (1.f - b1) * g;
    const float v = b2 * m2[p] + (1.f - b2) * g * g;
    m1[p] = m;
    m2[p] = v;
    const float mh = m / (1.f - powf(b1, (float)step));
    const float vh = v / (1.f - powf(b2, (float)step));
    P[p] -= lr * mh / (sqrtf(vh) + 1e-8f);
}

__global__ void rmi_pack_kernel(const float* __restrict__ P, RmiModel* __restrict__ m, double key_lo, double key_scale,
                                int n_leaves, int n_keys) {
    for (int i = threadIdx.x; i < kRmiHidden * kRmiHidden; i += blockDim.x) m->w2[i] = P[kOffW2 + i];
    for (int i = threadIdx.x; i < kRmiHidden; i += blockDim.x) {
        m->w1[i] = P[kOffW1 + i];
        m->b1[i] = P[kOffB1 + i];
        m->b2[i] = P[kOffB2 + i];
        m->w3[i] = P[kOffW3 + i];
    }
    if (threadIdx.x == 0) {
        m->b3 = P[kOffB3];
        m->key_lo = key_lo;
        m->key_scale = key_scale;
        m->n_leaves = n_leaves;
        m->n_keys = n_keys;
    }
}

// Tabulate the trained root over every ancestor key (one warp per key).
__global__ void __launch_bounds__(kThreads) rmi_table_kernel(const RmiModel* __restrict__ model, int64_t n_anc,
                                                             uint16_t* __restrict__ table) {
    __shared__ RmiShared sm;
    rmi_load_shared(&sm, model);
    __syncthreads();
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t c = warp; c < n_anc; c += nw) {
        const float y = rmi_root_warp(&sm, rmi_input((uint32_t)c, &sm));
        if ((threadIdx.x & 31) == 0) table[c] = (uint16_t)rmi_leaf(sm.n_leaves, y);
    }
}

__global__ void rmi_route_kernel(const uint16_t* __restrict__ table, const uint32_t* __restrict__ keys, int64_t n,
                                 int anc_shift, uint32_t* __restrict__ leaf_of) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        leaf_of[i] = table[keys[i] >> anc_shift];
}

__global__ void rmi_leaf_sums_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ leaf_of, int64_t n,
                                     double* __restrict__ sums) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t l = leaf_of[i];
        atomicAdd(&sums[3 * l + 0], 1.0);
        atomicAdd(&sums[3 * l + 1], (double)keys[i]);
        atomicAdd(&sums[3 * l + 2], (double)i);
    }
}

__global__ void rmi_leaf_cov_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ leaf_of, int64_t n,
                                    const double* __restrict__ sums, double* __restrict__ cov) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t l = leaf_of[i];
        const double c = sums[3 * l];
        const double mx = sums[3 * l + 1] / c, my = sums[3 * l + 2] / c;
        const double dx = (double)keys[i] - mx, dy = (double)i - my;
        atomicAdd(&cov[2 * l + 0], dx * dy);
        atomicAdd(&cov[2 * l + 1], dx * dx);
    }
}

__global__ void rmi_leaf_fit_kernel(const double* __restrict__ sums, const double* __restrict__ cov, int nl,
                                    double2* __restrict__ ab, int2* __restrict__ err) {
    for (int l = blockIdx.x * blockDim.x + threadIdx.x; l < nl; l += gridDim.x * blockDim.x) {
        const double c = sums[3 * l];
        double a = 0.0, b = 0.0;
        if (c > 0) {
            const double mx = sums[3 * l + 1] / c, my = sums[3 * l + 2] / c;
            b = cov[2 * l + 1] > 0 ? cov[2 * l + 0] / cov[2 * l + 1] : 0.0;
            a = my - b * mx;
        }
        ab[l] = make_double2(a, b);
        err[l] = make_int2(0x7fffffff, -0x7fffffff);
    }
}

// Error window of each leaf, measured over every stored key with the same
// routing table and leaf model the queries use.
__global__ void rmi_err_kernel(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ leaf_of, int64_t n,
                               const double2* __restrict__ ab, int2* __restrict__ err) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t l = leaf_of[i];
        long long e = (long long)i - rmi_predict(ab[l], keys[i]);
        e = e < -0x7ffffffe ? -0x7ffffffe : (e > 0x7ffffffe ? 0x7ffffffe : e);
        atomicMin(&err[l].x, (int)e);
        atomicMax(&err[l].y, (int)e);
    }
}

__global__ void rmi_window_stats_kernel(const uint32_t* __restrict__ leaf_of, int64_t n, const int2* __restrict__ err,
                                        unsigned long long* __restrict__ acc) {
    unsigned long long s = 0, mx = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int2 e = err[leaf_of[i]];
        const unsigned long long w = (unsigned long long)((long long)e.y - (long long)e.x + 1);
        s += w;
        mx = mx > w ? mx : w;
    }
    s = warp_sum(s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long t = __shfl_xor_sync(0xffffffffu, mx, o);
        mx = mx > t ? mx : t;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc[0], s);
        atomicMax(&acc[1], mx);
    }
}

// Frame fields of the query descriptor, computed exactly as the build
// quantised (frame_q), so query-side cell keys match the registered ones.
__global__ void learned_desc_kernel(const double* __restrict__ fr, LearnedJob* __restrict__ d) {
    double lox, loy, sx, sy;
    frame_q(fr, lox, loy, sx, sy);
    d->lox = lox;
    d->loy = loy;
    d->hix = fr[2];
    d->hiy = fr[3];
    d->sx = sx;
    d->sy = sy;
    // a level-L cell spans 2^(32-L) grid units of 1/scale each
    const double units = ldexp(1.0, 32 - d->L);
    d->cwx = units / sx;
    d->cwy = units / sy;
}

template <class T>
int dalloc(T** p, size_t n, int64_t& bytes) {
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        set_error("cudaMalloc(%zu bytes) failed: %s", n * sizeof(T), cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? VS_E_OOM : VS_E_CUDA;
    }
    bytes += (int64_t)(n * sizeof(T));
    return VS_OK;
}

// Registrations (E), distinct cells (n_cells) and the sum over cells of
// their squared entry counts (sum_sq) of the slot boxes at grid level L, on
// scratch only: the count, emit, sort and unique-flag steps of the build.
int probe_level(cudaStream_t s, const vs_box* boxes, int64_t M, const double* frame, int L, uint32_t* cnt,
                unsigned long long* tot, unsigned long long& E, uint32_t& n_cells, unsigned long long& sum_sq) {
    VS_CUDA_TRY(cudaMemsetAsync(tot, 0, sizeof(unsigned long long), s));
    cell_count_kernel<<<grid_for(M, 256), 256, 0, s>>>(boxes, M, frame, L, cnt, tot);
    VS_CUDA_TRY(cudaMemcpyAsync(&E, tot, sizeof(E), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    n_cells = 0;
    sum_sq = 0;
    if (E == 0 || E >= 0x7fffffffull) return VS_OK;
    Scratch<uint32_t> off, keys, vals, flag, nc;
    VS_TRY(off.alloc((size_t)M, s));
    VS_TRY(keys.alloc((size_t)E, s));
    VS_TRY(vals.alloc((size_t)E, s));
    VS_TRY(flag.alloc((size_t)E, s));
    VS_TRY(nc.alloc(1, s));
    VS_TRY(exclusive_scan_u32(cnt, off.p, M, nullptr, s));
    cell_emit_kernel<<<grid_for(M, 256), 256, 0, s>>>(boxes, M, frame, L, off.p, keys.p, vals.p);
    VS_CUDA_TRY(cudaGetLastError());
    VS_TRY(radix_sort_u32_u32(keys.p, vals.p, (int64_t)E, 2 * L, s));
    cell_flag_kernel<<<grid_for((int64_t)E, 256), 256, 0, s>>>(keys.p, (int64_t)E, flag.p);
    VS_TRY(exclusive_scan_u32(flag.p, flag.p, (int64_t)E, nc.p, s));
    VS_CUDA_TRY(cudaMemsetAsync(tot, 0, sizeof(unsigned long long), s));
    cell_run_sq_kernel<<<grid_for((int64_t)E, 256), 256, 0, s>>>(keys.p, (int64_t)E, tot);
    VS_CUDA_TRY(cudaMemcpyAsync(&n_cells, nc.p, sizeof(n_cells), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaMemcpyAsync(&sum_sq, tot, sizeof(sum_sq), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    return VS_OK;
}

int train_rmi(vs_context* ctx, vs_index* idx, int steps) {
    LearnedIndex& li = idx->learned;
    cudaStream_t s = ctx->stream;
    const int64_t n = li.n_cells;
    const int anc_shift = 2 * (li.level - li.root_level);
    // ancestor-key range and quantile knots (33 keys read back)
    std::vector<uint32_t> q(33);
    for (int j = 0; j <= 32; ++j) {
        const int64_t pos = (int64_t)((double)j * (double)(n - 1) / 32.0);
        VS_CUDA_TRY(cudaMemcpyAsync(&q[j], li.cell_keys + pos, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    }
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    for (auto& v : q) v >>= anc_shift;
    const double key_lo = (double)q[0];
    const double span = (double)q[32] - key_lo;
    const double key_scale = span > 0 ? 1.0 / span : 0.0;
    // Initial root: a piecewise-linear interpolant of the key CDF through the
    // 33 quantile knots (h1_j = relu(x - c_j), W2 = I, w3_j = slope change).
    std::vector<float> P(kRmiP, 0.f);
    std::vector<double> c(33), yk(33);
    for (int j = 0; j <= 32; ++j) {
        c[j] = ((double)q[j] - key_lo) * key_scale;
        yk[j] = (double)j / 32.0;
    }
    double prev_slope = 0.0;
    for (int j = 0; j < 32; ++j) {
        const double dx = c[j + 1] - c[j];
        const double slope = dx > 1e-12 ? (yk[j + 1] - yk[j]) / dx : 0.0;
        P[kOffW1 + j] = 1.0f;
        P[kOffB1 + j] = (float)-c[j];
        P[kOffW3 + j] = (float)(slope - prev_slope);
        prev_slope = slope;
        P[kOffW2 + j * kRmiHidden + j] = 1.0f;
        P[kOffB2 + j] = 0.0f;
    }
    P[kOffB3] = 0.0f;
    const int S = (int)std::min<int64_t>(n, 16384);
    Scratch<float> dP, m1, m2, xs, ts, part, loss;
    VS_TRY(dP.alloc(kRmiP, s));
    VS_TRY(m1.alloc(kRmiP, s));
    VS_TRY(m2.alloc(kRmiP, s));
    VS_TRY(xs.alloc(S, s));
    VS_TRY(ts.alloc(S, s));
    VS_TRY(part.alloc((size_t)kTrainBlocks * kRmiP, s));
    VS_TRY(loss.alloc(1, s));
    VS_CUDA_TRY(cudaMemcpyAsync(dP.p, P.data(), kRmiP * sizeof(float), cudaMemcpyHostToDevice, s));
    VS_CUDA_TRY(cudaMemsetAsync(m1.p, 0, kRmiP * sizeof(float), s));
    VS_CUDA_TRY(cudaMemsetAsync(m2.p, 0, kRmiP * sizeof(float), s));
    rmi_samples_kernel<<<div_up(S, 256), 256, 0, s>>>(li.cell_keys, n, S, anc_shift, key_lo, key_scale, xs.p, ts.p);
    VS_CUDA_TRY(cudaGetLastError());
    for (int step = 1; step <= steps; ++step) {
        VS_CUDA_TRY(cudaMemsetAsync(loss.p, 0, sizeof(float), s));
        rmi_grad_kernel<<<kTrainBlocks, kThreads, 0, s>>>(dP.p, xs.p, ts.p, S, part.p, loss.p);
        const float lr = 2e-3f * (step < steps / 2 ? 1.0f : 0.3f);
        rmi_adam_kernel<<<div_up(kRmiP, 256), 256, 0, s>>>(dP.p, m1.p, m2.p, part.p, kTrainBlocks, step, lr);
    }
    VS_CUDA_TRY(cudaGetLastError());
    VS_CUDA_TRY(cudaMemcpyAsync(&li.rmi_final_loss, loss.p, sizeof(float), cudaMemcpyDeviceToHost, s));
    int64_t& bytes = idx->device_bytes;
    if (!li.model) VS_TRY(dalloc(&li.model, 1, bytes));
    rmi_pack_kernel<<<1, 256, 0, s>>>(dP.p, li.model, key_lo, key_scale, li.n_leaves, (int)n);
    VS_CUDA_TRY(cudaGetLastError());
    // tabulate the root over all 4^R ancestor keys
    const int64_t n_anc = 1ll << (2 * li.root_level);
    VS_TRY(dalloc(&li.root_table, (size_t)n_anc, bytes));
    rmi_table_kernel<<<grid_for(n_anc * 32, kThreads, 8), kThreads, 0, s>>>(li.model, n_anc, li.root_table);
    VS_CUDA_TRY(cudaGetLastError());
    return VS_OK;
}

int fit_leaves(vs_context* ctx, vs_index* idx) {
    LearnedIndex& li = idx->learned;
    cudaStream_t s = ctx->stream;
    const int64_t n = li.n_cells;
    const int nl = li.n_leaves;
    const int anc_shift = 2 * (li.level - li.root_level);
    int64_t& bytes = idx->device_bytes;
    VS_TRY(dalloc(&li.leaf_ab, (size_t)nl, bytes));
    VS_TRY(dalloc(&li.leaf_err, (size_t)nl, bytes));
    Scratch<uint32_t> leaf_of;
    Scratch<double> sums, cov;
    Scratch<unsigned long long> acc;
    VS_TRY(leaf_of.alloc((size_t)n, s));
    VS_TRY(sums.alloc((size_t)3 * nl, s));
    VS_TRY(cov.alloc((size_t)2 * nl, s));
    VS_TRY(acc.alloc(2, s));
    VS_CUDA_TRY(cudaMemsetAsync(sums.p, 0, 3 * nl * sizeof(double), s));
    VS_CUDA_TRY(cudaMemsetAsync(cov.p, 0, 2 * nl * sizeof(double), s));
    VS_CUDA_TRY(cudaMemsetAsync(acc.p, 0, 2 * sizeof(unsigned long long), s));
    rmi_route_kernel<<<grid_for(n, 256), 256, 0, s>>>(li.root_table, li.cell_keys, n, anc_shift, leaf_of.p);
    rmi_leaf_sums_kernel<<<grid_for(n, 256), 256, 0, s>>>(li.cell_keys, leaf_of.p, n, sums.p);
    rmi_leaf_cov_kernel<<<grid_for(n, 256), 256, 0, s>>>(li.cell_keys, leaf_of.p, n, sums.p, cov.p);
    rmi_leaf_fit_kernel<<<div_up(nl, 256), 256, 0, s>>>(sums.p, cov.p, nl, li.leaf_ab, li.leaf_err);
    rmi_err_kernel<<<grid_for(n, 256), 256, 0, s>>>(li.cell_keys, leaf_of.p, n, li.leaf_ab, li.leaf_err);
    rmi_window_stats_kernel<<<grid_for(n, 256), 256, 0, s>>>(leaf_of.p, n, li.leaf_err, acc.p);
    VS_TRY(dalloc(&li.leaves, (size_t)nl, bytes));
    pack_leaves_kernel<<<div_up(nl, 256), 256, 0, s>>>(nl, li.leaf_ab, li.leaf_err, li.leaves);
    VS_CUDA_TRY(cudaGetLastError());
    unsigned long long h[2];
    VS_CUDA_TRY(cudaMemcpyAsync(h, acc.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    li.mean_window = n > 0 ? (float)((double)h[0] / (double)n) : 0.f;
    li.max_window = (int32_t)h[1];
    return VS_OK;
}

}  // namespace

void free_learned_index(vs_index* idx) {
    LearnedIndex& li = idx->learned;
    cudaFree(li.cell_keys);
    cudaFree(li.cell_start);
    cudaFree(li.entries);
    cudaFree(li.occ);
    cudaFree(li.model);
    cudaFree(li.root_table);
    cudaFree(li.leaf_ab);
    cudaFree(li.leaf_err);
    cudaFree(li.origin);
    cudaFree(li.err32);
    cudaFree(li.c01);
    cudaFree(li.ring_box32);
    cudaFree(li.ib32);
    cudaFree(li.xy32);
    cudaFree(li.leaves);
    cudaFree(li.recs);
    cudaFree(li.desc);
    li = LearnedIndex{};
}

static int auto_leaves(int64_t n_keys) {
    int64_t l = 4096;
    while (l < 65536 && l * 64 < n_keys) l *= 2;
    return (int)std::min<int64_t>(l, 65535);
}

int build_learned_index(vs_context* ctx, vs_index* idx, const vs_index_options* opts) {
    LearnedIndex& li = idx->learned;
    cudaStream_t s = ctx->stream;
    const int64_t M = idx->n_geoms;
    int64_t& bytes = idx->device_bytes;
    if (M == 0 || !(idx->h_frame[0] <= idx->h_frame[2])) return VS_OK;  // nothing to index: joins use the R-tree
    const vs_box* boxes = idx->nodes;  // level 0 = slot boxes
    // 1. grid level
    int L = opts ? opts->cell_level : 0;
    const bool auto_level = L <= 0;
    if (L <= 0) {
        Scratch<double> acc;
        VS_TRY(acc.alloc(2, s));
        VS_CUDA_TRY(cudaMemsetAsync(acc.p, 0, 2 * sizeof(double), s));
        box_side_kernel<<<grid_for(M, 256), 256, 0, s>>>(boxes, M, acc.p);
        double h[2];
        VS_CUDA_TRY(cudaMemcpyAsync(h, acc.p, sizeof(h), cudaMemcpyDeviceToHost, s));
        VS_CUDA_TRY(cudaStreamSynchronize(s));
        const double mean_side = h[1] > 0 ? h[0] / h[1] : 1.0;
        const double extent = std::max(idx->h_frame[2] - idx->h_frame[0], idx->h_frame[3] - idx->h_frame[1]);
        L = mean_side > 0 ? (int)std::lround(std::log2(extent / mean_side)) : 15;
    }
    L = std::max(1, std::min(L, 15));
    // 2. registrations; coarsen while the entry count is out of proportion
    Scratch<uint32_t> cnt;
    Scratch<unsigned long long> tot;
    VS_TRY(cnt.alloc((size_t)M, s));
    VS_TRY(tot.alloc(1, s));
    unsigned long long E = 0;
    for (;;) {
        VS_CUDA_TRY(cudaMemsetAsync(tot.p, 0, sizeof(unsigned long long), s));
        cell_count_kernel<<<grid_for(M, 256), 256, 0, s>>>(boxes, M, idx->frame, L, cnt.p, tot.p);
        VS_CUDA_TRY(cudaMemcpyAsync(&E, tot.p, sizeof(E), cudaMemcpyDeviceToHost, s));
        VS_CUDA_TRY(cudaStreamSynchronize(s));
        if (L <= 1 || E <= (unsigned long long)(16 * M + (1 << 20))) break;
        --L;
    }
    // An automatic level is then refined (at most 3 levels) while the mean
    // list length seen from an entry (sum over cells of count^2 / E) is above
    // 2.5 and the finer level's registrations stay within the budget.  The
    // refine tests every entry of a point's cell, and query points crowd
    // where the boxes crowd, so the lists that matter are the long ones of
    // the dense cells, which the plain mean E / n_cells hides under the many
    // one-entry cells around them.  (A box side mean is also pulled up by a
    // few wide boxes, such as multipolygons with spread parts, which leaves
    // the cells too coarse for the rest.)
    if (auto_level && E > 0) {
        uint32_t nc = 0;
        unsigned long long sq = 0;
        VS_TRY(probe_level(s, boxes, M, idx->frame, L, cnt.p, tot.p, E, nc, sq));
        const int l_max = std::min(15, L + 3);
        while (L < l_max && nc > 0 && (double)sq > 2.5 * (double)E) {
            unsigned long long e1 = 0, sq1 = 0;
            uint32_t nc1 = 0;
            VS_TRY(probe_level(s, boxes, M, idx->frame, L + 1, cnt.p, tot.p, e1, nc1, sq1));
            if (e1 > (unsigned long long)(16 * M + (1 << 20)) || e1 >= 0x7fffffffull) break;
            ++L;
            E = e1;
            nc = nc1;
            sq = sq1;
        }
        // the counts of the chosen level, for the emit below
        VS_CUDA_TRY(cudaMemsetAsync(tot.p, 0, sizeof(unsigned long long), s));
        cell_count_kernel<<<grid_for(M, 256), 256, 0, s>>>(boxes, M, idx->frame, L, cnt.p, tot.p);
        VS_CUDA_TRY(cudaMemcpyAsync(&E, tot.p, sizeof(E), cudaMemcpyDeviceToHost, s));
        VS_CUDA_TRY(cudaStreamSynchronize(s));
    }
    if (E >= 0x7fffffffull) {
        set_error("learned index: too many cell registrations (%llu)", E);
        return VS_E_ARG;
    }
    li.level = L;
    li.n_entries = (int64_t)E;
    Scratch<uint32_t> off, keys, flag;
    VS_TRY(off.alloc((size_t)M, s));
    VS_TRY(keys.alloc((size_t)E, s));
    VS_TRY(flag.alloc((size_t)E, s));
    VS_TRY(dalloc(&li.entries, (size_t)E, bytes));
    VS_TRY(exclusive_scan_u32(cnt.p, off.p, M, nullptr, s));
    cell_emit_kernel<<<grid_for(M, 256), 256, 0, s>>>(boxes, M, idx->frame, L, off.p, keys.p, li.entries);
    VS_CUDA_TRY(cudaGetLastError());
    VS_TRY(radix_sort_u32_u32(keys.p, li.entries, (int64_t)E, 2 * L, s));
    // 3. unique cells + CSR
    Scratch<uint32_t> ncell;
    VS_TRY(ncell.alloc(1, s));
    cell_flag_kernel<<<grid_for(E, 256), 256, 0, s>>>(keys.p, (int64_t)E, flag.p);
    VS_TRY(exclusive_scan_u32(flag.p, flag.p, (int64_t)E, ncell.p, s));
    uint32_t nc = 0;
    VS_CUDA_TRY(cudaMemcpyAsync(&nc, ncell.p, sizeof(nc), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    li.n_cells = nc;
    VS_TRY(dalloc(&li.cell_keys, (size_t)nc, bytes));
    VS_TRY(dalloc(&li.cell_start, (size_t)nc + 1, bytes));
    cell_compact_kernel<<<grid_for(E, 256), 256, 0, s>>>(keys.p, flag.p, (int64_t)E, li.cell_keys, li.cell_start);
    const uint32_t Eu = (uint32_t)E;
    VS_CUDA_TRY(cudaMemcpyAsync(li.cell_start + nc, &Eu, sizeof(Eu), cudaMemcpyHostToDevice, s));
    // 4. occupancy bitmap
#ifndef VS_OCC_MAX_LEVEL
#define VS_OCC_MAX_LEVEL 13  // 8 MB at level 13, L2-resident
#endif
    li.occ_level = std::min(L, VS_OCC_MAX_LEVEL);
    const int64_t occ_bits = 1ll << (2 * li.occ_level);
    VS_TRY(dalloc(&li.occ, (size_t)((occ_bits + 31) / 32), bytes));
    VS_CUDA_TRY(cudaMemsetAsync(li.occ, 0, (size_t)((occ_bits + 31) / 32) * sizeof(uint32_t), s));
    occ_kernel<<<grid_for(nc, 256), 256, 0, s>>>(li.cell_keys, nc, 2 * (L - li.occ_level), li.occ);
    VS_CUDA_TRY(cudaGetLastError());
    // 5. RMI (root tabulated over level-R ancestors)
    // leaves: 4096, or one per 64 stored keys (to the next power of two, at
    // most 65535, the root table's 16-bit leaf ids) when there are more than
    // 256k keys, so that a leaf's error window stays a few dozen keys wide
    li.n_leaves = (opts && opts->rmi_leaves > 0) ? std::min(opts->rmi_leaves, 65535) : auto_leaves((int64_t)nc);
    li.root_level = std::min(L, 10);
    const int steps = (opts && opts->rmi_train_steps > 0) ? opts->rmi_train_steps : 300;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    int st = train_rmi(ctx, idx, steps);
    if (st == VS_OK) st = fit_leaves(ctx, idx);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&li.rmi_train_ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    VS_TRY(st);
    // 6. the query descriptor (one job, cells numbered from 0); its frame
    // fields and cell widths are computed on the device
    LearnedJob d{};
    d.L = L;
    d.occ_shift = 2 * (L - li.occ_level);
    d.root_shift = 2 * (L - li.root_level);
    d.cell_base = 0;
    d.n_cells = li.n_cells;
    d.occ = li.occ;
    d.root_table = li.root_table;
    d.leaves = li.leaves;
    d.cell_keys = li.cell_keys;
    d.cell_start = li.cell_start;
    d.xy = idx->xy;
    d.item_geom = idx->item_geom;
    d.geom_off = idx->geom_off;
    d.part_off = idx->part_off;
    d.ring_off = idx->ring_off;
    d.boxes = idx->nodes;
    d.rings = idx->ring_index();
    // 7. FP32 slot-relative vertices, per-slot ring ranges, per-entry records
    VS_TRY(dalloc(&li.origin, (size_t)M, bytes));
    VS_TRY(dalloc(&li.err32, (size_t)M, bytes));
    VS_TRY(dalloc(&li.c01, (size_t)M, bytes));
    VS_TRY(dalloc(&li.ring_box32, (size_t)std::max<int32_t>(idx->n_rings, 1), bytes));
    VS_TRY(dalloc(&li.ib32, (size_t)M, bytes));
    VS_TRY(dalloc(&li.xy32, (size_t)std::max<int64_t>(idx->n_coords, 1), bytes));
    VS_TRY(dalloc(&li.recs, (size_t)E, bytes));
    VS_TRY(dalloc(&li.desc, 1, bytes));
    d.recs = li.recs;
    d.c01 = li.c01;
    d.ring_box32 = li.ring_box32;
    d.ib32 = li.ib32;
    d.xy32 = li.xy32;
    VS_CUDA_TRY(cudaMemcpyAsync(li.desc, &d, sizeof(d), cudaMemcpyHostToDevice, s));
    learned_desc_kernel<<<1, 1, 0, s>>>(idx->frame, li.desc);
    VS_CUDA_TRY(cudaGetLastError());
    split_copy_kernel<<<grid_for(M * 32, 256), 256, 0, s>>>(boxes, M, idx->geom_off, idx->part_off, idx->ring_off,
                                                            idx->xy, li.origin, li.err32, li.xy32);
    VS_CUDA_TRY(cudaGetLastError());
    Scratch<unsigned> n_extra;
    VS_TRY(n_extra.alloc(1, s));
    VS_CUDA_TRY(cudaMemsetAsync(n_extra.p, 0, sizeof(unsigned), s));
    slot_c01_kernel<<<grid_for(M, 256), 256, 0, s>>>(M, idx->geom_off, idx->part_off, idx->ring_off, idx->ring_bin,
                                                     li.c01, n_extra.p);
    VS_CUDA_TRY(cudaGetLastError());
    interior_box_kernel<<<grid_for(M * 32, 256), 256, 0, s>>>(boxes, M, idx->geom_off, idx->part_off, idx->ring_off,
                                                              idx->xy, idx->ring_index(), li.origin, li.ib32);
    VS_CUDA_TRY(cudaGetLastError());
    if (idx->n_rings > 0) {
        ring_box_kernel<<<grid_for((int64_t)idx->n_rings * 32, 256), 256, 0, s>>>(idx->ring_off, idx->n_rings, li.xy32,
                                                                                 li.ring_box32);
        VS_CUDA_TRY(cudaGetLastError());
    }
    Scratch<unsigned> bad;
    VS_TRY(bad.alloc(1, s));
    VS_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(unsigned), s));
    entry_recs_kernel<<<grid_for(E, 256), 256, 0, s>>>((int64_t)E, keys.p, li.entries, li.desc, boxes, li.origin,
                                                       li.err32, li.ib32, li.recs, bad.p);
    VS_CUDA_TRY(cudaGetLastError());
    unsigned h_bad = 0, h_extra = 0;
    VS_CUDA_TRY(cudaMemcpyAsync(&h_bad, bad.p, sizeof(h_bad), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaMemcpyAsync(&h_extra, n_extra.p, sizeof(h_extra), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaMemcpyAsync(&li.h_desc, li.desc, sizeof(LearnedJob), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    idx->n_split_binned_rings += (int64_t)h_extra;  // single rings the split walk also takes binned
    if (h_bad) {
        set_error("learned index: a cell key did not decode to its cell");
        return VS_E_CUDA;
    }
    idx->has_learned = true;
    return VS_OK;
}

}  // namespace vs
