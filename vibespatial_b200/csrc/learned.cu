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
// Query, three passes over the points (a counting sort keyed by the learned
// index's own positions, so no general sort is needed):
//   map      input order: level-L cell key -> occupancy bit -> root table ->
//            leaf model -> binary search inside the leaf's error window ->
//            cell index (or none); warp-aggregated atomics on the per-cell
//            counts return each point's rank within its cell
//   scatter  after an exclusive scan of the counts, each matched point
//            writes one aligned 32-byte record (x, y, row, cell) at
//            start[cell] + rank; points in empty cells drop out
//   join     a warp takes 32 consecutive records, which share a polygon list
//            except at cell boundaries, so the lanes read each polygon's data
//            together (broadcast); each candidate is box-filtered in FP32
//            (rounded outward) and refined with the FP32 crossing test on
//            tile-relative coordinates; only edges whose FP32 decision lies
//            within the rounding-error bound are re-decided in FP64, and a
//            pair the FP64 filter cannot certify is deferred to the exact
//            pass.
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
                                  float4* __restrict__ box32, float* __restrict__ err32, float2* __restrict__ xy32) {
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
            if (ok) {
                const double a = b.minx - ox, c = b.miny - oy, d = b.maxx - ox, e = b.maxy - oy;
                box32[s] = make_float4(__double2float_rd(a - fabs(a) * u64), __double2float_rd(c - fabs(c) * u64),
                                       __double2float_ru(d + fabs(d) * u64), __double2float_ru(e + fabs(e) * u64));
            } else {
                box32[s] = make_float4(INFINITY, INFINITY, -INFINITY, -INFINITY);
            }
        }
    }
}

__global__ void pack_slots_kernel(int64_t M, const double2* __restrict__ origin, const float4* __restrict__ box32,
                                  const float* __restrict__ err32, const int32_t* __restrict__ item_geom,
                                  const int32_t* __restrict__ geom_off, const int32_t* __restrict__ part_off,
                                  const int32_t* __restrict__ ring_off, SlotRecord* __restrict__ out) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < M; s += (int64_t)gridDim.x * blockDim.x) {
        SlotRecord r;
        r.ox = origin[s].x;
        r.oy = origin[s].y;
        r.box = box32[s];
        r.err = err32[s];
        r.slot = (int32_t)s;
        const int32_t p0 = geom_off[s], p1 = geom_off[s + 1];
        r.c0 = -1;
        r.c1 = -1;
        if (p1 - p0 == 1 && part_off[p0 + 1] - part_off[p0] == 1) {
            r.c0 = ring_off[part_off[p0]];
            r.c1 = ring_off[part_off[p0] + 1];
        }
        out[s] = r;
    }
}

// One record per (cell, polygon) entry, in cell order.
__global__ void entry_recs_kernel(int64_t E, const uint32_t* __restrict__ entries,
                                  const SlotRecord* __restrict__ slots, SlotRecord* __restrict__ out) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < E; e += (int64_t)gridDim.x * blockDim.x)
        out[e] = slots[entries[e]];
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

// ----------------------------------------------------------------- query ---
// One grouped point: a full 32-byte sector, so the scatter writes whole
// sectors (no read-modify-write of partially written ones).
// A matched query point as the map pass leaves it: coordinates, row, cell
// index and its rank among the cell's points.
struct __align__(32) StagedPoint {
    double x, y;
    int32_t row;
    int32_t cell;
    uint32_t rank;
    int32_t pad;
};

// The map pass appends matched points to kStripes regions of the staging
// array, region s taking the packets p with p % kStripes == s, so each
// region's append counter sees 1/kStripes of the atomics and a region never
// holds more than 32 * ceil(packets / kStripes) points.
constexpr int kStripes = 2048;

// A query point in cell order, with its cell's candidate range
// [lo, lo + len) of the per-entry records.
struct __align__(32) GroupedPoint {
    double x, y;
    int32_t row;
    uint32_t lo;
    uint32_t len;
    int32_t pad;
};

struct LearnedArgs {
    const double* px;
    const double* py;
    const uint8_t* pvalid;
    int64_t n;
    const double* frame;
    int L;
    int occ_shift;             // cell key >> occ_shift = occupancy bit
    int root_shift;            // cell key >> root_shift = root-table index
    const uint32_t* occ;
    const uint16_t* root_table;
    const uint32_t* cell_keys;
    const uint32_t* cell_start;
    const uint32_t* entries;
    int64_t n_cells;
    const RmiLeaf* leaves;
    const SlotRecord* recs;          // [n_entries] per-entry slot records
    const vs_box* boxes;       // FP64 slot boxes (R-tree level 0)
    const double2* origin;
    const float4* box32;
    const float* err32;
    const float2* xy32;
    const double2* xy;
    const int32_t* item_geom;
    const int32_t* geom_off;
    const int32_t* part_off;
    const int32_t* ring_off;
    int accept_mask;
    PairSink sink;
    DeferSink defer;
    unsigned long long* counters;
    // grouping scratch (per join)
    StagedPoint* staged;       // [kStripes * stripe_cap] matched points, striped
    uint32_t* stripe_count;    // [kStripes] points appended to each region
    int64_t stripe_cap;        // points one region can hold
    uint32_t* cell_count;      // [n_cells] counts, then (after the scan) start offsets
    GroupedPoint* grouped;     // [n_grouped] points grouped by cell
    const uint32_t* n_grouped;
    unsigned long long* work;  // refine work queue (grouped points handed out)
};

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

__device__ __forceinline__ int ring_location_split(double px, double py, float qx, float qy, float t,
                                                   const float2* __restrict__ xy32, const double2* __restrict__ xy,
                                                   int start, int end, unsigned& n32, unsigned& n64) {
    if (end - start < 2) return LOC_OUTSIDE;
    bool inside = false;
    float2 a = xy32[end - 1];
    int ia = end - 1;
    for (int i = start; i < end; ++i) {
        const float2 b = xy32[i];
        if (edge_step_fp32(a.x, a.y, b.x, b.y, qx, qy, t, inside)) {
            ++n32;
        } else {
            ++n64;
            const double2 A = xy[ia], B = xy[i];
            const int r = edge_step_filtered(A.x, A.y, B.x, B.y, px, py, inside);
            if (r == 1) return LOC_BOUNDARY;
            if (r == 2) return LOC_UNDECIDED;
        }
        a = b;
        ia = i;
    }
    return inside ? LOC_INTERIOR : LOC_OUTSIDE;
}

__device__ __forceinline__ int geometry_location_split(double px, double py, float qx, float qy, float t,
                                                       const LearnedArgs& a, int g, unsigned& n32, unsigned& n64) {
    const int p0 = a.geom_off[g], p1 = a.geom_off[g + 1];
    for (int part = p0; part < p1; ++part) {
        bool inside = false;
        const int r0 = a.part_off[part], r1 = a.part_off[part + 1];
        for (int ring = r0; ring < r1; ++ring) {
            const int k = ring_location_split(px, py, qx, qy, t, a.xy32, a.xy, a.ring_off[ring], a.ring_off[ring + 1],
                                              n32, n64);
            if (k == LOC_BOUNDARY || k == LOC_UNDECIDED) return k;
            if (k == LOC_INTERIOR) inside = !inside;
        }
        if (inside) return LOC_INTERIOR;
    }
    return LOC_OUTSIDE;
}

// Exact lookup of a point's cell in the learned index: level-L cell key ->
// occupancy bit -> root table -> leaf model -> binary search inside the
// leaf's error window.  Returns the cell's index, or -1 when no stored cell
// matches (no polygon box overlaps the point's cell).
__device__ __forceinline__ int learned_lookup(const LearnedArgs& a, double x, double y, double lox, double loy,
                                              double sx, double sy, const uint16_t* lut,
                                              unsigned long long& n_wide) {
    const uint32_t cell = hilbert_key_lut(quantize(x, lox, sx), quantize(y, loy, sy), a.L, lut);
    const uint32_t ob = cell >> a.occ_shift;
    if (!((a.occ[ob >> 5] >> (ob & 31)) & 1u)) return -1;
    const RmiLeaf lf = a.leaves[a.root_table[cell >> a.root_shift]];
    if (lf.lo > lf.hi) return -1;  // no stored key routes to this leaf
    const long long pred = rmi_predict(make_double2(lf.a, lf.b), cell);
    long long l0 = pred + lf.lo, h0 = pred + lf.hi + 1;  // search [l0, h0)
    l0 = l0 < 0 ? 0 : l0;
    h0 = h0 > a.n_cells ? a.n_cells : h0;
    if (h0 - l0 > 256) ++n_wide;
    const long long h1 = h0;
    while (l0 < h0) {
        const long long mid = (l0 + h0) >> 1;
        if (a.cell_keys[mid] < cell) l0 = mid + 1;
        else h0 = mid;
    }
    return (l0 < h1 && a.cell_keys[l0] == cell) ? (int)l0 : -1;
}

// Pass 1 (map), points in input order: each point's cell and its rank among
// the cell's points (warp-aggregated atomics on the per-cell counts); the
// matched points are appended to the staging regions.
__global__ void __launch_bounds__(kThreads, 8) learned_map_kernel(const LearnedArgs a) {
    __shared__ uint16_t s_lut[kHilbertLutSize];
    hilbert_lut_init(s_lut);
    __syncthreads();
    double lox, loy, sx, sy;
    frame_q(a.frame, lox, loy, sx, sy);
    const double fx1 = a.frame[2], fy1 = a.frame[3];
    unsigned long long n_wide = 0;
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    // Warp-uniform loop: the whole warp reaches the match and shuffle together.
    for (int64_t b0 = gw * 32; b0 < a.n; b0 += nw * 32) {
        const int64_t i = b0 + lane;
        int c = -1;
        double x = 0.0, y = 0.0;
        if (i < a.n) {
            x = a.px[i];
            y = a.py[i];
            if ((a.pvalid == nullptr || a.pvalid[i]) && x >= lox && x <= fx1 && y >= loy && y <= fy1)
                c = learned_lookup(a, x, y, lox, loy, sx, sy, s_lut, n_wide);
        }
        const unsigned lt = (1u << lane) - 1u;
        const unsigned peers = __match_any_sync(0xffffffffu, c);
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (c >= 0 && lane == leader) base = atomicAdd(&a.cell_count[c], (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        // append the matched points of this packet to its stripe region
        const unsigned mm = __ballot_sync(0xffffffffu, c >= 0);
        if (mm) {
            const int64_t stripe = (b0 >> 5) % kStripes;
            uint32_t sb = 0;
            if (lane == 0) sb = atomicAdd(&a.stripe_count[stripe], (uint32_t)__popc(mm));
            sb = __shfl_sync(0xffffffffu, sb, 0);
            if (c >= 0) {
                StagedPoint p;
                p.x = x;
                p.y = y;
                p.row = (int32_t)i;
                p.cell = c;
                p.rank = base + __popc(peers & lt);
                p.pad = 0;
                a.staged[stripe * a.stripe_cap + sb + __popc(mm & lt)] = p;
            }
        }
    }
    add_counter(a.counters, 6, n_wide);
}

// Pass 2 (scatter): after the exclusive scan of the counts, every staged
// point writes one aligned 32-byte record at start[cell] + rank, carrying its
// cell's candidate range.  A block walks whole stripe regions (coalesced
// reads, every lane busy); each thread keeps kScatterUnroll records in flight.
#ifndef VS_SCATTER_UNROLL
#define VS_SCATTER_UNROLL 4
#endif
constexpr int kScatterUnroll = VS_SCATTER_UNROLL;

__global__ void __launch_bounds__(kThreads) learned_scatter_kernel(const LearnedArgs a) {
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
                    const int c = p[u].cell;
                    g[u].x = p[u].x;
                    g[u].y = p[u].y;
                    g[u].row = p[u].row;
                    g[u].lo = a.cell_start[c];
                    g[u].len = a.cell_start[c + 1] - g[u].lo;
                    g[u].pad = 0;
                    pos[u] = a.cell_count[c] + p[u].rank;
                }
            }
#pragma unroll
            for (int u = 0; u < kScatterUnroll; ++u)
                if (k0 + u * blockDim.x < cnt) a.grouped[pos[u]] = g[u];
        }
    }
}

// Pass 3 (join): a warp takes 32 consecutive grouped points, which share a
// cell (and so a polygon list: broadcast reads) except at cell boundaries.
#ifndef VS_JOIN_MIN_BLOCKS
#define VS_JOIN_MIN_BLOCKS 5
#endif
#ifndef VS_JOIN_GRAB
#define VS_JOIN_GRAB 32
#endif
constexpr int64_t kJoinGrab = VS_JOIN_GRAB;  // grouped points per work-queue grab (multiple of 32)
__global__ void __launch_bounds__(kThreads, VS_JOIN_MIN_BLOCKS) learned_join_kernel(const LearnedArgs a) {
    __shared__ int2 s_buf[kThreads / 32][kWarpBuf];
    __shared__ unsigned s_cnt[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_cnt[warp] = 0;
    __syncwarp();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    const int64_t n = (int64_t)*a.n_grouped;
    unsigned long long n_cand = 0;
    unsigned n32 = 0, n64 = 0;
    for (;;) {
        const int64_t b0 = warp_grab(a.work, kJoinGrab);
        if (b0 >= n) break;
        const int64_t e0 = b0 + kJoinGrab < n ? b0 + kJoinGrab : n;
        for (int64_t base = b0; base < e0; base += 32) {
            const int64_t j = base + lane;
            GroupedPoint g{0.0, 0.0, 0, 0, 0, 0};
            if (j < e0) g = a.grouped[j];
            const double x = g.x, y = g.y;
            const uint32_t lo = g.lo, len = g.len;
            // Candidate loop with one trip count for the whole warp (the longest
            // list among its lanes; in grouped order the lanes mostly share one).
            uint32_t maxlen = len;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const uint32_t t = __shfl_xor_sync(0xffffffffu, maxlen, o);
                maxlen = t > maxlen ? t : maxlen;
            }
            for (uint32_t k = 0; k < maxlen; ++k) {
                bool want = false;
                int32_t right = 0;
                if (k < len) {
                    const SlotRecord r = a.recs[lo + k];
                    const int slot = r.slot;
                    const float qx = __double2float_rn(x - r.ox), qy = __double2float_rn(y - r.oy);
                    const float dp = __fmaf_ru(fmaxf(fabsf(qx), fabsf(qy)), 6.1e-8f, 1e-37f);
                    // FP32 box filter (rounded outward: never rejects a point of the box)
                    if (!(__fadd_ru(qx, dp) < r.box.x || __fsub_rd(qx, dp) > r.box.z || __fadd_ru(qy, dp) < r.box.y ||
                          __fsub_rd(qy, dp) > r.box.w)) {
                        bool cand = true;
                        int loc = 0;
                        if (a.accept_mask) {
                            // The exact location rejects points outside the box by itself.
                            const float t = __fmul_ru(__fadd_ru(r.err, dp), 1.0001f);
                            loc = r.c0 >= 0 ? ring_location_split(x, y, qx, qy, t, a.xy32, a.xy, r.c0, r.c1, n32, n64)
                                            : geometry_location_split(x, y, qx, qy, t, a, slot, n32, n64);
                        } else {
                            // Box candidates only: decide the box exactly in FP64.
                            const vs_box bb = a.boxes[slot];
                            cand = x >= bb.minx && x <= bb.maxx && y >= bb.miny && y <= bb.maxy;
                        }
                        if (cand) {
                            ++n_cand;
                            if (loc == LOC_UNDECIDED) {
                                defer(a.defer, g.row, slot);
                            } else if (!a.accept_mask || ((a.accept_mask >> loc) & 1)) {
                                want = true;
                                right = a.item_geom[slot];
                            }
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
    add_counter(a.counters, 2, n32);
    add_counter(a.counters, 3, n64);
}

// Pass 3 with candidate compaction (predicates with a location test): the
// warp walks its grouped points' candidate lists, and every (point,
// candidate) pair that passes the FP32 box filter is appended to a warp-local
// queue in shared memory.  Each time 32 pairs are queued, every lane refines
// one of them.  So the ring walks, which dominate, run with all lanes busy
// instead of only the lanes whose point lies in the current candidate's box.
// Neighbouring queue entries mostly share a polygon, so vertex reads stay
// broadcasts.
struct QueuedPair {
    double x, y;
    int32_t row;
    uint32_t rec;  // index into the per-entry records
};
constexpr int kQueue = 64;  // >= 31 left over + 32 appended in one step

__device__ __forceinline__ void refine_queued(const LearnedArgs& a, const WarpOut& out, const QueuedPair* q, int nq,
                                              int lane, unsigned& n32, unsigned& n64) {
    bool want = false;
    int32_t row = 0, right = 0;
    if (lane < nq) {
        const QueuedPair jb = q[lane];
        row = jb.row;
        const SlotRecord r = a.recs[jb.rec];
        const float qx = __double2float_rn(jb.x - r.ox), qy = __double2float_rn(jb.y - r.oy);
        const float dp = __fmaf_ru(fmaxf(fabsf(qx), fabsf(qy)), 6.1e-8f, 1e-37f);
        const float t = __fmul_ru(__fadd_ru(r.err, dp), 1.0001f);
        const int loc = r.c0 >= 0 ? ring_location_split(jb.x, jb.y, qx, qy, t, a.xy32, a.xy, r.c0, r.c1, n32, n64)
                                  : geometry_location_split(jb.x, jb.y, qx, qy, t, a, r.slot, n32, n64);
        if (loc == LOC_UNDECIDED) {
            defer(a.defer, jb.row, r.slot);
        } else if ((a.accept_mask >> loc) & 1) {
            want = true;
            right = a.item_geom[r.slot];
        }
    }
    wemit_sync(out, a.sink, want, row, right);
}

__global__ void __launch_bounds__(kThreads, VS_JOIN_MIN_BLOCKS) learned_refine_kernel(const LearnedArgs a) {
    __shared__ int2 s_buf[kThreads / 32][kWarpBuf];
    __shared__ unsigned s_cnt[kThreads / 32];
    __shared__ QueuedPair s_q[kThreads / 32][kQueue];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_cnt[warp] = 0;
    __syncwarp();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    QueuedPair* q = s_q[warp];
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
            for (uint32_t k = 0; k < maxlen; ++k) {
                bool inbox = false;
                if (k < g.len) {
                    const SlotRecord* rp = a.recs + g.lo + k;
                    const double2 o = *reinterpret_cast<const double2*>(&rp->ox);
                    const float4 bx = rp->box;
                    const float qx = __double2float_rn(g.x - o.x), qy = __double2float_rn(g.y - o.y);
                    const float dp = __fmaf_ru(fmaxf(fabsf(qx), fabsf(qy)), 6.1e-8f, 1e-37f);
                    // FP32 box filter (rounded outward: never rejects a point of the box)
                    inbox = !(__fadd_ru(qx, dp) < bx.x || __fsub_rd(qx, dp) > bx.z || __fadd_ru(qy, dp) < bx.y ||
                              __fsub_rd(qy, dp) > bx.w);
                }
                const unsigned m = __ballot_sync(0xffffffffu, inbox);
                if (inbox) {
                    QueuedPair& e = q[nq + __popc(m & lt)];
                    e.x = g.x;
                    e.y = g.y;
                    e.row = g.row;
                    e.rec = g.lo + k;
                    ++n_cand;
                }
                nq += __popc(m);
                __syncwarp();
                if (nq >= 32) {
                    refine_queued(a, out, q, 32, lane, n32, n64);
                    __syncwarp();
                    if (lane < nq - 32) q[lane] = q[32 + lane];
                    nq -= 32;
                    __syncwarp();
                }
            }
            wflush(out, a.sink, false);
        }
    }
    if (nq > 0) refine_queued(a, out, q, nq, lane, n32, n64);
    wflush(out, a.sink, true);
    add_counter(a.counters, 5, n_cand);
    add_counter(a.counters, 2, n32);
    add_counter(a.counters, 3, n64);
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
    cudaFree(li.box32);
    cudaFree(li.err32);
    cudaFree(li.xy32);
    cudaFree(li.leaves);
    cudaFree(li.recs);
    li = LearnedIndex{};
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
    li.occ_level = std::min(L, 11);
    const int64_t occ_bits = 1ll << (2 * li.occ_level);
    VS_TRY(dalloc(&li.occ, (size_t)((occ_bits + 31) / 32), bytes));
    VS_CUDA_TRY(cudaMemsetAsync(li.occ, 0, (size_t)((occ_bits + 31) / 32) * sizeof(uint32_t), s));
    occ_kernel<<<grid_for(nc, 256), 256, 0, s>>>(li.cell_keys, nc, 2 * (L - li.occ_level), li.occ);
    VS_CUDA_TRY(cudaGetLastError());
    // 5. RMI (root tabulated over level-R ancestors)
    li.n_leaves = (opts && opts->rmi_leaves > 0) ? std::min(opts->rmi_leaves, 65535) : 4096;
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
    // 6. FP32 tile-relative copies
    VS_TRY(dalloc(&li.origin, (size_t)M, bytes));
    VS_TRY(dalloc(&li.box32, (size_t)M, bytes));
    VS_TRY(dalloc(&li.err32, (size_t)M, bytes));
    VS_TRY(dalloc(&li.xy32, (size_t)std::max<int64_t>(idx->n_coords, 1), bytes));
    split_copy_kernel<<<grid_for(M * 32, 256), 256, 0, s>>>(boxes, M, idx->geom_off, idx->part_off, idx->ring_off,
                                                            idx->xy, li.origin, li.box32, li.err32, li.xy32);
    VS_CUDA_TRY(cudaGetLastError());
    Scratch<SlotRecord> slots;
    VS_TRY(slots.alloc((size_t)M, s));
    VS_TRY(dalloc(&li.recs, (size_t)E, bytes));
    pack_slots_kernel<<<grid_for(M, 256), 256, 0, s>>>(M, li.origin, li.box32, li.err32, idx->item_geom, idx->geom_off,
                                                       idx->part_off, idx->ring_off, slots.p);
    VS_CUDA_TRY(cudaGetLastError());
    entry_recs_kernel<<<grid_for(E, 256), 256, 0, s>>>((int64_t)E, li.entries, slots.p, li.recs);
    VS_CUDA_TRY(cudaGetLastError());
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    idx->has_learned = true;
    return VS_OK;
}

int launch_learned_join(vs_context* ctx, const vs_index* idx, const vs_points* pts, int accept_mask, int32_t* d_left,
                        int32_t* d_right, int64_t capacity, const DeferSink& dsink) {
    const LearnedIndex& li = idx->learned;
    cudaStream_t s = ctx->stream;
    const int64_t n = pts->n;
    const int64_t packets = (n + 31) / 32;
    const int64_t stripe_cap = 32 * ((packets + kStripes - 1) / kStripes);
    Scratch<StagedPoint> staged;
    Scratch<uint32_t> cell_count, n_grouped, stripe_count;
    Scratch<GroupedPoint> grouped;
    VS_TRY(staged.alloc((size_t)(kStripes * stripe_cap), s));
    VS_TRY(grouped.alloc((size_t)n, s));
    VS_TRY(cell_count.alloc((size_t)li.n_cells, s));
    VS_TRY(n_grouped.alloc(1, s));
    VS_TRY(stripe_count.alloc((size_t)kStripes, s));
    VS_CUDA_TRY(cudaMemsetAsync(cell_count.p, 0, (size_t)li.n_cells * sizeof(uint32_t), s));
    VS_CUDA_TRY(cudaMemsetAsync(stripe_count.p, 0, (size_t)kStripes * sizeof(uint32_t), s));
    LearnedArgs a{};
    a.px = pts->d_x;
    a.py = pts->d_y;
    a.pvalid = pts->d_valid;
    a.n = n;
    a.frame = idx->frame;
    a.L = li.level;
    a.occ_shift = 2 * (li.level - li.occ_level);
    a.root_shift = 2 * (li.level - li.root_level);
    a.occ = li.occ;
    a.root_table = li.root_table;
    a.cell_keys = li.cell_keys;
    a.cell_start = li.cell_start;
    a.entries = li.entries;
    a.n_cells = li.n_cells;
    a.leaves = li.leaves;
    a.recs = li.recs;
    a.boxes = idx->nodes;
    a.origin = li.origin;
    a.box32 = li.box32;
    a.err32 = li.err32;
    a.xy32 = li.xy32;
    a.xy = idx->xy;
    a.item_geom = idx->item_geom;
    a.geom_off = idx->geom_off;
    a.part_off = idx->part_off;
    a.ring_off = idx->ring_off;
    a.accept_mask = accept_mask;
    a.sink = PairSink{d_left, d_right, (unsigned long long)(capacity > 0 ? capacity : 0), &ctx->d_counters[0]};
    a.defer = dsink;
    a.counters = ctx->d_counters;
    a.staged = staged.p;
    a.stripe_count = stripe_count.p;
    a.stripe_cap = stripe_cap;
    a.cell_count = cell_count.p;
    a.grouped = grouped.p;
    a.n_grouped = n_grouped.p;
    a.work = &ctx->d_counters[kWorkCounter];
#ifndef VS_LEARNED_BLOCKS_PER_SM
#define VS_LEARNED_BLOCKS_PER_SM 8  // map and scatter blocks per SM (0: one resident wave)
#endif
    auto grid = [&](auto kernel, int64_t items) {
        return VS_LEARNED_BLOCKS_PER_SM > 0 ? grid_for(items, kThreads, VS_LEARNED_BLOCKS_PER_SM)
                                            : resident_grid(kernel, items, kThreads);
    };
    learned_map_kernel<<<grid(learned_map_kernel, n), kThreads, 0, s>>>(a);
    VS_LAUNCHED("learned_map", s);
    VS_TRY(exclusive_scan_u32(cell_count.p, cell_count.p, li.n_cells, n_grouped.p, s));
    phase_mark(ctx, 1);
    learned_scatter_kernel<<<kStripes, kThreads, 0, s>>>(a);
    VS_LAUNCHED("learned_scatter", s);
    phase_mark(ctx, 2);
#ifndef VS_REFINE_QUEUE
#define VS_REFINE_QUEUE 1
#endif
    if (VS_REFINE_QUEUE && accept_mask) {
        learned_refine_kernel<<<resident_grid(learned_refine_kernel, n, kThreads), kThreads, 0, s>>>(a);
        VS_LAUNCHED("learned_refine", s);
    } else {
        learned_join_kernel<<<resident_grid(learned_join_kernel, n, kThreads), kThreads, 0, s>>>(a);
        VS_LAUNCHED("learned_join", s);
    }
    return VS_OK;
}

}  // namespace vs
