// Packed Hilbert R-tree build for the polygon (tree) side.
//
// Replaces the reference's flat index build (build_flat_spatial_index,
// src/vibespatial/spatial/indexing.py:1357-1448: device bounds, a D2H fence
// for the total bounds, Morton keys, CCCL sort_pairs).  Here:
//   1. geom_bounds_kernel   one warp per polygon, coalesced min/max over its
//                           contiguous coordinate span (all parts and rings)
//   2. frame_kernel         total bounds of the valid boxes, kept on device
//   3. hilbert_key_kernel   64-bit Hilbert key of each box centre on the 2^32
//                           grid of the frame (no host fence in between)
//   4. radix sort           in-house, (key, row) pairs
//   5. slot kernels         polygons re-laid out in key order with interleaved
//                           double2 vertices, so a leaf's polygons are
//                           contiguous in HBM
//   6. level kernels        bottom-up box unions, fanout 16
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "hilbert.cuh"
#include "index.cuh"
#include "primitives.cuh"

namespace vs {
namespace {

__global__ void geom_bounds_kernel(vs_polygons p, vs_box* __restrict__ box, uint32_t* __restrict__ n_parts,
                                   uint32_t* __restrict__ n_rings, uint32_t* __restrict__ n_coords) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g = warp; g < p.n_geoms; g += nwarps) {
        const bool valid = p.d_valid == nullptr || p.d_valid[g] != 0;
        int32_t p0 = p.d_geom_off[g], p1 = p.d_geom_off[g + 1];
        if (!valid) p1 = p0;
        const int32_t r0 = p.d_part_off[p0], r1 = p.d_part_off[p1];
        const int32_t c0 = p.d_ring_off[r0], c1 = p.d_ring_off[r1];
        double mnx = INFINITY, mny = INFINITY, mxx = -INFINITY, mxy = -INFINITY;
        for (int32_t c = c0 + lane; c < c1; c += 32) {
            const double x = p.d_x[c], y = p.d_y[c];
            mnx = fmin(mnx, x);
            mny = fmin(mny, y);
            mxx = fmax(mxx, x);
            mxy = fmax(mxy, y);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mnx = fmin(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
            mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
            mxx = fmax(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
            mxy = fmax(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
        }
        if (lane == 0) {
            // A box with NaN coordinates is unusable; make it empty.
            if (!(mnx <= mxx && mny <= mxy)) {
                mnx = mny = INFINITY;
                mxx = mxy = -INFINITY;
            }
            box[g] = vs_box{mnx, mny, mxx, mxy};
            n_parts[g] = (uint32_t)(p1 - p0);
            n_rings[g] = (uint32_t)(r1 - r0);
            n_coords[g] = (uint32_t)(c1 - c0);
        }
    }
}

__global__ void frame_init_kernel(long long* f) {
    f[0] = dbl_to_ordered(INFINITY);
    f[1] = dbl_to_ordered(INFINITY);
    f[2] = dbl_to_ordered(-INFINITY);
    f[3] = dbl_to_ordered(-INFINITY);
}

__global__ void frame_kernel(const vs_box* __restrict__ box, int64_t n, long long* __restrict__ f) {
    double mnx = INFINITY, mny = INFINITY, mxx = -INFINITY, mxy = -INFINITY;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const vs_box b = box[i];
        if (b.minx <= b.maxx) {
            mnx = fmin(mnx, b.minx);
            mny = fmin(mny, b.miny);
            mxx = fmax(mxx, b.maxx);
            mxy = fmax(mxy, b.maxy);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mnx = fmin(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
        mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
        mxx = fmax(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
        mxy = fmax(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
    }
    if ((threadIdx.x & 31) == 0 && mnx <= mxx) {
        atomicMin(&f[0], dbl_to_ordered(mnx));
        atomicMin(&f[1], dbl_to_ordered(mny));
        atomicMax(&f[2], dbl_to_ordered(mxx));
        atomicMax(&f[3], dbl_to_ordered(mxy));
    }
}

// Decode the ordered-int frame into doubles in place.
__global__ void frame_finish_kernel(long long* f) {
    const int i = threadIdx.x;
    if (i < 4) {
        const double v = ordered_to_dbl(f[i]);
        reinterpret_cast<double*>(f)[i] = v;
    }
}

__device__ __forceinline__ void frame_scale(const double* fr, double& lox, double& loy, double& sx, double& sy) {
    lox = fr[0];
    loy = fr[1];
    const double wx = fr[2] - fr[0], wy = fr[3] - fr[1];
    sx = wx > 0.0 ? 4294967295.0 / wx : 0.0;
    sy = wy > 0.0 ? 4294967295.0 / wy : 0.0;
}

__global__ void hilbert_box_key_kernel(const vs_box* __restrict__ box, int64_t n, const double* __restrict__ fr,
                                       uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    double lox, loy, sx, sy;
    frame_scale(fr, lox, loy, sx, sy);
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const vs_box b = box[i];
        uint64_t k = ~0ull;  // empty boxes sort last
        if (b.minx <= b.maxx) {
            const double cx = 0.5 * b.minx + 0.5 * b.maxx, cy = 0.5 * b.miny + 0.5 * b.maxy;
            k = hilbert_key(quantize(cx, lox, sx), quantize(cy, loy, sy), 32);
        }
        keys[i] = k;
        vals[i] = (uint32_t)i;
    }
}

__global__ void hilbert_point_key_kernel(const double* __restrict__ x, const double* __restrict__ y, int64_t n,
                                         double lox, double loy, double sx, double sy, uint64_t* __restrict__ keys) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        keys[i] = hilbert_key(quantize(x[i], lox, sx), quantize(y[i], loy, sy), 32);
}

// slot s <- row order[s]: gather boxes and per-slot counts.
__global__ void slot_gather_kernel(const uint32_t* __restrict__ order, int64_t n, const vs_box* __restrict__ box,
                                   const uint32_t* __restrict__ np, const uint32_t* __restrict__ nr,
                                   const uint32_t* __restrict__ nc, vs_box* __restrict__ leaf,
                                   int32_t* __restrict__ item_geom, uint32_t* __restrict__ sp,
                                   uint32_t* __restrict__ sr, uint32_t* __restrict__ sc) {
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < n; s += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t g = order[s];
        leaf[s] = box[g];
        item_geom[s] = (int32_t)g;
        sp[s] = np[g];
        sr[s] = nr[g];
        sc[s] = nc[g];
    }
}

// One warp per slot: copy offsets (rebased) and interleave vertices.
__global__ void slot_copy_kernel(vs_polygons p, const int32_t* __restrict__ item_geom, int64_t n,
                                 const uint32_t* __restrict__ pbase, const uint32_t* __restrict__ rbase,
                                 const uint32_t* __restrict__ cbase, const uint32_t* __restrict__ np,
                                 int32_t* __restrict__ geom_off, int32_t* __restrict__ part_off,
                                 int32_t* __restrict__ ring_off, double2* __restrict__ xy,
                                 const uint32_t* __restrict__ totals) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t s = warp; s < n; s += nwarps) {
        const int32_t g = item_geom[s];
        const uint32_t pb = pbase[s], rb = rbase[s], cb = cbase[s];
        const int32_t nparts = (int32_t)np[g];
        const int32_t p0 = p.d_geom_off[g];
        const int32_t r0 = p.d_part_off[p0], r1 = p.d_part_off[p0 + nparts];
        const int32_t c0 = p.d_ring_off[r0], c1 = p.d_ring_off[r1];
        if (lane == 0) geom_off[s] = (int32_t)pb;
        for (int32_t k = lane; k < nparts; k += 32) part_off[pb + k] = p.d_part_off[p0 + k] - r0 + (int32_t)rb;
        for (int32_t k = lane; k < r1 - r0; k += 32) ring_off[rb + k] = p.d_ring_off[r0 + k] - c0 + (int32_t)cb;
        for (int32_t k = lane; k < c1 - c0; k += 32) xy[cb + k] = make_double2(p.d_x[c0 + k], p.d_y[c0 + k]);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        geom_off[n] = (int32_t)totals[0];
        part_off[totals[0]] = (int32_t)totals[1];
        ring_off[totals[1]] = (int32_t)totals[2];
    }
}

__global__ void level_kernel(const vs_box* __restrict__ child, int64_t nchild, vs_box* __restrict__ parent,
                             int64_t nparent) {
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < nparent;
         n += (int64_t)gridDim.x * blockDim.x) {
        double mnx = INFINITY, mny = INFINITY, mxx = -INFINITY, mxy = -INFINITY;
        const int64_t c0 = n * kFanout;
        const int64_t c1 = c0 + kFanout < nchild ? c0 + kFanout : nchild;
        for (int64_t c = c0; c < c1; ++c) {
            const vs_box b = child[c];
            if (b.minx <= b.maxx) {
                mnx = fmin(mnx, b.minx);
                mny = fmin(mny, b.miny);
                mxx = fmax(mxx, b.maxx);
                mxy = fmax(mxy, b.maxy);
            }
        }
        parent[n] = vs_box{mnx, mny, mxx, mxy};
    }
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


// ------------------------------------------------------------ ring bins ---
// Pass 1, one thread per ring: is it binned (enough vertices, finite y,
// positive height), its (y0, scale), and how many (bin, edge) entries it
// needs (an edge is listed in every bin its closed y-range meets).
__global__ void ring_bin_size_kernel(int64_t n_rings, const int32_t* __restrict__ ring_off,
                                     const double2* __restrict__ xy, int min_vertices,
                                     uint32_t* __restrict__ entries, uint32_t* __restrict__ binned,
                                     double2* __restrict__ yinfo, unsigned long long* __restrict__ n_long) {
    unsigned long long long_rings = 0;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rings;
         r += (int64_t)gridDim.x * blockDim.x) {
        const int s0 = ring_off[r], s1 = ring_off[r + 1], nv = s1 - s0;
        uint32_t cnt = 0, flag = 0;
        double y0 = 0.0, sc = 0.0;
        if (nv >= min_vertices && nv <= 65535) {
            double lo = INFINITY, hi = -INFINITY;
            bool finite = true;
            for (int i = s0; i < s1; ++i) {
                const double y = xy[i].y;
                finite = finite && isfinite(y);
                lo = fmin(lo, y);
                hi = fmax(hi, y);
            }
            if (finite && hi > lo) {
                sc = __ddiv_rn((double)kRingBins, __dsub_rn(hi, lo));
                if (isfinite(sc) && sc > 0.0) {
                    flag = 1;
                    y0 = lo;
                    long_rings += nv >= kSplitBinMinVertices ? 1 : 0;
                    for (int e = 0; e < nv; ++e) {
                        const double a = xy[e == 0 ? s1 - 1 : s0 + e - 1].y, b = xy[s0 + e].y;
                        cnt += (uint32_t)(ring_bin_of(fmax(a, b), y0, sc) - ring_bin_of(fmin(a, b), y0, sc) + 1);
                    }
                }
            }
        }
        entries[r] = cnt;
        binned[r] = flag;
        yinfo[r] = make_double2(y0, sc);
    }
    if (long_rings) atomicAdd(n_long, long_rings);
}

// Pass 2, one thread per binned ring: bin offsets, then the edge lists in
// ring order within each bin.
__global__ void ring_bin_fill_kernel(int64_t n_rings, const int32_t* __restrict__ ring_off,
                                     const double2* __restrict__ xy, const uint32_t* __restrict__ entry_off,
                                     const uint32_t* __restrict__ bin_idx, const uint32_t* __restrict__ binned,
                                     const double2* __restrict__ yinfo, int32_t* __restrict__ ring_bin,
                                     RingBins* __restrict__ bins, uint16_t* __restrict__ edges) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rings;
         r += (int64_t)gridDim.x * blockDim.x) {
        if (!binned[r]) {
            ring_bin[r] = -1;
            continue;
        }
        const int s0 = ring_off[r], s1 = ring_off[r + 1], nv = s1 - s0;
        const double y0 = yinfo[r].x, sc = yinfo[r].y;
        uint32_t cnt[kRingBins];
#pragma unroll
        for (int k = 0; k < kRingBins; ++k) cnt[k] = 0;
        for (int e = 0; e < nv; ++e) {
            const double a = xy[e == 0 ? s1 - 1 : s0 + e - 1].y, b = xy[s0 + e].y;
            const int k0 = ring_bin_of(fmin(a, b), y0, sc), k1 = ring_bin_of(fmax(a, b), y0, sc);
            for (int k = k0; k <= k1; ++k) ++cnt[k];
        }
        RingBins rb;
        rb.y0 = y0;
        rb.scale = sc;
        uint32_t o = entry_off[r];
        for (int k = 0; k < kRingBins; ++k) {
            rb.off[k] = o;
            o += cnt[k];
        }
        rb.off[kRingBins] = o;
        rb.pad[0] = rb.pad[1] = rb.pad[2] = 0;
        const uint32_t b_i = bin_idx[r];
        bins[b_i] = rb;
        ring_bin[r] = (int32_t)b_i;
        uint32_t cur[kRingBins];
#pragma unroll
        for (int k = 0; k < kRingBins; ++k) cur[k] = rb.off[k];
        for (int e = 0; e < nv; ++e) {
            const double a = xy[e == 0 ? s1 - 1 : s0 + e - 1].y, b = xy[s0 + e].y;
            const int k0 = ring_bin_of(fmin(a, b), y0, sc), k1 = ring_bin_of(fmax(a, b), y0, sc);
            for (int k = k0; k <= k1; ++k) edges[cur[k]++] = (uint16_t)e;
        }
    }
}

}  // namespace

int hilbert_point_keys(const double* x, const double* y, int64_t n, double minx, double miny, double maxx,
                       double maxy, uint64_t* keys, cudaStream_t s) {
    const double wx = maxx - minx, wy = maxy - miny;
    const double sx = wx > 0 ? 4294967295.0 / wx : 0.0, sy = wy > 0 ? 4294967295.0 / wy : 0.0;
    hilbert_point_key_kernel<<<grid_for(n, 256), 256, 0, s>>>(x, y, n, minx, miny, sx, sy, keys);
    VS_CUDA_TRY(cudaGetLastError());
    return VS_OK;
}

void free_index_memory(vs_index* idx) {
    cudaFree(idx->nodes);
    cudaFree(idx->item_geom);
    cudaFree(idx->geom_off);
    cudaFree(idx->part_off);
    cudaFree(idx->ring_off);
    cudaFree(idx->xy);
    cudaFree(idx->frame);
    cudaFree(idx->ring_bin);
    cudaFree(idx->ring_bins);
    cudaFree(idx->bin_edges);
    free_learned_index(idx);
}

int build_rtree(vs_context* ctx, const vs_polygons* P, vs_index* idx) {
    cudaStream_t s = ctx->stream;
    const int64_t M = P->n_geoms;
    idx->n_geoms = P->n_geoms;
    idx->n_parts = P->n_parts;
    idx->n_rings = P->n_rings;
    idx->n_coords = P->n_coords;

    // level layout (host arithmetic only)
    int64_t off = 0, size = M;
    int L = 0;
    for (;;) {
        idx->level_off[L] = off;
        idx->level_size[L] = size;
        off += size;
        ++L;
        if (size <= 1) break;
        size = (size + kFanout - 1) / kFanout;
        if (L >= kMaxLevels) {
            set_error("too many polygons for the R-tree layout");
            return VS_E_ARG;
        }
    }
    idx->levels = L;
    int64_t& bytes = idx->device_bytes;
    VS_TRY(dalloc(&idx->nodes, (size_t)off, bytes));
    VS_TRY(dalloc(&idx->item_geom, (size_t)M, bytes));
    VS_TRY(dalloc(&idx->geom_off, (size_t)M + 1, bytes));
    VS_TRY(dalloc(&idx->part_off, (size_t)P->n_parts + 1, bytes));
    VS_TRY(dalloc(&idx->ring_off, (size_t)P->n_rings + 1, bytes));
    VS_TRY(dalloc(&idx->xy, (size_t)P->n_coords, bytes));
    VS_TRY(dalloc(&idx->frame, 4, bytes));

    Scratch<vs_box> box;
    Scratch<uint32_t> np, nr, nc, sp, sr, sc, vals, totals;
    Scratch<uint64_t> keys;
    VS_TRY(box.alloc((size_t)M, s));
    VS_TRY(np.alloc((size_t)M, s));
    VS_TRY(nr.alloc((size_t)M, s));
    VS_TRY(nc.alloc((size_t)M, s));
    VS_TRY(sp.alloc((size_t)M, s));
    VS_TRY(sr.alloc((size_t)M, s));
    VS_TRY(sc.alloc((size_t)M, s));
    VS_TRY(vals.alloc((size_t)M, s));
    VS_TRY(keys.alloc((size_t)M, s));
    VS_TRY(totals.alloc(4, s));
    VS_CUDA_TRY(cudaMemsetAsync(totals.p, 0, 4 * sizeof(uint32_t), s));

    if (M > 0) {
        geom_bounds_kernel<<<grid_for(M * 32, 256), 256, 0, s>>>(*P, box.p, np.p, nr.p, nc.p);
        VS_CUDA_TRY(cudaGetLastError());
    }
    frame_init_kernel<<<1, 1, 0, s>>>((long long*)idx->frame);
    if (M > 0) frame_kernel<<<grid_for(M, 256), 256, 0, s>>>(box.p, M, (long long*)idx->frame);
    frame_finish_kernel<<<1, 32, 0, s>>>((long long*)idx->frame);
    VS_CUDA_TRY(cudaGetLastError());
    if (M > 0) {
        hilbert_box_key_kernel<<<grid_for(M, 256), 256, 0, s>>>(box.p, M, idx->frame, keys.p, vals.p);
        VS_CUDA_TRY(cudaGetLastError());
        VS_TRY(radix_sort_u64_u32(keys.p, vals.p, M, 64, s));
        slot_gather_kernel<<<grid_for(M, 256), 256, 0, s>>>(vals.p, M, box.p, np.p, nr.p, nc.p, idx->nodes,
                                                            idx->item_geom, sp.p, sr.p, sc.p);
        VS_CUDA_TRY(cudaGetLastError());
    }
    VS_TRY(exclusive_scan_u32(sp.p, sp.p, M, totals.p + 0, s));
    VS_TRY(exclusive_scan_u32(sr.p, sr.p, M, totals.p + 1, s));
    VS_TRY(exclusive_scan_u32(sc.p, sc.p, M, totals.p + 2, s));
    slot_copy_kernel<<<grid_for(M * 32 > 0 ? M * 32 : 32, 256), 256, 0, s>>>(
        *P, idx->item_geom, M, sp.p, sr.p, sc.p, np.p, idx->geom_off, idx->part_off, idx->ring_off, idx->xy,
        totals.p);
    VS_CUDA_TRY(cudaGetLastError());
    for (int l = 1; l < L; ++l) {
        level_kernel<<<grid_for(idx->level_size[l], 256), 256, 0, s>>>(
            idx->nodes + idx->level_off[l - 1], idx->level_size[l - 1], idx->nodes + idx->level_off[l],
            idx->level_size[l]);
        VS_CUDA_TRY(cudaGetLastError());
    }
    if (M == 0) {
        // A single empty root so traversal has a well-formed (empty) tree.
        const vs_box empty{INFINITY, INFINITY, -INFINITY, -INFINITY};
        VS_CUDA_TRY(cudaMemcpyAsync(idx->nodes, &empty, sizeof(empty), cudaMemcpyHostToDevice, s));
    }
    VS_CUDA_TRY(cudaMemcpyAsync(idx->h_frame, idx->frame, 4 * sizeof(double), cudaMemcpyDeviceToHost, s));
    uint32_t laid[3] = {0, 0, 0};
    VS_CUDA_TRY(cudaMemcpyAsync(laid, totals.p, sizeof(laid), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    // Null polygons own no parts, rings or vertices in the slot layout: the
    // index's counts are those laid out, which is what every later pass over
    // part_off / ring_off / xy may read.
    idx->n_parts = (int32_t)laid[0];
    idx->n_rings = (int32_t)laid[1];
    idx->n_coords = (int64_t)laid[2];
    return VS_OK;
}

int build_ring_bins(vs_context* ctx, vs_index* idx, int min_vertices) {
    if (min_vertices < 0 || idx->n_rings <= 0) return VS_OK;
    if (idx->n_coords * kRingBins >= 0xffffffffLL) return VS_OK;  // entry offsets are 32-bit
    if (min_vertices == 0) min_vertices = kRingBinMinVertices;
    if (min_vertices < 3) min_vertices = 3;
    cudaStream_t s = ctx->stream;
    const int64_t R = idx->n_rings;
    Scratch<uint32_t> entries, entry_off, binned, bin_idx, totals;
    Scratch<double2> yinfo;
    Scratch<unsigned long long> n_long;
    VS_TRY(n_long.alloc(1, s));
    VS_CUDA_TRY(cudaMemsetAsync(n_long.p, 0, sizeof(unsigned long long), s));
    VS_TRY(entries.alloc((size_t)R, s));
    VS_TRY(entry_off.alloc((size_t)R, s));
    VS_TRY(binned.alloc((size_t)R, s));
    VS_TRY(bin_idx.alloc((size_t)R, s));
    VS_TRY(yinfo.alloc((size_t)R, s));
    VS_TRY(totals.alloc(2, s));
    ring_bin_size_kernel<<<grid_for(R, 256), 256, 0, s>>>(R, idx->ring_off, idx->xy, min_vertices, entries.p,
                                                          binned.p, yinfo.p, n_long.p);
    VS_CUDA_TRY(cudaGetLastError());
    VS_TRY(exclusive_scan_u32(entries.p, entry_off.p, R, totals.p + 0, s));
    VS_TRY(exclusive_scan_u32(binned.p, bin_idx.p, R, totals.p + 1, s));
    uint32_t tot[2] = {0, 0};
    unsigned long long h_long = 0;
    VS_CUDA_TRY(cudaMemcpyAsync(tot, totals.p, sizeof(tot), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaMemcpyAsync(&h_long, n_long.p, sizeof(h_long), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    if (tot[1] == 0) return VS_OK;  // no ring qualifies
    int64_t& bytes = idx->device_bytes;
    VS_TRY(dalloc(&idx->ring_bin, (size_t)R, bytes));
    VS_TRY(dalloc(&idx->ring_bins, (size_t)tot[1], bytes));
    VS_TRY(dalloc(&idx->bin_edges, (size_t)tot[0], bytes));
    ring_bin_fill_kernel<<<grid_for(R, 256), 256, 0, s>>>(R, idx->ring_off, idx->xy, entry_off.p, bin_idx.p, binned.p,
                                                          yinfo.p, idx->ring_bin, idx->ring_bins, idx->bin_edges);
    VS_CUDA_TRY(cudaGetLastError());
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    idx->n_binned_rings = tot[1];
    idx->n_bin_edges = tot[0];
    idx->n_split_binned_rings = (int64_t)h_long;
    return VS_OK;
}

}  // namespace vs
