// Join export on the device: the row indexers of a relation join for
// how = inner / left / right / outer, after on_attribute filtering.
//
// Replaces the reference's host export (src/vibespatial/api/_native_results.py:395-470,
// _adjust_join_indexers) and its shared-attribute filter
// (src/vibespatial/api/tools/sjoin.py:826-888, filter_by_equal_columns).
// Input pairs are sorted by (left, right), as every join here returns them.
//
//   1. keep flags (equal attribute codes, missing codes never match), scan,
//      ordered compaction of the pairs and their source positions
//   2. how = right: the kept pairs re-sorted by (right, left) (radix sort)
//   3. per driving row (left rows; right rows for how = right) its pair
//      count; per tile of 2048 driving rows its pairs and unmatched rows,
//      scanned: a tile's output is one contiguous range, which one block
//      writes in order (a row's pairs, or one row with -1 on the other side
//      when it has none)
//   4. how = outer: right rows no pair reaches are appended in order
#include <cuda_runtime.h>
#include <stdint.h>

#include "primitives.cuh"
#include "vs_common.cuh"

namespace vs {
namespace {

// Pairs whose rows fall outside [0, n_left) x [0, n_right) are counted.
__global__ void export_check_kernel(const int32_t* __restrict__ l, const int32_t* __restrict__ r, int64_t n,
                                    int64_t n_left, int64_t n_right, uint32_t* __restrict__ bad) {
    uint32_t b = 0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        b += (l[k] < 0 || l[k] >= n_left || r[k] < 0 || r[k] >= n_right) ? 1u : 0u;
    if (b) atomicAdd(bad, b);
}

// Keep flags of the attribute filter; pairs outside the row ranges are
// counted (and not kept) as export_check_kernel counts them.
__global__ void export_keep_kernel(const int32_t* __restrict__ l, const int32_t* __restrict__ r, int64_t n,
                                   int64_t n_left, int64_t n_right, const int64_t* __restrict__ lc,
                                   const int64_t* __restrict__ rc, uint32_t* __restrict__ keep,
                                   uint32_t* __restrict__ bad) {
    uint32_t b = 0;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t li = l[k], ri = r[k];
        const bool ok = li >= 0 && li < n_left && ri >= 0 && ri < n_right;
        b += ok ? 0u : 1u;
        const int64_t a = ok ? lc[li] : -1;
        keep[k] = a >= 0 && a == rc[ri] ? 1u : 0u;
    }
    if (b) atomicAdd(bad, b);
}

__global__ void export_compact_kernel(const int32_t* __restrict__ l, const int32_t* __restrict__ r, int64_t n,
                                      const uint32_t* __restrict__ keep, const uint32_t* __restrict__ pos,
                                      int32_t* __restrict__ ol, int32_t* __restrict__ orr, uint32_t* __restrict__ osrc) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        if (keep[k]) {
            const uint32_t p = pos[k];
            ol[p] = l[k];
            orr[p] = r[k];
            osrc[p] = (uint32_t)k;
        }
}

// (right, left) keys for how = right; vals = position in the kept pairs
__global__ void export_right_keys_kernel(const int32_t* __restrict__ l, const int32_t* __restrict__ r, int64_t n,
                                         uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        keys[k] = ((uint64_t)(uint32_t)r[k] << 32) | (uint32_t)l[k];
        vals[k] = (uint32_t)k;
    }
}

__global__ void export_count_kernel(const int32_t* __restrict__ drive, const uint32_t* __restrict__ perm, int64_t n,
                                    uint32_t* __restrict__ cnt) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(&cnt[drive[perm ? perm[k] : (uint32_t)k]], 1u);
}

constexpr int kTileThreads = 256;
constexpr int kTileRows = 2048;
constexpr int kRowsPerThread = kTileRows / kTileThreads;

// A driving row's share of the output, packed: its pairs in the low word,
// 1 in the high word when it has none (it then owns one unmatched row).
// Neither word carries into the other: pairs and rows are below 2^31.
__device__ __forceinline__ uint64_t row_pack(uint32_t c) { return (uint64_t)c | ((uint64_t)(c == 0u) << 32); }

__global__ void __launch_bounds__(kTileThreads) export_tile_sum_kernel(const uint32_t* __restrict__ cnt, int64_t n,
                                                                       uint64_t* __restrict__ tile_sum) {
    __shared__ uint64_t s_w[kTileThreads / 32];
    const int64_t base = (int64_t)blockIdx.x * kTileRows;
    uint64_t v = 0;
    if (base + kTileRows <= n) {
        // a full tile: 16-byte loads (cnt is allocation-aligned, tiles are 8 KB apart)
        const uint4* c4 = reinterpret_cast<const uint4*>(cnt + base);
#pragma unroll
        for (int k = 0; k < kTileRows / (4 * kTileThreads); ++k) {
            const uint4 w = c4[threadIdx.x + k * kTileThreads];
            v += row_pack(w.x) + row_pack(w.y) + row_pack(w.z) + row_pack(w.w);
        }
    } else {
        for (int k = threadIdx.x; k < kTileRows; k += kTileThreads)
            if (base + k < n) v += row_pack(cnt[base + k]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint64_t t = 0;
#pragma unroll
        for (int w = 0; w < kTileThreads / 32; ++w) t += s_w[w];
        tile_sum[blockIdx.x] = t;
    }
}

// One block per tile of driving rows. The tile's output is the range that
// starts at its scanned offset (pairs before it + unmatched rows before it);
// row k of the tile owns [s_start[k], s_start[k + 1]) of it and its pairs
// are [s_first[k], s_first[k + 1]) of the tile's pairs in driving order.
// Output positions go to consecutive threads, so the stores are contiguous.
__global__ void __launch_bounds__(kTileThreads) export_write_kernel(
    const uint32_t* __restrict__ cnt, int64_t n, const uint64_t* __restrict__ tile_off,
    const int32_t* __restrict__ other, const uint32_t* __restrict__ perm, const uint32_t* __restrict__ src,
    int64_t* __restrict__ o_drive, int64_t* __restrict__ o_other, int64_t* __restrict__ o_src) {
    __shared__ uint32_t s_start[kTileRows + 1];
    __shared__ uint32_t s_first[kTileRows + 1];
    __shared__ uint64_t s_w[kTileThreads / 32];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int64_t base = (int64_t)blockIdx.x * kTileRows;
    const int64_t r0 = base + (int64_t)t * kRowsPerThread;
    uint64_t v[kRowsPerThread];
    uint64_t sum = 0;
    static_assert(kRowsPerThread == 8, "two 16-byte loads per thread");
    if (r0 + kRowsPerThread <= n) {
        // both loads stay 16-byte aligned: r0 is a multiple of 8 rows
        const uint4 w0 = *reinterpret_cast<const uint4*>(cnt + r0);
        const uint4 w1 = *reinterpret_cast<const uint4*>(cnt + r0 + 4);
        const uint32_t c[kRowsPerThread] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
        for (int k = 0; k < kRowsPerThread; ++k) v[k] = row_pack(c[k]);
    } else {
#pragma unroll
        for (int k = 0; k < kRowsPerThread; ++k)
            v[k] = r0 + k < n ? row_pack(cnt[r0 + k]) : 0ull;  // rows past the end own nothing
    }
#pragma unroll
    for (int k = 0; k < kRowsPerThread; ++k) sum += v[k];
    uint64_t incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint64_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_w[warp] = incl;
    __syncthreads();
    uint64_t run = incl - sum;
    for (int w = 0; w < warp; ++w) run += s_w[w];
#pragma unroll
    for (int k = 0; k < kRowsPerThread; ++k) {
        s_first[t * kRowsPerThread + k] = (uint32_t)run;
        s_start[t * kRowsPerThread + k] = (uint32_t)run + (uint32_t)(run >> 32);
        run += v[k];
    }
    if (t == kTileThreads - 1) {
        s_first[kTileRows] = (uint32_t)run;
        s_start[kTileRows] = (uint32_t)run + (uint32_t)(run >> 32);
    }
    __syncthreads();
    const uint64_t off = tile_off[blockIdx.x];
    const int64_t pair_base = (int64_t)(uint32_t)off;
    const int64_t out_base = pair_base + (int64_t)(off >> 32);
    const uint32_t total = s_start[kTileRows];
    for (uint32_t o = t; o < total; o += kTileThreads) {
        // the row that owns o: s_start[lo] <= o < s_start[hi]
        int lo = 0, hi = kTileRows;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (s_start[mid] <= o) lo = mid;
            else hi = mid;
        }
        const uint32_t f0 = s_first[lo];
        const int64_t p = out_base + o;
        o_drive[p] = base + lo;
        if (s_first[lo + 1] == f0) {
            o_other[p] = -1;
            if (o_src) o_src[p] = -1;
        } else {
            const int64_t k = pair_base + f0 + (o - s_start[lo]);
            const uint32_t j = perm ? perm[k] : (uint32_t)k;
            o_other[p] = other[j];
            if (o_src) o_src[p] = src ? (int64_t)src[j] : (int64_t)j;
        }
    }
}

__global__ void export_mark_kernel(const int32_t* __restrict__ r, int64_t n, uint32_t* __restrict__ matched) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        matched[r[k]] = 1u;
}

__global__ void export_flip_kernel(uint32_t* __restrict__ v, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v[i] = v[i] ? 0u : 1u;
}

__global__ void export_append_kernel(const uint32_t* __restrict__ missing, const uint32_t* __restrict__ pos,
                                     int64_t n, int64_t base, int64_t* __restrict__ o_left,
                                     int64_t* __restrict__ o_right, int64_t* __restrict__ o_src) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (missing[i]) {
            const int64_t p = base + pos[i];
            o_left[p] = -1;
            o_right[p] = i;
            if (o_src) o_src[p] = -1;
        }
}

__global__ void export_copy_kernel(const int32_t* __restrict__ l, const int32_t* __restrict__ r,
                                   const uint32_t* __restrict__ src, int64_t n, int64_t* __restrict__ ol,
                                   int64_t* __restrict__ orr, int64_t* __restrict__ osrc) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        ol[k] = l[k];
        orr[k] = r[k];
        if (osrc) osrc[k] = src ? (int64_t)src[k] : k;
    }
}

template <class K>
int grid_of(K kernel, int64_t n) {
    return resident_grid(kernel, n > 0 ? n : 1, 256);
}

}  // namespace
}  // namespace vs

using namespace vs;

extern "C" {

int vs_join_export(vs_context* ctx, const int32_t* d_left, const int32_t* d_right, int64_t n_pairs, int64_t n_left,
                   int64_t n_right, int32_t how, const int64_t* d_left_code, const int64_t* d_right_code,
                   int64_t* d_out_left, int64_t* d_out_right, int64_t* d_out_src, int64_t capacity,
                   int64_t* n_out) {
    if (!ctx || !n_out || (n_pairs > 0 && (!d_left || !d_right))) {
        set_error("ctx/n_out/pairs is NULL");
        return VS_E_ARG;
    }
    *n_out = 0;
    if (how < VS_HOW_INNER || how > VS_HOW_OUTER) {
        set_error("unknown how code %d", how);
        return VS_E_ARG;
    }
    if (n_pairs < 0 || n_pairs > 0x7fffffffLL || n_left < 0 || n_left > 0x7fffffffLL || n_right < 0 ||
        n_right > 0x7fffffffLL) {
        set_error("sizes outside the 32-bit ranges (pairs %lld, left %lld, right %lld)", (long long)n_pairs,
                  (long long)n_left, (long long)n_right);
        return VS_E_ARG;
    }
    // codes for one side imply codes for the other (an empty side may pass NULL)
    const bool with_codes = d_left_code || d_right_code;
    if (with_codes && ((n_left > 0 && !d_left_code) || (n_right > 0 && !d_right_code))) {
        set_error("attribute codes must be given for both sides or neither");
        return VS_E_ARG;
    }
    if (capacity < 0 || (capacity > 0 && (!d_out_left || !d_out_right))) {
        set_error("invalid output buffers (capacity %lld)", (long long)capacity);
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    cudaStream_t s = ctx->stream;
    // 1. attribute filter (ordered compaction); without codes the pairs are used in place
    const int32_t* kl = d_left;
    const int32_t* kr = d_right;
    const uint32_t* ksrc = nullptr;  // null: position k is its own source
    int64_t m = n_pairs;
    Scratch<uint32_t> keep, kpos, ksrc_buf;
    Scratch<int32_t> kl_buf, kr_buf;
    Scratch<uint32_t> totals;
    VS_TRY(totals.alloc(4, s));
    VS_CUDA_TRY(cudaMemsetAsync(totals.p, 0, 4 * sizeof(uint32_t), s));
    auto bad_pairs = [&](uint32_t bad) {
        set_error("%u pairs name rows outside [0, %lld) x [0, %lld)", bad, (long long)n_left, (long long)n_right);
        return VS_E_ARG;
    };
    if (n_pairs > 0 && !with_codes) {
        export_check_kernel<<<grid_of(export_check_kernel, n_pairs), 256, 0, s>>>(d_left, d_right, n_pairs, n_left,
                                                                                  n_right, totals.p + 3);
        VS_LAUNCHED("export_check", s);
        uint32_t bad = 0;
        VS_CUDA_TRY(cudaMemcpyAsync(&bad, totals.p + 3, sizeof(bad), cudaMemcpyDeviceToHost, s));
        VS_CUDA_TRY(cudaStreamSynchronize(s));
        if (bad) return bad_pairs(bad);
    }
    if (with_codes && n_pairs > 0) {
        VS_TRY(keep.alloc((size_t)n_pairs, s));
        VS_TRY(kpos.alloc((size_t)n_pairs, s));
        // the filter checks the row ranges too (before it reads a code)
        export_keep_kernel<<<grid_of(export_keep_kernel, n_pairs), 256, 0, s>>>(
            d_left, d_right, n_pairs, n_left, n_right, d_left_code, d_right_code, keep.p, totals.p + 3);
        VS_LAUNCHED("export_keep", s);
        VS_TRY(exclusive_scan_u32(keep.p, kpos.p, n_pairs, totals.p, s));
        uint32_t h4[4] = {0, 0, 0, 0};
        VS_CUDA_TRY(cudaMemcpyAsync(h4, totals.p, sizeof(h4), cudaMemcpyDeviceToHost, s));
        VS_CUDA_TRY(cudaStreamSynchronize(s));
        if (h4[3]) return bad_pairs(h4[3]);
        m = h4[0];
        VS_TRY(kl_buf.alloc((size_t)m, s));
        VS_TRY(kr_buf.alloc((size_t)m, s));
        VS_TRY(ksrc_buf.alloc((size_t)m, s));
        export_compact_kernel<<<grid_of(export_compact_kernel, n_pairs), 256, 0, s>>>(
            d_left, d_right, n_pairs, keep.p, kpos.p, kl_buf.p, kr_buf.p, ksrc_buf.p);
        VS_LAUNCHED("export_compact", s);
        kl = kl_buf.p;
        kr = kr_buf.p;
        ksrc = ksrc_buf.p;
    }
    if (how == VS_HOW_INNER) {
        *n_out = m;
        if (m > capacity) {
            set_error("output holds %lld rows, %lld required", (long long)capacity, (long long)m);
            return VS_E_CAPACITY;
        }
        if (m > 0) {
            export_copy_kernel<<<grid_of(export_copy_kernel, m), 256, 0, s>>>(kl, kr, ksrc, m, d_out_left,
                                                                              d_out_right, d_out_src);
            VS_LAUNCHED("export_copy", s);
        }
        VS_CUDA_TRY(cudaStreamSynchronize(s));
        return VS_OK;
    }
    // 2. the driving side: left rows, or right rows (pairs re-sorted by (right, left))
    const bool right = how == VS_HOW_RIGHT;
    const int32_t* drive = right ? kr : kl;
    const int32_t* other = right ? kl : kr;
    const int64_t n_drive = right ? n_right : n_left;
    Scratch<uint64_t> rkeys;
    Scratch<uint32_t> perm;
    if (right && m > 1) {
        VS_TRY(rkeys.alloc((size_t)m, s));
        VS_TRY(perm.alloc((size_t)m, s));
        export_right_keys_kernel<<<grid_of(export_right_keys_kernel, m), 256, 0, s>>>(kl, kr, m, rkeys.p, perm.p);
        VS_LAUNCHED("export_right_keys", s);
        VS_TRY(radix_sort_u64_u32(rkeys.p, perm.p, m, 64, s));
    }
    const uint32_t* p_perm = right && m > 1 ? perm.p : nullptr;
    // 3. counts per driving row, tile sums and their scan
    const size_t nd = (size_t)(n_drive > 0 ? n_drive : 1);
    const int64_t n_tiles = (n_drive + kTileRows - 1) / kTileRows;
    Scratch<uint32_t> cnt;
    Scratch<uint64_t> tile_sum, tile_off, body_total;
    VS_TRY(cnt.alloc(nd, s));
    VS_TRY(tile_sum.alloc((size_t)(n_tiles > 0 ? n_tiles : 1), s));
    VS_TRY(tile_off.alloc((size_t)(n_tiles > 0 ? n_tiles : 1), s));
    VS_TRY(body_total.alloc(1, s));
    VS_CUDA_TRY(cudaMemsetAsync(cnt.p, 0, nd * sizeof(uint32_t), s));
    VS_CUDA_TRY(cudaMemsetAsync(body_total.p, 0, sizeof(uint64_t), s));
    if (m > 0) {
        export_count_kernel<<<grid_of(export_count_kernel, m), 256, 0, s>>>(drive, p_perm, m, cnt.p);
        VS_LAUNCHED("export_count", s);
    }
    if (n_tiles > 0) {
        export_tile_sum_kernel<<<(unsigned)n_tiles, kTileThreads, 0, s>>>(cnt.p, n_drive, tile_sum.p);
        VS_LAUNCHED("export_tile_sum", s);
        VS_TRY(exclusive_scan_u64(tile_sum.p, tile_off.p, n_tiles, body_total.p, s));
    }
    // 4. outer: right rows no pair reaches
    Scratch<uint32_t> missing, mpos;
    if (how == VS_HOW_OUTER && n_right > 0) {
        const size_t nr = (size_t)(n_right > 0 ? n_right : 1);
        VS_TRY(missing.alloc(nr, s));
        VS_TRY(mpos.alloc(nr, s));
        VS_CUDA_TRY(cudaMemsetAsync(missing.p, 0, nr * sizeof(uint32_t), s));
        if (m > 0) {
            export_mark_kernel<<<grid_of(export_mark_kernel, m), 256, 0, s>>>(kr, m, missing.p);
            VS_LAUNCHED("export_mark", s);
        }
        export_flip_kernel<<<grid_of(export_flip_kernel, n_right), 256, 0, s>>>(missing.p, n_right);
        VS_LAUNCHED("export_flip", s);
        VS_TRY(exclusive_scan_u32(missing.p, mpos.p, n_right, totals.p + 2, s));
    }
    uint64_t packed = 0;
    uint32_t appended = 0;
    VS_CUDA_TRY(cudaMemcpyAsync(&packed, body_total.p, sizeof(packed), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaMemcpyAsync(&appended, totals.p + 2, sizeof(appended), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    const int64_t body = (int64_t)(uint32_t)packed + (int64_t)(packed >> 32);
    const int64_t total = body + (how == VS_HOW_OUTER && n_right > 0 ? (int64_t)appended : 0);
    *n_out = total;
    if (total > capacity) {
        set_error("output holds %lld rows, %lld required", (long long)capacity, (long long)total);
        return VS_E_CAPACITY;
    }
    int64_t* o_drive = right ? d_out_right : d_out_left;
    int64_t* o_other = right ? d_out_left : d_out_right;
    if (n_tiles > 0) {
        export_write_kernel<<<(unsigned)n_tiles, kTileThreads, 0, s>>>(cnt.p, n_drive, tile_off.p, other, p_perm,
                                                                       ksrc, o_drive, o_other, d_out_src);
        VS_LAUNCHED("export_write", s);
    }
    if (how == VS_HOW_OUTER && n_right > 0) {
        export_append_kernel<<<grid_of(export_append_kernel, n_right), 256, 0, s>>>(
            missing.p, mpos.p, n_right, body, d_out_left, d_out_right, d_out_src);
        VS_LAUNCHED("export_append", s);
    }
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    return VS_OK;
}

}  // extern "C"
