// Row reductions of a join's pairs on the device: the relation flow of the
// index (match counts, semijoin / antijoin row sets, per-row sums, pairs
// shared by two relations) without exporting the pairs.
//
// The reference's native index reduces its relation pairs inside its own
// carriers (sindex.query_left_semijoin / query_left_antijoin /
// query_right_semijoin / query_left_match_count_expression and
// query_pair_aggregate, src/vibespatial/api/sindex.py:973, 1592-1760); here
// the pairs are the int32 device arrays the join wrote, and each reduction is
// one or two kernels plus the in-house scan.
#include <cuda_runtime.h>
#include <stdint.h>

#include "primitives.cuh"
#include "vs_common.cuh"

namespace vs {
namespace {

constexpr int kRThreads = 256;

// counts[r] += occurrences of r in rows, over the pairs whose mask byte is
// set when a mask is given (warp-aggregated increments: the rows
// of a join's pairs come sorted, so neighbouring lanes mostly share a row).
// Rows outside [0, n_rows) set *bad.
__global__ void row_count_kernel(const int32_t* __restrict__ rows, const uint8_t* __restrict__ mask, int64_t n,
                                 int64_t n_rows, unsigned long long* __restrict__ counts, unsigned* __restrict__ bad) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // warp-uniform loop so the whole warp reaches the match
    for (int64_t base = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) & ~(int64_t)31; base < n; base += stride) {
        const int64_t k = base + lane;
        int r = -1;
        if (k < n && (mask == nullptr || mask[k] != 0)) {
            r = rows[k];
            if (r < 0 || r >= n_rows) {
                atomicOr(bad, 1u);
                r = -1;
            }
        }
        const unsigned peers = __match_any_sync(0xffffffffu, r);
        if (r >= 0 && (peers & lt) == 0) atomicAdd(&counts[r], (unsigned long long)__popc(peers));
    }
}

// flag[k] = 1 where rows[k] < rows[k - 1] (rows must ascend for the sums).
__global__ void descent_kernel(const int32_t* __restrict__ rows, int64_t n, unsigned* __restrict__ bad) {
    for (int64_t k = 1 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        if (rows[k] < rows[k - 1]) atomicOr(bad, 2u);
}

// Thread per row: the row's pairs are the contiguous run [off[r], off[r+1])
// of ascending rows; their values are summed in pair order, the order in
// which numpy's bincount(weights=...) accumulates, so the sums match it bit
// for bit.  cols outside [0, n_values) set *bad.
__global__ void row_sum_kernel(const uint64_t* __restrict__ off, int64_t n_rows, const int32_t* __restrict__ cols,
                               const double* __restrict__ values, int64_t n_values, double* __restrict__ sums,
                               unsigned* __restrict__ bad) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (uint64_t k = off[r]; k < off[r + 1]; ++k) {
            const int32_t c = cols[k];
            if (c < 0 || c >= n_values) {
                atomicOr(bad, 4u);
                continue;
            }
            acc = __dadd_rn(acc, values[c]);
        }
        sums[r] = acc;
    }
}

// keep[r] = (counts[r] > 0) == want_matched
__global__ void keep_kernel(const unsigned long long* __restrict__ counts, int64_t n_rows, int want_matched,
                            uint32_t* __restrict__ keep) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * blockDim.x)
        keep[r] = ((counts[r] > 0ull) == (want_matched != 0)) ? 1u : 0u;
}

__global__ void select_kernel(const uint32_t* __restrict__ keep, const uint32_t* __restrict__ pos, int64_t n_rows,
                              int32_t* __restrict__ out) {
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_rows; r += (int64_t)gridDim.x * blockDim.x)
        if (keep[r]) out[pos[r]] = (int32_t)r;
}

// Sets *bad when b is not sorted by (left, right).
__global__ void pair_order_kernel(const int32_t* __restrict__ bl, const int32_t* __restrict__ br, int64_t n,
                                  unsigned* __restrict__ bad) {
    for (int64_t k = 1 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
        if (bl[k] < bl[k - 1] || (bl[k] == bl[k - 1] && br[k] < br[k - 1])) atomicOr(bad, 2u);
}

// flags[k] = 1 when pair (a_left[k], a_right[k]) is one of b's pairs; b is
// sorted by (left, right), and b_off[l] .. b_off[l+1] is left row l's run in
// it, which is binary-searched for the right row.
__global__ void member_kernel(const int32_t* __restrict__ al, const int32_t* __restrict__ ar, int64_t n_a,
                              const int32_t* __restrict__ br, const uint64_t* __restrict__ b_off, int64_t n_left,
                              uint8_t* __restrict__ flags, unsigned* __restrict__ bad) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_a; k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t l = al[k], r = ar[k];
        uint8_t hit = 0;
        if (l < 0 || l >= n_left) {
            atomicOr(bad, 1u);
        } else {
            uint64_t lo = b_off[l], hi = b_off[l + 1];
            while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if (br[mid] < r) lo = mid + 1;
                else hi = mid;
            }
            hit = (lo < b_off[l + 1] && br[lo] == r) ? 1 : 0;
        }
        flags[k] = hit;
    }
}

int check_rows_args(vs_context* ctx, const void* d_rows, int64_t n_pairs, int64_t n_rows) {
    if (!ctx) {
        set_error("ctx is NULL");
        return VS_E_ARG;
    }
    if (n_pairs < 0 || n_rows < 0 || n_rows > 0x7fffffffLL || (n_pairs > 0 && !d_rows)) {
        set_error("invalid pair or row counts (n_pairs %lld, n_rows %lld)", (long long)n_pairs, (long long)n_rows);
        return VS_E_ARG;
    }
    return VS_OK;
}

// Counts of every row into d_counts (cleared first); checks the rows' range.
int count_rows(cudaStream_t s, const int32_t* rows, int64_t n, int64_t n_rows, unsigned long long* counts,
               unsigned* bad, const uint8_t* mask = nullptr) {
    VS_CUDA_TRY(cudaMemsetAsync(counts, 0, (size_t)(n_rows > 0 ? n_rows : 1) * sizeof(unsigned long long), s));
    if (n > 0) {
        row_count_kernel<<<grid_for(n, kRThreads), kRThreads, 0, s>>>(rows, mask, n, n_rows, counts, bad);
        VS_LAUNCHED("row_count", s);
    }
    return VS_OK;
}

int read_bad(cudaStream_t s, const unsigned* d_bad, unsigned* h_bad) {
    VS_CUDA_TRY(cudaMemcpyAsync(h_bad, d_bad, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    return VS_OK;
}

}  // namespace
}  // namespace vs

using namespace vs;

extern "C" int vs_row_counts(vs_context* ctx, const int32_t* d_rows, const uint8_t* d_mask, int64_t n_pairs,
                             int64_t n_rows, int64_t* d_counts) {
    VS_TRY(check_rows_args(ctx, d_rows, n_pairs, n_rows));
    if (n_rows > 0 && !d_counts) {
        set_error("d_counts is NULL");
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    if (n_rows == 0) return VS_OK;
    cudaStream_t s = ctx->stream;
    Scratch<unsigned> bad;
    VS_TRY(bad.alloc(1, s));
    VS_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(unsigned), s));
    VS_TRY(count_rows(s, d_rows, n_pairs, n_rows, reinterpret_cast<unsigned long long*>(d_counts), bad.p, d_mask));
    unsigned h = 0;
    VS_TRY(read_bad(s, bad.p, &h));
    if (h) {
        set_error("a pair row lies outside [0, %lld)", (long long)n_rows);
        return VS_E_ARG;
    }
    return VS_OK;
}

extern "C" int vs_row_sums(vs_context* ctx, const int32_t* d_rows, const int32_t* d_cols, int64_t n_pairs,
                           int64_t n_rows, const double* d_values, int64_t n_values, double* d_sums) {
    VS_TRY(check_rows_args(ctx, d_rows, n_pairs, n_rows));
    if ((n_pairs > 0 && (!d_cols || !d_values)) || (n_rows > 0 && !d_sums) || n_values < 0) {
        set_error("d_cols / d_values / d_sums is NULL or n_values is negative");
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    if (n_rows == 0) return VS_OK;
    cudaStream_t s = ctx->stream;
    Scratch<unsigned> bad;
    Scratch<unsigned long long> off;
    VS_TRY(bad.alloc(1, s));
    VS_TRY(off.alloc((size_t)n_rows + 1, s));
    VS_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(unsigned), s));
    VS_TRY(count_rows(s, d_rows, n_pairs, n_rows, off.p, bad.p));
    if (n_pairs > 1) {
        descent_kernel<<<grid_for(n_pairs, kRThreads), kRThreads, 0, s>>>(d_rows, n_pairs, bad.p);
        VS_LAUNCHED("row_descent", s);
    }
    VS_TRY(exclusive_scan_u64(reinterpret_cast<uint64_t*>(off.p), reinterpret_cast<uint64_t*>(off.p), n_rows,
                              reinterpret_cast<uint64_t*>(off.p) + n_rows, s));
    unsigned h = 0;
    VS_TRY(read_bad(s, bad.p, &h));  // nothing below runs on unchecked rows
    if (h & 1u) {
        set_error("a pair row lies outside [0, %lld)", (long long)n_rows);
        return VS_E_ARG;
    }
    if (h & 2u) {
        set_error("vs_row_sums needs the pairs sorted by row (ascending)");
        return VS_E_ARG;
    }
    row_sum_kernel<<<grid_for(n_rows, kRThreads), kRThreads, 0, s>>>(
        reinterpret_cast<const uint64_t*>(off.p), n_rows, d_cols, d_values, n_values, d_sums, bad.p);
    VS_LAUNCHED("row_sum", s);
    VS_TRY(read_bad(s, bad.p, &h));
    if (h & 4u) {
        set_error("a pair column lies outside [0, %lld)", (long long)n_values);
        return VS_E_ARG;
    }
    return VS_OK;
}

extern "C" int vs_select_rows(vs_context* ctx, const int64_t* d_counts, int64_t n_rows, int32_t matched,
                              int32_t* d_out, int64_t* n_out) {
    if (!ctx || !n_out || n_rows < 0 || n_rows > 0x7fffffffLL || (n_rows > 0 && (!d_counts || !d_out))) {
        set_error("invalid arguments (n_rows %lld)", (long long)n_rows);
        return VS_E_ARG;
    }
    *n_out = 0;
    VS_TRY(use_device(ctx->device));
    if (n_rows == 0) return VS_OK;
    cudaStream_t s = ctx->stream;
    Scratch<uint32_t> keep, pos;
    VS_TRY(keep.alloc((size_t)n_rows, s));
    VS_TRY(pos.alloc((size_t)n_rows + 1, s));
    keep_kernel<<<grid_for(n_rows, kRThreads), kRThreads, 0, s>>>(
        reinterpret_cast<const unsigned long long*>(d_counts), n_rows, matched, keep.p);
    VS_LAUNCHED("row_keep", s);
    VS_TRY(exclusive_scan_u32(keep.p, pos.p, n_rows, pos.p + n_rows, s));
    select_kernel<<<grid_for(n_rows, kRThreads), kRThreads, 0, s>>>(keep.p, pos.p, n_rows, d_out);
    VS_LAUNCHED("row_select", s);
    uint32_t total = 0;
    VS_CUDA_TRY(cudaMemcpyAsync(&total, pos.p + n_rows, sizeof(total), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    *n_out = (int64_t)total;
    return VS_OK;
}

extern "C" int vs_pairs_member(vs_context* ctx, const int32_t* d_a_left, const int32_t* d_a_right, int64_t n_a,
                               const int32_t* d_b_left, const int32_t* d_b_right, int64_t n_b, int64_t n_left_rows,
                               uint8_t* d_flags) {
    if (!ctx || n_a < 0 || n_b < 0 || n_left_rows < 0 || n_left_rows > 0x7fffffffLL ||
        (n_a > 0 && (!d_a_left || !d_a_right || !d_flags)) || (n_b > 0 && (!d_b_left || !d_b_right))) {
        set_error("invalid arguments (n_a %lld, n_b %lld, n_left_rows %lld)", (long long)n_a, (long long)n_b,
                  (long long)n_left_rows);
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    if (n_a == 0) return VS_OK;
    cudaStream_t s = ctx->stream;
    Scratch<unsigned> bad;
    Scratch<unsigned long long> off;
    VS_TRY(bad.alloc(1, s));
    VS_TRY(off.alloc((size_t)n_left_rows + 1, s));
    VS_CUDA_TRY(cudaMemsetAsync(bad.p, 0, sizeof(unsigned), s));
    VS_TRY(count_rows(s, d_b_left, n_b, n_left_rows, off.p, bad.p));
    if (n_b > 1) {
        pair_order_kernel<<<grid_for(n_b, kRThreads), kRThreads, 0, s>>>(d_b_left, d_b_right, n_b, bad.p);
        VS_LAUNCHED("pair_order", s);
    }
    VS_TRY(exclusive_scan_u64(reinterpret_cast<uint64_t*>(off.p), reinterpret_cast<uint64_t*>(off.p), n_left_rows,
                              reinterpret_cast<uint64_t*>(off.p) + n_left_rows, s));
    unsigned h = 0;
    VS_TRY(read_bad(s, bad.p, &h));
    if (h & 1u) {
        set_error("a pair of the second relation has a left row outside [0, %lld)", (long long)n_left_rows);
        return VS_E_ARG;
    }
    if (h & 2u) {
        set_error("vs_pairs_member needs the second relation's pairs sorted by (left, right)");
        return VS_E_ARG;
    }
    member_kernel<<<grid_for(n_a, kRThreads), kRThreads, 0, s>>>(d_a_left, d_a_right, n_a, d_b_right,
                                                                   reinterpret_cast<const uint64_t*>(off.p),
                                                                   n_left_rows, d_flags, bad.p);
    VS_LAUNCHED("pairs_member", s);
    VS_TRY(read_bad(s, bad.p, &h));
    if (h) {
        set_error("a pair of the first relation has a left row outside [0, %lld)", (long long)n_left_rows);
        return VS_E_ARG;
    }
    return VS_OK;
}
