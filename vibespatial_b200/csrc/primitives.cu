// Exclusive scan (reduce -> scan of block sums -> downsweep) and a stable
// LSD radix sort of (u32/u64 key, u32 value) pairs, 8 bits per pass.
//
// Radix sort per pass: (1) per-tile digit histograms with shared atomics,
// written digit-major so that one exclusive scan over [digit][tile] gives
// every (digit, tile) its global output offset; (2) a scatter that loads the
// tile into registers, ranks each key stably with __match_any_sync (peers with
// the same digit in a warp) plus per-warp digit counts scanned in shared
// memory, sorts the tile by digit in shared memory and then writes each
// digit's run contiguously (coalesced), as in one-sweep radix sorts.
#include <cuda_runtime.h>
#include <stdint.h>

#include "primitives.cuh"

namespace vs {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <class T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread.
template <class T>
__device__ __forceinline__ void block_exclusive_scan(T v, T& excl) {
    __shared__ T warp_tot[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T inc = warp_inclusive_scan(v);
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        T w = lane < kScanThreads / 32 ? warp_tot[lane] : T(0);
        T wi = warp_inclusive_scan(w);
        if (lane < kScanThreads / 32) warp_tot[lane] = wi - w;
    }
    __syncthreads();
    excl = warp_tot[warp] + inc - v;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const T* __restrict__ in, int64_t n,
                                                                   T* __restrict__ sums) {
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    T acc = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
        if (i < n) acc += in[i];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ T ws[kScanThreads / 32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        T t = 0;
        for (int w = 0; w < kScanThreads / 32; ++w) t += ws[w];
        sums[blockIdx.x] = t;
    }
}

// Each thread owns kScanItems consecutive items.
template <class T>
__global__ void __launch_bounds__(kScanThreads) scan_downsweep_kernel(const T* in, T* out, int64_t n,
                                                                      const T* __restrict__ offsets,
                                                                      T* __restrict__ d_total) {
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    T v[kScanItems];
    T local = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        v[k] = i < n ? in[i] : T(0);
        local += v[k];
    }
    T excl;
    block_exclusive_scan<T>(local, excl);
    T run = excl + (offsets ? offsets[blockIdx.x] : T(0));
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k;
        if (i < n) out[i] = run;
        run += v[k];
        if (d_total && i == n - 1) *d_total = run;
    }
}

template <class T>
int exclusive_scan_impl(const T* in, T* out, int64_t n, T* d_total, cudaStream_t s) {
    if (n <= 0) {
        if (d_total) VS_CUDA_TRY(cudaMemsetAsync(d_total, 0, sizeof(T), s));
        return VS_OK;
    }
    const int64_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb > 0x7fffffff) {
        set_error("scan too large (%lld items)", (long long)n);
        return VS_E_ARG;
    }
    if (nb == 1) {
        scan_downsweep_kernel<T><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, d_total);
        VS_LAUNCHED("scan_downsweep", s);
        return VS_OK;
    }
    Scratch<T> sums;
    VS_TRY(sums.alloc((size_t)nb, s));
    scan_reduce_kernel<T><<<(unsigned)nb, kScanThreads, 0, s>>>(in, n, sums.p);
    VS_LAUNCHED("scan_reduce", s);
    VS_TRY(exclusive_scan_impl<T>(sums.p, sums.p, nb, (T*)nullptr, s));
    scan_downsweep_kernel<T><<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, n, sums.p, d_total);
    VS_LAUNCHED("scan_downsweep", s);
    return VS_OK;
}

// ------------------------------------------------------------------------
// Radix sort
// ------------------------------------------------------------------------
constexpr int kRsThreads = 256;
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRadix = 256;
// 16 keys per thread for 32-bit keys, 8 for 64-bit keys (keeps the tile's
// shared-memory staging under 48 KB).
template <class K>
struct RsTile {
    static constexpr int kRounds = sizeof(K) == 8 ? 8 : 16;
    static constexpr int kTile = kRsThreads * kRounds;
};

template <class K>
__global__ void __launch_bounds__(kRsThreads) rs_histogram_kernel(const K* __restrict__ keys, int64_t n, int shift,
                                                                  uint32_t* __restrict__ hist, int ntiles) {
    __shared__ uint32_t h[kRadix];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * RsTile<K>::kTile;
#pragma unroll 4
    for (int r = 0; r < RsTile<K>::kRounds; ++r) {
        const int64_t i = base + (int64_t)r * kRsThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(unsigned)(keys[i] >> shift) & 0xffu], 1u);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one tile: the tile is ranked and sorted by digit in
// shared memory first, then written out in digit runs so that consecutive
// threads write consecutive addresses.
template <class K>
__global__ void __launch_bounds__(kRsThreads) rs_scatter_kernel(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                                K* __restrict__ kout, uint32_t* __restrict__ vout,
                                                                int64_t n, int shift,
                                                                const uint32_t* __restrict__ offsets, int ntiles) {
    constexpr int R = RsTile<K>::kRounds;
    constexpr int T = RsTile<K>::kTile;
    __shared__ uint32_t gbase[kRadix];   // global start of (digit, this tile)
    __shared__ uint32_t lstart[kRadix];  // tile-local start of digit
    __shared__ uint32_t run[kRadix];     // keys of digit placed by earlier rounds
    __shared__ uint32_t wcnt[kRsWarps][kRadix];
    __shared__ uint32_t wsum[kRsWarps];
    __shared__ K skey[T];
    __shared__ uint32_t sval[T];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int64_t tile0 = (int64_t)blockIdx.x * T;
    const int count = (int)((n - tile0) < T ? (n - tile0) : T);

    K k[R];
    uint32_t v[R];
    unsigned d[R];
    lstart[tid] = 0;
#pragma unroll
    for (int w = 0; w < kRsWarps; ++w) wcnt[w][tid] = 0;
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int j = r * kRsThreads + tid;
        d[r] = kRadix;
        if (j < count) {
            k[r] = kin[tile0 + j];
            v[r] = vin[tile0 + j];
            d[r] = (unsigned)(k[r] >> shift) & 0xffu;
            atomicAdd(&lstart[d[r]], 1u);
        }
    }
    __syncthreads();
    // exclusive scan of the tile's digit counts (256 entries, one per thread)
    {
        const uint32_t c = lstart[tid];
        uint32_t inc = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += t;
        }
        if (lane == 31) wsum[warp] = inc;
        __syncthreads();
        uint32_t wpre = 0;
        for (int w = 0; w < warp; ++w) wpre += wsum[w];
        lstart[tid] = wpre + inc - c;
        gbase[tid] = offsets[(int64_t)tid * ntiles + blockIdx.x];
        run[tid] = 0;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const unsigned dd = d[r];
        const unsigned peers = __match_any_sync(0xffffffffu, dd);
        const unsigned rank = __popc(peers & lt_mask);
        if (dd < kRadix && (__ffs(peers) - 1) == lane) wcnt[warp][dd] = __popc(peers);
        __syncthreads();
        uint32_t acc = 0;
#pragma unroll
        for (int w = 0; w < kRsWarps; ++w) {
            const uint32_t c = wcnt[w][tid];
            wcnt[w][tid] = acc;
            acc += c;
        }
        __syncthreads();
        if (dd < kRadix) {
            const uint32_t pos = lstart[dd] + run[dd] + wcnt[warp][dd] + rank;
            skey[pos] = k[r];
            sval[pos] = v[r];
        }
        __syncthreads();
        run[tid] += acc;
#pragma unroll
        for (int w = 0; w < kRsWarps; ++w) wcnt[w][tid] = 0;
        __syncthreads();
    }
    for (int j = tid; j < count; j += kRsThreads) {
        const K key = skey[j];
        const unsigned dd = (unsigned)(key >> shift) & 0xffu;
        const uint32_t pos = gbase[dd] + (uint32_t)j - lstart[dd];
        kout[pos] = key;
        vout[pos] = sval[j];
    }
}

template <class K>
int radix_sort_impl(K* keys, uint32_t* vals, int64_t n, int begin_bit, int end_bit, cudaStream_t s) {
    if (n <= 1) return VS_OK;
    if (n > 0xffffffffLL) {
        set_error("radix sort supports at most 2^32-1 items (got %lld)", (long long)n);
        return VS_E_ARG;
    }
    const int max_bits = (int)(8 * sizeof(K));
    if (end_bit <= 0 || end_bit > max_bits) end_bit = max_bits;
    if (begin_bit < 0 || begin_bit >= end_bit) begin_bit = 0;
    const int passes = (end_bit - begin_bit + 7) / 8;
    constexpr int T = RsTile<K>::kTile;
    const int ntiles = (int)((n + T - 1) / T);
    Scratch<K> kalt;
    Scratch<uint32_t> valt, hist;
    VS_TRY(kalt.alloc((size_t)n, s));
    VS_TRY(valt.alloc((size_t)n, s));
    VS_TRY(hist.alloc((size_t)kRadix * ntiles, s));
    K* ka = keys;
    uint32_t* va = vals;
    K* kb = kalt.p;
    uint32_t* vb = valt.p;
    for (int p = 0; p < passes; ++p) {
        // the last pass may overlap the previous one's bits: it still sorts stably
        int shift = begin_bit + 8 * p;
        if (shift + 8 > max_bits) shift = max_bits - 8;
        rs_histogram_kernel<K><<<ntiles, kRsThreads, 0, s>>>(ka, n, shift, hist.p, ntiles);
        VS_LAUNCHED("rs_histogram", s);
        VS_TRY(exclusive_scan_u32(hist.p, hist.p, (int64_t)kRadix * ntiles, nullptr, s));
        rs_scatter_kernel<K><<<ntiles, kRsThreads, 0, s>>>(ka, va, kb, vb, n, shift, hist.p, ntiles);
        VS_LAUNCHED("rs_scatter", s);
        K* tk = ka;
        ka = kb;
        kb = tk;
        uint32_t* tv = va;
        va = vb;
        vb = tv;
    }
    if (ka != keys) {
        VS_CUDA_TRY(cudaMemcpyAsync(keys, ka, (size_t)n * sizeof(K), cudaMemcpyDeviceToDevice, s));
        VS_CUDA_TRY(cudaMemcpyAsync(vals, va, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    }
    return VS_OK;
}

}  // namespace

int exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* d_total, cudaStream_t s) {
    return exclusive_scan_impl<uint32_t>(in, out, n, d_total, s);
}
int exclusive_scan_u64(const uint64_t* in, uint64_t* out, int64_t n, uint64_t* d_total, cudaStream_t s) {
    return exclusive_scan_impl<uint64_t>(in, out, n, d_total, s);
}

int radix_sort_u64_u32(uint64_t* keys, uint32_t* vals, int64_t n, int key_bits, cudaStream_t s, int begin_bit) {
    return radix_sort_impl<uint64_t>(keys, vals, n, begin_bit, key_bits, s);
}

int radix_sort_u32_u32(uint32_t* keys, uint32_t* vals, int64_t n, int key_bits, cudaStream_t s, int begin_bit) {
    return radix_sort_impl<uint32_t>(keys, vals, n, begin_bit, key_bits, s);
}

}  // namespace vs
