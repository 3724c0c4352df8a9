// Block-buffered pair emission shared by the join kernels.
//
// Accepted pairs go to a shared-memory buffer (shared atomics); once per block
// iteration the block reserves one contiguous range of the output with a
// single global atomic and copies the buffer out coalesced.  When the buffer
// is full a pair is written directly.  Writes beyond `capacity` are dropped
// but still counted, so the host learns the exact size it needs.  This
// replaces the reference's count pass -> exclusive_sum -> host fence ->
// scatter pass (src/vibespatial/spatial/spatial_index_device.py:975-1017).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace vs {

constexpr int kOutBuf = 1024;  // pairs buffered per block iteration

struct PairSink {
    int32_t* out_left;
    int32_t* out_right;
    unsigned long long capacity;
    unsigned long long* counter;  // global pair counter
};

struct BlockOut {
    int2* buf;
    unsigned* cnt;
};

__device__ __forceinline__ void emit(const BlockOut& o, const PairSink& k, int32_t l, int32_t r) {
    const unsigned pos = atomicAdd(o.cnt, 1u);
    if (pos < (unsigned)kOutBuf) {
        o.buf[pos] = make_int2(l, r);
    } else {
        const unsigned long long gp = atomicAdd(k.counter, 1ull);
        if (gp < k.capacity) {
            k.out_left[gp] = l;
            k.out_right[gp] = r;
        }
    }
}

// Every thread of the block must call flush (it synchronises the block).
__device__ __forceinline__ void flush(const BlockOut& o, const PairSink& k, unsigned long long* s_base, unsigned* s_n) {
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned c = *o.cnt < (unsigned)kOutBuf ? *o.cnt : (unsigned)kOutBuf;
        *s_n = c;
        *s_base = c ? atomicAdd(k.counter, (unsigned long long)c) : 0ull;
        *o.cnt = 0;
    }
    __syncthreads();
    const unsigned c = *s_n;
    const unsigned long long b = *s_base;
    for (unsigned i = threadIdx.x; i < c; i += blockDim.x) {
        const unsigned long long gp = b + i;
        if (gp < k.capacity) {
            const int2 v = o.buf[i];
            k.out_left[gp] = v.x;
            k.out_right[gp] = v.y;
        }
    }
    __syncthreads();
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// counters layout (see vs_context): [1] exact fallbacks, [2] fp32 edges,
// [3] fp64 edges, [5] candidates, [6] rmi window misses
__device__ __forceinline__ void add_counter(unsigned long long* counters, int slot, unsigned long long v) {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(&counters[slot], v);
}

}  // namespace vs
