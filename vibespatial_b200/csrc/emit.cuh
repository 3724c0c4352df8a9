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

// ---------------------------------------------------------------------------
// Warp-private buffering: the same idea without block barriers, so a warp
// that finishes early never waits for the slowest warp of its block.
// ---------------------------------------------------------------------------
constexpr int kWarpBuf = 128;  // pairs buffered per warp

struct WarpOut {
    int2* buf;
    unsigned* cnt;
};

// Copy `c` buffered pairs out with one global atomic.  Whole warp, converged.
__device__ __forceinline__ void wdrain(const WarpOut& o, const PairSink& k, unsigned c) {
    const int lane = threadIdx.x & 31;
    unsigned long long b = 0;
    if (lane == 0 && c) b = atomicAdd(k.counter, (unsigned long long)c);
    b = __shfl_sync(0xffffffffu, b, 0);
    for (unsigned j = lane; j < c; j += 32) {
        const unsigned long long gp = b + j;
        if (gp < k.capacity) {
            const int2 v = o.buf[j];
            k.out_left[gp] = v.x;
            k.out_right[gp] = v.y;
        }
    }
    __syncwarp();
}

// Warp-synchronous emission: every lane of the warp calls it at a converged
// point; the lanes with `want` set append (l, r).  Positions come from a
// ballot, so the buffer count is only ever written by lane 0 between
// __syncwarp()s and there are no shared-memory atomics in divergent code.
__device__ __forceinline__ void wemit_sync(const WarpOut& o, const PairSink& k, bool want, int32_t l, int32_t r) {
    const unsigned m = __ballot_sync(0xffffffffu, want);
    if (m == 0u) return;
    const int lane = threadIdx.x & 31;
    unsigned base = *o.cnt;
    const unsigned add = (unsigned)__popc(m);
    if (base + add > (unsigned)kWarpBuf) {
        wdrain(o, k, base);
        base = 0;
    }
    if (want) o.buf[base + (unsigned)__popc(m & ((1u << lane) - 1u))] = make_int2(l, r);
    __syncwarp();
    if (lane == 0) *o.cnt = base + add;
    __syncwarp();
}

// Call with the whole warp converged.  Drains when at least half full, or
// always when `force`.
__device__ __forceinline__ void wflush(const WarpOut& o, const PairSink& k, bool force) {
    __syncwarp();
    const unsigned c = *o.cnt;
    if (c == 0u || (!force && c < (unsigned)(kWarpBuf / 2))) return;
    wdrain(o, k, c);
    if ((threadIdx.x & 31) == 0) *o.cnt = 0;
    __syncwarp();
}

// Pairs whose location the filters could not certify; resolved exactly by a
// separate pass.  Entries beyond `capacity` are counted, not stored, and the
// host re-runs the join with a larger buffer.
struct DeferSink {
    int2* buf;                    // (point row, polygon slot)
    unsigned long long capacity;
    unsigned long long* counter;
};

__device__ __forceinline__ void defer(const DeferSink& d, int32_t row, int32_t slot) {
    const unsigned long long p = atomicAdd(d.counter, 1ull);
    if (p < d.capacity) d.buf[p] = make_int2(row, slot);
}

// Warp-level dynamic work queue: lane 0 takes `grab` consecutive items from
// *counter and the first one is broadcast to the warp (>= the item count
// once the queue is drained).  Warps that finish early keep taking work, so
// uneven per-item costs do not leave SMs idle at the end of a launch.
__device__ __forceinline__ int64_t warp_grab(unsigned long long* counter, int64_t grab) {
    unsigned long long b = 0;
    if ((threadIdx.x & 31) == 0) b = atomicAdd(counter, (unsigned long long)grab);
    return (int64_t)__shfl_sync(0xffffffffu, b, 0);
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
