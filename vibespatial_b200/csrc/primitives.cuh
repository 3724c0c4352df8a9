// In-house device primitives (scan, radix sort) and stream-ordered scratch.
//
// The reference calls CCCL for these (exclusive_sum, radix sort_pairs,
// select, lower/upper_bound: src/vibespatial/cuda/cccl_primitives.py:523-1167);
// the build forbids CCCL/CUB on the hot path, so they are written here.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "vs_common.cuh"

namespace vs {

// Stream-ordered scratch buffer (cudaMallocAsync / cudaFreeAsync on the
// context stream; the device pool keeps freed blocks, so steady-state calls do
// not reach the driver).
template <class T>
struct Scratch {
    T* p = nullptr;
    cudaStream_t s = nullptr;
    Scratch() = default;
    Scratch(const Scratch&) = delete;
    Scratch& operator=(const Scratch&) = delete;
    int alloc(size_t n, cudaStream_t stream) {
        release();
        s = stream;
        if (n == 0) n = 1;
        cudaError_t e = cudaMallocAsync((void**)&p, n * sizeof(T), stream);
        if (e != cudaSuccess) {
            p = nullptr;
            set_error("cudaMallocAsync(%zu bytes) failed: %s", n * sizeof(T), cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? VS_E_OOM : VS_E_CUDA;
        }
        return VS_OK;
    }
    void release() {
        if (p) cudaFreeAsync(p, s);
        p = nullptr;
    }
    T* release_ownership() {
        T* q = p;
        p = nullptr;
        return q;
    }
    ~Scratch() { release(); }
};

// out[i] = sum(in[0..i)), n items; in == out allowed.  If d_total is non-null
// it receives sum(in[0..n)).
int exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* d_total, cudaStream_t s);
int exclusive_scan_u64(const uint64_t* in, uint64_t* out, int64_t n, uint64_t* d_total, cudaStream_t s);

// Stable LSD radix sort of (key, value) pairs by key bits [begin_bit,
// key_bits) (8 bits per pass).  Sorted data ends in keys / vals.
int radix_sort_u64_u32(uint64_t* keys, uint32_t* vals, int64_t n, int key_bits, cudaStream_t s, int begin_bit = 0);
int radix_sort_u32_u32(uint32_t* keys, uint32_t* vals, int64_t n, int key_bits, cudaStream_t s, int begin_bit = 0);

}  // namespace vs
