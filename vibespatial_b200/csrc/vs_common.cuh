// Shared definitions for the vsjoin CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/vsjoin.h"

namespace vs {

// Thread-local last-error message, exported through vs_last_error().
void set_error(const char* fmt, ...);

// Make `device` current (VS_OK or VS_E_CUDA).
int use_device(int device);
// Argument checks shared by the entry points (VS_OK or VS_E_ARG).
int check_points(const vs_points* p);
int check_polygons(const vs_polygons* p);

// Pinned host words of a context (read-back of the device counters and of
// per-call extras).
constexpr int kHostCounters = 16;
constexpr int kDevCounters = 16;
constexpr int kWorkCounter = 8;

#define VS_CUDA_TRY(expr)                                                        \
    do {                                                                         \
        cudaError_t _e = (expr);                                                 \
        if (_e != cudaSuccess) {                                                 \
            ::vs::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), \
                            __FILE__, __LINE__);                                 \
            return VS_E_CUDA;                                                    \
        }                                                                        \
    } while (0)

// Kernels this thread has enqueued (every launch site ends in VS_LAUNCHED);
// entry points report the difference as vs_join_stats.kernel_launches.
extern thread_local long long g_launches;

// After a kernel launch: count it and report launch errors.  Debug builds compiled with
// -DVS_DEBUG_SYNC also wait for the kernel and name it in the error message.
#ifdef VS_DEBUG_SYNC
#define VS_LAUNCHED(name, stream)                                                        \
    do {                                                                                 \
        ++::vs::g_launches;                                                              \
        cudaError_t _e = cudaGetLastError();                                             \
        if (_e == cudaSuccess) _e = cudaStreamSynchronize(stream);                       \
        if (_e != cudaSuccess) {                                                         \
            ::vs::set_error("kernel %s failed: %s", name, cudaGetErrorString(_e));       \
            return VS_E_CUDA;                                                            \
        }                                                                                \
    } while (0)
#else
#define VS_LAUNCHED(name, stream) \
    do {                          \
        ++::vs::g_launches;       \
        VS_CUDA_TRY(cudaGetLastError()); \
    } while (0)
#endif

#define VS_TRY(expr)                 \
    do {                             \
        int _s = (expr);             \
        if (_s != VS_OK) return _s;  \
    } while (0)

constexpr int kNumSMs = 148;  // B200: 2 dies x 74 SMs

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// Grid size for a grid-stride kernel: a multiple of the SM count, at most
// enough blocks to cover n items once.
inline int grid_for(int64_t n, int block, int per_sm = 8) {
    int64_t need = (n + block - 1) / block;
    int64_t cap = (int64_t)kNumSMs * per_sm;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

// Grid for a grid-stride kernel: at most one full wave of resident blocks
// (blocks per SM from the occupancy calculator x SMs), so no partial second
// wave runs on a fraction of the SMs.
template <class Kernel>
int resident_grid(Kernel kernel, int64_t n_items, int block, size_t smem = 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, smem) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    int64_t need = (n_items + block - 1) / block;
    const int64_t cap = (int64_t)kNumSMs * per_sm;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

// Order-preserving map from double to int64 so atomicMin/atomicMax on
// long long order doubles correctly (NaN excluded by the callers).
__device__ __forceinline__ long long dbl_to_ordered(double v) {
    long long i = __double_as_longlong(v);
    return i >= 0 ? i : (i ^ 0x7fffffffffffffffLL);
}
__device__ __forceinline__ double ordered_to_dbl(long long i) {
    return __longlong_as_double(i >= 0 ? i : (i ^ 0x7fffffffffffffffLL));
}
inline long long host_dbl_to_ordered(double v) {
    long long i;
    static_assert(sizeof(i) == sizeof(v), "");
    __builtin_memcpy(&i, &v, sizeof(i));
    return i >= 0 ? i : (i ^ 0x7fffffffffffffffLL);
}

// Growable device scratch owned by a context; every allocation is stream
// ordered on the context stream.
struct Arena {
    void* base = nullptr;
    size_t cap = 0;
    size_t used = 0;
};

}  // namespace vs

// Axis-aligned box; an inverted box (min > max) contains nothing.
struct __align__(32) vs_box {
    double minx, miny, maxx, maxy;
};

namespace vs {
struct HostPipe;
}

// Opaque handles of the C-ABI.
struct vs_context {
    int device;
    cudaStream_t stream;
    bool owns_stream;
    vs::Arena arena;
    // Pinned host words (kHostCounters) used to read back counts.
    unsigned long long* h_counter;
    // Device counters (kDevCounters, zeroed at the start of every join):
    // [0] pair count, [1] exact-fallback count, [2] fp32-filter decided
    // edges, [3] edges sent past the fp32 filter, [4] error flags,
    // [5] candidate (bbox) count, [6] wide learned-index windows,
    // [7] deferred pairs, [8] work queue of the refine kernel.
    unsigned long long* d_counters;
    // Pairs deferred to the exact pass (grown on demand).
    int2* defer_buf;
    unsigned long long defer_cap;
    // Phase boundaries of one join (vs_join_stats.phase_ms): marks 0..4
    // around locate / group / refine / exact; recorded only while phase_on.
    cudaEvent_t phase_ev[5];
    bool phase_on;
    // Streams and double buffers of vs_join_host, kept between calls.
    vs::HostPipe* host_pipe;
};

namespace vs {
// Two events bracketing device work on a stream; ms() after both completed.
struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
    EventPair() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~EventPair() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
    EventPair(const EventPair&) = delete;
    EventPair& operator=(const EventPair&) = delete;
    float ms() {
        float t = 0.f;
        cudaEventElapsedTime(&t, a, b);
        return t;
    }
};
}  // namespace vs

// Record phase boundary k of the current join on the context stream.
inline void phase_mark(vs_context* ctx, int k) {
    if (ctx->phase_on) cudaEventRecord(ctx->phase_ev[k], ctx->stream);
}
