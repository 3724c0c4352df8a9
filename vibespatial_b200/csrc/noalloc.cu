// vs_join_brute_noalloc: the brute-force point x polygon join with no device
// allocation at all, for callers that cannot allocate.
//
// Some hosts own every byte of device memory themselves: an engine that
// carves one fixed arena at start-up and forbids later cudaMalloc, or a
// process held to a hard memory budget that a hidden allocation would break.
// This entry point serves them: the caller passes inputs and the output pair
// buffers, and the only scratch the kernels need (one box per polygon and a
// pair counter) lives in a file-scope device array of fixed size, reserved
// when the library is loaded and held by every GPU that loads it until the
// process exits.
//
// Limits and rules:
//   * at most kNoAllocMaxPolygons (65,536) polygon rows; larger inputs are
//     rejected with VS_E_ARG before any device work;
//   * the scratch is shared by every call: concurrent calls whose kernels
//     overlap on the GPU (different streams, threads or processes sharing a
//     context) race on it and must be serialised by the caller; each call
//     clears the counter it needs before use;
//   * every call blocks the calling thread: it ends by copying the pair count
//     back to the host and waiting for `stream`;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current) and keeps it for the
//     life of the process; make that first call before any stream capture.
//     The address belongs to the device's primary context: call this entry
//     point with the primary context current (the CUDA runtime's default),
//     and not after cudaDeviceReset, which invalidates the kept address;
//   * a polygon's box spans its finite coordinates (fmin/fmax skip NaN), as
//     the index builder computes it; null and empty rows get a box that
//     contains nothing;
//   * pairs come back unordered (left = point row, right = polygon row).
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "emit.cuh"
#include "exact.cuh"
#include "vs_common.cuh"

namespace vs {
namespace {

constexpr int kNoAllocMaxPolygons = 65536;
constexpr size_t kNoAllocCounterBytes = 256;  // [0] pair counter, rest spare; keeps the boxes 256-B aligned
constexpr size_t kNoAllocScratchBytes = kNoAllocCounterBytes + sizeof(vs_box) * (size_t)kNoAllocMaxPolygons;

// The scratch (2 MiB + 256 B).  Host code must not use this name as an
// address: it is a host-side stand-in; the device address comes from
// cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

int scratch_address(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) {
        set_error("device ordinal %d outside [0, %d)", device, kMaxDevices);
        return VS_E_ARG;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) {
            set_error("cudaGetSymbolAddress(no-alloc scratch) failed on device %d: %s", device,
                      cudaGetErrorString(e));
            return VS_E_CUDA;
        }
        g_scratch_addr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[device];
    return VS_OK;
}

// One warp per polygon row: box of its coordinate span (null / empty rows get
// an inverted box that contains nothing).
__global__ void noalloc_bounds_kernel(vs_polygons p, vs_box* __restrict__ boxes) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t g = warp; g < p.n_geoms; g += nwarps) {
        const bool valid = p.d_valid == nullptr || p.d_valid[g] != 0;
        int32_t p0 = p.d_geom_off[g], p1 = p.d_geom_off[g + 1];
        if (!valid) p1 = p0;
        const int32_t c0 = p.d_ring_off[p.d_part_off[p0]], c1 = p.d_ring_off[p.d_part_off[p1]];
        double mnx = INFINITY, mny = INFINITY, mxx = -INFINITY, mxy = -INFINITY;
        for (int32_t c = c0 + lane; c < c1; c += 32) {
            mnx = fmin(mnx, p.d_x[c]);
            mny = fmin(mny, p.d_y[c]);
            mxx = fmax(mxx, p.d_x[c]);
            mxy = fmax(mxy, p.d_y[c]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mnx = fmin(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
            mny = fmin(mny, __shfl_xor_sync(0xffffffffu, mny, o));
            mxx = fmax(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
            mxy = fmax(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
        }
        if (lane == 0) {
            if (!(mnx <= mxx && mny <= mxy)) {
                mnx = mny = INFINITY;
                mxx = mxy = -INFINITY;
            }
            boxes[g] = vs_box{mnx, mny, mxx, mxy};
        }
    }
}

// Every point against every polygon box, exact location in line; points in a
// warp-uniform loop so emission is warp-synchronous.
__global__ void __launch_bounds__(256) noalloc_join_kernel(vs_points pts, vs_polygons polys,
                                                           const vs_box* __restrict__ boxes, int accept_mask,
                                                           PairSink sink) {
    __shared__ int2 s_buf[8][kWarpBuf];
    __shared__ unsigned s_cnt[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_cnt[warp] = 0;
    __syncwarp();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    const int64_t M = polys.n_geoms;
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = gw * 32; base < pts.n; base += nw * 32) {
        const int64_t i = base + lane;
        const bool act = i < pts.n && (pts.d_valid == nullptr || pts.d_valid[i]);
        const double x = act ? pts.d_x[i] : 0.0, y = act ? pts.d_y[i] : 0.0;
        for (int64_t g = 0; g < M; ++g) {  // the same trip count in every lane
            bool want = false;
            const vs_box b = boxes[g];
            if (act && x >= b.minx && x <= b.maxx && y >= b.miny && y <= b.maxy) {
                if (accept_mask == 0) {
                    want = true;
                } else {
                    unsigned n_exact = 0;
                    const int loc = geometry_location_soa(x, y, polys.d_x, polys.d_y, polys.d_ring_off,
                                                          polys.d_part_off, polys.d_geom_off, (int)g, n_exact);
                    want = (accept_mask >> loc) & 1;
                }
            }
            wemit_sync(out, sink, want, (int32_t)i, (int32_t)g);
        }
        wflush(out, sink, false);
    }
    wflush(out, sink, true);
}

}  // namespace

int accept_mask_for(int predicate, int* mask);

}  // namespace vs

using namespace vs;

extern "C" int vs_join_brute_noalloc(const vs_points* pts, const vs_polygons* polys, int32_t predicate,
                                     int32_t* d_left, int32_t* d_right, int64_t capacity, int64_t* n_pairs,
                                     void* stream) {
    if (!pts || !polys || !n_pairs) {
        set_error("points/polygons/n_pairs is NULL");
        return VS_E_ARG;
    }
    *n_pairs = 0;
    if (pts->n < 0 || pts->n > 0x7fffffffLL || polys->n_geoms < 0) {
        set_error("invalid input sizes");
        return VS_E_ARG;
    }
    if (polys->n_geoms > kNoAllocMaxPolygons) {
        set_error("vs_join_brute_noalloc takes at most %d polygons (got %d): its scratch is a fixed %zu-byte "
                  "device array",
                  kNoAllocMaxPolygons, polys->n_geoms, kNoAllocScratchBytes);
        return VS_E_ARG;
    }
    if (capacity < 0 || (capacity > 0 && (!d_left || !d_right))) {
        set_error("invalid pair buffers (capacity %lld)", (long long)capacity);
        return VS_E_ARG;
    }
    if ((pts->n > 0 && (!pts->d_x || !pts->d_y)) ||
        (polys->n_geoms > 0 && (!polys->d_geom_off || !polys->d_part_off || !polys->d_ring_off)) ||
        (polys->n_coords > 0 && (!polys->d_x || !polys->d_y))) {
        set_error("input buffers must not be NULL");
        return VS_E_ARG;
    }
    int mask = 0;
    VS_TRY(accept_mask_for(predicate, &mask));
    if (pts->n == 0 || polys->n_geoms == 0) return VS_OK;
    int device = 0;
    VS_CUDA_TRY(cudaGetDevice(&device));
    unsigned char* scratch = nullptr;
    VS_TRY(scratch_address(device, &scratch));
    unsigned long long* counter = reinterpret_cast<unsigned long long*>(scratch);
    vs_box* boxes = reinterpret_cast<vs_box*>(scratch + kNoAllocCounterBytes);
    cudaStream_t s = (cudaStream_t)stream;
    VS_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s));
    noalloc_bounds_kernel<<<grid_for((int64_t)polys->n_geoms * 32, 256), 256, 0, s>>>(*polys, boxes);
    VS_LAUNCHED("noalloc_bounds", s);
    const PairSink sink{d_left, d_right, (unsigned long long)capacity, counter};
    noalloc_join_kernel<<<grid_for(pts->n, 256, 8), 256, 0, s>>>(*pts, *polys, boxes, mask, sink);
    VS_LAUNCHED("noalloc_join", s);
    unsigned long long total = 0;
    VS_CUDA_TRY(cudaMemcpyAsync(&total, counter, sizeof(total), cudaMemcpyDeviceToHost, s));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    *n_pairs = (int64_t)total;
    if ((int64_t)total > capacity) {
        set_error("pair buffer holds %lld pairs, %llu required", (long long)capacity, total);
        return VS_E_CAPACITY;
    }
    return VS_OK;
}
