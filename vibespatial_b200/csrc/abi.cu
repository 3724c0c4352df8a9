// extern "C" entry points of libvsjoin.so (declared in include/vsjoin.h).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdint.h>
#include <string.h>

#include <new>

#include "index.cuh"
#include "join.cuh"
#include "primitives.cuh"

namespace vs {

static thread_local char g_err[1024] = "";
thread_local long long g_launches = 0;

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int use_device(int device) {
    int cur = -1;
    VS_CUDA_TRY(cudaGetDevice(&cur));
    if (cur != device) VS_CUDA_TRY(cudaSetDevice(device));
    return VS_OK;
}

int check_polygons(const vs_polygons* p) {
    if (!p) {
        set_error("polygons is NULL");
        return VS_E_ARG;
    }
    if (p->n_geoms < 0 || p->n_parts < 0 || p->n_rings < 0 || p->n_coords < 0) {
        set_error("negative polygon sizes");
        return VS_E_ARG;
    }
    if (p->n_coords > 0x7fffffffLL) {
        set_error("more than 2^31-1 polygon coordinates (int32 offsets)");
        return VS_E_ARG;
    }
    if (!p->d_geom_off || !p->d_part_off || !p->d_ring_off) {
        set_error("polygon offset buffers must not be NULL");
        return VS_E_ARG;
    }
    if (p->n_coords > 0 && (!p->d_x || !p->d_y)) {
        set_error("polygon coordinate buffers must not be NULL");
        return VS_E_ARG;
    }
    return VS_OK;
}

int check_points(const vs_points* p) {
    if (!p) {
        set_error("points is NULL");
        return VS_E_ARG;
    }
    if (p->n < 0 || p->n > 0x7fffffffLL) {
        set_error("point count %lld outside [0, 2^31-1]", (long long)p->n);
        return VS_E_ARG;
    }
    if (p->n > 0 && (!p->d_x || !p->d_y)) {
        set_error("point coordinate buffers must not be NULL");
        return VS_E_ARG;
    }
    return VS_OK;
}

int ensure_defer_capacity(vs_context* ctx, unsigned long long want) {
    if (ctx->defer_cap >= want) return VS_OK;
    if (ctx->defer_buf) {
        VS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        cudaFree(ctx->defer_buf);
        ctx->defer_buf = nullptr;
        ctx->defer_cap = 0;
    }
    cudaError_t e = cudaMalloc((void**)&ctx->defer_buf, want * sizeof(int2));
    if (e != cudaSuccess) {
        ctx->defer_buf = nullptr;
        set_error("cudaMalloc of the deferred-pair buffer (%llu pairs) failed: %s", want, cudaGetErrorString(e));
        return VS_E_OOM;
    }
    ctx->defer_cap = want;
    return VS_OK;
}

}  // namespace vs

using namespace vs;

extern "C" {

int vs_version(void) { return VSJOIN_ABI_VERSION; }

const char* vs_last_error(void) { return g_err; }

long long vs_thread_kernel_launches(void) { return g_launches; }

int vs_context_create(int device, void* stream, vs_context** out) {
    if (!out) {
        set_error("out is NULL");
        return VS_E_ARG;
    }
    *out = nullptr;
    int ndev = 0;
    VS_CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) {
        set_error("device %d out of range (%d devices)", device, ndev);
        return VS_E_ARG;
    }
    VS_TRY(use_device(device));
    vs_context* ctx = new (std::nothrow) vs_context{};
    if (!ctx) {
        set_error("host allocation failed");
        return VS_E_OOM;
    }
    ctx->device = device;
    if (stream) {
        ctx->stream = (cudaStream_t)stream;
        ctx->owns_stream = false;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            delete ctx;
            set_error("cudaStreamCreate failed: %s", cudaGetErrorString(e));
            return VS_E_CUDA;
        }
        ctx->owns_stream = true;
    }
    // Keep freed stream-ordered scratch in the pool between calls.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    bool ok = cudaMallocHost((void**)&ctx->h_counter, kHostCounters * sizeof(unsigned long long)) == cudaSuccess &&
              cudaMalloc((void**)&ctx->d_counters, kDevCounters * sizeof(unsigned long long)) == cudaSuccess;
    for (int k = 0; k < 5 && ok; ++k) ok = cudaEventCreate(&ctx->phase_ev[k]) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        set_error("context buffer allocation failed");
        for (int k = 0; k < 5; ++k)
            if (ctx->phase_ev[k]) cudaEventDestroy(ctx->phase_ev[k]);
        if (ctx->d_counters) cudaFree(ctx->d_counters);
        if (ctx->h_counter) cudaFreeHost(ctx->h_counter);
        if (ctx->owns_stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return VS_E_OOM;
    }
    *out = ctx;
    return VS_OK;
}

int vs_context_destroy(vs_context* ctx) {
    if (!ctx) return VS_OK;
    use_device(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    free_host_pipe(ctx);
    cudaFree(ctx->d_counters);
    cudaFree(ctx->defer_buf);
    cudaFreeHost(ctx->h_counter);
    for (int k = 0; k < 5; ++k) cudaEventDestroy(ctx->phase_ev[k]);
    if (ctx->owns_stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
    return VS_OK;
}

int vs_context_synchronize(vs_context* ctx) {
    if (!ctx) {
        set_error("ctx is NULL");
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    VS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return VS_OK;
}

int vs_index_build(vs_context* ctx, const vs_polygons* polys, const vs_index_options* opts, vs_index** out) {
    if (!ctx || !out) {
        set_error("ctx/out is NULL");
        return VS_E_ARG;
    }
    *out = nullptr;
    VS_TRY(check_polygons(polys));
    VS_TRY(use_device(ctx->device));
    vs_index* idx = new (std::nothrow) vs_index{};
    if (!idx) {
        set_error("host allocation failed");
        return VS_E_OOM;
    }
    idx->device = ctx->device;
    EventPair ev;
    cudaEventRecord(ev.a, ctx->stream);
    int st = build_rtree(ctx, polys, idx);
    if (st == VS_OK) st = build_ring_bins(ctx, idx, opts ? opts->ring_bin_min_vertices : 0);
    if (st == VS_OK && opts && (opts->method_mask & 2)) st = build_learned_index(ctx, idx, opts);
    if (st != VS_OK) {
        cudaStreamSynchronize(ctx->stream);
        free_index_memory(idx);
        delete idx;
        return st;
    }
    cudaEventRecord(ev.b, ctx->stream);
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        set_error("index build failed: %s", cudaGetErrorString(e));
        free_index_memory(idx);
        delete idx;
        return VS_E_CUDA;
    }
    idx->build_ms = ev.ms();
    *out = idx;
    return VS_OK;
}

int vs_index_info_get(const vs_index* idx, vs_index_info* info) {
    if (!idx || !info) {
        set_error("index/info is NULL");
        return VS_E_ARG;
    }
    memset(info, 0, sizeof(*info));
    info->n_geoms = idx->n_geoms;
    info->fanout = kFanout;
    info->levels = idx->levels;
    info->cell_level = idx->has_learned ? idx->learned.level : 0;
    info->n_cells = idx->has_learned ? idx->learned.n_cells : 0;
    info->n_cell_entries = idx->has_learned ? idx->learned.n_entries : 0;
    info->device_bytes = idx->device_bytes;
    info->build_ms = idx->build_ms;
    info->rmi_train_ms = idx->learned.rmi_train_ms;
    info->rmi_mean_window = idx->learned.mean_window;
    info->rmi_max_window = idx->learned.max_window;
    info->n_binned_rings = idx->n_binned_rings;
    info->n_bin_edges = idx->n_bin_edges;
    info->rmi_leaves = idx->has_learned ? idx->learned.n_leaves : 0;
    return VS_OK;
}

int vs_index_free(vs_index* idx) {
    if (!idx) return VS_OK;
    use_device(idx->device);
    cudaDeviceSynchronize();
    free_index_memory(idx);
    delete idx;
    return VS_OK;
}

int vs_join(vs_context* ctx, const vs_index* idx, const vs_points* pts, int32_t predicate, int32_t method,
            uint32_t flags, int32_t* d_left, int32_t* d_right, int64_t capacity, int64_t* n_pairs,
            vs_join_stats* stats) {
    if (!ctx || !idx || !n_pairs) {
        set_error("ctx/index/n_pairs is NULL");
        return VS_E_ARG;
    }
    *n_pairs = 0;
    if (stats) memset(stats, 0, sizeof(*stats));
    VS_TRY(check_points(pts));
    if (capacity < 0 || (capacity > 0 && (!d_left || !d_right))) {
        set_error("invalid pair buffers (capacity %lld)", (long long)capacity);
        return VS_E_ARG;
    }
    if (idx->device != ctx->device) {
        set_error("index lives on device %d, context on device %d", idx->device, ctx->device);
        return VS_E_ARG;
    }
    int mask = 0;
    VS_TRY(accept_mask_for(predicate, &mask));
    if (method != VS_METHOD_RTREE && method != VS_METHOD_LEARNED && method != VS_METHOD_BRUTE) {
        set_error("unknown method %d", method);
        return VS_E_ARG;
    }
    // The plain R-tree is the learned index's fallback: an index built without
    // the learned cell index (or with nothing to index) answers with the R-tree.
    if (method == VS_METHOD_LEARNED && !idx->has_learned) method = VS_METHOD_RTREE;
    VS_TRY(use_device(ctx->device));
    if (pts->n == 0 || idx->n_geoms == 0 || !(idx->h_frame[0] <= idx->h_frame[2])) return VS_OK;
    cudaStream_t s = ctx->stream;
    const long long launches0 = g_launches;
    EventPair ev;
    // Pairs the filters cannot certify go to the context's deferred buffer
    // and are resolved exactly after the join kernel; if more were deferred
    // than the buffer holds, the join runs once more with a buffer that fits.
    LearnedShape shape{};
    shape.flags = ((flags & VS_JOIN_LEARNED_BSEARCH) ? kLearnedBsearch : 0u) |
                  ((flags & VS_JOIN_LEARNED_FP64_WALK) ? kLearnedFp64Walk : 0u) |
                  ((flags & VS_JOIN_LEARNED_NO_STAGE) ? kLearnedNoStage : 0u) |
                  ((flags & VS_JOIN_LEARNED_NO_INTERIOR) ? kLearnedNoInterior : 0u);
    unsigned long long want = (unsigned long long)(pts->n / 64 + 65536);
    for (int attempt = 0; attempt < 2; ++attempt) {
        VS_TRY(ensure_defer_capacity(ctx, want));
        VS_CUDA_TRY(cudaMemsetAsync(ctx->d_counters, 0, kDevCounters * sizeof(unsigned long long), s));
        const DeferSink ds{ctx->defer_buf, ctx->defer_cap, &ctx->d_counters[7]};
        ctx->phase_on = stats != nullptr;
        cudaEventRecord(ev.a, s);
        phase_mark(ctx, 0);
        int st;
        if (method == VS_METHOD_LEARNED)
            st = launch_learned_join(ctx, idx, pts, mask, d_left, d_right, capacity, ds, 0, shape);
        else
            st = launch_rtree_join(ctx, idx, pts, mask, method == VS_METHOD_BRUTE, (flags & VS_JOIN_BULK_LEAVES) != 0,
                                   d_left, d_right, capacity, ds);
        phase_mark(ctx, 3);
        if (st == VS_OK && mask) st = launch_resolve_deferred(ctx, idx, pts, mask, d_left, d_right, capacity, ds);
        phase_mark(ctx, 4);
        ctx->phase_on = false;
        VS_TRY(st);
        cudaEventRecord(ev.b, s);
        VS_CUDA_TRY(cudaMemcpyAsync(ctx->h_counter, ctx->d_counters, 8 * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, s));
        VS_CUDA_TRY(cudaStreamSynchronize(s));
        if (ctx->h_counter[7] <= ctx->defer_cap) break;
        want = ctx->h_counter[7];
    }
    const unsigned long long* c = ctx->h_counter;
    if (c[7] > ctx->defer_cap) {
        set_error("deferred-pair buffer did not converge (%llu pairs)", c[7]);
        return VS_E_STATE;
    }
    const int64_t n = (int64_t)c[0];
    *n_pairs = n;
    if (stats) {
        stats->exact_fallbacks = (int64_t)c[1];
        stats->fp32_edges = (int64_t)c[2];
        stats->fp64_edges = (int64_t)c[3];
        stats->candidates = (int64_t)c[5];
        stats->rmi_fallbacks = (int64_t)c[6];
        stats->kernel_ms = ev.ms();
        stats->kernel_launches = g_launches - launches0;
        for (int k = 0; k < 4; ++k) cudaEventElapsedTime(&stats->phase_ms[k], ctx->phase_ev[k], ctx->phase_ev[k + 1]);
    }
    if (c[4] & 2) {
        set_error("a bounded device wait (bulk copy) gave up; the join's result is incomplete");
        return VS_E_TIMEOUT;
    }
    if (c[4] != 0) {
        set_error("device-side consistency check failed (flags 0x%llx)", (unsigned long long)c[4]);
        return VS_E_STATE;
    }
    if (n > capacity) {
        set_error("pair buffer holds %lld pairs, %lld required", (long long)capacity, (long long)n);
        return VS_E_CAPACITY;
    }
    if (flags & VS_JOIN_SORT) {
        EventPair es;
        cudaEventRecord(es.a, s);
        VS_TRY(sort_pairs(ctx, d_left, d_right, n, (uint64_t)pts->n, (uint64_t)idx->n_geoms));
        cudaEventRecord(es.b, s);
        VS_CUDA_TRY(cudaStreamSynchronize(s));
        if (stats) {
            stats->sort_ms = es.ms();
            stats->kernel_launches = g_launches - launches0;
        }
    }
    return VS_OK;
}

int vs_locate_aligned(vs_context* ctx, const vs_points* pts, const vs_polygons* polys, uint8_t* d_out) {
    if (!ctx) {
        set_error("ctx is NULL");
        return VS_E_ARG;
    }
    VS_TRY(check_points(pts));
    VS_TRY(check_polygons(polys));
    if ((int64_t)polys->n_geoms != pts->n) {
        set_error("aligned arrays differ in length (%lld points, %d polygons)", (long long)pts->n, polys->n_geoms);
        return VS_E_ARG;
    }
    if (pts->n > 0 && !d_out) {
        set_error("d_out is NULL");
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    VS_CUDA_TRY(cudaMemsetAsync(ctx->d_counters, 0, kDevCounters * sizeof(unsigned long long), ctx->stream));
    VS_TRY(launch_locate_aligned(ctx, pts, polys, d_out));
    VS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return VS_OK;
}

int vs_sort_pairs(vs_context* ctx, int32_t* d_left, int32_t* d_right, int64_t n) {
    if (!ctx || n < 0 || (n > 0 && (!d_left || !d_right))) {
        set_error("invalid arguments to vs_sort_pairs");
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    VS_TRY(sort_pairs(ctx, d_left, d_right, n, 0xffffffffull, 0xffffffffull));
    VS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return VS_OK;
}

int vs_radix_sort_pairs(vs_context* ctx, uint64_t* d_keys, uint32_t* d_vals, int64_t n, int32_t key_bits) {
    if (!ctx || n < 0 || (n > 0 && (!d_keys || !d_vals))) {
        set_error("invalid arguments to vs_radix_sort_pairs");
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    VS_TRY(radix_sort_u64_u32(d_keys, d_vals, n, key_bits, ctx->stream));
    VS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return VS_OK;
}

int vs_hilbert_keys(vs_context* ctx, const double* d_x, const double* d_y, int64_t n, double minx, double miny,
                    double maxx, double maxy, uint64_t* d_keys) {
    if (!ctx || n < 0 || (n > 0 && (!d_x || !d_y || !d_keys))) {
        set_error("invalid arguments to vs_hilbert_keys");
        return VS_E_ARG;
    }
    VS_TRY(use_device(ctx->device));
    if (n == 0) return VS_OK;
    VS_TRY(hilbert_point_keys(d_x, d_y, n, minx, miny, maxx, maxy, d_keys, ctx->stream));
    VS_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return VS_OK;
}

}  // extern "C"
