// vs_join_host: the join on HOST point and pair buffers, pipelined.
//
// The points are streamed in chunks of millions of points: while the device joins
// chunk k (on the context stream), chunk k+1 is copied in on one stream and
// chunk k-1's pairs are copied out on another, so the PCIe transfers that
// bound a host-to-host join overlap the kernels instead of adding to them.
// Every chunk reuses the single-join launchers with a row base (its first
// point's row), so pair rows are global; with VS_JOIN_SORT each chunk is
// sorted on the device before it is copied out, and because chunks cover
// increasing row ranges the concatenation is sorted.  Replaces the
// reference's host round trip around its device join (H2D at move_to,
// D2H of the pair arrays, src/vibespatial/spatial/query.py:124).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "index.cuh"
#include "join.cuh"
#include "vs_common.cuh"

#include <new>

namespace vs {

// Points per chunk.  Smaller chunks overlap more of the copies, larger ones
// keep more of a join's cross-warp locality (all chunks span the whole
// polygon set); measured on the 50M x 1M workload: 8M points is best for the
// learned method (16.8 ms vs 14.4 ms for the bare 800 MB copy), 16M for the
// R-tree (19.7 ms; 4M chunks took 34 ms).
constexpr int64_t kHostChunkLearned = 1 << 23;
constexpr int64_t kHostChunkRtree = 1 << 24;

struct Streams {
    cudaStream_t in = nullptr, out = nullptr;
    cudaEvent_t h2d[2] = {nullptr, nullptr}, comp[2] = {nullptr, nullptr}, d2h[2] = {nullptr, nullptr};
    cudaEvent_t start = nullptr, t0 = nullptr, t1 = nullptr;
    ~Streams() {
        if (in) cudaStreamDestroy(in);
        if (out) cudaStreamDestroy(out);
        for (int b = 0; b < 2; ++b) {
            if (h2d[b]) cudaEventDestroy(h2d[b]);
            if (comp[b]) cudaEventDestroy(comp[b]);
            if (d2h[b]) cudaEventDestroy(d2h[b]);
        }
        if (start) cudaEventDestroy(start);
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
    }
    int create() {
        VS_CUDA_TRY(cudaStreamCreateWithFlags(&in, cudaStreamNonBlocking));
        VS_CUDA_TRY(cudaStreamCreateWithFlags(&out, cudaStreamNonBlocking));
        for (int b = 0; b < 2; ++b) {
            VS_CUDA_TRY(cudaEventCreateWithFlags(&h2d[b], cudaEventDisableTiming));
            VS_CUDA_TRY(cudaEventCreateWithFlags(&comp[b], cudaEventDisableTiming));
            VS_CUDA_TRY(cudaEventCreateWithFlags(&d2h[b], cudaEventDisableTiming));
        }
        VS_CUDA_TRY(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
        VS_CUDA_TRY(cudaEventCreate(&t0));
        VS_CUDA_TRY(cudaEventCreate(&t1));
        return VS_OK;
    }
};

// Double-buffered device memory of the pipeline.
struct Buffers {
    double* x[2] = {nullptr, nullptr};
    double* y[2] = {nullptr, nullptr};
    uint8_t* valid[2] = {nullptr, nullptr};
    int32_t* left[2] = {nullptr, nullptr};
    int32_t* right[2] = {nullptr, nullptr};
    int64_t cap[2] = {0, 0};  // pair capacity of each pair buffer
    ~Buffers() {
        for (int b = 0; b < 2; ++b) {
            cudaFree(x[b]);
            cudaFree(y[b]);
            cudaFree(valid[b]);
            cudaFree(left[b]);
            cudaFree(right[b]);
        }
    }
};

// The pipeline's streams, events and double buffers, created on the first
// vs_join_host of a context and reused (allocation would otherwise
// synchronise the device and cost more than the copies it overlaps).
struct HostPipe {
    Streams st;
    Buffers bf;
    int64_t point_cap = 0;  // points each point (and validity) buffer holds
    bool ready = false;
};

namespace {

int grow_pairs(Buffers& bf, int b, int64_t want) {
    cudaFree(bf.left[b]);
    cudaFree(bf.right[b]);
    bf.left[b] = bf.right[b] = nullptr;
    bf.cap[b] = 0;
    if (cudaMalloc((void**)&bf.left[b], sizeof(int32_t) * want) != cudaSuccess ||
        cudaMalloc((void**)&bf.right[b], sizeof(int32_t) * want) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaMalloc of a %lld-pair chunk buffer failed", (long long)want);
        return VS_E_OOM;
    }
    bf.cap[b] = want;
    return VS_OK;
}

}  // namespace

void free_host_pipe(vs_context* ctx) {
    delete ctx->host_pipe;  // the members release their streams, events and buffers
    ctx->host_pipe = nullptr;
}

}  // namespace vs

using namespace vs;

extern "C" {

int vs_join_host(vs_context* ctx, const vs_index* idx, const double* h_x, const double* h_y, const uint8_t* h_valid,
                 int64_t n, int32_t predicate, int32_t method, uint32_t flags, int32_t* h_left, int32_t* h_right,
                 int64_t capacity, int64_t* n_pairs, vs_join_stats* stats) {
    if (!ctx || !idx || !n_pairs) {
        set_error("ctx/index/n_pairs is NULL");
        return VS_E_ARG;
    }
    *n_pairs = 0;
    if (stats) memset(stats, 0, sizeof(*stats));
    if (n < 0 || n > 0x7fffffffLL || (n > 0 && (!h_x || !h_y))) {
        set_error("invalid host point buffers (n %lld)", (long long)n);
        return VS_E_ARG;
    }
    if (capacity < 0 || (capacity > 0 && (!h_left || !h_right))) {
        set_error("invalid host pair buffers (capacity %lld)", (long long)capacity);
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
    if (method == VS_METHOD_LEARNED && !idx->has_learned) method = VS_METHOD_RTREE;
    VS_TRY(use_device(ctx->device));
    if (n == 0 || idx->n_geoms == 0 || !(idx->h_frame[0] <= idx->h_frame[2])) return VS_OK;

    cudaStream_t s = ctx->stream;
    if (!ctx->host_pipe) {
        ctx->host_pipe = new (std::nothrow) HostPipe();
        if (!ctx->host_pipe) {
            set_error("host allocation failed");
            return VS_E_OOM;
        }
    }
    HostPipe& hp = *ctx->host_pipe;
    if (!hp.ready) {
        VS_TRY(hp.st.create());
        hp.ready = true;
    }
    Streams& st = hp.st;
    Buffers& bf = hp.bf;
    int64_t chunk_max = method == VS_METHOD_LEARNED ? kHostChunkLearned : kHostChunkRtree;
    // VSJOIN_HOST_CHUNK (points) overrides the chunk size, e.g. to bound the
    // device memory the pipeline holds
    if (const char* env = getenv("VSJOIN_HOST_CHUNK")) {
        const long long v = atoll(env);
        if (v > 0) chunk_max = v;
    }
    const int64_t chunk = n < chunk_max ? n : chunk_max;
    const int64_t n_chunks = (n + chunk - 1) / chunk;
    if (hp.point_cap < chunk) {
        // (re)allocate the point buffers for this chunk size
        VS_CUDA_TRY(cudaStreamSynchronize(s));
        for (int b = 0; b < 2; ++b) {
            cudaFree(bf.x[b]);
            cudaFree(bf.y[b]);
            cudaFree(bf.valid[b]);
            bf.x[b] = bf.y[b] = nullptr;
            bf.valid[b] = nullptr;
        }
        hp.point_cap = 0;
        for (int b = 0; b < 2; ++b) {
            if (cudaMalloc((void**)&bf.x[b], sizeof(double) * chunk) != cudaSuccess ||
                cudaMalloc((void**)&bf.y[b], sizeof(double) * chunk) != cudaSuccess ||
                cudaMalloc((void**)&bf.valid[b], chunk) != cudaSuccess) {
                cudaGetLastError();
                set_error("cudaMalloc of the chunk buffers failed");
                return VS_E_OOM;
            }
        }
        hp.point_cap = chunk;
    }
    for (int b = 0; b < 2; ++b)
        if (bf.cap[b] < 1024) VS_TRY(grow_pairs(bf, b, chunk > 1024 ? chunk : 1024));
    VS_TRY(ensure_defer_capacity(ctx, (unsigned long long)(chunk / 64 + 65536)));
    // order the pipeline after earlier work on the context stream
    VS_CUDA_TRY(cudaEventRecord(st.start, s));
    VS_CUDA_TRY(cudaStreamWaitEvent(st.in, st.start, 0));
    VS_CUDA_TRY(cudaEventRecord(st.t0, st.in));

    auto copy_in = [&](int64_t k) -> int {
        const int b = (int)(k & 1);
        const int64_t first = k * chunk, m = (n - first) < chunk ? (n - first) : chunk;
        VS_CUDA_TRY(cudaStreamWaitEvent(st.in, st.comp[b], 0));  // chunk k-2 has left the buffer
        VS_CUDA_TRY(cudaMemcpyAsync(bf.x[b], h_x + first, sizeof(double) * m, cudaMemcpyHostToDevice, st.in));
        VS_CUDA_TRY(cudaMemcpyAsync(bf.y[b], h_y + first, sizeof(double) * m, cudaMemcpyHostToDevice, st.in));
        if (h_valid) VS_CUDA_TRY(cudaMemcpyAsync(bf.valid[b], h_valid + first, m, cudaMemcpyHostToDevice, st.in));
        VS_CUDA_TRY(cudaEventRecord(st.h2d[b], st.in));
        return VS_OK;
    };

    unsigned long long totals[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // summed context counters
    int64_t total = 0;
    bool over = false;
    const long long launches0 = g_launches;
    VS_TRY(copy_in(0));
    for (int64_t k = 0; k < n_chunks; ++k) {
        const int b = (int)(k & 1);
        const int64_t first = k * chunk, m = (n - first) < chunk ? (n - first) : chunk;
        if (k + 1 < n_chunks) VS_TRY(copy_in(k + 1));
        const vs_points pts{bf.x[b], bf.y[b], h_valid ? bf.valid[b] : nullptr, m};
        VS_CUDA_TRY(cudaStreamWaitEvent(s, st.h2d[b], 0));
        VS_CUDA_TRY(cudaStreamWaitEvent(s, st.d2h[b], 0));  // chunk k-2's pairs have left the buffer
        unsigned long long* c = ctx->h_counter;
        for (int attempt = 0;; ++attempt) {
            const DeferSink ds{ctx->defer_buf, ctx->defer_cap, &ctx->d_counters[7]};
            VS_CUDA_TRY(cudaMemsetAsync(ctx->d_counters, 0, kDevCounters * sizeof(unsigned long long), s));
            if (method == VS_METHOD_LEARNED)
                VS_TRY(launch_learned_join(ctx, idx, &pts, mask, bf.left[b], bf.right[b], bf.cap[b], ds, first));
            else
                VS_TRY(launch_rtree_join(ctx, idx, &pts, mask, method == VS_METHOD_BRUTE, false, bf.left[b],
                                         bf.right[b], bf.cap[b], ds, first));
            if (mask)
                VS_TRY(launch_resolve_deferred(ctx, idx, &pts, mask, bf.left[b], bf.right[b], bf.cap[b], ds, first));
            VS_CUDA_TRY(cudaMemcpyAsync(c, ctx->d_counters, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                        s));
            VS_CUDA_TRY(cudaEventRecord(st.comp[b], s));
            VS_CUDA_TRY(cudaEventSynchronize(st.comp[b]));
            if (c[4] & 2) {
                set_error("a bounded device wait (bulk copy) gave up; the join's result is incomplete");
                return VS_E_TIMEOUT;
            }
            if (c[4]) {
                set_error("device-side consistency check failed (flags 0x%llx)", c[4]);
                return VS_E_STATE;
            }
            const bool defer_over = c[7] > ctx->defer_cap, pair_over = (int64_t)c[0] > bf.cap[b];
            if (!defer_over && !pair_over) break;
            if (attempt == 2) {
                set_error("chunk buffers did not converge");
                return VS_E_STATE;
            }
            if (defer_over) VS_TRY(ensure_defer_capacity(ctx, c[7] + c[7] / 8 + 65536));
            if (pair_over) {
                VS_CUDA_TRY(cudaEventSynchronize(st.d2h[b]));
                VS_TRY(grow_pairs(bf, b, (int64_t)(c[0] + c[0] / 8 + 1024)));
            }
        }
        const int64_t cnt = (int64_t)c[0];
        for (int q = 1; q < 8; ++q) totals[q] += c[q];
        if (cnt > 0 && (flags & VS_JOIN_SORT)) {
            VS_TRY(sort_pairs(ctx, bf.left[b], bf.right[b], cnt, (uint64_t)n, (uint64_t)idx->n_geoms));
            VS_CUDA_TRY(cudaEventRecord(st.comp[b], s));
        }
        if (!over && total + cnt <= capacity) {
            VS_CUDA_TRY(cudaStreamWaitEvent(st.out, st.comp[b], 0));
            VS_CUDA_TRY(cudaMemcpyAsync(h_left + total, bf.left[b], sizeof(int32_t) * cnt, cudaMemcpyDeviceToHost,
                                        st.out));
            VS_CUDA_TRY(cudaMemcpyAsync(h_right + total, bf.right[b], sizeof(int32_t) * cnt,
                                        cudaMemcpyDeviceToHost, st.out));
            VS_CUDA_TRY(cudaEventRecord(st.d2h[b], st.out));
        } else {
            over = true;  // keep counting the pairs; the caller gets the required size
        }
        total += cnt;
    }
    VS_CUDA_TRY(cudaEventRecord(st.t1, st.out));
    VS_CUDA_TRY(cudaStreamSynchronize(st.out));
    VS_CUDA_TRY(cudaStreamSynchronize(st.in));
    VS_CUDA_TRY(cudaStreamSynchronize(s));
    *n_pairs = total;
    if (stats) {
        stats->exact_fallbacks = (int64_t)totals[1];
        stats->fp32_edges = (int64_t)totals[2];
        stats->fp64_edges = (int64_t)totals[3];
        stats->candidates = (int64_t)totals[5];
        stats->rmi_fallbacks = (int64_t)totals[6];
        cudaEventElapsedTime(&stats->kernel_ms, st.t0, st.t1);
        stats->kernel_launches = g_launches - launches0;
    }
    if (over) {
        set_error("pair buffer holds %lld pairs, %lld required", (long long)capacity, (long long)total);
        return VS_E_CAPACITY;
    }
    return VS_OK;
}

}  // extern "C"
