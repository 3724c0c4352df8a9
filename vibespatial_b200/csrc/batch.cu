// Batched joins: many independent point x polygon joins of uneven sizes in one
// persistent launch, replayed from a CUDA graph.
//
// A batch plan holds, for every job, a device descriptor of that job's
// packed R-tree (built by vs_index_build) and the job's slice of one
// concatenated point array.  One run is:
//   1. batch_key_kernel   key = job id (top bits) | Hilbert cell of the point
//                         in its job's frame; points outside their frame,
//                         null or NaN get the sentinel key
//   2. radix sort         of all jobs' points at once (in-house, top bits only)
//   3. batch_join_kernel  persistent: warps take packets of 32 sorted points
//                         from an atomic work counter (several packets per
//                         grab) and walk the packet's job tree exactly as the
//                         single join does; a packet that straddles two jobs
//                         is walked once per job
//   4. batch_resolve      exact pass over the pairs the filter deferred
// All four are captured once into a CUDA graph per (predicate, output
// buffers) and replayed; nothing in between needs the host.  The tile shape
// (blocks per SM, packets per grab, Hilbert levels sorted) comes from the
// caller, normally the autotuner in vibespatial_b200/autotune.py.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <new>
#include <vector>

#include "emit.cuh"
#include "exact.cuh"
#include "hilbert.cuh"
#include "index.cuh"
#include "join.cuh"
#include "learned.cuh"
#include "primitives.cuh"

namespace vs {
namespace {

constexpr int kBThreads = 256;
constexpr int kBWarps = kBThreads / 32;
constexpr int kBStack = 112;
constexpr int kMaxJobs = 4096;

struct JobTree {
    const vs_box* nodes;
    const int32_t* item_geom;
    const int32_t* geom_off;
    const int32_t* part_off;
    const int32_t* ring_off;
    const double2* xy;
    int64_t level_off[kMaxLevels];
    int64_t level_size[kMaxLevels];
    double frame[4];
    int32_t levels;
    int32_t n_geoms;
    RingIndex rings;
};

struct BatchArgs {
    const double* px;
    const double* py;
    const uint8_t* pvalid;     // nullable
    const int64_t* job_start;  // [n_jobs + 1]
    int n_jobs;
    int job_shift;             // key >> job_shift = job id
    int key_levels;            // Hilbert levels in the key's low bits
    const JobTree* jobs;
    uint32_t* keys;
    uint32_t* order;
    uint32_t* n_valid;
    unsigned long long* work;  // packets handed out
    int packets_per_grab;
    int accept_mask;
    PairSink sink;
    DeferSink defer;
    unsigned long long* counters;
};

__device__ __forceinline__ int job_of(const int64_t* js, int n_jobs, int64_t i) {
    int lo = 0, hi = n_jobs;  // last job with js[job] <= i
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (js[mid] <= i) lo = mid;
        else hi = mid;
    }
    return lo;
}

__global__ void batch_key_kernel(const BatchArgs a, int64_t n) {
    extern __shared__ int64_t s_js[];
    __shared__ uint16_t s_lut[kHilbertLutSize];
    hilbert_lut_init(s_lut);
    for (int k = threadIdx.x; k <= a.n_jobs; k += blockDim.x) s_js[k] = a.job_start[k];
    __syncthreads();
    uint32_t cnt = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int job = job_of(s_js, a.n_jobs, i);
        const JobTree& t = a.jobs[job];
        const double f0 = t.frame[0], f1 = t.frame[1], f2 = t.frame[2], f3 = t.frame[3];
        const double x = a.px[i], y = a.py[i];
        uint32_t k = 0xffffffffu;
        if ((a.pvalid == nullptr || a.pvalid[i]) && t.n_geoms > 0 && f0 <= f2 && x >= f0 && x <= f2 && y >= f1 &&
            y <= f3) {
            const double sx = f2 > f0 ? 4294967295.0 / (f2 - f0) : 0.0;
            const double sy = f3 > f1 ? 4294967295.0 / (f3 - f1) : 0.0;
            const uint32_t h = hilbert_key_lut(quantize(x, f0, sx), quantize(y, f1, sy), a.key_levels, s_lut);
            k = ((uint32_t)job << a.job_shift) | h;
            ++cnt;
        }
        a.keys[i] = k;
        a.order[i] = (uint32_t)i;
    }
    cnt = (uint32_t)warp_sum(cnt);
    __shared__ uint32_t wsum[32];
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += wsum[w];
        if (t) atomicAdd(a.n_valid, t);
    }
}

__device__ __forceinline__ bool box_has_b(const vs_box& b, double x, double y) {
    return x >= b.minx && x <= b.maxx && y >= b.miny && y <= b.maxy;
}

__device__ __forceinline__ bool box_overlaps_b(const vs_box& b, double x0, double y0, double x1, double y1) {
    return b.minx <= x1 && b.maxx >= x0 && b.miny <= y1 && b.maxy >= y0;
}

__global__ void __launch_bounds__(kBThreads) batch_join_kernel(const BatchArgs a) {
    __shared__ int2 s_buf[kBWarps][kWarpBuf];
    __shared__ unsigned s_cnt[kBWarps];
    __shared__ int s_stack[kBWarps][kBStack];
    __shared__ vs_box s_items[kBWarps][kFanout];
    __shared__ int64_t s_loff[kBWarps][kMaxLevels];
    __shared__ int64_t s_lsize[kBWarps][kMaxLevels];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_cnt[warp] = 0;
    __syncwarp();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    const unsigned lt = (1u << lane) - 1u;
    const int64_t n = (int64_t)*a.n_valid;
    const int64_t grab = 32ll * a.packets_per_grab;
    unsigned long long n_cand = 0;
    for (;;) {
        unsigned long long g0 = 0;
        if (lane == 0) g0 = atomicAdd(a.work, (unsigned long long)grab);
        g0 = __shfl_sync(0xffffffffu, g0, 0);
        if ((int64_t)g0 >= n) break;
        const int64_t gend = (int64_t)g0 + grab < n ? (int64_t)g0 + grab : n;
        for (int64_t base = (int64_t)g0; base < gend; base += 32) {
            const int64_t i = base + lane;
            const bool active = i < gend;
            double x = 0.0, y = 0.0;
            int32_t row = -1;
            int job = -1;
            if (active) {
                row = (int32_t)a.order[i];
                job = (int)(a.keys[i] >> a.job_shift);
                x = a.px[row];
                y = a.py[row];
            }
            unsigned pending = __ballot_sync(0xffffffffu, active);
            while (pending) {
                const int J = __shfl_sync(0xffffffffu, job, __ffs(pending) - 1);
                const bool mine = active && job == J;
                pending &= ~__ballot_sync(0xffffffffu, mine);
                const JobTree& t = a.jobs[J];
                if (lane < kMaxLevels) {
                    s_loff[warp][lane] = t.level_off[lane];
                    s_lsize[warp][lane] = t.level_size[lane];
                }
                const vs_box* nodes = t.nodes;
                const int32_t* item_geom = t.item_geom;
                const int top = t.levels - 1;
                __syncwarp();
                double x0 = mine ? x : INFINITY, x1 = mine ? x : -INFINITY;
                double y0 = mine ? y : INFINITY, y1 = mine ? y : -INFINITY;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    x0 = fmin(x0, __shfl_xor_sync(0xffffffffu, x0, o));
                    x1 = fmax(x1, __shfl_xor_sync(0xffffffffu, x1, o));
                    y0 = fmin(y0, __shfl_xor_sync(0xffffffffu, y0, o));
                    y1 = fmax(y1, __shfl_xor_sync(0xffffffffu, y1, o));
                }
                int sp = 0;
                const vs_box root = nodes[s_loff[warp][top]];
                if (box_overlaps_b(root, x0, y0, x1, y1)) {
                    if (top == 0) {
                        bool want = false;
                        if (mine && box_has_b(root, x, y)) {
                            ++n_cand;
                            const int loc = a.accept_mask ? geometry_location_filtered(x, y, t.xy, t.ring_off,
                                                                                       t.part_off, t.geom_off, 0,
                                                                                       t.rings)
                                                          : 0;
                            if (loc == LOC_UNDECIDED) defer(a.defer, row, 0);
                            else want = !a.accept_mask || ((a.accept_mask >> loc) & 1);
                        }
                        wemit_sync(out, a.sink, want, row, item_geom[0]);
                    } else {
                        if (lane == 0) s_stack[warp][0] = top;
                        sp = 1;
                    }
                }
                __syncwarp();
                while (sp > 0) {
                    --sp;
                    const int e = s_stack[warp][sp];
                    __syncwarp();
                    const int cl = (e & 15) - 1;
                    const int64_t c = (int64_t)(e >> 4) * kFanout + (lane & 15);
                    const bool in_range = lane < kFanout && c < s_lsize[warp][cl];
                    vs_box b{INFINITY, INFINITY, -INFINITY, -INFINITY};
                    if (in_range) b = nodes[s_loff[warp][cl] + c];
                    const bool hit = in_range && box_overlaps_b(b, x0, y0, x1, y1);
                    const unsigned m = __ballot_sync(0xffffffffu, hit);
                    if (cl > 0) {
                        if (hit) {
                            const int pos = sp + __popc(m & lt);
                            if (pos < kBStack) s_stack[warp][pos] = (int)(c << 4) | cl;
                        }
                        int add = __popc(m);
                        if (sp + add > kBStack) {
                            if (lane == 0) atomicOr(&a.counters[4], 1ull);
                            add = kBStack - sp;
                        }
                        sp += add;
                        __syncwarp();
                    } else {
                        if (lane < kFanout) s_items[warp][lane] = b;
                        __syncwarp();
                        unsigned mm = m;
                        const int64_t slot0 = (int64_t)(e >> 4) * kFanout;
                        while (mm) {
                            const int j = __ffs(mm) - 1;
                            mm &= mm - 1;
                            const vs_box ib = s_items[warp][j];
                            const int slot = (int)(slot0 + j);
                            bool want = false;
                            if (mine && box_has_b(ib, x, y)) {
                                ++n_cand;
                                int loc = 0;
                                if (a.accept_mask)
                                    loc = geometry_location_filtered(x, y, t.xy, t.ring_off, t.part_off, t.geom_off,
                                                                     slot, t.rings);
                                if (loc == LOC_UNDECIDED) defer(a.defer, row, slot);
                                else want = !a.accept_mask || ((a.accept_mask >> loc) & 1);
                            }
                            wemit_sync(out, a.sink, want, row, item_geom[slot]);
                        }
                        __syncwarp();
                    }
                }
            }
            wflush(out, a.sink, false);
        }
    }
    wflush(out, a.sink, true);
    add_counter(a.counters, 5, n_cand);
}

// Exact pass over deferred (global point row, slot) pairs; the job is found
// from the row.
__global__ void __launch_bounds__(kBThreads) batch_resolve_kernel(const BatchArgs a) {
    __shared__ int2 s_buf[kBWarps][kWarpBuf];
    __shared__ unsigned s_cnt[kBWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_cnt[warp] = 0;
    __syncwarp();
    const WarpOut out{s_buf[warp], &s_cnt[warp]};
    const unsigned long long cnt = *a.defer.counter;
    const int64_t n = (int64_t)(cnt < a.defer.capacity ? cnt : a.defer.capacity);
    const int64_t gw = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    unsigned n_exact = 0;
    for (int64_t base = gw * 32; base < n; base += nw * 32) {
        const int64_t k = base + lane;
        bool want = false;
        int2 pr = make_int2(0, 0);
        int32_t right = 0;
        if (k < n) {
            pr = a.defer.buf[k];
            const JobTree& t = a.jobs[job_of(a.job_start, a.n_jobs, pr.x)];
            const int loc = geometry_location(a.px[pr.x], a.py[pr.x], t.xy, t.ring_off, t.part_off, t.geom_off, pr.y,
                                              t.rings, n_exact);
            want = (a.accept_mask >> loc) & 1;
            right = want ? t.item_geom[pr.y] : 0;
        }
        wemit_sync(out, a.sink, want, pr.x, right);
        wflush(out, a.sink, false);
    }
    wflush(out, a.sink, true);
    add_counter(a.counters, 1, n_exact);
}

int bits_needed(int64_t v) {  // smallest b with 2^b > v
    int b = 1;
    while (b < 31 && (1ll << b) <= v) ++b;
    return b;
}

}  // namespace
}  // namespace vs

struct vs_batch_plan {
    vs_context* ctx = nullptr;
    int n_jobs = 0;
    int64_t n_points = 0;
    vs_batch_options opts{};
    vs_points pts{};
    vs::JobTree* d_jobs = nullptr;
    int64_t* d_job_start = nullptr;
    uint32_t* keys = nullptr;
    uint32_t* order = nullptr;
    int2* defer = nullptr;
    unsigned long long defer_cap = 0;
    unsigned long long* d_work = nullptr;  // [0] packets handed out, [1] deferred pairs
    uint32_t* d_n_valid = nullptr;
    int job_shift = 0, key_levels = 0, sort_begin = 0;
    // graph replay: captured on a private stream (the legacy default stream
    // cannot be captured) and ordered after / before the context stream by events
    cudaStream_t gstream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr, t0 = nullptr, t1 = nullptr;
    cudaGraphExec_t graph = nullptr;
    int32_t g_pred = -1;
    int32_t* g_left = nullptr;
    int32_t* g_right = nullptr;
    int64_t g_cap = -1;
    long long g_kernels = 0;  // kernels in the captured graph
    // learned method: per-job query descriptors and the pipeline's scratch
    bool learned = false;
    vs::LearnedJob* d_ljobs = nullptr;
    vs::LearnedJob h_single{};  // the descriptor when the batch has one job
    int64_t n_cells = 0;        // batch-wide learned cells
    bool has_ring_bins = false; // some job's index has binned rings long enough for the split walk
    void* lscratch = nullptr;
    vs::LearnedScratch lsc{};
};

namespace vs {
namespace {

void free_plan(vs_batch_plan* p) {
    if (p->graph) cudaGraphExecDestroy(p->graph);
    if (p->gstream) cudaStreamDestroy(p->gstream);
    if (p->ev_in) cudaEventDestroy(p->ev_in);
    if (p->ev_out) cudaEventDestroy(p->ev_out);
    if (p->t0) cudaEventDestroy(p->t0);
    if (p->t1) cudaEventDestroy(p->t1);
    cudaFree(p->d_jobs);
    cudaFree(p->d_job_start);
    cudaFree(p->keys);
    cudaFree(p->order);
    cudaFree(p->defer);
    cudaFree(p->d_work);
    cudaFree(p->d_n_valid);
    cudaFree(p->d_ljobs);
    cudaFree(p->lscratch);
}

BatchArgs plan_args(vs_batch_plan* p, int mask, int32_t* left, int32_t* right, int64_t capacity) {
    BatchArgs a{};
    a.px = p->pts.d_x;
    a.py = p->pts.d_y;
    a.pvalid = p->pts.d_valid;
    a.job_start = p->d_job_start;
    a.n_jobs = p->n_jobs;
    a.job_shift = p->job_shift;
    a.key_levels = p->key_levels;
    a.jobs = p->d_jobs;
    a.keys = p->keys;
    a.order = p->order;
    a.n_valid = p->d_n_valid;
    a.work = p->d_work;
    a.packets_per_grab = p->opts.packets_per_grab;
    a.accept_mask = mask;
    a.sink = PairSink{left, right, (unsigned long long)(capacity > 0 ? capacity : 0), &p->ctx->d_counters[0]};
    a.defer = DeferSink{p->defer, p->defer_cap, &p->d_work[1]};
    a.counters = p->ctx->d_counters;
    return a;
}

// Enqueue one whole batched join on stream s (capturable: no host
// synchronisation, scratch from the stream-ordered allocator).
int enqueue_batch(vs_batch_plan* p, cudaStream_t s, int mask, int32_t* left, int32_t* right, int64_t capacity) {
    const BatchArgs a = plan_args(p, mask, left, right, capacity);
    VS_CUDA_TRY(cudaMemsetAsync(p->ctx->d_counters, 0, kDevCounters * sizeof(unsigned long long), s));
    VS_CUDA_TRY(cudaMemsetAsync(p->d_work, 0, 2 * sizeof(unsigned long long), s));
    if (p->learned) {
        LearnedQuery q{};
        q.px = p->pts.d_x;
        q.py = p->pts.d_y;
        q.pvalid = p->pts.d_valid;
        q.n = p->n_points;
        q.jobs = p->d_ljobs;
        q.n_jobs = p->n_jobs;
        q.job_start = p->d_job_start;
        q.n_cells = p->n_cells;
        q.accept_mask = mask;
        q.has_ring_bins = p->has_ring_bins;
        q.shape.map_blocks_per_sm = p->opts.learned_map_blocks_per_sm;
        q.shape.refine_blocks_per_sm = p->opts.learned_refine_blocks_per_sm;
        q.shape.grab = p->opts.learned_grab;
        q.shape.map_packets = p->opts.learned_map_packets;
        q.shape.flags = ((p->opts.learned_flags & VS_JOIN_LEARNED_BSEARCH) ? kLearnedBsearch : 0u) |
                        ((p->opts.learned_flags & VS_JOIN_LEARNED_FP64_WALK) ? kLearnedFp64Walk : 0u) |
                        ((p->opts.learned_flags & VS_JOIN_LEARNED_NO_STAGE) ? kLearnedNoStage : 0u) |
                        ((p->opts.learned_flags & VS_JOIN_LEARNED_NO_INTERIOR) ? kLearnedNoInterior : 0u);
        VS_TRY(enqueue_learned(s, nullptr, q, p->n_jobs == 1 ? &p->h_single : nullptr, p->lsc, a.sink, a.defer,
                               a.counters, &p->d_work[0]));
        if (mask) {
            batch_resolve_kernel<<<resident_grid(batch_resolve_kernel, (int64_t)1 << 30, kBThreads), kBThreads, 0,
                                   s>>>(a);
            VS_LAUNCHED("batch_resolve", s);
        }
        return VS_OK;
    }
    VS_CUDA_TRY(cudaMemsetAsync(p->d_n_valid, 0, sizeof(uint32_t), s));
    const size_t smem = (size_t)(p->n_jobs + 1) * sizeof(int64_t);
    batch_key_kernel<<<resident_grid(batch_key_kernel, p->n_points, 256, smem), 256, smem, s>>>(a, p->n_points);
    VS_LAUNCHED("batch_key", s);
    VS_TRY(radix_sort_u32_u32(p->keys, p->order, p->n_points, 32, s, p->sort_begin));
    // blocks per SM from the launch shape, capped at what can be resident
    const int resident = resident_grid(batch_join_kernel, (int64_t)1 << 30, kBThreads) / kNumSMs;
    const int per_sm = p->opts.blocks_per_sm < resident ? p->opts.blocks_per_sm : resident;
    batch_join_kernel<<<kNumSMs * per_sm, kBThreads, 0, s>>>(a);
    VS_LAUNCHED("batch_join", s);
    if (mask) {
        batch_resolve_kernel<<<resident_grid(batch_resolve_kernel, (int64_t)1 << 30, kBThreads), kBThreads, 0, s>>>(a);
        VS_LAUNCHED("batch_resolve", s);
    }
    return VS_OK;
}

int capture_graph(vs_batch_plan* p, int32_t predicate, int mask, int32_t* left, int32_t* right, int64_t capacity) {
    if (p->graph) {
        cudaGraphExecDestroy(p->graph);
        p->graph = nullptr;
    }
    p->g_pred = -1;
    cudaGraph_t g = nullptr;
    VS_CUDA_TRY(cudaStreamBeginCapture(p->gstream, cudaStreamCaptureModeThreadLocal));
    const long long l0 = g_launches;
    const int st = enqueue_batch(p, p->gstream, mask, left, right, capacity);
    p->g_kernels = g_launches - l0;
    const cudaError_t e = cudaStreamEndCapture(p->gstream, &g);
    if (st != VS_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) {
        set_error("stream capture of the batched join failed: %s", cudaGetErrorString(e));
        return VS_E_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiate(&p->graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        p->graph = nullptr;
        set_error("cudaGraphInstantiate failed: %s", cudaGetErrorString(ei));
        return VS_E_CUDA;
    }
    p->g_pred = predicate;
    p->g_left = left;
    p->g_right = right;
    p->g_cap = capacity;
    return VS_OK;
}

}  // namespace
}  // namespace vs

using namespace vs;

extern "C" {

int vs_batch_plan_create(vs_context* ctx, const vs_index* const* indexes, int32_t n_jobs, const vs_points* pts,
                         const int64_t* h_job_start, const vs_batch_options* opts, vs_batch_plan** out) {
    if (!ctx || !indexes || !pts || !h_job_start || !out) {
        set_error("ctx/indexes/pts/job_start/out is NULL");
        return VS_E_ARG;
    }
    *out = nullptr;
    if (n_jobs <= 0 || n_jobs > kMaxJobs) {
        set_error("n_jobs %d outside [1, %d]", n_jobs, kMaxJobs);
        return VS_E_ARG;
    }
    VS_TRY(check_points(pts));
    const int64_t N = pts->n;
    if (h_job_start[0] != 0 || h_job_start[n_jobs] != N) {
        set_error("job_start must run from 0 to the point count %lld", (long long)N);
        return VS_E_ARG;
    }
    for (int j = 0; j < n_jobs; ++j) {
        if (h_job_start[j + 1] < h_job_start[j]) {
            set_error("job %d: job_start is decreasing", j);
            return VS_E_ARG;
        }
        if (!indexes[j] || indexes[j]->device != ctx->device) {
            set_error("job %d: index is NULL or lives on another device", j);
            return VS_E_ARG;
        }
    }
    VS_TRY(use_device(ctx->device));
    vs_batch_plan* p = new (std::nothrow) vs_batch_plan{};
    if (!p) {
        set_error("host allocation failed");
        return VS_E_OOM;
    }
    p->ctx = ctx;
    p->n_jobs = n_jobs;
    p->n_points = N;
    p->pts = *pts;
    p->opts = opts ? *opts : vs_batch_options{};
    if (p->opts.blocks_per_sm <= 0) p->opts.blocks_per_sm = 4;
    if (p->opts.blocks_per_sm > 8) p->opts.blocks_per_sm = 8;
    if (p->opts.packets_per_grab <= 0) p->opts.packets_per_grab = 4;
    if (p->opts.sort_levels <= 0) p->opts.sort_levels = 8;
    if (p->opts.learned_map_blocks_per_sm < 0 || p->opts.learned_map_blocks_per_sm > 8 ||
        p->opts.learned_refine_blocks_per_sm < 0 || p->opts.learned_refine_blocks_per_sm > 8 ||
        p->opts.learned_grab < 0 || p->opts.learned_grab > 4096 || p->opts.learned_map_packets < 0 ||
        p->opts.learned_map_packets > 2 ||
        (p->opts.learned_flags &
         ~(VS_JOIN_LEARNED_BSEARCH | VS_JOIN_LEARNED_FP64_WALK | VS_JOIN_LEARNED_NO_STAGE |
           VS_JOIN_LEARNED_NO_INTERIOR)) != 0) {
        set_error("learned launch shape out of range (blocks per SM 0..8, grab 0..4096, map packets 0..2, flags 4|8|16|32)");
        delete p;
        return VS_E_ARG;
    }
    // key = job id in the top bits, Hilbert cell below; 2^job_bits > n_jobs,
    // so the all-ones sentinel never collides with a valid key
    const int job_bits = bits_needed(n_jobs);
    p->job_shift = 32 - job_bits;
    p->key_levels = p->job_shift / 2;
    const int sort_levels = p->opts.sort_levels < p->key_levels ? p->opts.sort_levels : p->key_levels;
    p->sort_begin = 2 * (p->key_levels - sort_levels);
    std::vector<JobTree> jobs(n_jobs);
    for (int j = 0; j < n_jobs; ++j) {
        const vs_index* ix = indexes[j];
        JobTree& t = jobs[j];
        t = JobTree{};
        t.nodes = ix->nodes;
        t.item_geom = ix->item_geom;
        t.geom_off = ix->geom_off;
        t.part_off = ix->part_off;
        t.ring_off = ix->ring_off;
        t.xy = ix->xy;
        for (int l = 0; l < kMaxLevels; ++l) {
            t.level_off[l] = ix->level_off[l];
            t.level_size[l] = ix->level_size[l];
        }
        for (int k = 0; k < 4; ++k) t.frame[k] = ix->h_frame[k];
        t.levels = ix->levels;
        t.n_geoms = ix->levels > 0 ? ix->n_geoms : 0;
        t.rings = ix->ring_index();
        p->has_ring_bins = p->has_ring_bins || ix->n_split_binned_rings > 0;
    }
    p->learned = p->opts.method == VS_METHOD_LEARNED;
    if (p->opts.method != VS_METHOD_RTREE && !p->learned) {
        set_error("batch method %d: use VS_METHOD_RTREE or VS_METHOD_LEARNED", p->opts.method);
        delete p;
        return VS_E_ARG;
    }
    std::vector<LearnedJob> ljobs;
    if (p->learned) {
        ljobs.resize(n_jobs);
        int64_t base = 0;
        for (int j = 0; j < n_jobs; ++j) {
            const vs_index* ix = indexes[j];
            LearnedJob& d = ljobs[j];
            d = LearnedJob{};
            const bool has_polys = ix->n_geoms > 0 && ix->h_frame[0] <= ix->h_frame[2];
            if (ix->has_learned) {
                d = ix->learned.h_desc;
                d.cell_base = (uint32_t)base;
                base += ix->learned.n_cells;
            } else if (has_polys) {
                set_error("job %d: index was built without its learned part", j);
                delete p;
                return VS_E_ARG;
            }
        }
        if (base >= 0x7fffffffLL) {
            set_error("batch has %lld learned cells (at most 2^31-1)", (long long)base);
            delete p;
            return VS_E_ARG;
        }
        p->n_cells = base;
        p->h_single = ljobs[0];
    }
    p->defer_cap = (unsigned long long)(N / 16 + (1 << 16));
    const size_t nn = (size_t)(N > 0 ? N : 1);
    if (cudaMalloc((void**)&p->d_jobs, sizeof(JobTree) * n_jobs) != cudaSuccess ||
        cudaMalloc((void**)&p->d_job_start, sizeof(int64_t) * (n_jobs + 1)) != cudaSuccess ||
        cudaMalloc((void**)&p->keys, sizeof(uint32_t) * nn) != cudaSuccess ||
        cudaMalloc((void**)&p->order, sizeof(uint32_t) * nn) != cudaSuccess ||
        cudaMalloc((void**)&p->defer, sizeof(int2) * p->defer_cap) != cudaSuccess ||
        cudaMalloc((void**)&p->d_work, 2 * sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc((void**)&p->d_n_valid, sizeof(uint32_t)) != cudaSuccess ||
        (p->learned && (cudaMalloc((void**)&p->d_ljobs, sizeof(LearnedJob) * n_jobs) != cudaSuccess ||
                        cudaMalloc(&p->lscratch, learned_scratch_bytes(N, p->n_cells)) != cudaSuccess))) {
        cudaGetLastError();
        set_error("batch plan allocation failed (%lld points)", (long long)N);
        free_plan(p);
        delete p;
        return VS_E_OOM;
    }
    if (cudaStreamCreateWithFlags(&p->gstream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&p->ev_out, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&p->t0) != cudaSuccess || cudaEventCreate(&p->t1) != cudaSuccess) {
        cudaGetLastError();
        set_error("batch plan stream/event creation failed");
        free_plan(p);
        delete p;
        return VS_E_CUDA;
    }
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaMemcpyAsync(p->d_jobs, jobs.data(), sizeof(JobTree) * n_jobs, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(p->d_job_start, h_job_start, sizeof(int64_t) * (n_jobs + 1), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && p->learned) {
        e = cudaMemcpyAsync(p->d_ljobs, ljobs.data(), sizeof(LearnedJob) * n_jobs, cudaMemcpyHostToDevice, s);
        learned_scratch_carve(p->lscratch, N, p->n_cells, p->lsc);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        set_error("batch plan upload failed: %s", cudaGetErrorString(e));
        free_plan(p);
        delete p;
        return VS_E_CUDA;
    }
    *out = p;
    return VS_OK;
}

int vs_batch_run(vs_batch_plan* p, int32_t predicate, int32_t* d_left, int32_t* d_right, int64_t capacity,
                 int32_t use_graph, int64_t* n_pairs, vs_join_stats* stats) {
    if (!p || !n_pairs) {
        set_error("plan/n_pairs is NULL");
        return VS_E_ARG;
    }
    *n_pairs = 0;
    if (stats) memset(stats, 0, sizeof(*stats));
    if (capacity < 0 || (capacity > 0 && (!d_left || !d_right))) {
        set_error("invalid pair buffers (capacity %lld)", (long long)capacity);
        return VS_E_ARG;
    }
    int mask = 0;
    VS_TRY(accept_mask_for(predicate, &mask));
    vs_context* ctx = p->ctx;
    VS_TRY(use_device(ctx->device));
    if (p->n_points == 0) return VS_OK;
    cudaStream_t s = ctx->stream;
    unsigned long long* h = ctx->h_counter;  // pinned: the context counters, then the plan's two
    long long launches = 0;
    // Pairs the filters cannot certify go to the plan's deferred buffer; if
    // more were deferred than it holds, it grows to fit and the batch runs
    // once more (the graph is captured again for the new buffer).
    for (int attempt = 0; attempt < 2; ++attempt) {
        launches = g_launches;
        if (use_graph) {
            if (!p->graph || p->g_pred != predicate || p->g_left != d_left || p->g_right != d_right ||
                p->g_cap != capacity)
                VS_TRY(capture_graph(p, predicate, mask, d_left, d_right, capacity));
            VS_CUDA_TRY(cudaEventRecord(p->ev_in, s));
            VS_CUDA_TRY(cudaStreamWaitEvent(p->gstream, p->ev_in, 0));
            VS_CUDA_TRY(cudaEventRecord(p->t0, p->gstream));
            VS_CUDA_TRY(cudaGraphLaunch(p->graph, p->gstream));
            VS_CUDA_TRY(cudaEventRecord(p->t1, p->gstream));
            VS_CUDA_TRY(cudaEventRecord(p->ev_out, p->gstream));
            VS_CUDA_TRY(cudaStreamWaitEvent(s, p->ev_out, 0));
            launches = p->g_kernels;
        } else {
            VS_CUDA_TRY(cudaEventRecord(p->t0, s));
            VS_TRY(enqueue_batch(p, s, mask, d_left, d_right, capacity));
            VS_CUDA_TRY(cudaEventRecord(p->t1, s));
            launches = g_launches - launches;
        }
        VS_CUDA_TRY(cudaMemcpyAsync(h, ctx->d_counters, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        VS_CUDA_TRY(cudaMemcpyAsync(h + 8, p->d_work, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        const cudaError_t e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            set_error("batched join failed: %s", cudaGetErrorString(e));
            return VS_E_CUDA;
        }
        if (h[9] <= p->defer_cap || attempt == 1) break;
        const unsigned long long want = h[9] + h[9] / 8 + (1 << 16);
        int2* grown = nullptr;
        if (cudaMalloc((void**)&grown, sizeof(int2) * want) != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaMalloc of the deferred-pair buffer (%llu pairs) failed", want);
            return VS_E_OOM;
        }
        cudaFree(p->defer);
        p->defer = grown;
        p->defer_cap = want;
        if (p->graph) {
            cudaGraphExecDestroy(p->graph);
            p->graph = nullptr;
        }
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p->t0, p->t1);
    *n_pairs = (int64_t)h[0];
    if (stats) {
        stats->exact_fallbacks = (int64_t)h[1];
        stats->fp32_edges = (int64_t)h[2];
        stats->fp64_edges = (int64_t)h[3];
        stats->candidates = (int64_t)h[5];
        stats->rmi_fallbacks = (int64_t)h[6];
        stats->kernel_ms = ms;
        stats->kernel_launches = launches;
    }
    if (h[4] & 2) {
        set_error("a bounded device wait (bulk copy) gave up; the batch's result is incomplete");
        return VS_E_TIMEOUT;
    }
    if (h[4]) {
        set_error("device-side consistency check failed (flags 0x%llx)", h[4]);
        return VS_E_STATE;
    }
    if (h[9] > p->defer_cap) {
        set_error("deferred-pair buffer of the batch plan did not converge (%llu > %llu pairs)", h[9], p->defer_cap);
        return VS_E_STATE;
    }
    if ((int64_t)h[0] > capacity) {
        set_error("pair buffer holds %lld pairs, %llu required", (long long)capacity, h[0]);
        return VS_E_CAPACITY;
    }
    return VS_OK;
}

int vs_batch_plan_free(vs_batch_plan* p) {
    if (!p) return VS_OK;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    if (p->gstream) cudaStreamSynchronize(p->gstream);
    free_plan(p);
    delete p;
    return VS_OK;
}

}  // extern "C"
