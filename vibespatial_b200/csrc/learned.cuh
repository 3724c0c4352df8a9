// Query side of the learned cell index, shared by single joins (vs_join) and
// batch plans (vs_batch_run).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "emit.cuh"
#include "index.cuh"

namespace vs {

// Per-query scratch of the learned pipeline (points n, batch-wide cells).
struct LearnedScratch {
    void* staged = nullptr;          // striped staging regions of matched points (CellPoint)
    uint32_t* stripe_count = nullptr;
    int64_t stripe_cap = 0;
    uint32_t* cell_count = nullptr;  // counts, then start offsets after the scan
    void* grouped = nullptr;         // matched points in cell order (CellPoint)
    uint32_t* n_grouped = nullptr;
};

// Bytes of scratch for n points and n_cells cells.
size_t learned_scratch_bytes(int64_t n, int64_t n_cells);
// Carve the scratch out of one device buffer of learned_scratch_bytes().
void learned_scratch_carve(void* base, int64_t n, int64_t n_cells, LearnedScratch& sc);

// Points and jobs of one learned query; job_start is null for one job.
struct LearnedQuery {
    const double* px;
    const double* py;
    const uint8_t* pvalid;
    int64_t n;
    const LearnedJob* jobs;
    int32_t n_jobs;
    const int64_t* job_start;
    int64_t n_cells;  // batch-wide cells
    int accept_mask;
    bool has_ring_bins;  // some job's index has y-binned rings long enough for the split walk
    int64_t row_base;    // added to every emitted / deferred point row (chunked joins)
    LearnedShape shape;  // launch shape and ablation switches (zero = defaults)
};

// Enqueue map -> scan -> place -> refine on stream s (no host
// synchronisation; capturable).  For one job, `single` is its descriptor
// (host copy, passed as a kernel parameter); q.jobs is used for batches.
// ctx (may be null) receives phase marks 1, 2.
int enqueue_learned(cudaStream_t s, vs_context* ctx, const LearnedQuery& q, const LearnedJob* single,
                    const LearnedScratch& sc, const PairSink& sink, const DeferSink& defer,
                    unsigned long long* counters, unsigned long long* work);

}  // namespace vs
