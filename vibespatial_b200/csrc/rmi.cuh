// Recursive model index (RMI) evaluation.
//
// The root MLP (FP32, 1 -> 32 -> 32 -> 1) maps a normalised ancestor-cell key
// to [0, 1); leaf = floor(y * n_leaves).  It is evaluated by a full warp for
// one input (lane j owns hidden unit j) when the root table is built; queries
// only read the table.  Leaf models predict a position from the full cell key
// in FP64.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "index.cuh"

namespace vs {

// Shared-memory copy of the root MLP with W2 transposed (w2t[k*32 + j] =
// W2[j][k]) so that lane j reading column k is bank-conflict free.
struct RmiShared {
    float w1[kRmiHidden], b1[kRmiHidden];
    float w2t[kRmiHidden * kRmiHidden];
    float b2[kRmiHidden], w3[kRmiHidden];
    float b3;
    double key_lo, key_scale;
    int n_leaves;
};

__device__ __forceinline__ void rmi_load_shared(RmiShared* s, const RmiModel* m) {
    for (int i = threadIdx.x; i < kRmiHidden * kRmiHidden; i += blockDim.x) {
        const int j = i / kRmiHidden, k = i % kRmiHidden;
        s->w2t[k * kRmiHidden + j] = m->w2[i];
    }
    for (int i = threadIdx.x; i < kRmiHidden; i += blockDim.x) {
        s->w1[i] = m->w1[i];
        s->b1[i] = m->b1[i];
        s->b2[i] = m->b2[i];
        s->w3[i] = m->w3[i];
    }
    if (threadIdx.x == 0) {
        s->b3 = m->b3;
        s->key_lo = m->key_lo;
        s->key_scale = m->key_scale;
        s->n_leaves = m->n_leaves;
    }
}

// Normalised root input of an ancestor-cell key.
__device__ __forceinline__ float rmi_input(uint32_t anc, const RmiShared* s) {
    return __double2float_rn(__dmul_rn((double)anc - s->key_lo, s->key_scale));
}

// Root MLP for ONE input, evaluated by the whole warp (lane j = hidden unit
// j); the xor-butterfly sum leaves the same bits in every lane.
__device__ __forceinline__ float rmi_root_warp(const RmiShared* s, float x) {
    const int j = threadIdx.x & 31;
    const float h1 = fmaxf(__fmaf_rn(s->w1[j], x, s->b1[j]), 0.0f);
    float z2 = s->b2[j];
#pragma unroll
    for (int k = 0; k < kRmiHidden; ++k) z2 = __fmaf_rn(s->w2t[k * kRmiHidden + j], __shfl_sync(0xffffffffu, h1, k), z2);
    float t = __fmul_rn(s->w3[j], fmaxf(z2, 0.0f));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t = __fadd_rn(t, __shfl_xor_sync(0xffffffffu, t, o));
    return __fadd_rn(t, s->b3);
}

__device__ __forceinline__ int rmi_leaf(int n_leaves, float y) {
    const float f = floorf(__fmul_rn(y, (float)n_leaves));
    // NaN lands in leaf 0 like any other value: routing only has to be deterministic.
    return (f >= 0.0f) ? (f < (float)n_leaves ? (int)f : n_leaves - 1) : 0;
}

// Leaf model: predicted position = floor(a + b * key) in FP64, clamped to
// +-2^40 so that adding an error bound cannot overflow.
__device__ __forceinline__ long long rmi_predict(const double2 ab, uint32_t key) {
    const double p = floor(__fma_rn(ab.y, (double)key, ab.x));
    const double c = 1099511627776.0;
    return (long long)(p >= -c ? (p <= c ? p : c) : -c);
}

}  // namespace vs
