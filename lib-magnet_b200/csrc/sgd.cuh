// Sampled SGD layout on the device (optimize_layout, src/layout.cpp:343-472).
#pragma once
#include "common.cuh"

namespace mgb {

// An edge's read-only fields, packed for the split form (one 8-byte load per sample)
struct alignas(8) EdgeRO {
    int32_t tail;
    float eps;
};

// Everything an epoch kernel reads (the reference's Ctx, src/layout.cpp:69-88), as device pointers plus the
// scalars derived once per call (src/layout.cpp:421-431).
struct SgdDev {
    float* Y; int64_t n; int dim;
    const int32_t* head; const int32_t* tail; const float* eps; float* eons; float* eonns; int64_t n_edges;
    const int32_t* indptr; const int32_t* indices; const int32_t* walk_lens;
    const int32_t* mid_pairs; int n_mid;
    const int32_t* jump_indptr; const int32_t* jump_indices; float mid_jump;
    float a, b, two_ab, two_b, negative_sample_rate, exaggeration, repulsion_strength, mid_rate;
    float rep_a, rep_b;
    bool b_is_one, rep_b_is_one, rep_coupled, use_mid;
    int m_neg, walk_len, loss, clip_mode, kernel, optimizer;
    int64_t n_fixed;
    const float* node_b;
    float* adam_m; float* adam_v; int32_t* adam_t; float beta1, beta2;
    uint64_t seed;
    // the split form's packed copies for one call: (eons, eonns) per edge, and (tail, eps) per edge
    float2* eo = nullptr;
    const EdgeRO* te = nullptr;
};

// launches F<2>, F<3> or the generic F<0> (dims up to kMaxDim) for a layout of `dim` columns
#define MGB_DIM_DISPATCH(dim, F, ...)                \
    switch (dim) {                                   \
        case 2: F<2>(__VA_ARGS__); break;            \
        case 3: F<3>(__VA_ARGS__); break;            \
        default: F<0>(__VA_ARGS__); break;           \
    }

// device scratch of the stream modes and of owner mode
struct SgdWork {
    DevBuf cnt, state, delta, eptr, flag;
    DevBuf samp;               // the epoch's sampled set (counter mode fast path)
    DevBuf pack;               // the split form's packed edge fields
    // owner mode: node rows, chunk bounds, per-edge negatives, per-node stream states, marked chunks, snapshots
    DevBuf o_row, o_own, o_neg, o_state, o_dirty, o_snap, o_snap_m, o_snap_v, o_snap_t;
};

void sgd_sched(const SgdDev& c, int epoch, int e0, int e1, float alpha0, float alpha1, float mid_w0, float mid_w1,
               float& alpha, float& mid_w);
// epochs [e0, e1) (one optimize_layout call), asynchronous on s
void sgd_run(SgdDev& c, SgdWork& w, int stream_mode, int e0, int e1, float alpha0, float alpha1, float mid_w0,
             float mid_w1, cudaStream_t s);
// draws of one epoch without updates (device outputs); advances eons / eonns
void sgd_record(SgdDev& c, SgdWork& w, int stream_mode, int epoch, float alpha, float mid_w, int32_t* n_neg_out,
                int64_t* off_out, int32_t* negs, int64_t negs_cap, int32_t* mid, int64_t* n_negs_dev,
                cudaStream_t s);

// owner mode (parallel = 1, src/layout.cpp:441-463): chunk count for E edges (chunk_edges 0: the reference's
// min(4096, max(1, E / 4096)); else max(1, E / chunk_edges)), the sorted-heads check (device heads; synchronises
// s), and epochs [e0, e1); the reverse mid pairs are device arrays or NULL
int owner_chunk_count(int64_t n_edges, int chunk_edges);
bool owner_heads_sorted(const int32_t* head_dev, int64_t n_edges, SgdWork& w, cudaStream_t s);
void owner_run(SgdDev& c, SgdWork& w, const int32_t* rev_indptr, const int32_t* rev_indices, int chunk_edges,
               int e0, int e1, float alpha0, float alpha1, float mid_w0, float mid_w1, cudaStream_t s);

}  // namespace mgb
