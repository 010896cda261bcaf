// The fuzzy neighbour graph on the device: smooth_knn (src/graph.cpp:29-78) and the fuzzy union of
// magnet/knn.py:215-230 (A + A^T - A o A^T over the kNN memberships).
#pragma once
#include "common.cuh"

namespace mgb {

// device scratch of the graph passes
struct GraphWork {
    DevBuf sigma, rho, part, acol, aval, alen, tcnt, tptr, tcur, trow, tval, ucnt, uptr, scan, flag;
};

// memberships (n_rows, k) of sorted neighbour distances; `target` = log2(n_neighbors) * bandwidth, computed by the
// caller with the host libm as the reference computes it
void smooth_knn_dev(const float* dist, int64_t n_rows, int k, float target, int n_iter, float* out, GraphWork& w,
                    cudaStream_t s);

// Fuzzy union of A = (i, ind[i, j], vals[i, j]) over an n x n graph (rows past n_rows empty): indptr (n + 1),
// indices / data (cap). Returns nnz (synchronises s); throws when an index is out of range or nnz exceeds cap.
int64_t fuzzy_union_dev(const int32_t* ind, const float* vals, int64_t n_rows, int k, int64_t n, float mix,
                        float one_minus_mix, int32_t* indptr, int32_t* indices, float* data, int64_t cap,
                        GraphWork& w, cudaStream_t s);

}  // namespace mgb
