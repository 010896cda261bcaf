// The fuzzy neighbour graph on the device: smooth_knn (src/graph.cpp:29-78) and the fuzzy union of
// magnet/knn.py:215-230 (A + A^T - A o A^T over the kNN memberships).
#pragma once
#include "common.cuh"

namespace mgb {

// device scratch of the graph passes
struct GraphWork {
    DevBuf sigma, rho, part, acol, aval, alen, tcnt, tptr, tcur, trow, tval, ucnt, uptr, scan, flag;
    DevBuf mid_state, mid_tab;   // mid-near partners: per-row stream states, jump tables and chunk tables
    DevBuf sched;                // the transform schedule's kept-edge count
    DevBuf s_part, s_flag, s_off, s_tmp;   // the fit schedule's block partials, keep flags, offsets, scan tiles
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

// Mid-near partners of dense rows X (n, d) (src/nndescent.cpp:731-768): out (n, n_pairs), for every row and pair
// the second closest (squared distance, index) of n_cand draws, with the reference's streams for `n_threads`
// threads (>= 1) and its squared-distance kernel `order` (0 AVX-512, 1 AVX2, 2 plain loop).
void mid_near_pairs_dev(const float* X, int64_t n, int d, int n_pairs, int n_cand, uint64_t seed, int n_threads,
                        int order, int32_t* out, GraphWork& w, cudaStream_t s);
// The edge schedule of MAGNET.transform (magnet/__init__.py:907-912) for memberships w (m, k) of m new rows and
// their neighbours ind (m, k): the kept edges in row order as (head = n_train + row, tail, eps = 1 / freq), with
// freq = min(1, s w) summing to samples_per_node * m and kept when freq >= 1 / n_epochs. head, tail and eps hold
// m * k entries; returns the number kept (synchronises s).
int64_t transform_schedule_dev(const float* w, const int64_t* ind, int64_t m, int k, int64_t n_train,
                               double samples_per_node, int n_epochs, int32_t* head, int32_t* tail, float* eps,
                               GraphWork& gw, cudaStream_t s);
// The edge schedule of a fit (MAGNET._edge_schedule, magnet/__init__.py:726-737) for the CSR graph (indptr, indices,
// data) of n nodes: freq = min(1, s w) over the nnz entries, summing to samples_per_node * n, the entries with
// freq >= 1 / n_epochs kept in CSR order as (head = row, tail = column, eps = 1 / freq) into arrays of nnz entries.
// s is bracketed by bisection with block-partial sums added on the host in block order (the same bits every call),
// then solved exactly on its segment. Returns the number kept (synchronises s).
int64_t edge_schedule_dev(const int32_t* indptr, const int32_t* indices, const float* w, int64_t n, int64_t nnz,
                          double samples_per_node, int n_epochs, int32_t* head, int32_t* tail, float* eps,
                          GraphWork& gw, cudaStream_t s);
// out[0..n] = exclusive scan of in[0..n) and, in out[n], the total (tmp: tile sums)
void exclusive_scan_i32(const int32_t* in, int64_t n, int64_t* out, DevBuf& tmp, cudaStream_t s);
// knn_search (src/nndescent.cpp:585-690): the beam search of queries Q (m, d) over the training rows X (n, d) and
// their neighbour graph (gptr, gidx), from the n_entry landmarks closest to each query, or from the given random
// entry rows (host array m x n_entry) without landmarks; out (m, k) rows and squared distances. ef <=
// knn_search_max_ef(). Synchronises s.
void knn_search_dev(const float* X, int64_t n, int d, const int32_t* gptr, const int32_t* gidx, const int32_t* land,
                    int64_t n_land, const int32_t* entries_host, const float* Q, int64_t m, int k, int ef,
                    int n_entry, int order, int32_t* out_i, float* out_d, cudaStream_t s);
int knn_search_max_ef();
// the reference's distance kernel on this host (its CPUID choice, src/nndescent.cpp:101-106)
int host_distance_order();

}  // namespace mgb
