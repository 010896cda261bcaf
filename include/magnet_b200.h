/*
 * magnet_b200 — C ABI of the B200 (sm_100a) layout pass of MAGNET.
 *
 * The entry points replace the native functions of the reference's pybind11 module `_magnet`
 * (kerighan/lib-magnet 3.0.2, src/bindings.cpp:8-83) that make up the layout pass. Arguments are plain
 * pointers and sizes. Every array pointer may be HOST memory (the call stages it through device buffers and
 * copies results back before returning) or DEVICE memory from cudaMalloc (used in place; the call is then
 * asynchronous on the calling thread's stream, see mg_set_stream). Arrays are C-contiguous, float32 / int32
 * unless stated otherwise, as the reference requires of its numpy arguments (src/layout.hpp:11-15).
 *
 * Every function returns MG_OK (0) or an error code; mg_last_error() then gives the message (thread-local).
 * The pybind11 shim `_magnet` raises RuntimeError with that message, like the reference's `require`
 * (src/layout.hpp:34).
 */
#ifndef MAGNET_B200_H
#define MAGNET_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    MG_OK = 0,
    MG_ERR_ARGUMENT = 1,      /* invalid argument (the reference's std::runtime_error from require) */
    MG_ERR_OUT_OF_MEMORY = 2, /* device allocation failed */
    MG_ERR_DEVICE = 3,        /* CUDA error */
    MG_ERR_TIMEOUT = 4,       /* a bounded device-side wait gave up */
    MG_ERR_NOT_SUPPORTED = 5, /* option not available on this path */
    MG_ERR_INTERNAL = 6
};

/* Message of the last failed call on this host thread ("" if none). */
const char* mg_last_error(void);
/* Library version (major*10000 + minor*100 + patch). */
int mg_version(void);
/* Stream used by this host thread's calls (a cudaStream_t; NULL = the legacy default stream). */
int mg_set_stream(void* stream);
/* Waits for all work of this host thread's stream. */
int mg_synchronize(void);
/* Number of device kernels this library has launched in the process so far (a CUDA-graph replay counts each
 * kernel node). */
uint64_t mg_launch_count(void);

/* ================================================================ FFT-interpolated repulsion
 * Persistent object with device buffers; replaces class FFTConv2D (src/fftconv.cpp:43-244).
 * Not reentrant: one object per stream, like the reference's object (its buffers are shared). */
typedef struct mg_fftconv mg_fftconv;

/* FFTConv2D(M, n_interp) (src/fftconv.cpp:45-47, bound at :241): M = padded FFT side, any 5-smooth M >= 2. */
int mg_fftconv_create(int M, int n_interp, mg_fftconv** out);
/* FFTConv2D.set_kernels(K1h, K2h) (src/fftconv.cpp:51-55): real spectra, (M, M/2+1) each, row-major. */
int mg_fftconv_set_kernels(mg_fftconv* h, const float* K1h, const float* K2h, int64_t rows, int64_t cols);
/* FFTConv2D.compute(Y, xmin, ymin, width, n_boxes) (src/fftconv.cpp:58-230): Y (n, 2) -> *sumQ (sum of the
 * kernel over all pairs, self terms removed, FP64-accumulated) and F (n, 2) = sum_j K2(y_i - y_j)(y_i - y_j).
 * The live grid is N = n_boxes * n_interp <= M nodes per side. sumQ may point to host or device memory. */
int mg_fftconv_compute(mg_fftconv* h, const float* Y, int64_t n, float xmin, float ymin, float width,
                       int n_boxes, float* sumQ, float* F);
void mg_fftconv_destroy(mg_fftconv* h);

/* No counterpart in the reference: FFTConv2D(M, n_interp).set_kernels(K1h, K2h).compute(Y, ...) in one call
 * that allocates nothing, for callers that must not allocate device memory, e.g. a process whose device memory
 * is already reserved up to its budget, or a thread that must not stall the other streams on the implicit
 * device synchronisation of cudaMalloc / cudaFree. Same arguments and results as mg_fftconv_create +
 * mg_fftconv_set_kernels + mg_fftconv_compute, with three limits:
 *   - M <= mg_fftconv_noalloc_max_side() (512, so n_boxes * n_interp <= 512); larger M returns MG_ERR_ARGUMENT.
 *   - K1h, K2h ((M, M/2+1) real each), Y, F ((n, 2)) and sumQ must be device memory; nothing is staged.
 *   - The scratch is one static device array (16.8 MB) per device, shared by all callers of this entry point:
 *     calls whose work overlaps on the device (two streams, or two host threads) race on it and must be
 *     serialised by the caller.
 * The first call on each device looks up the scratch's device address (cudaGetSymbolAddress, which may load
 * the library's module); make that first call before any stream capture. Asynchronous on the thread's stream
 * (mg_set_stream). */
int mg_fftconv_compute_noalloc(const float* K1h, const float* K2h, int M, int n_interp, const float* Y, int64_t n,
                               float xmin, float ymin, float width, int n_boxes, float* sumQ, float* F);
/* The largest FFT side M that mg_fftconv_compute_noalloc accepts. */
int mg_fftconv_noalloc_max_side(void);

/* ================================================================ t-SNE per-iteration kernels (src/fftrep.cpp) */
/* tsne_attraction (src/fftrep.cpp:129-177): out_i = sum_j p_ij (1 + |y_i - y_j|^2/dof)^-1 (y_i - y_j) over the
 * CSR rows (indptr n+1, indices / data nnz); Y and out (n, dim), 1 <= dim <= 64. */
int mg_tsne_attraction(const int32_t* indptr, const int32_t* indices, const float* data, int64_t nnz,
                       const float* Y, int64_t n, int dim, float dof, float* out);
/* tsne_step (src/fftrep.cpp:225-266): grad = rho*attr - F*inv_sumQ; delta-bar-delta gains, momentum update,
 * position update and recentring, in place on Y, update, gains (n, dim). */
int mg_tsne_step(float* Y, float* update, float* gains, const float* attr, const float* F, int64_t n, int dim,
                 float rho, float inv_sumQ, float lr, float momentum);
/* tsne_update (src/fftrep.cpp:181-220): the same update from a materialised gradient. */
int mg_tsne_update(float* Y, float* update, float* gains, const float* grad, int64_t n, int dim, float lr,
                   float momentum);
/* bbox_2d (src/fftrep.cpp:415-434): out4 = (xmin, ymin, xmax, ymax) of Y (n, 2), n >= 1. */
int mg_bbox_2d(const float* Y, int64_t n, float* out4);
/* mid_spring (src/fftrep.cpp:270-287): grad_i += w (Y_i - mean of the positions of the partners of i); Y and grad
 * (n, dim), pairs (n, m) with m >= 1. grad is updated in place. */
int mg_mid_spring(const float* Y, const int32_t* pairs, float* grad, int64_t n, int dim, int m, float w);

/* ================================================================ whole t-SNE pass on the device
 * optimize_tsne (magnet/tsne.py:132-214, the common path without mid-range or far-field terms): P is a
 * symmetric CSR affinity matrix (normalised to sum 1 inside), Y (n, 2) the initial layout, updated in place.
 * Each iteration (attraction, bounding box and grid choice, spread, FFT convolution, gather, gains/momentum
 * step, recentring) runs on the device without host synchronisation and is replayed as a CUDA graph. */
typedef struct {
    int n_iter;                  /* 750 */
    int early_iter;              /* 250 */
    float early_exaggeration;    /* 12 */
    float exaggeration;          /* 1 */
    float learning_rate;         /* <= 0: max(200, n / early_exaggeration) (magnet/tsne.py:152-153) */
    float momentum_early;        /* 0.5 */
    float momentum_late;         /* 0.8 */
    int n_interp;                /* 3 */
    float box_width;             /* 0.7 */
    int min_boxes;               /* 20 */
    int max_boxes;               /* 1000 */
    float dof;                   /* 1 (Student-t degrees of freedom) */
    int threads_per_row;         /* attraction lanes per point, 0 = chosen from the mean degree */
    int use_graph;               /* 1: replay each iteration as a CUDA graph (default), 0: plain launches */
} mg_tsne_params;

/* Fills p with the reference's defaults (the values in the comments above). */
void mg_tsne_params_default(mg_tsne_params* p);
int mg_optimize_tsne(const int32_t* indptr, const int32_t* indices, const float* P, int64_t n, int64_t nnz,
                     float* Y, const mg_tsne_params* p);
/* The same pass with per-stage timing: plain launches bracketed by CUDA events on the calling thread's stream.
 * stage_ms[9] receives the summed milliseconds of: 0 bbox + grid choice, 1 twiddles, 2 kernel spectra,
 * 3 spread, 4 forward row FFTs, 5 column FFT convolution, 6 inverse row FFTs, 7 gather + attraction + step,
 * 8 all; grid[4] receives the last iteration's (n_boxes, N, M, Mh). */
int mg_optimize_tsne_profiled(const int32_t* indptr, const int32_t* indices, const float* P, int64_t n, int64_t nnz,
                              float* Y, const mg_tsne_params* p, double* stage_ms, int* grid);
/* ================================================================ batched t-SNE layouts
 * Many independent optimize_tsne passes (magnet/tsne.py:132-214; the reference runs them as a loop of
 * optimize_tsne calls) of uneven size, run together: each layout keeps its own device state, and one CUDA graph
 * holds one iteration of every layout as independent branches (layout i on branch i mod `branches`), replayed
 * once per iteration. Every layout uses the same parameters p (n_iter, early_iter, schedule, n_interp, box width);
 * its grid is allocated for max_boxes[i] boxes per side (NULL: 64 + 2 ceil(sqrt(n_i)) rounded up to a multiple of
 * 4, capped by p->max_boxes), and a layout that outgrows it is clamped to that many boxes (wider boxes). The
 * arrays of layout i are indptr[i] (n[i] + 1), indices[i] / P[i] (nnz[i]), host or device; P is normalised to
 * sum 1 inside. */
typedef struct mg_tsne_batch mg_tsne_batch;
int mg_tsne_batch_create(int count, const int64_t* n, const int64_t* nnz, const int32_t* const* indptr,
                         const int32_t* const* indices, const float* const* P, const mg_tsne_params* p,
                         const int* max_boxes, int branches, mg_tsne_batch** out);
/* Runs p->n_iter iterations of every layout from Y[i] ((n[i], 2), host or device), updated in place. Synchronous.
 * The first run on a stream captures the iteration graph. */
int mg_tsne_batch_run(mg_tsne_batch* b, float* const* Y);
/* Layout count and kernels per replayed iteration (0 before the first run). */
int mg_tsne_batch_size(const mg_tsne_batch* b, int* count, uint64_t* kernels_per_iteration);
void mg_tsne_batch_destroy(mg_tsne_batch* b);

/* Hybrid hand-off (magnet/__init__.py:695-696): Y (n, dim) -= column means, then Y *= target_std / std(Y[:, 0]). */
int mg_center_scale(float* Y, int64_t n, int dim, double target_std);

/* ================================================================ sampled SGD
 * optimize_layout (src/layout.cpp:343-472, bound at src/bindings.cpp:11-23). Y (n, dim), eons / eonns and the
 * Adam state are updated in place; empty optional arrays are passed as NULL with length 0. */
typedef struct {
    float* Y; int64_t n; int dim;
    const int32_t* head; const int32_t* tail; const float* epochs_per_sample;
    float* epoch_of_next_sample; float* epoch_of_next_negative_sample; int64_t n_edges;
    const int32_t* indptr; const int32_t* indices; int64_t graph_nnz;       /* walks (n+1, nnz) or NULL */
    int epoch_start, epoch_end;
    float alpha0, alpha1, mid_w0, mid_w1;
    float a, b, rep_a, rep_b, negative_sample_rate;
    int loss;                    /* 0 umap, 1 infonce */
    float exaggeration, repulsion_strength;
    int walk_len; float mid_rate;
    int optimizer;               /* 0 sgd, 1 adam */
    int clip_mode;               /* 0 coord, 1 norm */
    int64_t n_fixed;
    float* adam_m; float* adam_v; int32_t* adam_t; float beta1, beta2;   /* (n, dim), (n, dim), (n) or NULL */
    const int32_t* walk_lens;                    /* (n) or NULL */
    const int32_t* mid_pairs; int n_mid;         /* (n, n_mid) or NULL */
    const int32_t* jump_indptr; const int32_t* jump_indices; int64_t jump_nnz; float mid_jump;
    int kernel;                  /* 0 power, 1 gaussian, 2 sech, 3 tanh */
    const float* node_b;         /* (n) or NULL */
    uint64_t seed;
    int n_threads;               /* accepted for signature parity; the device decides its own parallelism */
    int parallel;                /* 0 hogwild; 1 owner (src/layout.cpp:441-463): edges sorted by head, umap loss;
                                    one stream per chunk of about 4096 edges, reads from the epoch-start layout;
                                    deterministic, and bit-exact against the reference for the power kernel
                                    with b = rep_b = 1 under the sgd optimizer */
    int stream_mode;             /* hogwild only. 0 = counter-based draws per (epoch, edge, index) (fast, default);
                                    1 = the reference's single stream per epoch replayed exactly (serial mode),
                                        updates from an epoch snapshot in fixed point: deterministic */
    /* owner mode: who chose each node as a mid-range partner, CSR (n + 1, rev_nnz), or NULL
       (rev_indptr / rev_indices of src/bindings.cpp:23) */
    const int32_t* rev_indptr; const int32_t* rev_indices; int64_t rev_nnz;
    /* owner mode: edges per chunk; 0 = the reference's 4096 (src/layout.cpp:448). Smaller chunks give more
       independent streams (a deterministic result of its own, not the reference's owner stream assignment);
       the server uses them for small transforms. */
    int owner_chunk_edges;
} mg_layout_args;

/* Fills a with the reference's defaults for the scalars (pointers NULL). */
void mg_layout_args_default(mg_layout_args* a);
int mg_optimize_layout(const mg_layout_args* a);

/* Test hook: the draws of one epoch as the device makes them, without moving Y (eons / eonns advance as the
 * epoch would advance them). Outputs per edge: sampled (u8), n_neg (i32), neg_off (i64 offset into negs),
 * mid partner (i32: -1 none, -2 the partner was the head itself); negs receives up to negs_cap indices and
 * *n_negs the total drawn. */
int mg_layout_schedule(const mg_layout_args* a, int epoch, uint8_t* sampled, int32_t* n_neg, int64_t* neg_off,
                       int32_t* negs, int64_t negs_cap, int64_t* n_negs, int32_t* mid);

/* ================================================================ fuzzy neighbour graph
 * smooth_knn (src/graph.cpp:29-78, bound at src/bindings.cpp:73-74): dist (n, k) sorted distances to the
 * neighbours (self excluded) -> out (n, k) memberships in (0, 1]; the bisection of each row's bandwidth to
 * log2(n_neighbors) * bandwidth in n_iter steps at most. */
int mg_smooth_knn(const float* dist, int64_t n, int k, int n_neighbors, float bandwidth, int n_iter, float* out);

/* chebyshev_eigenvectors (src/spectral.cpp:141-241, bound at src/bindings.cpp; called by magnet/spectral.py:8-46,
 * the spectral initialisation): the Chebyshev-filtered subspace iteration with Rayleigh-Ritz for the leading
 * non-trivial eigenvectors of the lazy normalised adjacency (I + D^-1/2 A D^-1/2) / 2 of the graph (indptr,
 * indices, data; n nodes, nnz entries), the trivial eigenvector deflated per connected component (component
 * labels >= 0). X (n, p) row major: the start block in, the Ritz vectors out, columns by descending Ritz value.
 * inv_sqrt_deg: 1 / sqrt(degree) per node (0 where the degree is 0). 1 <= n_wanted < p <= 8 (larger p returns
 * MG_ERR_NOT_SUPPORTED), degree >= 2, max_iter >= 0, the reference's stopping rule with tol. FP64 on the device;
 * host or device arrays. Synchronises the stream. */
int mg_chebyshev_eigenvectors(const int32_t* indptr, const int32_t* indices, const float* data, int64_t n,
                              int64_t nnz, float* X, int p, const float* inv_sqrt_deg, const int32_t* component,
                              int n_wanted, int degree, int max_iter, float tol);

/* The edge schedule of a fit, MAGNET._edge_schedule (magnet/__init__.py:726-737, with _sampling_frequencies of
 * magnet/__init__.py:51-66), on the device: the CSR graph (indptr, indices, data) of n nodes -> the kept entries in
 * CSR order as head (row), tail (column) and eps = 1 / freq, with freq = min(1, s w) summing to
 * samples_per_node * n and kept when freq >= 1 / n_epochs; *n_kept their count. head, tail and eps hold nnz
 * entries. s is solved in FP64 (bisection with block sums added in a fixed order, then exactly on its segment), so
 * eps can differ from the host's sorted cumulative sum by FP64 rounding of s only. Host or device arrays. */
int mg_edge_schedule(const int32_t* indptr, const int32_t* indices, const float* data, int64_t n, int64_t nnz,
                     double samples_per_node, int n_epochs, int32_t* head, int32_t* tail, float* eps,
                     int64_t* n_kept);

/* The edge schedule of MAGNET.transform (magnet/__init__.py:907-912, with _sampling_frequencies of
 * magnet/__init__.py:51-66), on the device: w (m, k) memberships of m new rows and ind (m, k) their neighbours
 * among n_train fixed rows -> the kept edges in row order, head[e] = n_train + row, tail[e] = ind, eps[e] = 1 / freq,
 * with freq = min(1, s w) summing to samples_per_node * m and kept when freq >= 1 / n_epochs; *n_kept (host) their
 * count. head, tail and eps are device arrays of m * k entries. s is solved in FP64 (bisection, then exactly on
 * its segment), so eps can differ from the host's sorted cumulative sum by FP64 rounding only. Synchronises the
 * stream. */
int mg_transform_schedule(const float* w, const int64_t* ind, int64_t m, int k, int64_t n_train,
                          double samples_per_node, int n_epochs, int32_t* head, int32_t* tail, float* eps,
                          int64_t* n_kept);

/* mid_near_pairs_dense (src/nndescent.cpp:731-768, bound at src/bindings.cpp:58-59): X (n, d) dense rows -> out
 * (n, n_pairs), for every row and pair the second closest, by squared distance then index, of n_cand rows drawn
 * at random (the row itself replaced by the next row). The draws are the reference's streams for n_threads threads
 * (<= 0: the host's hardware threads, as the reference resolves it; the partners depend on it as the reference's
 * do) and the squared distances follow the reference's kernel for the host's instruction set, so out equals the
 * reference's output for the same n_threads on the same host. n_pairs >= 1, n_cand >= 2 and n > n_cand
 * (MG_ERR_ARGUMENT otherwise, with the reference's message). Synchronous. */
int mg_mid_near_pairs(const float* X, int64_t n, int d, int n_pairs, int n_cand, uint64_t seed, int n_threads,
                      int32_t* out);

/* knn_search (src/nndescent.cpp:585-690, bound at src/bindings.cpp:43-45; called by MAGNET.transform through
 * magnet/knn.py:131-152): the k nearest training rows of each query row by beam search over the training rows'
 * neighbour graph (gptr n + 1, gidx nnz), started from the n_entry landmarks closest to the query (n_land > 0) or
 * from n_entry random rows drawn as the reference draws them for n_threads threads. X (n, d) training rows, Q (m, d)
 * queries; out_i / out_d (m, k) rows and squared distances sorted by (distance, row), -1 / inf past the rows found.
 * Distances follow the reference's kernel for the host's instruction set, so the results equal the reference's
 * wherever no two distances tie. 1 <= k <= n, k <= ef <= 256. Synchronous. */
int mg_knn_search(const float* X, int64_t n, int d, const int32_t* gptr, const int32_t* gidx, int64_t nnz,
                  const int32_t* landmarks, int64_t n_land, const float* Q, int64_t m, int k, int ef, int n_entry,
                  uint64_t seed, int n_threads, int32_t* out_i, float* out_d);

/* The fuzzy union of fuzzy_graph (magnet/knn.py:215-230, after smooth_knn): A = the n x n matrix with rows
 * i < n_rows holding (ind[i, j], vals[i, j]) (duplicate columns summed, zeros dropped), and
 * P = mix (A + A^T - A o A^T) + (1 - mix) (A o A^T) with mix = set_op_mix_ratio, zeros dropped, columns sorted.
 * Outputs indptr (n + 1), indices / data of capacity cap (2 n_rows k always suffices); *nnz = entries. An index
 * outside [0, n) is MG_ERR_ARGUMENT. */
int mg_fuzzy_union(const int32_t* ind, const float* vals, int64_t n_rows, int k, int64_t n, double set_op_mix_ratio,
                   int32_t* indptr, int32_t* indices, float* data, int64_t cap, int64_t* nnz);

#ifdef __cplusplus
}
#endif

#endif /* MAGNET_B200_H */
