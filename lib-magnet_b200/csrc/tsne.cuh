// t-SNE pass on the device: the per-iteration kernels of src/fftrep.cpp (attraction, step, update, bbox) and
// the whole optimisation loop of magnet/tsne.py:132-214 (common path) kept on the device.
#pragma once
#include "fftrep.cuh"
#include <string>

namespace mgb {

// standalone kernels (one call = one reference call)
void tsne_attraction_dev(const int32_t* ip, const int32_t* ix, const float* P, const float* Y, int64_t n, int dim,
                         float dof, float* out, cudaStream_t s);
void tsne_step_dev(float* Y, float* U, float* G, const float* A, const float* F, int64_t n, int dim, float rho,
                   float inv_sumQ, float lr, float momentum, DevBuf& scratch, cudaStream_t s);
void tsne_update_dev(float* Y, float* U, float* G, const float* grad, int64_t n, int dim, float lr, float momentum,
                     DevBuf& scratch, cudaStream_t s);
void bbox_dev(const float* Y, int64_t n, float* out4_dev, DevBuf& scratch, cudaStream_t s);
void mid_spring_dev(const float* Y, const int32_t* pairs, float* grad, int64_t n, int dim, int m, float w,
                    cudaStream_t s);
void center_scale_dev(float* Y, int64_t n, int dim, double target_std, DevBuf& scratch, cudaStream_t s);

struct TsneSched {
    int early_iter;
    float early_exag, exag, mom0, mom1, lr, inv_dof;
    double box_width;
    int min_boxes, max_boxes, ni;
};

// Device-resident state of one t-SNE layout: the layout double buffer, the optimiser state, the normalised
// affinities and the repulsion buffers. One instance per stream.
struct TsneDev {
    int64_t n = 0, nnz = 0;
    int ni = 3, tpr = 8;
    float dof = 1.f;
    TsneSched sch{};
    DevBuf Ycur, Ynext, U, G, ip, ix, P, gdesc, bbox_part, mean_part;
    RepBuffers rb;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t graph_stream = nullptr;
    uint64_t graph_kernels = 0;         // kernel nodes of the captured iteration
    std::string graph_sig;              // sizes, schedule and buffer addresses the graph was captured with
    int blocks_iter = 0, blocks_bbox = 0;
    // spatial order of the points (the loop of a large layout): row r of every per-point array holds the caller's
    // point perm[r]; the affinity rows and their column indices are relabelled to match. Set by reorder(),
    // undone by set_layout / get_layout, so callers always see their own order.
    bool permuted = false;
    int reorder_every = 0;              // iterations between reorders (0: never)
    DevBuf perm, perm_t, okey, ocnt, ostart, osrc, onew, olen, oip, oscan, Yt, Ut, Gt, ipt, ixt, Pt;
    ~TsneDev();
    // P must already be normalised to sum 1 (done by the caller, as magnet/tsne.py:149-150)
    void init(const int32_t* ip_h, const int32_t* ix_h, const float* P_h, int64_t n, int64_t nnz, bool host_ptrs,
              const TsneSched& s, float dof, int threads_per_row, cudaStream_t st);
    void set_layout(const float* Y, bool host_ptr, cudaStream_t st);   // also resets update = 0, gains = 1
    void get_layout(float* Y, bool host_ptr, cudaStream_t st);         // applies the pending recentring
    // one iteration, plain launches; with ev (8 events) the stage boundaries are recorded
    void iterate(cudaStream_t st, cudaEvent_t* ev = nullptr);
    void run(int n_iter, bool use_graph, cudaStream_t st);
    // plain launches with per-stage event timing; stage_ms[0..7] += stage times, grid[4] = last grid
    void run_profiled(int n_iter, cudaStream_t st, double* stage_ms, int* grid);
    // sorts the points by grid box (Morton order of the boxes of the last iteration's grid), so that the rows a
    // warp handles touch nearby nodes of the grid and nearby positions; plain launches, outside any capture
    void reorder(cudaStream_t st);
    bool reorder_due(int i) const;
    std::string signature() const;
    GridDesc* g() { return gdesc.as<GridDesc>(); }
};

}  // namespace mgb
