// Batched t-SNE layouts: many independent layouts of uneven size optimised together (the loop of
// magnet/tsne.py:132-214 for each of them, as a loop of optimize_tsne calls would run them one after another).
//
// Every layout keeps its own device state (TsneDev: positions, optimiser state, normalised affinities, a repulsion
// grid sized for it). One CUDA graph holds one iteration of every layout: the capture stream forks into `branches`
// streams, layout i's kernels are captured on branch i mod branches, and the branches join at the end. The graph's
// branches are independent, so the device runs the layouts' kernels side by side (a small layout's kernels fill a
// few SMs only); the host replays the graph once per iteration, and the schedule (exaggeration, momentum) follows
// each layout's device-side iteration counter.
//
// A layout's grid is allocated for at most max_boxes boxes per side (by default 64 + 2 ceil(sqrt(n)), rounded up to
// a multiple of 4 and at most the caller's limit, about twice the side a t-SNE layout of n points reaches); a
// layout that grows past it is clamped to that many boxes with wider boxes, where the reference would take more.
#include "tsne.cuh"
#include <vector>
#include <memory>
#include <cmath>
#include <algorithm>

namespace mgb {

void tsne_prepare(TsneDev& d, const int32_t* indptr, const int32_t* indices, const float* P, int64_t n, int64_t nnz,
                  const mg_tsne_params& p, double box_width_exact, cudaStream_t s);

int batch_default_max_boxes(int64_t n, int limit) {
    int b = 64 + 2 * (int)std::ceil(std::sqrt((double)std::max<int64_t>(n, 1)));
    b = (b + 3) & ~3;
    return std::max(1, std::min(b, limit));
}

struct TsneBatch {
    std::vector<std::unique_ptr<TsneDev>> layouts;
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> joins;
    cudaEvent_t fork = nullptr;
    cudaGraphExec_t graph = nullptr;
    cudaStream_t graph_stream = nullptr;
    uint64_t graph_kernels = 0;
    int n_iter = 0;

    ~TsneBatch() {
        if (graph) cudaGraphExecDestroy(graph);
        for (auto b : branch) cudaStreamDestroy(b);
        for (auto e : joins) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
    }

    // one iteration of every layout as one graph: fork, layout i on branch i mod branches, join
    void capture(cudaStream_t st) {
        if (graph && graph_stream == st) return;
        if (graph) { cudaGraphExecDestroy(graph); graph = nullptr; }
        cudaStream_t cap;
        MGB_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        cudaGraph_t gr = nullptr;
        try {
            MGB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
            const uint64_t before = launch_count();
            MGB_CUDA(cudaEventRecord(fork, cap));
            for (auto b : branch) MGB_CUDA(cudaStreamWaitEvent(b, fork, 0));
            for (size_t i = 0; i < layouts.size(); ++i) layouts[i]->iterate(branch[i % branch.size()]);
            for (size_t j = 0; j < branch.size(); ++j) {
                MGB_CUDA(cudaEventRecord(joins[j], branch[j]));
                MGB_CUDA(cudaStreamWaitEvent(cap, joins[j], 0));
            }
            graph_kernels = launch_count() - before;
            MGB_CUDA(cudaStreamEndCapture(cap, &gr));
        } catch (...) {
            cudaGraph_t tmp = nullptr;
            cudaStreamEndCapture(cap, &tmp);
            if (tmp) cudaGraphDestroy(tmp);
            cudaStreamDestroy(cap);
            throw;
        }
        cudaStreamDestroy(cap);
        MGB_CUDA(cudaGraphInstantiate(&graph, gr, 0));
        cudaGraphDestroy(gr);
        graph_stream = st;
        count_launch(0 - graph_kernels);   // captured, not run: the replays count them
    }
};

}  // namespace mgb

struct mg_tsne_batch {
    mgb::TsneBatch b;
};

using namespace mgb;

extern "C" int mg_tsne_batch_create(int count, const int64_t* n, const int64_t* nnz, const int32_t* const* indptr,
                                    const int32_t* const* indices, const float* const* P, const mg_tsne_params* p,
                                    const int* max_boxes, int branches, mg_tsne_batch** out) {
    return guard_call([&] {
        require(out != nullptr, "out must not be NULL");
        *out = nullptr;
        require(count >= 1, "the batch needs at least one layout");
        require(n && nnz && indptr && indices && P, "n, nnz, indptr, indices and P must hold `count` entries");
        require(branches >= 1 && branches <= 1024, "branches must be between 1 and 1024");
        mg_tsne_params def;
        mg_tsne_params_default(&def);
        const mg_tsne_params& pp = p ? *p : def;
        std::unique_ptr<mg_tsne_batch> h(new mg_tsne_batch());
        cudaStream_t s = current_stream();
        for (int i = 0; i < count; ++i) {
            mg_tsne_params pi = pp;
            pi.max_boxes = max_boxes ? std::min(pp.max_boxes, max_boxes[i]) : batch_default_max_boxes(n[i], pp.max_boxes);
            require(pi.max_boxes >= pi.min_boxes, "max_boxes below min_boxes for layout " + std::to_string(i));
            h->b.layouts.emplace_back(new TsneDev());
            tsne_prepare(*h->b.layouts.back(), indptr[i], indices[i], P[i], n[i], nnz[i], pi, (double)pi.box_width, s);
        }
        h->b.n_iter = pp.n_iter;
        const int nb = std::min(branches, count);
        for (int j = 0; j < nb; ++j) {
            cudaStream_t b;
            MGB_CUDA(cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking));
            h->b.branch.push_back(b);
            cudaEvent_t e;
            MGB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            h->b.joins.push_back(e);
        }
        MGB_CUDA(cudaEventCreateWithFlags(&h->b.fork, cudaEventDisableTiming));
        MGB_CUDA(cudaStreamSynchronize(s));
        *out = h.release();
    });
}

extern "C" int mg_tsne_batch_run(mg_tsne_batch* h, float* const* Y) {
    return guard_call([&] {
        require(h != nullptr && Y != nullptr, "batch and Y must not be NULL");
        auto& b = h->b;
        cudaStream_t s = current_stream();
        for (size_t i = 0; i < b.layouts.size(); ++i) {
            require(Y[i] != nullptr, "Y must hold one (n, 2) array per layout");
            b.layouts[i]->set_layout(Y[i], !is_device_ptr(Y[i]), s);
        }
        if (b.n_iter > 0) {
            b.capture(s);
            for (int it = 0; it < b.n_iter; ++it) {
                MGB_CUDA(cudaGraphLaunch(b.graph, s));
                count_launch(b.graph_kernels);
            }
        }
        for (size_t i = 0; i < b.layouts.size(); ++i) b.layouts[i]->get_layout(Y[i], !is_device_ptr(Y[i]), s);
        MGB_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" int mg_tsne_batch_size(const mg_tsne_batch* h, int* count, uint64_t* kernels_per_iteration) {
    return guard_call([&] {
        require(h != nullptr, "batch must not be NULL");
        if (count) *count = (int)h->b.layouts.size();
        if (kernels_per_iteration) *kernels_per_iteration = h->b.graph_kernels;
    });
}

extern "C" void mg_tsne_batch_destroy(mg_tsne_batch* h) {
    delete h;
}
