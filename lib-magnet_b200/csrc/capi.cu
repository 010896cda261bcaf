// C ABI of the layout pass (include/magnet_b200.h): argument checks with the reference's rules and messages,
// staging of host arrays through per-thread device buffers, error codes with a thread-local message.
#include "common.cuh"
#include "fftrep.cuh"
#include "fft.cuh"
#include "tsne.cuh"
#include "sgd.cuh"
#include "graph.cuh"
#include "spectral.cuh"
#include <string>
#include <vector>
#include <memory>
#include <cstring>
#include <cmath>
#include <algorithm>
#include <atomic>
#include <thread>
#include <functional>

namespace mgb {

namespace {
thread_local std::string g_last_error;
thread_local cudaStream_t g_stream = nullptr;

// per-thread staging buffers (slots reused across calls)
struct Stage {
    DevBuf slot[24];
    DevBuf scratch;
};
thread_local std::unique_ptr<Stage> g_stage;
Stage& stage() {
    if (!g_stage) g_stage.reset(new Stage());
    return *g_stage;
}

template <class F>
int guard(F&& f) {
    try {
        f();
        g_last_error.clear();
        return MG_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host out of memory";
        return MG_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return MG_ERR_INTERNAL;
    }
}

}  // namespace

// the C-ABI convention for entry points defined in other files: status code and the thread's last error
int guard_call(const std::function<void()>& f) { return guard(f); }

namespace {
// device view of a caller array: the pointer itself when it is device memory, else a staged copy
template <class T>
T* in_dev(const T* p, int64_t count, int slot, cudaStream_t s) {
    if (!p || count <= 0) return nullptr;
    if (is_device_ptr(p)) return const_cast<T*>(p);
    DevBuf& b = stage().slot[slot];
    b.ensure(sizeof(T) * (size_t)count);
    MGB_CUDA(cudaMemcpyAsync(b.p, p, sizeof(T) * (size_t)count, cudaMemcpyHostToDevice, s));
    return b.as<T>();
}
template <class T>
T* out_dev(T* p, int64_t count, int slot) {
    if (!p || count <= 0) return nullptr;
    if (is_device_ptr(p)) return p;
    DevBuf& b = stage().slot[slot];
    b.ensure(sizeof(T) * (size_t)count);
    return b.as<T>();
}
template <class T>
void back(T* user, const T* dev, int64_t count, cudaStream_t s) {
    if (!user || count <= 0 || user == dev) return;
    MGB_CUDA(cudaMemcpyAsync(user, dev, sizeof(T) * (size_t)count, cudaMemcpyDeviceToHost, s));
}
bool any_host(std::initializer_list<const void*> ptrs) {
    for (const void* p : ptrs)
        if (p && !is_device_ptr(p)) return true;
    return false;
}

// The first i in [0, count) where ok(i) fails, or -1: large ranges are split over the host's cores (the checks of
// host arrays run once per element and call); each chunk stops at its own first failure and the smallest wins.
template <class F>
int64_t first_failure(int64_t count, F ok) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (count < (1 << 20) || hw == 1) {
        for (int64_t i = 0; i < count; ++i)
            if (!ok(i)) return i;
        return -1;
    }
    const int64_t chunk = (count + hw - 1) / hw;
    std::vector<int64_t> first(hw, -1);
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < hw; ++t) {
        const int64_t b = t * chunk, e = std::min<int64_t>(count, b + chunk);
        if (b >= e) break;
        pool.emplace_back([&, t, b, e] {
            for (int64_t i = b; i < e; ++i)
                if (!ok(i)) { first[t] = i; return; }
        });
    }
    for (auto& th : pool) th.join();
    for (int64_t f : first)
        if (f >= 0) return f;   // chunks are in index order
    return -1;
}
template <class F>
bool all_of_range(int64_t count, F ok) { return first_failure(count, ok) < 0; }

// validate_csr of src/layout.hpp:21-32 (host arrays only; device arrays are the caller's responsibility)
void validate_csr_host(const int32_t* ip, const int32_t* ix, int64_t nnz, int64_t n, int64_t n_cols,
                       const char* what) {
    if (!ip || is_device_ptr(ip)) return;
    if (n_cols < 0) n_cols = n;
    require(ip[0] == 0, std::string(what) + ": indptr[0] must be 0");
    if (!all_of_range(n, [&](int64_t i) { return ip[i + 1] >= ip[i]; }))
        require(false, std::string(what) + ": indptr must be non-decreasing");
    require((int64_t)ip[n] == nnz, std::string(what) + ": indices must have indptr[n] entries");
    if (ix && !is_device_ptr(ix))
        require(all_of_range(nnz, [&](int64_t j) { return ix[j] >= 0 && ix[j] < n_cols; }), "column index out of range");
}

// sum of P in FP64: per-block partials, the last block adds them in block order (deterministic)
__global__ void csr_sum_kernel(const float* __restrict__ P, int64_t nnz, double* __restrict__ part,
                               unsigned* __restrict__ counter, double* __restrict__ out) {
    __shared__ double red[32];
    __shared__ int is_last;
    double s = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x)
        s += (double)P[e];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        part[blockIdx.x] = t;
        __threadfence();
        is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last || threadIdx.x != 0) return;
    __threadfence();
    double t = 0.0;
    for (unsigned b = 0; b < gridDim.x; ++b) t += __ldcg(&part[b]);
    *out = t;
    *counter = 0u;
}
__global__ void csr_scale_kernel(const float* __restrict__ P, int64_t nnz, const double* __restrict__ sum,
                                 float* __restrict__ out) {
    const float s = (float)*sum;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x)
        out[e] = P[e] / s;
}
__global__ void read_sumq_kernel(const GridDesc* g, float* out) { *out = g->sumQ_f; }

}  // namespace

cudaStream_t current_stream() { return g_stream; }

namespace {
std::atomic<uint64_t> g_launches{0};
}
void count_launch(uint64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

}  // namespace mgb

using namespace mgb;

// ============================================================================================== general
extern "C" const char* mg_last_error(void) { return g_last_error.c_str(); }
extern "C" int mg_version(void) { return 100; }
extern "C" int mg_set_stream(void* stream) {
    g_stream = static_cast<cudaStream_t>(stream);
    return MG_OK;
}
extern "C" int mg_synchronize(void) {
    return guard([&] { MGB_CUDA(cudaStreamSynchronize(current_stream())); });
}
extern "C" uint64_t mg_launch_count(void) { return launch_count(); }

// ============================================================================================== FFTConv2D
struct mg_fftconv {
    int M = 0, ni = 3;
    RepBuffers rb;
    DevBuf gdesc;
    bool kernels_set = false;
};

extern "C" int mg_fftconv_create(int M, int n_interp, mg_fftconv** out) {
    return guard([&] {
        require(out != nullptr, "out must not be NULL");
        *out = nullptr;
        require(M >= 2 && fft::is_5smooth(M), "M must be a 5-smooth FFT size >= 2 (2^a 3^b 5^c)");
        require(M <= fft::kMaxLen, "M exceeds the supported maximum " + std::to_string(fft::kMaxLen));
        require(n_interp >= 1 && n_interp <= 8, "n_interp must be between 1 and 8");
        std::unique_ptr<mg_fftconv> h(new mg_fftconv());
        h->M = M; h->ni = n_interp;
        h->rb.alloc(M, M, n_interp);
        h->gdesc.ensure(sizeof(GridDesc));
        cudaStream_t s = current_stream();
        MGB_CUDA(cudaMemsetAsync(h->gdesc.p, 0, sizeof(GridDesc), s));
        rep_set_grid_host(h->gdesc.as<GridDesc>(), 0.f, 0.f, 1.f, 1, n_interp, M, s);
        rep_twiddles(h->gdesc.as<GridDesc>(), h->rb, s, true);
        MGB_CUDA(cudaStreamSynchronize(s));
        *out = h.release();
    });
}

extern "C" int mg_fftconv_set_kernels(mg_fftconv* h, const float* K1h, const float* K2h, int64_t rows, int64_t cols) {
    return guard([&] {
        require(h != nullptr, "null FFTConv2D handle");
        const int Mh = h->M / 2 + 1;
        require(rows == h->M && cols == Mh, "K1h must be (M, M/2+1) real");
        require(K1h && K2h, "K1h must be (M, M/2+1) real");
        cudaStream_t s = current_stream();
        const int64_t cnt = rows * cols;
        const float* d1 = in_dev(K1h, cnt, 0, s);
        const float* d2 = in_dev(K2h, cnt, 1, s);
        rep_set_spectra_from_host_layout(h->rb, d1, d2, h->M, s);
        MGB_CUDA(cudaStreamSynchronize(s));
        h->kernels_set = true;
    });
}

extern "C" int mg_fftconv_compute(mg_fftconv* h, const float* Y, int64_t n, float xmin, float ymin, float width,
                                  int n_boxes, float* sumQ, float* F) {
    return guard([&] {
        require(h != nullptr, "null FFTConv2D handle");
        require(n >= 0, "Y must be (n, 2)");
        const int64_t N = (int64_t)n_boxes * h->ni;
        require(n_boxes >= 1 && N <= h->M && width > 0, "grid larger than the buffer");
        require(h->kernels_set, "set_kernels must be called before compute");
        require(sumQ != nullptr && (F != nullptr || n == 0), "sumQ and F must not be NULL");
        cudaStream_t s = current_stream();
        GridDesc* g = h->gdesc.as<GridDesc>();
        rep_set_grid_host(g, xmin, ymin, width, n_boxes, h->ni, h->M, s);
        const float2* Yd = reinterpret_cast<const float2*>(in_dev(Y, 2 * n, 2, s));
        float2* Fd = reinterpret_cast<float2*>(out_dev(F, 2 * n, 3));
        if (n > 0) rep_spread(Yd, n, g, h->rb, s);
        rep_convolve(g, h->rb, n, s);
        if (n > 0) rep_gather_forces(Yd, n, g, h->rb, Fd, s);
        back(F, reinterpret_cast<float*>(Fd), 2 * n, s);
        float* sq = out_dev(sumQ, 1, 4);
        read_sumq_kernel<<<1, 1, 0, s>>>(g, sq);
        MGB_LAUNCH_CHECK();
        back(sumQ, sq, 1, s);
        if (any_host({Y, F, sumQ})) MGB_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" void mg_fftconv_destroy(mg_fftconv* h) { delete h; }

extern "C" int mg_fftconv_compute_noalloc(const float* K1h, const float* K2h, int M, int n_interp, const float* Y,
                                          int64_t n, float xmin, float ymin, float width, int n_boxes, float* sumQ,
                                          float* F) {
    return guard([&] { fftconv_compute_noalloc(K1h, K2h, M, n_interp, Y, n, xmin, ymin, width, n_boxes, sumQ, F); });
}

extern "C" int mg_fftconv_noalloc_max_side(void) { return noalloc_max_fft_side(); }

// ============================================================================================== t-SNE kernels
extern "C" int mg_tsne_attraction(const int32_t* indptr, const int32_t* indices, const float* data, int64_t nnz,
                                  const float* Y, int64_t n, int dim, float dof, float* out) {
    return guard([&] {
        require(dof > 0.f, "dof must be positive");
        require(dim >= 1 && dim <= kMaxDim, "dim out of range");
        require(n >= 0 && indptr != nullptr, "indptr must have n + 1 entries");
        validate_csr_host(indptr, indices, nnz, n, -1, "tsne_attraction");
        cudaStream_t s = current_stream();
        const int32_t* ip = in_dev(indptr, n + 1, 0, s);
        const int32_t* ix = in_dev(indices, nnz, 1, s);
        const float* P = in_dev(data, nnz, 2, s);
        const float* Yd = in_dev(Y, n * dim, 3, s);
        float* od = out_dev(out, n * dim, 4);
        tsne_attraction_dev(ip, ix, P, Yd, n, dim, dof, od, s);
        back(out, od, n * dim, s);
        if (any_host({indptr, indices, data, Y, out})) MGB_CUDA(cudaStreamSynchronize(s));
    });
}

static int step_impl(float* Y, float* update, float* gains, const float* A, const float* F, int64_t n, int dim,
                     float rho, float inv_sumQ, float lr, float momentum, bool fused) {
    return guard([&] {
        require(dim >= 1 && dim <= kMaxDim && n >= 1, "Y must be 2-d");
        require(Y && update && gains && A && (F || !fused), "arrays must match Y");
        cudaStream_t s = current_stream();
        const int64_t t = n * dim;
        float* Yd = in_dev(Y, t, 0, s);
        float* Ud = in_dev(update, t, 1, s);
        float* Gd = in_dev(gains, t, 2, s);
        const float* Ad = in_dev(A, t, 3, s);
        const float* Fd = fused ? in_dev(F, t, 4, s) : nullptr;
        if (fused) tsne_step_dev(Yd, Ud, Gd, Ad, Fd, n, dim, rho, inv_sumQ, lr, momentum, stage().scratch, s);
        else tsne_update_dev(Yd, Ud, Gd, Ad, n, dim, lr, momentum, stage().scratch, s);
        back(Y, Yd, t, s); back(update, Ud, t, s); back(gains, Gd, t, s);
        if (any_host({Y, update, gains, A, F})) MGB_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" int mg_tsne_step(float* Y, float* update, float* gains, const float* attr, const float* F, int64_t n,
                            int dim, float rho, float inv_sumQ, float lr, float momentum) {
    return step_impl(Y, update, gains, attr, F, n, dim, rho, inv_sumQ, lr, momentum, true);
}

extern "C" int mg_tsne_update(float* Y, float* update, float* gains, const float* grad, int64_t n, int dim, float lr,
                              float momentum) {
    return step_impl(Y, update, gains, grad, nullptr, n, dim, 0.f, 0.f, lr, momentum, false);
}

extern "C" int mg_bbox_2d(const float* Y, int64_t n, float* out4) {
    return guard([&] {
        require(n >= 1 && Y && out4, "Y must be (n, 2)");
        cudaStream_t s = current_stream();
        const float* Yd = in_dev(Y, 2 * n, 0, s);
        float* od = out_dev(out4, 4, 1);
        bbox_dev(Yd, n, od, stage().scratch, s);
        back(out4, od, 4, s);
        if (any_host({Y, out4})) MGB_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" int mg_mid_spring(const float* Y, const int32_t* pairs, float* grad, int64_t n, int dim, int m, float w) {
    return guard([&] {
        require(Y && pairs && grad && n >= 0 && dim >= 1 && dim <= kMaxDim && m >= 1, "bad shapes");
        cudaStream_t s = current_stream();
        const float* Yd = in_dev(Y, n * dim, 0, s);
        const int32_t* pd = in_dev(pairs, n * m, 1, s);
        float* gd = in_dev(grad, n * dim, 2, s);
        mid_spring_dev(Yd, pd, gd, n, dim, m, w, s);
        back(grad, gd, n * dim, s);
        if (any_host({Y, pairs, grad})) MGB_CUDA(cudaStreamSynchronize(s));
    });
}

// ============================================================================================== t-SNE loop
extern "C" void mg_tsne_params_default(mg_tsne_params* p) {
    if (!p) return;
    p->n_iter = 750; p->early_iter = 250; p->early_exaggeration = 12.f; p->exaggeration = 1.f;
    p->learning_rate = -1.f; p->momentum_early = 0.5f; p->momentum_late = 0.8f; p->n_interp = 3;
    p->box_width = 0.7f; p->min_boxes = 20; p->max_boxes = 1000; p->dof = 1.f; p->threads_per_row = 0;
    p->use_graph = 1;
}

namespace mgb {
// shared by the C ABI and the batch / serving layers
void tsne_prepare(TsneDev& d, const int32_t* indptr, const int32_t* indices, const float* P, int64_t n, int64_t nnz,
                  const mg_tsne_params& p, double box_width_exact, cudaStream_t s) {
    require(n >= 1, "the layout needs at least one point");
    require(p.n_iter >= 0 && p.early_iter >= 0, "iteration counts must be non-negative");
    require(p.dof > 0.f, "dof must be positive");
    require(p.box_width > 0.f, "box_width must be positive");
    validate_csr_host(indptr, indices, nnz, n, -1, "optimize_tsne");
    TsneSched sc{};
    sc.early_iter = p.early_iter; sc.early_exag = p.early_exaggeration; sc.exag = p.exaggeration;
    sc.mom0 = p.momentum_early; sc.mom1 = p.momentum_late;
    const double lr = p.learning_rate > 0.f ? (double)p.learning_rate
                                            : std::max(200.0, (double)n / (double)p.early_exaggeration);
    sc.lr = (float)lr;
    sc.inv_dof = 1.f / p.dof;
    sc.box_width = box_width_exact > 0 ? box_width_exact : (double)p.box_width;
    sc.min_boxes = p.min_boxes; sc.max_boxes = p.max_boxes; sc.ni = p.n_interp;
    const int32_t* ip = in_dev(indptr, n + 1, 0, s);
    const int32_t* ix = in_dev(indices, nnz, 1, s);
    const float* Pd = in_dev(P, nnz, 2, s);
    d.init(ip, ix, Pd, n, nnz, false, sc, p.dof, p.threads_per_row, s);
    // P / P.sum() (magnet/tsne.py:149-150)
    if (nnz > 0) {
        const int blocks = 2 * kNumSMs;
        char* base = static_cast<char*>(stage().scratch.ensure(64 + sizeof(double) * (blocks + 1)));
        unsigned* counter = reinterpret_cast<unsigned*>(base);
        double* sum = reinterpret_cast<double*>(base + 8);
        double* part = reinterpret_cast<double*>(base + 16);
        MGB_CUDA(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
        csr_sum_kernel<<<blocks, 1024, 0, s>>>(d.P.as<float>(), nnz, part, counter, sum);
        MGB_LAUNCH_CHECK();
        csr_scale_kernel<<<256, 256, 0, s>>>(d.P.as<float>(), nnz, sum, d.P.as<float>());
        MGB_LAUNCH_CHECK();
    }
}
}  // namespace mgb

namespace {
// the device state of the calling thread's last t-SNE pass: buffers and the captured iteration are reused by the
// next call with the same sizes (the reference keeps its FFTConv2D objects for the same reason)
thread_local std::unique_ptr<TsneDev> g_tsne;
TsneDev& tsne_state() {
    if (!g_tsne) g_tsne.reset(new TsneDev());
    return *g_tsne;
}
}  // namespace

static void optimize_tsne_impl(const int32_t* indptr, const int32_t* indices, const float* P, int64_t n, int64_t nnz,
                               float* Y, const mg_tsne_params* p, double* stage_ms, int* grid) {
    mg_tsne_params def;
    mg_tsne_params_default(&def);
    const mg_tsne_params& pp = p ? *p : def;
    require(Y != nullptr, "Y must be (n, 2)");
    cudaStream_t s = current_stream();
    TsneDev& d = tsne_state();
    tsne_prepare(d, indptr, indices, P, n, nnz, pp, (double)pp.box_width, s);
    const float* Yd = in_dev(Y, 2 * n, 3, s);
    d.set_layout(Yd, false, s);
    if (stage_ms) d.run_profiled(pp.n_iter, s, stage_ms, grid);
    else d.run(pp.n_iter, pp.use_graph != 0, s);
    d.get_layout(Y, !is_device_ptr(Y), s);
}

extern "C" int mg_optimize_tsne(const int32_t* indptr, const int32_t* indices, const float* P, int64_t n, int64_t nnz,
                                float* Y, const mg_tsne_params* p) {
    return guard([&] { optimize_tsne_impl(indptr, indices, P, n, nnz, Y, p, nullptr, nullptr); });
}

extern "C" int mg_optimize_tsne_profiled(const int32_t* indptr, const int32_t* indices, const float* P, int64_t n,
                                         int64_t nnz, float* Y, const mg_tsne_params* p, double* stage_ms, int* grid) {
    return guard([&] {
        require(stage_ms != nullptr, "stage_ms must hold 9 values");
        for (int k = 0; k < 9; ++k) stage_ms[k] = 0.0;
        optimize_tsne_impl(indptr, indices, P, n, nnz, Y, p, stage_ms, grid);
        MGB_CUDA(cudaStreamSynchronize(current_stream()));
    });
}

extern "C" int mg_center_scale(float* Y, int64_t n, int dim, double target_std) {
    return guard([&] {
        require(Y && n >= 1 && dim >= 1 && dim <= kMaxDim, "Y must be (n, dim)");
        cudaStream_t s = current_stream();
        float* Yd = in_dev(Y, n * dim, 0, s);
        center_scale_dev(Yd, n, dim, target_std, stage().scratch, s);
        back(Y, Yd, n * dim, s);
        if (!is_device_ptr(Y)) MGB_CUDA(cudaStreamSynchronize(s));
    });
}

// ============================================================================================== SGD
extern "C" void mg_layout_args_default(mg_layout_args* a) {
    if (!a) return;
    std::memset(a, 0, sizeof(*a));
    a->alpha0 = 1.f; a->alpha1 = 1.f; a->a = 1.577f; a->b = 0.895f; a->rep_a = 1.577f; a->rep_b = 1.f;
    a->negative_sample_rate = 5.f; a->exaggeration = 1.f; a->repulsion_strength = 2.f; a->walk_len = 4;
    a->mid_rate = 0.25f; a->beta1 = 0.9f; a->beta2 = 0.999f; a->n_threads = -1;
}

namespace {

// the reference's checks (src/layout.cpp:360-437) and derived scalars; stages the arrays
SgdDev prepare_sgd(const mg_layout_args& A, cudaStream_t s) {
    require(A.Y != nullptr && A.n >= 0, "Y must be 2-dimensional");
    const int64_t n = A.n;
    const int dim = A.dim;
    require(dim >= 1 && dim <= kMaxDim, "n_components must be between 1 and 64");
    const int64_t E = A.n_edges;
    require(E >= 0, "head must be 1-d");
    require(E == 0 || (A.head && A.tail && A.epochs_per_sample && A.epoch_of_next_sample && A.epoch_of_next_negative_sample),
            "head, tail and epoch arrays must have the same length");
    require(A.epoch_start >= 0 && A.epoch_end >= A.epoch_start, "invalid epoch range");
    require(A.negative_sample_rate > 0.0f, "negative_sample_rate must be positive");
    require(A.loss == 0 || A.loss == 1, "loss must be 0 (umap) or 1 (infonce)");
    require(A.kernel >= 0 && A.kernel <= 3, "kernel must be 0 (power), 1 (gaussian), 2 (sech) or 3 (tanh)");
    require(A.loss == 0 || A.kernel == 0, "the InfoNCE loss supports the power kernel only");
    require(A.parallel == 0 || A.parallel == 1, "parallel must be 0 (hogwild) or 1 (owner)");
    require(A.parallel == 0 || A.loss == 0, "parallel='owner' supports the umap loss only (InfoNCE moves the negatives)");
    require(A.owner_chunk_edges >= 0, "owner_chunk_edges must be 0 (the reference's chunks) or positive");
    require(A.n_fixed >= 0 && A.n_fixed <= n, "n_fixed out of range");
    require(A.stream_mode == 0 || A.stream_mode == 1, "stream_mode must be 0 (per-edge streams) or 1 (serial stream)");
    if (A.parallel == 0 && A.stream_mode == 1 && A.optimizer == 1)
        throw Error(MG_ERR_NOT_SUPPORTED, "the serial stream mode supports the sgd optimizer only");
    if (A.head && !is_device_ptr(A.head)) {
        // the reference's per-edge checks (src/layout.cpp:385-388); the first failing edge names the message
        const int32_t* hd = A.head; const int32_t* tl = A.tail; const float* ep = A.epochs_per_sample;
        const auto edge_ok = [&](int64_t i) { return hd[i] >= 0 && hd[i] < n && tl[i] >= 0 && tl[i] < n; };
        const int64_t f = first_failure(E, [&](int64_t i) { return edge_ok(i) && ep[i] > 0.0f; });
        if (f >= 0) {
            require(edge_ok(f), "edge index out of range");
            require(false, "epochs_per_sample must be positive");
        }
    }
    const bool adam = A.optimizer == 1;
    if (adam) require(A.adam_m && A.adam_v && A.adam_t, "Adam state arrays have the wrong shape");
    const bool has_pairs = A.mid_pairs != nullptr && A.n_mid > 0;
    if (has_pairs && !is_device_ptr(A.mid_pairs)) {
        const int32_t* mp = A.mid_pairs;
        require(all_of_range(n * A.n_mid, [&](int64_t i) { return mp[i] >= 0 && mp[i] < n; }),
                "mid_pairs index out of range");
    }
    const bool has_jumps = A.jump_indptr != nullptr && A.mid_jump > 0.0f;
    if (has_jumps) validate_csr_host(A.jump_indptr, A.jump_indices, A.jump_nnz, n, -1, "jump graph");
    const bool walks = has_jumps || !has_pairs;
    const bool use_mid = (A.mid_w0 > 0.0f || A.mid_w1 > 0.0f) && A.mid_rate > 0.0f && (has_pairs || A.walk_len > 0);
    if (use_mid && walks) {
        require(A.indptr != nullptr, "indptr must have n + 1 entries");
        validate_csr_host(A.indptr, A.indices, A.graph_nnz, n, -1, "graph");
    }
    if (use_mid && A.walk_lens && !is_device_ptr(A.walk_lens))
        for (int64_t i = 0; i < n; ++i) require(A.walk_lens[i] >= 0 && A.walk_lens[i] <= 64, "walk_lens out of range");
    float rep_a = A.rep_a, rep_b = A.rep_b;
    const bool rep_coupled = rep_b <= 0.0f;
    if (rep_b <= 0.0f) { rep_a = A.a; rep_b = A.b; }
    require(rep_a > 0.0f, "repulsion kernel a must be positive");
    if (A.node_b && !is_device_ptr(A.node_b))
        for (int64_t i = 0; i < n; ++i) require(A.node_b[i] > 0.05f && A.node_b[i] <= 2.0f, "node_b out of range");
    if (A.parallel == 1) {
        // src/layout.cpp:441-446; heads in device memory are checked on the device before the run
        if (A.head && !is_device_ptr(A.head)) {
            const int32_t* hd = A.head;
            require(E < 2 || all_of_range(E - 1, [&](int64_t i) { return hd[i] <= hd[i + 1]; }),
                    "parallel='owner' needs edges sorted by head");
        }
        if (A.rev_indptr) validate_csr_host(A.rev_indptr, A.rev_indices, A.rev_nnz, n, -1, "reverse pairs");
        if (A.rev_indptr && has_pairs && use_mid) {
            // the reverse pulls of an edge take p = mid_rate * row length / n_mid rounds of p -= 1
            // (src/layout.cpp:262-273); in float that loop stops shrinking p above 2^24, so the device run
            // requires a bound that keeps it short (the reference's loop would not end there either)
            std::vector<int32_t> ip_h;
            const int32_t* ip = A.rev_indptr;
            if (is_device_ptr(ip)) {
                ip_h.resize(n + 1);
                MGB_CUDA(cudaMemcpy(ip_h.data(), ip, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost));
                ip = ip_h.data();
            }
            int64_t longest = 0;
            for (int64_t i = 0; i < n; ++i) longest = std::max<int64_t>(longest, (int64_t)ip[i + 1] - ip[i]);
            require(std::isfinite(A.mid_rate) && A.mid_rate * (float)longest / (float)A.n_mid <= 65536.0f,
                    "reverse pairs: mid_rate * row length / n_mid must be at most 65536");
        }
    }

    SgdDev c{};
    c.n = n; c.dim = dim; c.n_edges = E;
    c.Y = in_dev(A.Y, n * dim, 0, s);
    c.head = in_dev(A.head, E, 1, s);
    c.tail = in_dev(A.tail, E, 2, s);
    c.eps = in_dev(A.epochs_per_sample, E, 3, s);
    c.eons = in_dev(A.epoch_of_next_sample, E, 4, s);
    c.eonns = in_dev(A.epoch_of_next_negative_sample, E, 5, s);
    c.mid_pairs = has_pairs && !has_jumps ? in_dev(A.mid_pairs, n * A.n_mid, 6, s) : nullptr;
    c.n_mid = has_pairs ? A.n_mid : 0;
    c.jump_indptr = has_jumps ? in_dev(A.jump_indptr, n + 1, 7, s) : nullptr;
    c.jump_indices = has_jumps ? in_dev(A.jump_indices, A.jump_nnz, 8, s) : nullptr;
    c.mid_jump = A.mid_jump;
    c.indptr = (use_mid && walks) ? in_dev(A.indptr, n + 1, 9, s) : nullptr;
    c.indices = (use_mid && walks) ? in_dev(A.indices, A.graph_nnz, 10, s) : nullptr;
    c.walk_lens = (use_mid && A.walk_lens) ? in_dev(A.walk_lens, n, 11, s) : nullptr;
    c.node_b = A.node_b ? in_dev(A.node_b, n, 12, s) : nullptr;
    if (adam) {
        c.adam_m = in_dev(A.adam_m, n * dim, 13, s);
        c.adam_v = in_dev(A.adam_v, n * dim, 14, s);
        c.adam_t = in_dev(A.adam_t, n, 15, s);
    }
    c.beta1 = A.beta1; c.beta2 = A.beta2;
    c.a = A.a; c.b = A.b; c.rep_a = rep_a; c.rep_b = rep_b;
    c.two_ab = 2.0f * A.a * A.b;
    c.two_b = 2.0f * rep_b * A.repulsion_strength;
    c.negative_sample_rate = A.negative_sample_rate; c.exaggeration = A.exaggeration;
    c.repulsion_strength = A.repulsion_strength; c.mid_rate = A.mid_rate;
    c.b_is_one = std::fabs(A.b - 1.0f) < 1e-6f;
    c.rep_b_is_one = std::fabs(rep_b - 1.0f) < 1e-6f;
    c.rep_coupled = rep_coupled;
    c.use_mid = use_mid;
    c.m_neg = (int)std::min<long>(64, std::max<long>(1, std::lround(A.negative_sample_rate)));
    c.walk_len = A.walk_len; c.loss = A.loss; c.clip_mode = A.clip_mode; c.kernel = A.kernel;
    c.optimizer = A.optimizer; c.n_fixed = A.n_fixed; c.seed = A.seed;
    return c;
}

void sgd_copy_back(const mg_layout_args& A, const SgdDev& c, cudaStream_t s) {
    back(A.Y, c.Y, c.n * c.dim, s);
    back(A.epoch_of_next_sample, c.eons, c.n_edges, s);
    back(A.epoch_of_next_negative_sample, c.eonns, c.n_edges, s);
    if (A.optimizer == 1) {
        back(A.adam_m, c.adam_m, c.n * c.dim, s);
        back(A.adam_v, c.adam_v, c.n * c.dim, s);
        back(A.adam_t, c.adam_t, c.n, s);
    }
}

thread_local std::unique_ptr<SgdWork> g_sgd_work;

}  // namespace

extern "C" int mg_optimize_layout(const mg_layout_args* a) {
    return guard([&] {
        require(a != nullptr, "args must not be NULL");
        cudaStream_t s = current_stream();
        SgdDev c = prepare_sgd(*a, s);
        if (!g_sgd_work) g_sgd_work.reset(new SgdWork());
        if (a->parallel == 1) {
            if (is_device_ptr(a->head))
                require(owner_heads_sorted(c.head, c.n_edges, *g_sgd_work, s), "parallel='owner' needs edges sorted by head");
            const int32_t* rp = a->rev_indptr ? in_dev(a->rev_indptr, c.n + 1, 21, s) : nullptr;
            const int32_t* rx = a->rev_indptr ? in_dev(a->rev_indices, a->rev_nnz, 22, s) : nullptr;
            if (c.n_edges > 0 && a->epoch_end > a->epoch_start)
                owner_run(c, *g_sgd_work, rp, rx, a->owner_chunk_edges, a->epoch_start, a->epoch_end, a->alpha0,
                          a->alpha1, a->mid_w0, a->mid_w1, s);
        } else if (c.n_edges > 0 && a->epoch_end > a->epoch_start) {
            sgd_run(c, *g_sgd_work, a->stream_mode, a->epoch_start, a->epoch_end, a->alpha0, a->alpha1, a->mid_w0,
                    a->mid_w1, s);
        }
        sgd_copy_back(*a, c, s);
        if (any_host({a->Y, a->epoch_of_next_sample, a->epoch_of_next_negative_sample, a->adam_m}))
            MGB_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" int mg_layout_schedule(const mg_layout_args* a, int epoch, uint8_t* sampled, int32_t* n_neg,
                                  int64_t* neg_off, int32_t* negs, int64_t negs_cap, int64_t* n_negs, int32_t* mid) {
    return guard([&] {
        require(a != nullptr, "args must not be NULL");
        require(sampled && n_neg && neg_off && mid && n_negs, "outputs must not be NULL");
        require(epoch >= a->epoch_start && epoch < std::max(a->epoch_end, a->epoch_start + 1), "epoch outside the call's range");
        if (a->parallel == 1) throw Error(MG_ERR_NOT_SUPPORTED, "the schedule hook records the hogwild draws only");
        cudaStream_t s = current_stream();
        SgdDev c = prepare_sgd(*a, s);
        if (!g_sgd_work) g_sgd_work.reset(new SgdWork());
        const int64_t E = c.n_edges;
        float alpha, mid_w;
        sgd_sched(c, epoch, a->epoch_start, a->epoch_end, a->alpha0, a->alpha1, a->mid_w0, a->mid_w1, alpha, mid_w);
        int32_t* cnt_d = out_dev(n_neg, E, 16);
        int64_t* off_d = out_dev(neg_off, E, 17);
        int32_t* negs_d = out_dev(negs, std::max<int64_t>(negs_cap, 1), 18);
        int32_t* mid_d = out_dev(mid, E, 19);
        int64_t* tot_d = out_dev(n_negs, 1, 20);
        sgd_record(c, *g_sgd_work, a->stream_mode, epoch, alpha, mid_w, cnt_d, off_d, negs_d, negs_cap, mid_d, tot_d, s);
        MGB_CUDA(cudaStreamSynchronize(s));
        std::vector<int32_t> cnt_h(E);
        if (E > 0) MGB_CUDA(cudaMemcpy(cnt_h.data(), cnt_d, sizeof(int32_t) * E, cudaMemcpyDeviceToHost));
        back(neg_off, off_d, E, s);
        back(mid, mid_d, E, s);
        back(n_negs, tot_d, 1, s);
        MGB_CUDA(cudaStreamSynchronize(s));
        int64_t tot = 0;
        if (is_device_ptr(n_negs)) MGB_CUDA(cudaMemcpy(&tot, n_negs, sizeof(int64_t), cudaMemcpyDeviceToHost));
        else tot = *n_negs;
        if (negs && negs_cap > 0) back(negs, negs_d, std::min(tot, negs_cap), s);
        // sampled flags and n_neg in the reference's recording convention (0 when not sampled)
        std::vector<uint8_t> sm(E);
        for (int64_t i = 0; i < E; ++i) { sm[i] = cnt_h[i] >= 0; cnt_h[i] = std::max(cnt_h[i], 0); }
        if (is_device_ptr(sampled)) MGB_CUDA(cudaMemcpy(sampled, sm.data(), E, cudaMemcpyHostToDevice));
        else std::memcpy(sampled, sm.data(), E);
        if (is_device_ptr(n_neg)) MGB_CUDA(cudaMemcpy(n_neg, cnt_h.data(), sizeof(int32_t) * E, cudaMemcpyHostToDevice));
        else std::memcpy(n_neg, cnt_h.data(), sizeof(int32_t) * E);
        sgd_copy_back(*a, c, s);
        MGB_CUDA(cudaStreamSynchronize(s));
    });
}

// ================================================================ fuzzy neighbour graph
namespace {
thread_local std::unique_ptr<GraphWork> g_graph_work;
GraphWork& graph_work() {
    if (!g_graph_work) g_graph_work.reset(new GraphWork());
    return *g_graph_work;
}
thread_local std::unique_ptr<SpecWork> g_spec_work;
SpecWork& spec_work() {
    if (!g_spec_work) g_spec_work.reset(new SpecWork());
    return *g_spec_work;
}
}  // namespace

extern "C" int mg_smooth_knn(const float* dist, int64_t n, int k, int n_neighbors, float bandwidth, int n_iter,
                             float* out) {
    return guard([&] {
        require(n >= 0 && k >= 0 && (n * (int64_t)k == 0 || (dist && out)), "dist must be (n, k)");
        require(n_neighbors >= 1, "n_neighbors must be positive");
        cudaStream_t s = current_stream();
        // src/graph.cpp:35, on the host libm as the reference evaluates it
        const float target = std::log2((float)n_neighbors) * bandwidth;
        const float* d = in_dev(dist, n * k, 0, s);
        float* o = out_dev(out, n * k, 1);
        smooth_knn_dev(d, n, k, target, n_iter, o, graph_work(), s);
        back(out, o, n * k, s);
        if (any_host({dist, out})) MGB_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" int mg_chebyshev_eigenvectors(const int32_t* indptr, const int32_t* indices, const float* data,
                                         int64_t n, int64_t nnz, float* X, int p, const float* inv_sqrt_deg,
                                         const int32_t* component, int n_wanted, int degree, int max_iter,
                                         float tol) {
    return guard([&] {
        // the argument rules of src/spectral.cpp:146-157
        require(X && n >= 1 && p >= 1, "X must be 2-d");
        require(n_wanted >= 1 && n_wanted < p, "X needs at least n_wanted + 1 columns");
        require(degree >= 2 && max_iter >= 0, "degree must be >= 2");
        require(indptr && (nnz == 0 || (indices && data)), "the graph must be a CSR matrix");
        require(inv_sqrt_deg, "inv_sqrt_deg must have n entries");
        require(component, "component must have n entries");
        require(n <= INT32_MAX, "n must fit 32-bit indices");
        if (p > kSpecMaxCols) throw Error(MG_ERR_NOT_SUPPORTED, "the device solver takes at most 8 columns");
        validate_csr_host(indptr, indices, nnz, n, -1, "chebyshev_eigenvectors");
        // the component labels on the host: their count sizes the per-component sums
        std::vector<int32_t> comp_h;
        const int32_t* ch = component;
        if (is_device_ptr(component)) {
            comp_h.resize((size_t)n);
            MGB_CUDA(cudaMemcpy(comp_h.data(), component, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToHost));
            ch = comp_h.data();
        }
        int32_t n_comp = 0;
        for (int64_t i = 0; i < n; ++i) {
            require(ch[i] >= 0, "component labels must be >= 0");
            n_comp = std::max(n_comp, ch[i] + 1);
        }
        cudaStream_t s = current_stream();
        const int32_t* ip = in_dev(indptr, n + 1, 0, s);
        const int32_t* ix = in_dev(indices, nnz, 1, s);
        const float* pd = in_dev(data, nnz, 2, s);
        const float* sd = in_dev(inv_sqrt_deg, n, 3, s);
        const int32_t* cd = in_dev(component, n, 4, s);
        float* xd = in_dev(X, n * p, 5, s);
        chebyshev_eigenvectors_dev(ip, ix, pd, n, sd, cd, n_comp, xd, p, n_wanted, degree, max_iter, (double)tol,
                                   spec_work(), s);
        back(X, xd, n * p, s);
        MGB_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" int mg_edge_schedule(const int32_t* indptr, const int32_t* indices, const float* data, int64_t n,
                                int64_t nnz, double samples_per_node, int n_epochs, int32_t* head, int32_t* tail,
                                float* eps, int64_t* n_kept) {
    return guard([&] {
        require(n >= 0 && nnz >= 0 && n_kept && (n == 0 || indptr), "need a CSR graph and n_kept");
        require(nnz == 0 || (indices && data && head && tail && eps), "indices, data, head, tail and eps must hold nnz entries");
        require(n_epochs >= 1 && samples_per_node > 0.0, "need n_epochs >= 1 and samples_per_node > 0");
        require(n <= INT32_MAX, "node indices must fit 32 bits");
        validate_csr_host(indptr, indices, nnz, n, -1, "edge_schedule");
        cudaStream_t s = current_stream();
        const int32_t* ip = in_dev(indptr, n + 1, 0, s);
        const int32_t* ix = in_dev(indices, nnz, 1, s);
        const float* w = in_dev(data, nnz, 2, s);
        int32_t* hd = out_dev(head, nnz, 3);
        int32_t* td = out_dev(tail, nnz, 4);
        float* ed = out_dev(eps, nnz, 5);
        const int64_t kept = edge_schedule_dev(ip, ix, w, n, nnz, samples_per_node, n_epochs, hd, td, ed, graph_work(), s);
        back(head, hd, kept, s);
        back(tail, td, kept, s);
        back(eps, ed, kept, s);
        MGB_CUDA(cudaStreamSynchronize(s));
        *n_kept = kept;
    });
}

extern "C" int mg_transform_schedule(const float* w, const int64_t* ind, int64_t m, int k, int64_t n_train,
                                     double samples_per_node, int n_epochs, int32_t* head, int32_t* tail, float* eps,
                                     int64_t* n_kept) {
    return guard([&] {
        require(m >= 0 && k >= 1 && n_train >= 0 && n_kept, "need m >= 0, k >= 1, n_train >= 0 and n_kept");
        require(n_epochs >= 1 && samples_per_node > 0.0, "need n_epochs >= 1 and samples_per_node > 0");
        require(n_train + m <= INT32_MAX, "node indices must fit 32 bits");
        const int64_t n = m * (int64_t)k;
        if (n > 0)
            for (const void* p : {(const void*)w, (const void*)ind, (const void*)head, (const void*)tail,
                                  (const void*)eps})
                require(p && is_device_ptr(p), "w, ind, head, tail and eps must be device arrays of m * k entries");
        *n_kept = n == 0 ? 0 : transform_schedule_dev(w, ind, m, k, n_train, samples_per_node, n_epochs, head,
                                                      tail, eps, graph_work(), current_stream());
    });
}

extern "C" int mg_mid_near_pairs(const float* X, int64_t n, int d, int n_pairs, int n_cand, uint64_t seed,
                                 int n_threads, int32_t* out) {
    return guard([&] {
        require(X && out && d >= 1, "X must be 2-d");
        // src/nndescent.cpp:737
        require(n_pairs >= 1 && n_cand >= 2 && n >= n_cand + 1, "need n_pairs >= 1, n_cand >= 2 and n > n_cand");
        require(n <= INT32_MAX, "n must fit 32-bit indices");
        if (n_threads <= 0) {   // the reference's resolve(): all hardware threads, 4 when unknown
            const unsigned h = std::thread::hardware_concurrency();
            n_threads = h == 0 ? 4 : (int)h;
        }
        cudaStream_t s = current_stream();
        const float* Xd = in_dev(X, n * (int64_t)d, 0, s);
        int32_t* od = out_dev(out, n * (int64_t)n_pairs, 1);
        mid_near_pairs_dev(Xd, n, d, n_pairs, n_cand, seed, n_threads, host_distance_order(), od, graph_work(), s);
        back(out, od, n * (int64_t)n_pairs, s);
        MGB_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" int mg_knn_search(const float* X, int64_t n, int d, const int32_t* gptr, const int32_t* gidx, int64_t nnz,
                             const int32_t* landmarks, int64_t n_land, const float* Q, int64_t m, int k, int ef,
                             int n_entry, uint64_t seed, int n_threads, int32_t* out_i, float* out_d) {
    return guard([&] {
        // src/nndescent.cpp:666-674
        require(X && d >= 1 && n >= 1 && m >= 0 && (m == 0 || Q), "X and Q must be 2-d with the same width");
        require(k >= 1 && k <= n && ef >= k, "need 1 <= k <= n and ef >= k");
        require(ef <= knn_search_max_ef(), "ef above " + std::to_string(knn_search_max_ef()) + " is not supported");
        require(n_entry >= 1, "n_entry must be positive");
        require(n <= INT32_MAX, "n must fit 32-bit indices");
        require(gptr && (nnz == 0 || gidx) && (m == 0 || (out_i && out_d)), "arrays must not be NULL");
        require(n_land == 0 || landmarks, "landmarks must not be NULL");
        validate_csr_host(gptr, gidx, nnz, n, -1, "knn_search");
        if (landmarks && !is_device_ptr(landmarks))
            for (int64_t l = 0; l < n_land; ++l)
                require(landmarks[l] >= 0 && landmarks[l] < n, "landmark out of range");
        std::vector<int32_t> entries;
        if (n_land == 0 && m > 0) {
            // the reference's random entry rows: thread t of nt draws for queries t, t + nt, ... from
            // Rng(seed + 7 (t + 1)) (src/nndescent.cpp:677-685)
            if (n_threads <= 0) {
                const unsigned h = std::thread::hardware_concurrency();
                n_threads = h == 0 ? 4 : (int)h;
            }
            const int64_t nt = std::min<int64_t>(n_threads, std::max<int64_t>(1, m / 64));
            entries.resize((size_t)m * n_entry);
            for (int64_t t = 0; t < nt; ++t) {
                Rng rng(seed + 7ULL * (uint64_t)(t + 1));
                for (int64_t q = t; q < m; q += nt)
                    for (int e = 0; e < n_entry; ++e) entries[(size_t)q * n_entry + e] = (int32_t)rng.below((uint32_t)n);
            }
        }
        cudaStream_t s = current_stream();
        const float* Xd = in_dev(X, n * (int64_t)d, 0, s);
        const int32_t* gp = in_dev(gptr, n + 1, 1, s);
        const int32_t* gx = in_dev(gidx, nnz, 2, s);
        const int32_t* ld = in_dev(landmarks, n_land, 3, s);
        const float* Qd = in_dev(Q, m * (int64_t)d, 4, s);
        int32_t* oi = out_dev(out_i, m * (int64_t)k, 5);
        float* od = out_dev(out_d, m * (int64_t)k, 6);
        knn_search_dev(Xd, n, d, gp, gx, ld, n_land, entries.data(), Qd, m, k, ef, n_entry, host_distance_order(), oi,
                       od, s);
        back(out_i, oi, m * (int64_t)k, s);
        back(out_d, od, m * (int64_t)k, s);
        MGB_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" int mg_fuzzy_union(const int32_t* ind, const float* vals, int64_t n_rows, int k, int64_t n,
                              double set_op_mix_ratio, int32_t* indptr, int32_t* indices, float* data, int64_t cap,
                              int64_t* nnz) {
    return guard([&] {
        require(n_rows >= 0 && k >= 0 && n >= n_rows, "ind must be (n_rows, k) with n_rows <= n");
        require(n_rows * (int64_t)k == 0 || (ind && vals), "ind and vals must not be NULL");
        require(indptr && nnz && cap >= 0 && (cap == 0 || (indices && data)), "outputs must not be NULL");
        require(n <= INT32_MAX, "n must fit 32-bit indices");
        cudaStream_t s = current_stream();
        const int32_t* id = in_dev(ind, n_rows * k, 0, s);
        const float* vd = in_dev(vals, n_rows * k, 1, s);
        int32_t* ipd = out_dev(indptr, n + 1, 2);
        int32_t* ixd = out_dev(indices, cap, 3);
        float* dd = out_dev(data, cap, 4);
        // scipy multiplies the float32 arrays by the python floats mix and 1 - mix as float32 scalars
        const float mix = (float)set_op_mix_ratio;
        const float one_minus_mix = (float)(1.0 - set_op_mix_ratio);
        const int64_t m = fuzzy_union_dev(id, vd, n_rows, k, n, mix, one_minus_mix, ipd, ixd, dd, cap, graph_work(), s);
        back(indptr, ipd, n + 1, s);
        back(indices, ixd, m, s);
        back(data, dd, m, s);
        *nnz = m;
        MGB_CUDA(cudaStreamSynchronize(s));
    });
}

