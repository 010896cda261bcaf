// pybind11 surface of the B200 layout pass, with the names, argument names and defaults of the reference's
// native module `_magnet` (src/bindings.cpp:8-83, FFTConv2D at src/fftconv.cpp:239-244), over the C ABI
// (include/magnet_b200.h). Host arrays are numpy arrays taken with the reference's convention (C-contiguous,
// forcecast: a wrong dtype is silently copied and in-place updates then land in the copy, src/layout.hpp:11-15);
// objects with __cuda_array_interface__ (torch / cupy device tensors) are passed as device pointers and used in
// place. Errors raise RuntimeError with the library's message, as the reference's `require` does.
#include <pybind11/pybind11.h>
#include <pybind11/numpy.h>
#include <pybind11/stl.h>
#include <cstring>
#include <string>
#include <vector>
#include <tuple>
#include "magnet_b200.h"

namespace py = pybind11;

namespace {

void check(int rc) {
    if (rc != MG_OK) throw std::runtime_error(mg_last_error());
}

template <class T> const char* typestr();
template <> const char* typestr<float>() { return "<f4"; }
template <> const char* typestr<int32_t>() { return "<i4"; }
template <> const char* typestr<uint8_t>() { return "|u1"; }
template <> const char* typestr<int64_t>() { return "<i8"; }

// A host (numpy) or device (__cuda_array_interface__) array view
template <class T>
struct View {
    T* ptr = nullptr;
    std::vector<int64_t> shape;
    py::object keep;
    int64_t size() const {
        int64_t s = 1;
        for (auto d : shape) s *= d;
        return shape.empty() ? 0 : s;
    }
    int ndim() const { return (int)shape.size(); }
    int64_t dim(int i) const { return i < (int)shape.size() ? shape[i] : 0; }
};

template <class T>
View<T> view(py::handle obj) {
    View<T> v;
    if (obj.is_none()) return v;
    if (py::hasattr(obj, "__cuda_array_interface__")) {
        py::dict cai = obj.attr("__cuda_array_interface__");
        std::string ts = py::str(cai["typestr"]);
        if (ts != typestr<T>())
            throw std::runtime_error("device array has dtype " + ts + ", expected " + typestr<T>());
        py::tuple shp = cai["shape"];
        for (auto d : shp) v.shape.push_back(d.cast<int64_t>());
        if (cai.contains("strides") && !cai["strides"].is_none()) {
            py::tuple st = cai["strides"];
            int64_t expect = sizeof(T);
            for (int i = (int)v.shape.size() - 1; i >= 0; --i) {
                if (v.shape[i] > 1 && st[i].cast<int64_t>() != expect)
                    throw std::runtime_error("device arrays must be C-contiguous");
                expect *= v.shape[i];
            }
        }
        py::tuple data = cai["data"];
        v.ptr = reinterpret_cast<T*>(data[0].cast<uintptr_t>());
        v.keep = py::reinterpret_borrow<py::object>(obj);
        return v;
    }
    auto a = py::array_t<T, py::array::c_style | py::array::forcecast>::ensure(obj);
    if (!a) throw std::runtime_error(std::string("expected an array of ") + typestr<T>());
    for (int i = 0; i < a.ndim(); ++i) v.shape.push_back(a.shape(i));
    v.ptr = const_cast<T*>(a.data());
    v.keep = a;
    return v;
}

bool is_device(py::handle obj) { return !obj.is_none() && py::hasattr(obj, "__cuda_array_interface__"); }

// ------------------------------------------------------------------------------------------ FFTConv2D
class FFTConv2DDevice {
public:
    FFTConv2DDevice(int M, int n_interp) : M_(M), ni_(n_interp) { check(mg_fftconv_create(M, n_interp, &h_)); }
    ~FFTConv2DDevice() { mg_fftconv_destroy(h_); }
    void set_kernels(py::object K1, py::object K2) {
        auto a = view<float>(K1), b = view<float>(K2);
        if (a.ndim() != 2 || a.dim(0) != M_ || a.dim(1) != M_ / 2 + 1) throw std::runtime_error("K1h must be (M, M/2+1) real");
        if (b.ndim() != 2 || b.dim(0) != M_ || b.dim(1) != M_ / 2 + 1) throw std::runtime_error("K2h must be (M, M/2+1) real");
        py::gil_scoped_release rel;
        check(mg_fftconv_set_kernels(h_, a.ptr, b.ptr, a.dim(0), a.dim(1)));
    }
    std::tuple<float, py::object> compute(py::object Y, float xmin, float ymin, float width, int n_boxes, int) {
        auto y = view<float>(Y);
        if (y.ndim() != 2 || y.dim(1) != 2) throw std::runtime_error("Y must be (n, 2)");
        const int64_t n = y.dim(0);
        float sumQ = 0.f;
        if (is_device(Y)) {
            py::module_ torch = py::module_::import("torch");
            py::object F = torch.attr("empty")(py::make_tuple(n, 2), py::arg("dtype") = torch.attr("float32"),
                                               py::arg("device") = Y.attr("device"));
            auto f = view<float>(F);
            {
                py::gil_scoped_release rel;
                check(mg_fftconv_compute(h_, y.ptr, n, xmin, ymin, width, n_boxes, &sumQ, f.ptr));
            }
            return std::make_tuple(sumQ, F);
        }
        py::array_t<float> F({n, (int64_t)2});
        {
            py::gil_scoped_release rel;
            check(mg_fftconv_compute(h_, y.ptr, n, xmin, ymin, width, n_boxes, &sumQ, F.mutable_data()));
        }
        return std::make_tuple(sumQ, py::object(F));
    }

private:
    mg_fftconv* h_ = nullptr;
    int M_, ni_;
};

// ------------------------------------------------------------------------------------------ helpers
py::object like(py::object ref, std::vector<int64_t> shape) {
    if (is_device(ref)) {
        py::module_ torch = py::module_::import("torch");
        return torch.attr("empty")(py::cast(shape), py::arg("dtype") = torch.attr("float32"),
                                   py::arg("device") = ref.attr("device"));
    }
    return py::array_t<float>(shape);
}

void optimize_layout(py::object Y, py::object head, py::object tail, py::object eps, py::object eons,
                     py::object eonns, py::object indptr, py::object indices, int epoch_start, int epoch_end,
                     float alpha0, float alpha1, float mid_w0, float mid_w1, float a, float b, float rep_a,
                     float rep_b, float negative_sample_rate, int loss, float exaggeration, float repulsion_strength,
                     int walk_len, float mid_rate, int optimizer, int clip_mode, int64_t n_fixed, py::object adam_m,
                     py::object adam_v, py::object adam_t, float beta1, float beta2, py::object walk_lens,
                     py::object mid_pairs, py::object jump_indptr, py::object jump_indices, float mid_jump, int kernel,
                     py::object node_b, uint64_t seed, int n_threads, int parallel, py::object rev_indptr,
                     py::object rev_indices, int stream_mode, int owner_chunk_edges) {
    auto y = view<float>(Y);
    if (y.ndim() != 2) throw std::runtime_error("Y must be 2-dimensional");
    auto h = view<int32_t>(head), t = view<int32_t>(tail);
    auto e = view<float>(eps), en = view<float>(eons), enn = view<float>(eonns);
    auto ip = view<int32_t>(indptr), ix = view<int32_t>(indices);
    auto am = view<float>(adam_m), av = view<float>(adam_v);
    auto at = view<int32_t>(adam_t);
    auto wl = view<int32_t>(walk_lens), mp = view<int32_t>(mid_pairs);
    auto jp = view<int32_t>(jump_indptr), jx = view<int32_t>(jump_indices);
    auto nb = view<float>(node_b);
    const int64_t E = h.size();
    if (h.ndim() != 1) throw std::runtime_error("head must be 1-d");
    if (t.size() != E || e.size() != E || en.size() != E || enn.size() != E)
        throw std::runtime_error("head, tail and epoch arrays must have the same length");
    const int64_t n = y.dim(0);
    const int dim = (int)y.dim(1);
    if (optimizer == 1 && (am.ndim() != 2 || am.dim(0) != n || am.dim(1) != dim || av.ndim() != 2 ||
                           av.dim(0) != n || av.dim(1) != dim || at.ndim() != 1 || at.dim(0) != n))
        throw std::runtime_error("Adam state arrays have the wrong shape");
    if (mp.size() > 0 && (mp.ndim() != 2 || mp.dim(0) != n || mp.dim(1) < 1))
        throw std::runtime_error("mid_pairs must be (n, m)");
    if (wl.size() > 0 && (wl.ndim() != 1 || wl.dim(0) != n)) throw std::runtime_error("walk_lens must have n entries");
    if (nb.size() > 0 && (nb.ndim() != 1 || nb.dim(0) != n)) throw std::runtime_error("node_b must have n entries");
    if (ip.size() > 0 && ip.size() != n + 1) throw std::runtime_error("indptr must have n + 1 entries");
    if (jp.size() > 0 && jp.size() != n + 1) throw std::runtime_error("indptr must have n + 1 entries");
    auto rp = view<int32_t>(rev_indptr), rx = view<int32_t>(rev_indices);
    if (rp.size() > 0 && rp.size() != n + 1) throw std::runtime_error("indptr must have n + 1 entries");
    mg_layout_args A;
    mg_layout_args_default(&A);
    A.Y = y.ptr; A.n = n; A.dim = dim;
    A.head = h.ptr; A.tail = t.ptr; A.epochs_per_sample = e.ptr; A.epoch_of_next_sample = en.ptr;
    A.epoch_of_next_negative_sample = enn.ptr; A.n_edges = E;
    A.indptr = ip.size() > 0 ? ip.ptr : nullptr; A.indices = ix.size() > 0 ? ix.ptr : nullptr; A.graph_nnz = ix.size();
    A.epoch_start = epoch_start; A.epoch_end = epoch_end;
    A.alpha0 = alpha0; A.alpha1 = alpha1; A.mid_w0 = mid_w0; A.mid_w1 = mid_w1;
    A.a = a; A.b = b; A.rep_a = rep_a; A.rep_b = rep_b; A.negative_sample_rate = negative_sample_rate; A.loss = loss;
    A.exaggeration = exaggeration; A.repulsion_strength = repulsion_strength; A.walk_len = walk_len;
    A.mid_rate = mid_rate; A.optimizer = optimizer; A.clip_mode = clip_mode; A.n_fixed = n_fixed;
    A.adam_m = optimizer == 1 ? am.ptr : nullptr; A.adam_v = optimizer == 1 ? av.ptr : nullptr;
    A.adam_t = optimizer == 1 ? at.ptr : nullptr; A.beta1 = beta1; A.beta2 = beta2;
    A.walk_lens = wl.size() > 0 ? wl.ptr : nullptr;
    A.mid_pairs = mp.size() > 0 ? mp.ptr : nullptr; A.n_mid = mp.size() > 0 ? (int)mp.dim(1) : 0;
    A.jump_indptr = jp.size() > 0 ? jp.ptr : nullptr; A.jump_indices = jx.size() > 0 ? jx.ptr : nullptr;
    A.jump_nnz = jx.size(); A.mid_jump = mid_jump;
    A.kernel = kernel; A.node_b = nb.size() > 0 ? nb.ptr : nullptr; A.seed = seed; A.n_threads = n_threads;
    A.parallel = parallel; A.stream_mode = stream_mode; A.owner_chunk_edges = owner_chunk_edges;
    if (parallel == 1 && rp.size() > 0) {
        A.rev_indptr = rp.ptr; A.rev_indices = rx.size() > 0 ? rx.ptr : nullptr; A.rev_nnz = rx.size();
    }
    py::gil_scoped_release rel;
    check(mg_optimize_layout(&A));
}

py::tuple layout_schedule(py::object Y, py::object head, py::object tail, py::object eps, py::object eons,
                          py::object eonns, int epoch, int epoch_start, int epoch_end, float alpha0, float alpha1,
                          float mid_w0, float mid_w1, float negative_sample_rate, int loss, float mid_rate,
                          int walk_len, int64_t n_fixed, py::object mid_pairs, py::object indptr, py::object indices,
                          uint64_t seed, int stream_mode, py::object walk_lens, py::object jump_indptr,
                          py::object jump_indices, float mid_jump) {
    auto y = view<float>(Y);
    auto h = view<int32_t>(head), t = view<int32_t>(tail);
    auto e = view<float>(eps), en = view<float>(eons), enn = view<float>(eonns);
    auto mp = view<int32_t>(mid_pairs);
    auto ip = view<int32_t>(indptr), ix = view<int32_t>(indices);
    auto wl = view<int32_t>(walk_lens);
    auto jp = view<int32_t>(jump_indptr), jx = view<int32_t>(jump_indices);
    const int64_t E = h.size();
    mg_layout_args A;
    mg_layout_args_default(&A);
    A.Y = y.ptr; A.n = y.dim(0); A.dim = (int)y.dim(1);
    A.head = h.ptr; A.tail = t.ptr; A.epochs_per_sample = e.ptr; A.epoch_of_next_sample = en.ptr;
    A.epoch_of_next_negative_sample = enn.ptr; A.n_edges = E;
    A.epoch_start = epoch_start; A.epoch_end = epoch_end; A.alpha0 = alpha0; A.alpha1 = alpha1;
    A.mid_w0 = mid_w0; A.mid_w1 = mid_w1; A.negative_sample_rate = negative_sample_rate; A.loss = loss;
    A.mid_rate = mid_rate; A.walk_len = walk_len; A.n_fixed = n_fixed; A.seed = seed; A.stream_mode = stream_mode;
    A.mid_pairs = mp.size() > 0 ? mp.ptr : nullptr; A.n_mid = mp.size() > 0 ? (int)mp.dim(1) : 0;
    A.indptr = ip.size() > 0 ? ip.ptr : nullptr; A.indices = ix.size() > 0 ? ix.ptr : nullptr; A.graph_nnz = ix.size();
    A.walk_lens = wl.size() > 0 ? wl.ptr : nullptr;
    A.jump_indptr = jp.size() > 0 ? jp.ptr : nullptr; A.jump_indices = jx.size() > 0 ? jx.ptr : nullptr;
    A.jump_nnz = jx.size(); A.mid_jump = mid_jump;
    const int64_t cap = E * ((int64_t)negative_sample_rate + 2) + 64;
    py::array_t<uint8_t> sampled(E);
    py::array_t<int32_t> n_neg(E), mid(E), negs(cap);
    py::array_t<int64_t> off(E);
    int64_t tot = 0;
    {
        py::gil_scoped_release rel;
        check(mg_layout_schedule(&A, epoch, sampled.mutable_data(), n_neg.mutable_data(), off.mutable_data(),
                                 negs.mutable_data(), cap, &tot, mid.mutable_data()));
    }
    if (tot > cap) throw std::runtime_error("negative buffer too small");
    return py::make_tuple(sampled, n_neg, off, negs[py::slice(0, tot, 1)], mid);
}

// smooth_knn of src/graph.cpp:29-78 on the device (signature of src/bindings.cpp:73-74)
py::array_t<float> smooth_knn(py::object dist, int n_neighbors, float bandwidth, int n_iter, int n_threads) {
    (void)n_threads;
    auto d = view<float>(dist);
    if (d.ndim() != 2) throw std::runtime_error("dist must be (n, k)");
    const int64_t n = d.dim(0);
    const int k = (int)d.dim(1);
    py::array_t<float> out({n, (int64_t)k});
    {
        py::gil_scoped_release rel;
        check(mg_smooth_knn(d.ptr, n, k, n_neighbors, bandwidth, n_iter, out.mutable_data()));
    }
    return out;
}

// mid_near_pairs_dense of src/nndescent.cpp:731-768 on the device (signature of src/bindings.cpp:58-59)
py::array_t<int32_t> mid_near_pairs_dense(py::object X, int n_pairs, int n_cand, uint64_t seed, int n_threads) {
    auto x = view<float>(X);
    if (x.ndim() != 2 || x.dim(1) < 1) throw std::runtime_error("X must be 2-d");
    const int64_t n = x.dim(0);
    py::array_t<int32_t> out({n, (int64_t)n_pairs});
    {
        py::gil_scoped_release rel;
        check(mg_mid_near_pairs(x.ptr, n, (int)x.dim(1), n_pairs, n_cand, seed, n_threads, out.mutable_data()));
    }
    return out;
}

// knn_search of src/nndescent.cpp:660-690 on the device (signature of src/bindings.cpp:43-45)
py::tuple knn_search(py::object X, py::object gptr, py::object gidx, py::object landmarks, py::object Q, int k, int ef,
                     int n_entry, uint64_t seed, int n_threads) {
    auto x = view<float>(X), q = view<float>(Q);
    auto gp = view<int32_t>(gptr), gx = view<int32_t>(gidx), ld = view<int32_t>(landmarks);
    if (x.ndim() != 2 || q.ndim() != 2 || x.dim(1) != q.dim(1)) throw std::runtime_error("X and Q must be 2-d with the same width");
    const int64_t m = q.dim(0);
    py::array_t<int32_t> oi({m, (int64_t)k});
    py::array_t<float> od({m, (int64_t)k});
    {
        py::gil_scoped_release rel;
        check(mg_knn_search(x.ptr, x.dim(0), (int)x.dim(1), gp.ptr, gx.ptr, gx.size(), ld.ptr, ld.size(), q.ptr, m, k,
                            ef, n_entry, seed, n_threads, oi.mutable_data(), od.mutable_data()));
    }
    return py::make_tuple(oi, od);
}

// MAGNET._edge_schedule (magnet/__init__.py:726-737) on the device: (head, tail, eps) of the kept entries of the
// CSR graph, in CSR order, as host arrays
py::tuple edge_schedule_device(py::object indptr, py::object indices, py::object data, int n_epochs,
                               double samples_per_node) {
    auto ip = view<int32_t>(indptr), ix = view<int32_t>(indices);
    auto pd = view<float>(data);
    if (ip.ndim() != 1 || ip.size() < 1) throw std::runtime_error("indptr must have n + 1 entries");
    if (ix.size() != pd.size()) throw std::runtime_error("indices and data must have the same length");
    const int64_t n = ip.size() - 1, nnz = ix.size();
    py::array_t<int32_t> head(std::max<int64_t>(nnz, 1)), tail(std::max<int64_t>(nnz, 1));
    py::array_t<float> eps(std::max<int64_t>(nnz, 1));
    int64_t kept = 0;
    {
        py::gil_scoped_release rel;
        check(mg_edge_schedule(ip.ptr, ix.ptr, pd.ptr, n, nnz, samples_per_node, n_epochs, head.mutable_data(),
                               tail.mutable_data(), eps.mutable_data(), &kept));
    }
    return py::make_tuple(head[py::slice(0, kept, 1)], tail[py::slice(0, kept, 1)], eps[py::slice(0, kept, 1)]);
}

// chebyshev_eigenvectors (src/spectral.cpp:141-241) on the device; X is updated in place and returned, as the
// reference returns its X argument
py::object chebyshev_eigenvectors(py::object indptr, py::object indices, py::object data, py::object X,
                                  py::object inv_sqrt_deg, py::object component, int n_wanted, int degree,
                                  int max_iter, float tol, int n_threads) {
    (void)n_threads;   // the device solver does not take a host thread count
    auto ip = view<int32_t>(indptr), ix = view<int32_t>(indices), cp = view<int32_t>(component);
    auto pd = view<float>(data), sd = view<float>(inv_sqrt_deg);
    auto x = view<float>(X);
    if (x.ndim() != 2) throw std::runtime_error("X must be 2-d");
    const int64_t n = x.dim(0);
    if (ip.size() != n + 1) throw std::runtime_error("indptr must have n + 1 entries");
    if (ix.size() != pd.size()) throw std::runtime_error("indices and data must have the same length");
    if (sd.ndim() != 1 || sd.dim(0) != n) throw std::runtime_error("inv_sqrt_deg must have n entries");
    if (cp.ndim() != 1 || cp.dim(0) != n) throw std::runtime_error("component must have n entries");
    {
        py::gil_scoped_release rel;
        check(mg_chebyshev_eigenvectors(ip.ptr, ix.ptr, pd.ptr, n, ix.size(), x.ptr, (int)x.dim(1), sd.ptr, cp.ptr,
                                        n_wanted, degree, max_iter, tol));
    }
    return x.keep;
}

// the fuzzy union of magnet/knn.py:221-230 on the device: (indptr, indices, data) of the n x n CSR
py::tuple fuzzy_union(py::object ind, py::object vals, int64_t n, double set_op_mix_ratio) {
    auto id = view<int32_t>(ind);
    auto v = view<float>(vals);
    if (id.ndim() != 2 || v.ndim() != 2 || id.dim(0) != v.dim(0) || id.dim(1) != v.dim(1))
        throw std::runtime_error("ind and vals must be (n, k) of the same shape");
    const int64_t rows = id.dim(0);
    const int k = (int)id.dim(1);
    if (n < 0) n = rows;
    const int64_t cap = std::max<int64_t>(2 * rows * k, 1);
    py::array_t<int32_t> indptr(n + 1), indices(cap);
    py::array_t<float> data(cap);
    int64_t nnz = 0;
    {
        py::gil_scoped_release rel;
        check(mg_fuzzy_union(id.ptr, v.ptr, rows, k, n, set_op_mix_ratio, indptr.mutable_data(),
                             indices.mutable_data(), data.mutable_data(), cap, &nnz));
    }
    return py::make_tuple(indptr, indices[py::slice(0, nnz, 1)], data[py::slice(0, nnz, 1)]);
}

// many t-SNE layouts run together (mg_tsne_batch_*): one CUDA graph per iteration holds every layout's kernels
class TsneBatch {
  public:
    TsneBatch(py::list graphs, int n_iter, int early_iter, float early_exaggeration, float exaggeration,
              float learning_rate, float momentum_early, float momentum_late, int n_interp, float box_width, float dof,
              int min_boxes, int max_boxes, int threads_per_row, py::object layout_max_boxes, int branches) {
        const size_t count = graphs.size();
        std::vector<int64_t> n(count), nnz(count);
        std::vector<const int32_t*> ip(count), ix(count);
        std::vector<const float*> P(count);
        std::vector<View<int32_t>> keep_i;
        std::vector<View<float>> keep_f;
        for (size_t i = 0; i < count; ++i) {
            py::tuple t = graphs[i].cast<py::tuple>();
            if (t.size() != 3) throw std::runtime_error("each layout is (indptr, indices, data)");
            keep_i.push_back(view<int32_t>(t[0]));
            keep_i.push_back(view<int32_t>(t[1]));
            keep_f.push_back(view<float>(t[2]));
            const auto& a = keep_i[keep_i.size() - 2];
            const auto& b = keep_i.back();
            n[i] = a.size() - 1; nnz[i] = b.size();
            ip[i] = a.ptr; ix[i] = b.ptr; P[i] = keep_f.back().ptr;
        }
        std::vector<int> mb;
        if (!layout_max_boxes.is_none()) mb = layout_max_boxes.cast<std::vector<int>>();
        if (!mb.empty() && mb.size() != count) throw std::runtime_error("max_boxes needs one entry per layout");
        mg_tsne_params p;
        mg_tsne_params_default(&p);
        p.n_iter = n_iter; p.early_iter = early_iter; p.early_exaggeration = early_exaggeration;
        p.exaggeration = exaggeration; p.learning_rate = learning_rate; p.momentum_early = momentum_early;
        p.momentum_late = momentum_late; p.n_interp = n_interp; p.box_width = box_width; p.dof = dof;
        p.min_boxes = min_boxes; p.max_boxes = max_boxes; p.threads_per_row = threads_per_row;
        py::gil_scoped_release rel;
        check(mg_tsne_batch_create((int)count, n.data(), nnz.data(), ip.data(), ix.data(), P.data(), &p,
                                   mb.empty() ? nullptr : mb.data(), branches, &h_));
    }
    ~TsneBatch() { mg_tsne_batch_destroy(h_); }
    void run(py::list Ys) {
        std::vector<View<float>> keep;
        std::vector<float*> y;
        for (size_t i = 0; i < Ys.size(); ++i) {
            keep.push_back(view<float>(Ys[i]));
            if (keep.back().ndim() != 2 || keep.back().dim(1) != 2) throw std::runtime_error("each Y must be (n, 2)");
            y.push_back(keep.back().ptr);
        }
        int count = 0;
        check(mg_tsne_batch_size(h_, &count, nullptr));
        if ((int)y.size() != count) throw std::runtime_error("run needs one layout per graph of the batch");
        py::gil_scoped_release rel;
        check(mg_tsne_batch_run(h_, y.data()));
    }
    uint64_t kernels_per_iteration() const {
        uint64_t k = 0;
        check(mg_tsne_batch_size(h_, nullptr, &k));
        return k;
    }

  private:
    mg_tsne_batch* h_ = nullptr;
};

}  // namespace

PYBIND11_MODULE(_native, m) {
    m.doc() = "MAGNET layout pass on B200 (sm_100a): reference-compatible native entry points";
    py::class_<FFTConv2DDevice>(m, "FFTConv2D", "FFT repulsion with persistent device buffers: spread, FFTs, kernel products, gather")
        .def(py::init<int, int>(), py::arg("M"), py::arg("n_interp"))
        .def("set_kernels", &FFTConv2DDevice::set_kernels, py::arg("K1h"), py::arg("K2h"))
        .def("compute", &FFTConv2DDevice::compute, py::arg("Y"), py::arg("xmin"), py::arg("ymin"), py::arg("width"),
             py::arg("n_boxes"), py::arg("n_threads") = -1);
    m.def("optimize_layout", &optimize_layout, "SGD layout optimisation on the device (in place)",
          py::arg("Y"), py::arg("head"), py::arg("tail"), py::arg("epochs_per_sample"),
          py::arg("epoch_of_next_sample"), py::arg("epoch_of_next_negative_sample"),
          py::arg("indptr"), py::arg("indices"),
          py::arg("epoch_start"), py::arg("epoch_end"), py::arg("alpha0"), py::arg("alpha1"),
          py::arg("mid_w0"), py::arg("mid_w1"),
          py::arg("a"), py::arg("b"), py::arg("rep_a"), py::arg("rep_b"), py::arg("negative_sample_rate"), py::arg("loss"),
          py::arg("exaggeration"), py::arg("repulsion_strength"), py::arg("walk_len"), py::arg("mid_rate"),
          py::arg("optimizer"), py::arg("clip_mode"), py::arg("n_fixed"),
          py::arg("adam_m"), py::arg("adam_v"), py::arg("adam_t"), py::arg("beta1"), py::arg("beta2"),
          py::arg("walk_lens"), py::arg("mid_pairs"), py::arg("jump_indptr"), py::arg("jump_indices"),
          py::arg("mid_jump"), py::arg("kernel"), py::arg("node_b"), py::arg("seed"), py::arg("n_threads"),
          py::arg("parallel") = 0, py::arg("rev_indptr") = py::none(), py::arg("rev_indices") = py::none(),
          py::arg("stream_mode") = 0, py::arg("owner_chunk_edges") = 0);
    m.def("layout_schedule", &layout_schedule, "draws of one SGD epoch (test hook): (sampled, n_neg, neg_off, negs, mid)",
          py::arg("Y"), py::arg("head"), py::arg("tail"), py::arg("epochs_per_sample"), py::arg("epoch_of_next_sample"),
          py::arg("epoch_of_next_negative_sample"), py::arg("epoch"), py::arg("epoch_start"), py::arg("epoch_end"),
          py::arg("alpha0"), py::arg("alpha1"), py::arg("mid_w0"), py::arg("mid_w1"),
          py::arg("negative_sample_rate") = 5.0f, py::arg("loss") = 0, py::arg("mid_rate") = 0.25f,
          py::arg("walk_len") = 4, py::arg("n_fixed") = 0, py::arg("mid_pairs") = py::none(),
          py::arg("indptr") = py::none(), py::arg("indices") = py::none(), py::arg("seed") = 0,
          py::arg("stream_mode") = 0, py::arg("walk_lens") = py::none(), py::arg("jump_indptr") = py::none(),
          py::arg("jump_indices") = py::none(), py::arg("mid_jump") = 0.0f);
    m.def("smooth_knn", &smooth_knn, "UMAP smooth-kNN memberships (n, k) from sorted neighbour distances (device)",
          py::arg("dist"), py::arg("n_neighbors"), py::arg("bandwidth") = 1.0f, py::arg("n_iter") = 64,
          py::arg("n_threads") = -1);
    m.def("mid_near_pairs_dense", &mid_near_pairs_dense, "PaCMAP-style mid-near partners (dense rows, device)",
          py::arg("X"), py::arg("n_pairs") = 5, py::arg("n_cand") = 6, py::arg("seed") = 0, py::arg("n_threads") = -1);
    m.def("knn_search", &knn_search, "Beam search of queries over a neighbour graph (dense data, device)",
          py::arg("X"), py::arg("gptr"), py::arg("gidx"), py::arg("landmarks"), py::arg("Q"), py::arg("k"),
          py::arg("ef") = 64, py::arg("n_entry") = 10, py::arg("seed") = 0, py::arg("n_threads") = -1);
    m.def("edge_schedule_device", &edge_schedule_device,
          "the edge schedule of a fit on the device: (head, tail, epochs_per_sample) of the kept CSR entries",
          py::arg("indptr"), py::arg("indices"), py::arg("data"), py::arg("n_epochs"),
          py::arg("samples_per_node") = 5.0);
    m.def("chebyshev_eigenvectors", &chebyshev_eigenvectors,
          "Chebyshev-filtered subspace iteration for the leading non-trivial eigenvectors (device)",
          py::arg("indptr"), py::arg("indices"), py::arg("data"), py::arg("X"), py::arg("inv_sqrt_deg"),
          py::arg("component"), py::arg("n_wanted"), py::arg("degree"), py::arg("max_iter"), py::arg("tol"),
          py::arg("n_threads") = -1);
    m.def("fuzzy_union", &fuzzy_union, "fuzzy union A + A^T - A o A^T of kNN memberships (device): (indptr, indices, data)",
          py::arg("ind"), py::arg("vals"), py::arg("n") = -1, py::arg("set_op_mix_ratio") = 1.0);
    m.def("tsne_attraction", [](py::object indptr, py::object indices, py::object data, py::object Y, float dof, int) {
              auto ip = view<int32_t>(indptr), ix = view<int32_t>(indices);
              auto P = view<float>(data);
              auto y = view<float>(Y);
              if (y.ndim() != 2) throw std::runtime_error("Y must be 2-d");
              const int64_t n = y.dim(0);
              const int dim = (int)y.dim(1);
              if (ip.ndim() != 1 || ip.size() != n + 1) throw std::runtime_error("indptr must have n + 1 entries");
              if (ix.size() != P.size()) throw std::runtime_error("data must have indptr[n] entries");
              py::object out = like(Y, {n, (int64_t)dim});
              auto o = view<float>(out);
              {
                  py::gil_scoped_release rel;
                  check(mg_tsne_attraction(ip.ptr, ix.ptr, P.ptr, ix.size(), y.ptr, n, dim, dof, o.ptr));
              }
              return out;
          }, "sum_j p_ij (1 + d^2/dof)^-1 (y_i - y_j) over a CSR graph",
          py::arg("indptr"), py::arg("indices"), py::arg("data"), py::arg("Y"), py::arg("dof") = 1.0f, py::arg("n_threads") = -1);
    m.def("tsne_step", [](py::object Y, py::object update, py::object gains, py::object attr, py::object F, float rho,
                          float inv_sumQ, float lr, float momentum, int) {
              auto y = view<float>(Y), u = view<float>(update), g = view<float>(gains), a = view<float>(attr), f = view<float>(F);
              if (y.ndim() != 2) throw std::runtime_error("Y must be 2-d");
              const int64_t t = y.size();
              if (u.size() != t || g.size() != t || a.size() != t || f.size() != t) throw std::runtime_error("arrays must match Y");
              py::gil_scoped_release rel;
              check(mg_tsne_step(y.ptr, u.ptr, g.ptr, a.ptr, f.ptr, y.dim(0), (int)y.dim(1), rho, inv_sumQ, lr, momentum));
          }, "Fused t-SNE iteration: gradient combination, gains, momentum, update, recentring",
          py::arg("Y"), py::arg("update"), py::arg("gains"), py::arg("attr"), py::arg("F"), py::arg("rho"),
          py::arg("inv_sumQ"), py::arg("lr"), py::arg("momentum"), py::arg("n_threads") = -1);
    m.def("tsne_update", [](py::object Y, py::object update, py::object gains, py::object grad, float lr, float momentum, int) {
              auto y = view<float>(Y), u = view<float>(update), g = view<float>(gains), d = view<float>(grad);
              if (y.ndim() != 2) throw std::runtime_error("Y must be 2-d");
              const int64_t t = y.size();
              if (u.size() != t || g.size() != t || d.size() != t) throw std::runtime_error("arrays must match Y");
              py::gil_scoped_release rel;
              check(mg_tsne_update(y.ptr, u.ptr, g.ptr, d.ptr, y.dim(0), (int)y.dim(1), lr, momentum));
          }, "Fused gains / momentum / position update / recentring",
          py::arg("Y"), py::arg("update"), py::arg("gains"), py::arg("grad"), py::arg("lr"), py::arg("momentum"),
          py::arg("n_threads") = -1);
    m.def("bbox_2d", [](py::object Y, int) {
              auto y = view<float>(Y);
              if (y.ndim() != 2 || y.dim(1) != 2 || y.dim(0) < 1) throw std::runtime_error("Y must be (n, 2)");
              float out[4];
              {
                  py::gil_scoped_release rel;
                  check(mg_bbox_2d(y.ptr, y.dim(0), out));
              }
              return py::make_tuple(out[0], out[1], out[2], out[3]);
          }, "Bounding box of a (n, 2) array", py::arg("Y"), py::arg("n_threads") = -1);
    m.def("mid_spring", [](py::object Y, py::object pairs, py::object grad, float w, int) {
              auto y = view<float>(Y);
              auto p = view<int32_t>(pairs);
              auto g = view<float>(grad);
              if (y.ndim() != 2 || g.ndim() != 2 || p.ndim() != 2) throw std::runtime_error("bad shapes");
              if (p.dim(0) != y.dim(0) || g.dim(0) != y.dim(0) || g.dim(1) != y.dim(1) || p.dim(1) < 1)
                  throw std::runtime_error("bad shapes");
              py::gil_scoped_release rel;
              check(mg_mid_spring(y.ptr, p.ptr, g.ptr, y.dim(0), (int)y.dim(1), (int)p.dim(1), w));
          }, "grad += w (Y_i - mean of partner positions)",
          py::arg("Y"), py::arg("pairs"), py::arg("grad"), py::arg("w"), py::arg("n_threads") = -1);
    m.def("optimize_tsne", [](py::object indptr, py::object indices, py::object data, py::object Y, int n_iter,
                              int early_iter, float early_exaggeration, float exaggeration, float learning_rate,
                              float momentum_early, float momentum_late, int n_interp, float box_width, float dof,
                              int min_boxes, int max_boxes, int threads_per_row, bool use_graph) {
              auto ip = view<int32_t>(indptr), ix = view<int32_t>(indices);
              auto P = view<float>(data);
              auto y = view<float>(Y);
              if (y.ndim() != 2 || y.dim(1) != 2) throw std::runtime_error("Y must be (n, 2)");
              mg_tsne_params p;
              mg_tsne_params_default(&p);
              p.n_iter = n_iter; p.early_iter = early_iter; p.early_exaggeration = early_exaggeration;
              p.exaggeration = exaggeration; p.learning_rate = learning_rate; p.momentum_early = momentum_early;
              p.momentum_late = momentum_late; p.n_interp = n_interp; p.box_width = box_width; p.dof = dof;
              p.min_boxes = min_boxes; p.max_boxes = max_boxes; p.threads_per_row = threads_per_row;
              p.use_graph = use_graph ? 1 : 0;
              py::gil_scoped_release rel;
              check(mg_optimize_tsne(ip.ptr, ix.ptr, P.ptr, y.dim(0), ix.size(), y.ptr, &p));
          }, "Whole t-SNE pass on the device (in place on Y; P is normalised to sum 1 inside)",
          py::arg("indptr"), py::arg("indices"), py::arg("data"), py::arg("Y"), py::arg("n_iter") = 750,
          py::arg("early_iter") = 250, py::arg("early_exaggeration") = 12.0f, py::arg("exaggeration") = 1.0f,
          py::arg("learning_rate") = -1.0f, py::arg("momentum_early") = 0.5f, py::arg("momentum_late") = 0.8f,
          py::arg("n_interp") = 3, py::arg("box_width") = 0.7f, py::arg("dof") = 1.0f, py::arg("min_boxes") = 20,
          py::arg("max_boxes") = 1000, py::arg("threads_per_row") = 0, py::arg("use_graph") = true);
    m.def("optimize_tsne_profiled", [](py::object indptr, py::object indices, py::object data, py::object Y, int n_iter,
                                       int early_iter, float early_exaggeration, float exaggeration,
                                       float learning_rate, int n_interp, float box_width, float dof) {
              auto ip = view<int32_t>(indptr), ix = view<int32_t>(indices);
              auto P = view<float>(data);
              auto y = view<float>(Y);
              mg_tsne_params p;
              mg_tsne_params_default(&p);
              p.n_iter = n_iter; p.early_iter = early_iter; p.early_exaggeration = early_exaggeration;
              p.exaggeration = exaggeration; p.learning_rate = learning_rate; p.n_interp = n_interp;
              p.box_width = box_width; p.dof = dof;
              double ms[9];
              int grid[4];
              {
                  py::gil_scoped_release rel;
                  check(mg_optimize_tsne_profiled(ip.ptr, ix.ptr, P.ptr, y.dim(0), ix.size(), y.ptr, &p, ms, grid));
              }
              py::dict out;
              const char* names[9] = {"bbox_grid", "twiddles", "spectra", "spread", "row_fwd", "col_conv", "row_inv",
                                      "gather_attr_step", "iteration"};
              for (int k = 0; k < 9; ++k) out[names[k]] = ms[k];
              out["grid"] = py::make_tuple(grid[0], grid[1], grid[2], grid[3]);
              return out;
          }, "t-SNE pass with per-stage CUDA-event timing (plain launches); returns the summed ms per stage",
          py::arg("indptr"), py::arg("indices"), py::arg("data"), py::arg("Y"), py::arg("n_iter"),
          py::arg("early_iter") = 0, py::arg("early_exaggeration") = 12.0f, py::arg("exaggeration") = 1.0f,
          py::arg("learning_rate") = -1.0f, py::arg("n_interp") = 3, py::arg("box_width") = 0.7f, py::arg("dof") = 1.0f);
    py::class_<TsneBatch>(m, "TsneBatch", "many t-SNE layouts run together, one CUDA graph per iteration")
        .def(py::init<py::list, int, int, float, float, float, float, float, int, float, float, int, int, int,
                      py::object, int>(),
             py::arg("graphs"), py::arg("n_iter") = 750, py::arg("early_iter") = 250,
             py::arg("early_exaggeration") = 12.0f, py::arg("exaggeration") = 1.0f, py::arg("learning_rate") = -1.0f,
             py::arg("momentum_early") = 0.5f, py::arg("momentum_late") = 0.8f, py::arg("n_interp") = 3,
             py::arg("box_width") = 0.7f, py::arg("dof") = 1.0f, py::arg("min_boxes") = 20, py::arg("max_boxes") = 1000,
             py::arg("threads_per_row") = 0, py::arg("layout_max_boxes") = py::none(), py::arg("branches") = 32)
        .def("run", &TsneBatch::run, py::arg("Ys"))
        .def_property_readonly("kernels_per_iteration", &TsneBatch::kernels_per_iteration);
    m.def("center_scale", [](py::object Y, double target_std) {
              auto y = view<float>(Y);
              if (y.ndim() != 2) throw std::runtime_error("Y must be (n, dim)");
              py::gil_scoped_release rel;
              check(mg_center_scale(y.ptr, y.dim(0), (int)y.dim(1), target_std));
          }, "Y -= column means; Y *= target_std / std(Y[:, 0]) (the hybrid hand-off)", py::arg("Y"), py::arg("target_std"));
    m.def("launch_count", []() { return mg_launch_count(); });
    m.def("synchronize", []() { check(mg_synchronize()); });
    m.def("set_stream", [](uintptr_t s) { check(mg_set_stream(reinterpret_cast<void*>(s))); }, py::arg("stream"));
    m.attr("__version__") = mg_version();
}
