// Owner mode of optimize_layout (parallel = 1): src/layout.cpp:118-276 with OWNER = true, :300-330 (owner epochs),
// :441-463 (chunks), :31-40 (the owner attraction scale 1.5).
//
// The reference splits the nodes at the edge quantiles into n_chunks = min(4096, max(1, E / 4096)) chunks (edges
// sorted by head). In epoch e, chunk k draws from its own stream stream_seed(seed, e, k) over its edges in order,
// moves only its own heads u (no step on the tail or on the partners) and reads every other position from the
// layout as it was at the start of the epoch; with the reverse mid pairs, u also takes, after each edge, the pulls
// of the nodes that chose it. The result is a function of the inputs alone, whatever the thread count.
//
// On the device one epoch is four steps on the caller's stream:
//  1. snapshot: the layout (and the Adam state) is copied aside; it is the "start of the epoch" every read uses;
//  2. schedule, one thread per edge: advances eons / eonns as the reference does and records each sampled edge's
//     negatives count; then the chain pass, one warp per chunk: consumes the chunk's stream in edge order as
//     the edge loop would (n_neg draws, the mid-range test and walk, the reverse-pull draws), recording at each
//     head's first sampled edge the stream state where its draws start. It reads no position: the draws depend
//     on positions only through a negative at distance 0 exactly (src/layout.cpp:181), which draws dim extra
//     uniforms;
//  3. node pass, one thread per head node: from its recorded state, replays the node's edges as the reference
//     does (other positions from the snapshot, its own in registers) and writes its row. A negative at distance 0
//     marks the node's chunk, since the states recorded after it are then off by dim draws;
//  4. fallback, one thread per chunk, doing work for marked chunks only: restores the rows of the chunk's heads
//     (and their Adam state) from the snapshot and replays the whole chunk serially from the chunk's seed.
// This file is compiled without FMA contraction (-fmad=false): every product and sum rounds on its own, as in
// the reference's plain x86-64 build. The power kernel with b = rep_b = 1 under the sgd optimizer uses +, *, / and
// sqrt only and reproduces the reference bit for bit; powf, expf, tanhf and coshf may differ from the host libm
// in the last place.
#include "sgd.cuh"
#include <algorithm>
#include <climits>

namespace mgb {

namespace {

constexpr int32_t kNotSampled = INT32_MIN;   // n_neg record of an edge skipped this epoch
constexpr float kOwnerAttraction = 1.5f;     // OWNER_ATT, src/layout.cpp:40

struct OwnerDev {
    const int64_t* own; const int64_t* eown; int n_chunks;   // first node / first edge of each chunk (+1 entry)
    const int64_t* row;                                       // first edge of each node (n + 1 entries)
    const int32_t* rev_indptr; const int32_t* rev_indices;    // reverse mid pairs or NULL
    int32_t* n_neg;                                           // per edge: this epoch's negatives, kNotSampled
    uint64_t* node_state;                                     // stream state at each node's first edge
    int* dirty;                                               // per chunk: a distance-0 negative was drawn
    const float* Yr;                                          // the layout at the start of the epoch
    const float* snap_m; const float* snap_v; const int32_t* snap_t;   // the Adam state at the start
};

// the mid-range partner of edge (u, v) (src/layout.cpp:225-249), after the mid_rate test succeeded
__device__ __forceinline__ int32_t mid_partner(const SgdDev& c, Rng& r, int64_t u, int32_t v) {
    int32_t w = v;
    if (c.jump_indptr) {
        const int L = c.walk_lens ? c.walk_lens[v] : c.walk_len;
        for (int h = 0; h < L; ++h) {
            const int32_t js = c.jump_indptr[w], je = c.jump_indptr[w + 1];
            if (je > js && r.uniform() < c.mid_jump) {
                w = c.jump_indices[js + (int32_t)r.below((uint32_t)(je - js))];
            } else {
                const int32_t s0 = c.indptr[w], e0 = c.indptr[w + 1];
                if (e0 <= s0) break;
                w = c.indices[s0 + (int32_t)r.below((uint32_t)(e0 - s0))];
            }
        }
    } else if (c.mid_pairs) {
        w = c.mid_pairs[u * c.n_mid + r.below((uint32_t)c.n_mid)];
    } else {
        const int L = c.walk_lens ? c.walk_lens[v] : c.walk_len;
        for (int h = 0; h < L; ++h) {
            const int32_t s0 = c.indptr[w], e0 = c.indptr[w + 1];
            if (e0 <= s0) break;
            w = c.indices[s0 + (int32_t)r.below((uint32_t)(e0 - s0))];
        }
    }
    return w;
}

// apply_step (src/layout.cpp:90-116) on a row held in registers; the Adam state of u belongs to this thread
template <int DM>
__device__ __forceinline__ void owner_step(const SgdDev& c, float* yu, const float* g, float alpha, int64_t u,
                                           int dim) {
    float step[DM];
    if (c.optimizer == 1) {
        const int32_t t = ++c.adam_t[u];
        const float c1 = 1.0f - powf(c.beta1, (float)t), c2 = 1.0f - powf(c.beta2, (float)t);
        float* m = c.adam_m + u * dim;
        float* v = c.adam_v + u * dim;
        for (int d = 0; d < dim; ++d) {
            m[d] = c.beta1 * m[d] + (1.0f - c.beta1) * g[d];
            v[d] = c.beta2 * v[d] + (1.0f - c.beta2) * g[d] * g[d];
            step[d] = alpha * (m[d] / c1) / (sqrtf(v[d] / c2) + 1e-7f);
        }
    } else {
#pragma unroll
        for (int d = 0; d < DM; ++d)
            if (d < dim) step[d] = alpha * g[d];
    }
    const float cap = 4.0f * alpha;
    if (c.clip_mode == 1) {
        float n2 = 0.0f;
#pragma unroll
        for (int d = 0; d < DM; ++d)
            if (d < dim) n2 += step[d] * step[d];
        if (n2 > cap * cap) {
            const float f = cap / sqrtf(n2);
#pragma unroll
            for (int d = 0; d < DM; ++d)
                if (d < dim) step[d] *= f;
        }
    } else {
#pragma unroll
        for (int d = 0; d < DM; ++d)
            if (d < dim) step[d] = step[d] > cap ? cap : (step[d] < -cap ? -cap : step[d]);
    }
#pragma unroll
    for (int d = 0; d < DM; ++d)
        if (d < dim) yu[d] += step[d];
}

// The edges of head node u in one epoch, from stream state `state`; returns the state after them. The row is read
// from the snapshot and written back to Y (when u may move). `jitter` is set when a negative lands at distance 0.
template <int D>
__device__ uint64_t owner_node(const SgdDev& c, const OwnerDev& o, int64_t u, uint64_t state, float alpha,
                               float mid_w, bool& jitter) {
    constexpr int DM = D ? D : kMaxDim;
    const int dim = D ? D : c.dim;
    Rng r(0);
    r.s = state;
    const bool move_u = u >= c.n_fixed;
    const float inv_n_mid = c.n_mid > 0 ? 1.0f / (float)c.n_mid : 0.0f;
    float yu[DM], diff[DM], gu[DM], gk[DM];
#pragma unroll
    for (int d = 0; d < DM; ++d)
        if (d < dim) yu[d] = o.Yr[u * dim + d];
    const int64_t row1 = o.row[u + 1];
    for (int64_t w0 = o.row[u]; w0 < row1; w0 += 64) {
        // the sampled edges of a window of 64 as a bit mask, taken in edge order
        const int cnt = (int)(row1 - w0 < 64 ? row1 - w0 : 64);
        uint64_t mask = 0;
        for (int t = 0; t < cnt; ++t)
            if (o.n_neg[w0 + t] != kNotSampled) mask |= 1ull << t;
        while (mask) {
            const int64_t i = w0 + (__ffsll((long long)mask) - 1);
            mask &= mask - 1;
            const int n_neg = o.n_neg[i];
            const int32_t v = c.tail[i];
            const float* yv = o.Yr + (int64_t)v * dim;
            float d2 = 0.0f;
#pragma unroll
            for (int d = 0; d < DM; ++d)
                if (d < dim) { gu[d] = 0.0f; diff[d] = yu[d] - yv[d]; d2 += diff[d] * diff[d]; }
            const float b_u = c.node_b ? c.node_b[u] : c.b;
            const float b_uv = c.node_b ? 0.5f * (c.node_b[u] + c.node_b[v]) : c.b;
            const float pw_v = (c.b_is_one && !c.node_b) ? d2 : (d2 > 0.0f ? powf(d2, b_uv) : 0.0f);
            // attraction along the edge, the head only, scaled by 1.5
            if (d2 > 0.0f) {
                float coeff;
                if (c.kernel == 0) coeff = -kOwnerAttraction * c.exaggeration * 2.0f * c.a * b_uv * pw_v / (d2 * (c.a * pw_v + 1.0f));
                else if (c.kernel == 1) coeff = -kOwnerAttraction * c.exaggeration * 2.0f * c.a;
                else if (c.kernel == 2) { const float dd = sqrtf(d2); coeff = -kOwnerAttraction * c.exaggeration * c.a * tanhf(c.a * dd) / dd; }
                else coeff = -kOwnerAttraction * c.exaggeration * 2.0f * c.a * (1.0f + tanhf(c.a * d2));
#pragma unroll
                for (int d = 0; d < DM; ++d)
                    if (d < dim) gu[d] += coeff * diff[d];
            }
            // repulsion from the negatives, read from the snapshot
            for (int p = 0; p < n_neg; ++p) {
                const int32_t k = (int32_t)r.below((uint32_t)c.n);
                if (k == u) continue;
                const float* yk = o.Yr + (int64_t)k * dim;
                float dd = 0.0f;
#pragma unroll
                for (int d = 0; d < DM; ++d)
                    if (d < dim) { diff[d] = yu[d] - yk[d]; dd += diff[d] * diff[d]; }
                if (dd > 0.0f) {
                    float coeff;
                    if (c.kernel == 0) {
                        if (c.node_b && c.rep_coupled) { const float pw = powf(dd, b_u); coeff = 2.0f * b_u * c.repulsion_strength / ((0.001f + dd) * (c.a * pw + 1.0f)); }
                        else { const float pw = c.rep_b_is_one ? dd : powf(dd, c.rep_b); coeff = c.two_b / ((0.001f + dd) * (c.rep_a * pw + 1.0f)); }
                    } else if (c.kernel == 1) {
                        const float q = expf(-c.a * dd);
                        coeff = c.repulsion_strength * 2.0f * c.a * q / fmaxf(1.0f - q, 1e-3f);
                    } else if (c.kernel == 2) {
                        const float rr = sqrtf(dd); const float q = 1.0f / coshf(c.a * rr);
                        coeff = c.repulsion_strength * c.a * q * tanhf(c.a * rr) / (rr * fmaxf(1.0f - q, 1e-3f));
                    } else {
                        const float th = fmaxf(tanhf(c.a * dd), 1e-3f);
                        coeff = c.repulsion_strength * 2.0f * c.a * (1.0f - th * th) / th;
                    }
#pragma unroll
                    for (int d = 0; d < DM; ++d)
                        if (d < dim) gu[d] += coeff * diff[d];
                } else {
                    jitter = true;
                    for (int d = 0; d < dim; ++d) gu[d] += (r.uniform() - 0.5f) * 1e-3f / fmaxf(alpha, 1e-6f);
                }
            }
            // mid-range partner, read from the snapshot
            if (mid_w > 0.0f && r.uniform() < c.mid_rate) {
                const int32_t w = mid_partner(c, r, u, v);
                if (w != u) {
                    const float* yw = o.Yr + (int64_t)w * dim;
#pragma unroll
                    for (int d = 0; d < DM; ++d)
                        if (d < dim) { const float g = -mid_w * (yu[d] - yw[d]); gu[d] += g; }
                }
            }
            if (move_u) owner_step<DM>(c, yu, gu, alpha, u, dim);
            // the pulls of the nodes that chose u as their partner, each its own step
            if (move_u && mid_w > 0.0f && o.rev_indptr) {
                const int32_t rs = o.rev_indptr[u], re = o.rev_indptr[u + 1];
                float p = c.mid_rate * (float)(re - rs) * inv_n_mid;
                while (p > 0.0f && re > rs) {
                    if (r.uniform() < p) {
                        const int32_t x = o.rev_indices[rs + (int32_t)r.below((uint32_t)(re - rs))];
                        if (x != u) {
                            const float* yx = o.Yr + (int64_t)x * dim;
#pragma unroll
                            for (int d = 0; d < DM; ++d)
                                if (d < dim) gk[d] = -mid_w * (yu[d] - yx[d]);
                            owner_step<DM>(c, yu, gk, alpha, u, dim);
                        }
                    }
                    p -= 1.0f;
                }
            }
        }
    }
    if (move_u) {
#pragma unroll
        for (int d = 0; d < DM; ++d)
            if (d < dim) c.Y[u * dim + d] = yu[d];
    }
    return r.s;
}

// ---------------------------------------------------------------------------------------------- set-up kernels
// first edge of every node (lower bound of u in the sorted heads), u in [0, n]
__global__ void owner_rows_kernel(const int32_t* __restrict__ head, int64_t E, int64_t n, int64_t* __restrict__ row) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u > n) return;
    int64_t lo = 0, hi = E;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)head[mid] < u) lo = mid + 1; else hi = mid;
    }
    row[u] = lo;
}

// chunk boundaries (src/layout.cpp:448-462): own[t] = max(head[E t / nc], own[t - 1]), which is head[E t / nc]
// itself for sorted heads; eown[t] is the first edge of own[t]
__global__ void owner_chunks_kernel(const int32_t* __restrict__ head, int64_t E, int64_t n, int nc,
                                    const int64_t* __restrict__ row, int64_t* __restrict__ own,
                                    int64_t* __restrict__ eown) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > nc) return;
    const int64_t node = t == 0 ? 0 : (t == nc ? n : (int64_t)head[E * t / nc]);
    own[t] = node;
    eown[t] = t == nc ? E : row[node];
}

__global__ void owner_sorted_kernel(const int32_t* __restrict__ head, int64_t E, int* __restrict__ unsorted) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; i < E; i += (int64_t)gridDim.x * blockDim.x)
        if (head[i - 1] > head[i]) { atomicExch(unsorted, 1); return; }
}

// ---------------------------------------------------------------------------------------------- epoch kernels
// the epoch's schedule, one thread per edge (coalesced): eons / eonns advanced as src/layout.cpp:135,160-163,184
// advance them, and each edge's negatives count recorded (kNotSampled when eons[i] > epoch)
__global__ void __launch_bounds__(256) owner_schedule_kernel(SgdDev c, OwnerDev o, int epoch) {
    const float fepoch = (float)epoch;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c.n_edges;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float eo = c.eons[i];
        if (eo > fepoch) { o.n_neg[i] = kNotSampled; continue; }
        const float ep = c.eps[i];
        c.eons[i] = eo + ep;
        const float epn = ep / c.negative_sample_rate;
        const float en = c.eonns[i];
        const int n_neg = (int)((fepoch - en) / epn);
        c.eonns[i] = en + (float)n_neg * epn;
        o.n_neg[i] = n_neg;
    }
}

// One warp per chunk: the chunk's stream consumed in edge order from the recorded negatives counts. The lanes
// read 32 edges' counts and heads at a time (coalesced) and take the sampled ones in order from a ballot; every
// lane holds the same stream state and makes the same draws, so control flow stays uniform across the warp.
// A head's state is recorded at its first sampled edge (edges that are not sampled draw nothing, and a head
// without sampled edges draws nothing in the node pass), so heads without edges, such as the fixed training rows
// of a transform, cost nothing. No position is read and nothing is stored but the per-node states.
constexpr int kChainWarps = 4;   // chunks per block

__global__ void __launch_bounds__(32 * kChainWarps) owner_chain_kernel(SgdDev c, OwnerDev o, int epoch,
                                                                        float mid_w) {
    const int k = blockIdx.x * kChainWarps + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= o.n_chunks) return;
    Rng r(stream_seed(c.seed, epoch, (uint64_t)k));
    const float inv_n_mid = c.n_mid > 0 ? 1.0f / (float)c.n_mid : 0.0f;
    const int32_t* __restrict__ rec = o.n_neg;
    const int64_t e0 = o.eown[k], e1 = o.eown[k + 1];
    int64_t u = -1;
    float p0 = 0.0f;
    for (int64_t base = e0; base < e1; base += 32) {
        const int64_t i = base + lane;
        const int mine = i < e1 ? __ldg(rec + i) : kNotSampled;
        const int32_t my_head = i < e1 ? c.head[i] : -1;
        unsigned todo = __ballot_sync(0xffffffffu, mine != kNotSampled);
        while (todo) {
            const int b = __ffs(todo) - 1;
            todo &= todo - 1;
            const int n_neg = __shfl_sync(0xffffffffu, mine, b);
            const int32_t h = __shfl_sync(0xffffffffu, my_head, b);
            if (h != u) {
                u = h;
                if (lane == 0) o.node_state[u] = r.s;
                // the reverse-pull rounds of each of u's edges: the same p for every edge of u
                p0 = 0.0f;
                if (u >= c.n_fixed && mid_w > 0.0f && o.rev_indptr) {
                    const int32_t rs = o.rev_indptr[u], re = o.rev_indptr[u + 1];
                    if (re > rs) p0 = c.mid_rate * (float)(re - rs) * inv_n_mid;
                }
            }
            for (int p = 0; p < n_neg; ++p) r.next();
            if (mid_w > 0.0f && r.uniform() < c.mid_rate) (void)mid_partner(c, r, u, c.tail[base + b]);
            for (float p = p0; p > 0.0f; p -= 1.0f)
                if (r.uniform() < p) (void)r.next();
        }
    }
}

template <int D>
__global__ void __launch_bounds__(128) owner_node_kernel(SgdDev c, OwnerDev o, int epoch, float alpha, float mid_w) {
    const int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= c.n || o.row[u] == o.row[u + 1]) return;
    bool jitter = false;
    owner_node<D>(c, o, u, o.node_state[u], alpha, mid_w, jitter);
    if (jitter) {
        // the chunk holding u: the last k with own[k] <= u (empty chunks share their bound with the next one)
        int lo = 0, hi = o.n_chunks;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (o.own[mid] <= u) lo = mid; else hi = mid;
        }
        atomicExch(&o.dirty[lo], 1);
    }
}

template <int D>
__global__ void __launch_bounds__(32) owner_fallback_kernel(SgdDev c, OwnerDev o, int epoch, float alpha,
                                                            float mid_w) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= o.n_chunks || !o.dirty[k]) return;
    o.dirty[k] = 0;
    // the heads of the chunk's edges (a marked chunk has at least one); rows without edges never move
    const int64_t u0 = c.head[o.eown[k]], u1 = (int64_t)c.head[o.eown[k + 1] - 1] + 1;
    const int dim = c.dim;
    for (int64_t j = u0 * dim; j < u1 * dim; ++j) c.Y[j] = o.Yr[j];
    if (c.optimizer == 1) {
        for (int64_t j = u0 * dim; j < u1 * dim; ++j) { c.adam_m[j] = o.snap_m[j]; c.adam_v[j] = o.snap_v[j]; }
        for (int64_t u = u0; u < u1; ++u) c.adam_t[u] = o.snap_t[u];
    }
    uint64_t state = Rng(stream_seed(c.seed, epoch, (uint64_t)k)).s;
    bool jitter = false;
    for (int64_t u = u0; u < u1; ++u) state = owner_node<D>(c, o, u, state, alpha, mid_w, jitter);
}

template <int D>
void owner_epoch_launch(const SgdDev& c, const OwnerDev& o, int epoch, float alpha, float mid_w, cudaStream_t s) {
    owner_node_kernel<D><<<ceil_div(c.n, 128), 128, 0, s>>>(c, o, epoch, alpha, mid_w);
    MGB_LAUNCH_CHECK();
    owner_fallback_kernel<D><<<ceil_div(o.n_chunks, 32), 32, 0, s>>>(c, o, epoch, alpha, mid_w);
    MGB_LAUNCH_CHECK();
}

}  // namespace

int owner_chunk_count(int64_t n_edges, int chunk_edges) {
    const int64_t per = chunk_edges > 0 ? chunk_edges : 4096;
    return (int)std::min<int64_t>(chunk_edges > 0 ? INT32_MAX / 2 : 4096, std::max<int64_t>(1, n_edges / per));
}

bool owner_heads_sorted(const int32_t* head_dev, int64_t n_edges, SgdWork& w, cudaStream_t s) {
    if (n_edges < 2) return true;
    int* flag = static_cast<int*>(w.flag.ensure(sizeof(int)));
    MGB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
    owner_sorted_kernel<<<std::min(ceil_div(n_edges, 256), 4 * kNumSMs), 256, 0, s>>>(head_dev, n_edges, flag);
    MGB_LAUNCH_CHECK();
    int h = 0;
    MGB_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    MGB_CUDA(cudaStreamSynchronize(s));
    return h == 0;
}

void owner_run(SgdDev& c, SgdWork& w, const int32_t* rev_indptr, const int32_t* rev_indices, int chunk_edges,
               int e0, int e1, float alpha0, float alpha1, float mid_w0, float mid_w1, cudaStream_t s) {
    const int64_t n = c.n, E = c.n_edges;
    const int dim = c.dim;
    const int nc = owner_chunk_count(E, chunk_edges);
    OwnerDev o{};
    int64_t* row = static_cast<int64_t*>(w.o_row.ensure(sizeof(int64_t) * (n + 1)));
    int64_t* own = static_cast<int64_t*>(w.o_own.ensure(sizeof(int64_t) * (nc + 1) * 2));
    int64_t* eown = own + (nc + 1);
    o.row = row; o.own = own; o.eown = eown; o.n_chunks = nc;
    o.rev_indptr = rev_indptr; o.rev_indices = rev_indices;
    o.n_neg = static_cast<int32_t*>(w.o_neg.ensure(sizeof(int32_t) * std::max<int64_t>(E, 1)));
    o.node_state = static_cast<uint64_t*>(w.o_state.ensure(sizeof(uint64_t) * std::max<int64_t>(n, 1)));
    o.dirty = static_cast<int*>(w.o_dirty.ensure(sizeof(int) * nc));
    float* snap = static_cast<float*>(w.o_snap.ensure(sizeof(float) * std::max<int64_t>(n * dim, 1)));
    o.Yr = snap;
    float* snap_m = nullptr; float* snap_v = nullptr; int32_t* snap_t = nullptr;
    if (c.optimizer == 1) {
        snap_m = static_cast<float*>(w.o_snap_m.ensure(sizeof(float) * std::max<int64_t>(n * dim, 1)));
        snap_v = static_cast<float*>(w.o_snap_v.ensure(sizeof(float) * std::max<int64_t>(n * dim, 1)));
        snap_t = static_cast<int32_t*>(w.o_snap_t.ensure(sizeof(int32_t) * std::max<int64_t>(n, 1)));
    }
    o.snap_m = snap_m; o.snap_v = snap_v; o.snap_t = snap_t;
    MGB_CUDA(cudaMemsetAsync(o.dirty, 0, sizeof(int) * nc, s));
    owner_rows_kernel<<<ceil_div(n + 1, 256), 256, 0, s>>>(c.head, E, n, row);
    MGB_LAUNCH_CHECK();
    owner_chunks_kernel<<<ceil_div(nc + 1, 256), 256, 0, s>>>(c.head, E, n, nc, row, own, eown);
    MGB_LAUNCH_CHECK();
    for (int epoch = e0; epoch < e1; ++epoch) {
        float alpha, mid_w;
        sgd_sched(c, epoch, e0, e1, alpha0, alpha1, mid_w0, mid_w1, alpha, mid_w);
        MGB_CUDA(cudaMemcpyAsync(snap, c.Y, sizeof(float) * n * dim, cudaMemcpyDeviceToDevice, s));
        if (c.optimizer == 1) {
            MGB_CUDA(cudaMemcpyAsync(snap_m, c.adam_m, sizeof(float) * n * dim, cudaMemcpyDeviceToDevice, s));
            MGB_CUDA(cudaMemcpyAsync(snap_v, c.adam_v, sizeof(float) * n * dim, cudaMemcpyDeviceToDevice, s));
            MGB_CUDA(cudaMemcpyAsync(snap_t, c.adam_t, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, s));
        }
        owner_schedule_kernel<<<std::min(ceil_div(E, 256), 8 * kNumSMs), 256, 0, s>>>(c, o, epoch);
        MGB_LAUNCH_CHECK();
        owner_chain_kernel<<<ceil_div(nc, kChainWarps), 32 * kChainWarps, 0, s>>>(c, o, epoch, mid_w);
        MGB_LAUNCH_CHECK();
        MGB_DIM_DISPATCH(dim, owner_epoch_launch, c, o, epoch, alpha, mid_w, s);
    }
}

}  // namespace mgb
