// Sampled SGD layout on the device: optimize_layout of src/layout.cpp:343-472 (epoch_worker :118-276,
// apply_step :90-116, run_epochs :281-339).
//
// Two stream modes:
//  * counter-based (stream_mode 0, default): every draw of a sample is addressed by (seed, epoch, edge, index).
//    The sample of edge i in epoch e has a 32-bit key, the hash of the reference's stream seed
//    (src/layout.cpp:123) stream_seed(seed, e, i); its draw j is hash32(key + j * 0x9E3779B9) in the high 32
//    bits of a 64-bit draw, so below(n) and uniform() read it as they read the reference's 64-bit outputs.
//    Negative p is draw p; the mid-range draws are draws 1024, 1025, ...; the distance-0 jitter of negative p
//    in dimension d is draw 2048 + 64 p + d. Any lane can take any draw directly with one 32-bit hash, so the
//    draws of a sample need no coordination. With the edges sorted by head (the reference's schedule is the COO of a
//    sorted CSR) one thread owns a head row and applies the head's steps one after another, as the reference's
//    loop does; the tails and partners move through hogwild float2 atomics. At most n / 8 rows are in flight.
//  * serial (stream_mode 1): the reference's single stream per epoch (n_threads = 1) is replayed exactly. The
//    schedule (eons / eonns) is computed in parallel; one thread walks the sampled edges in order to find where
//    each edge's draws start in the stream (its RNG state is recorded), then the head rows run in parallel from
//    their recorded states in 8 sub-steps per epoch (sub-step p: the p-th sampled edge of every row). Within a
//    sub-step every position is read as committed by the previous one and all displacements are summed in 2^-32
//    fixed point (order-independent integer atomics), so the result does not depend on scheduling: the same
//    inputs give the same bits on every run.
//    Assumption stated for the replay: no negative sample lands at exactly the head's position (distance 0);
//    the reference draws extra uniforms in that case (src/layout.cpp:181), which the replay does not.
#include "sgd.cuh"
#include <vector>
#include <cmath>
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <unordered_map>

namespace mgb {

namespace {

constexpr int kThreads = 256;
constexpr double kFix = 4294967296.0;   // 2^32
constexpr int kMidDraw = 1024;          // first draw index of the mid-range draws (counter mode)
constexpr int kJitterDraw = 2048;       // first draw index of the distance-0 jitter (counter mode)

int blocks_for(int64_t work, int per_block, int cap_per_sm = 16) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((work + per_block - 1) / per_block, (int64_t)cap_per_sm * kNumSMs));
}

// ---------------------------------------------------------------------------------------------- draws
__device__ __forceinline__ uint32_t below_of(uint64_t x, uint32_t n) { return (uint32_t)(((x >> 32) * (uint64_t)n) >> 32); }
__device__ __forceinline__ float uniform_of(uint64_t x) { return (float)(x >> 40) * (1.0f / 16777216.0f); }
// 32-bit integer hash: "lowbias32" of C. Wellons' hash-prospector (xorshift-multiply rounds, full avalanche)
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
// key of a sample from its 64-bit stream seed
__device__ __forceinline__ uint32_t sample_key(uint64_t ss) {
    return hash32((uint32_t)ss ^ hash32((uint32_t)(ss >> 32)));
}
// draw j of a sample, in the high half of a 64-bit draw
__device__ __forceinline__ uint64_t counter_draw(uint32_t key, int j) {
    return (uint64_t)hash32(key + (uint32_t)j * 0x9E3779B9u) << 32;
}

// the reference's order: one stream, consumed in sequence
struct SerialDraws {
    Rng r;
    __device__ __forceinline__ uint64_t neg() { return r.next(); }
    __device__ __forceinline__ uint64_t mid() { return r.next(); }
    __device__ __forceinline__ uint64_t jitter(int, int) { return r.next(); }
};
// the counter-based draws of the fast mode
struct CounterDraws {
    uint32_t key;
    int p = 0, t = 0;
    __device__ __forceinline__ explicit CounterDraws(uint32_t k) : key(k) {}
    __device__ __forceinline__ uint64_t neg() { return counter_draw(key, p++); }
    __device__ __forceinline__ uint64_t mid() { return counter_draw(key, kMidDraw + t++); }
    __device__ __forceinline__ uint64_t jitter(int pi, int d) { return counter_draw(key, kJitterDraw + 64 * pi + d); }
};

// ---------------------------------------------------------------------------------------------- steps
// apply_step (src/layout.cpp:90-116): optional lazy Adam, step = alpha * g, clip per coordinate at 4 alpha or by
// norm. The sinks differ in how y += step lands.
template <int D>
__device__ __forceinline__ void make_step(const SgdDev& c, const float* g, float alpha, int64_t node, int dim,
                                          float* step) {
    if (c.optimizer == 1) {
        const int32_t t = atomicAdd(&c.adam_t[node], 1) + 1;
        const float c1 = 1.0f - powf(c.beta1, (float)t), c2 = 1.0f - powf(c.beta2, (float)t);
        float* m = c.adam_m + node * dim;
        float* v = c.adam_v + node * dim;
        for (int d = 0; d < dim; ++d) {
            // the moments are read from L2 (__ldcg): other SMs write them during the epoch, and an L1 copy would
            // hold the value this SM saw first (lost updates, measured as 11 points of purity on a 600-node layout)
            const float md = c.beta1 * __ldcg(&m[d]) + (1.0f - c.beta1) * g[d];
            const float vd = c.beta2 * __ldcg(&v[d]) + (1.0f - c.beta2) * g[d] * g[d];
            m[d] = md; v[d] = vd;
            step[d] = alpha * (md / c1) / (sqrtf(vd / c2) + 1e-7f);
        }
    } else {
#pragma unroll
        for (int d = 0; d < D; ++d)
            if (d < dim) step[d] = __fmul_rn(alpha, g[d]);
    }
    const float cap = 4.0f * alpha;
    if (c.clip_mode == 1) {
        float n2 = 0.0f;
        for (int d = 0; d < dim; ++d) n2 = __fadd_rn(n2, __fmul_rn(step[d], step[d]));
        if (n2 > cap * cap) {
            const float f = cap / sqrtf(n2);
            for (int d = 0; d < dim; ++d) step[d] *= f;
        }
    } else {
#pragma unroll
        for (int d = 0; d < D; ++d)
            if (d < dim) step[d] = step[d] > cap ? cap : (step[d] < -cap ? -cap : step[d]);
    }
}

struct HogwildSink {
    template <int D>
    __device__ __forceinline__ void apply(const SgdDev& c, int64_t node, const float* g, float alpha, int dim) const {
        float step[D];
        make_step<D>(c, g, alpha, node, dim, step);
        if (D == 2) atomicAdd(reinterpret_cast<float2*>(c.Y) + node, make_float2(step[0], step[1]));
        else for (int d = 0; d < dim; ++d) atomicAdd(&c.Y[node * dim + d], step[d]);
    }
};

struct FixedSink {
    unsigned long long* delta;
    template <int D>
    __device__ __forceinline__ void apply(const SgdDev& c, int64_t node, const float* g, float alpha, int dim) const {
        float step[D];
        make_step<D>(c, g, alpha, node, dim, step);
        for (int d = 0; d < dim; ++d)
            atomicAdd(&delta[node * dim + d], (unsigned long long)llrint((double)step[d] * kFix));
    }
};

struct NullSink {
    template <int D>
    __device__ __forceinline__ void apply(const SgdDev&, int64_t, const float*, float, int) const {}
};

// record of the draws (schedule test hook)
struct Rec {
    int32_t* negs;          // at neg_off[i]
    const int64_t* neg_off;
    int64_t negs_cap;
    int32_t* mid;           // per edge: -1 no mid-range draw succeeded, -2 the partner was the head, else the partner
};

// the head's own step, applied to its registers (the thread or group that owns the row holds its position)
template <int D>
__device__ __forceinline__ void local_step(const SgdDev& c, float* yu, const float* g, float alpha, int64_t node,
                                           int dim) {
    float step[D];
    make_step<D>(c, g, alpha, node, dim, step);
#pragma unroll
    for (int d = 0; d < D; ++d)
        if (d < dim) yu[d] += step[d];
}

// the mid-range partner of src/layout.cpp:226-249, after the mid-range uniform succeeded
template <class Draws>
__device__ __forceinline__ int32_t mid_partner(const SgdDev& c, int32_t u, int32_t v, Draws& dr) {
    int32_t w = v;
    if (c.jump_indptr) {
        const int L = c.walk_lens ? c.walk_lens[v] : c.walk_len;
        for (int h = 0; h < L; ++h) {
            const int32_t js = c.jump_indptr[w], je = c.jump_indptr[w + 1];
            if (je > js && uniform_of(dr.mid()) < c.mid_jump) {
                w = c.jump_indices[js + (int32_t)below_of(dr.mid(), (uint32_t)(je - js))];
            } else {
                const int32_t s0 = c.indptr[w], e0 = c.indptr[w + 1];
                if (e0 <= s0) break;
                w = c.indices[s0 + (int32_t)below_of(dr.mid(), (uint32_t)(e0 - s0))];
            }
        }
    } else if (c.mid_pairs) {
        w = c.mid_pairs[(int64_t)u * c.n_mid + below_of(dr.mid(), (uint32_t)c.n_mid)];
    } else {
        const int L = c.walk_lens ? c.walk_lens[v] : c.walk_len;
        for (int h = 0; h < L; ++h) {
            const int32_t s0 = c.indptr[w], e0 = c.indptr[w + 1];
            if (e0 <= s0) break;
            w = c.indices[s0 + (int32_t)below_of(dr.mid(), (uint32_t)(e0 - s0))];
        }
    }
    return w;
}

// repulsion coefficient of a negative at squared distance dd > 0 (src/layout.cpp:166-179)
__device__ __forceinline__ float repulsion_coeff(const SgdDev& c, float dd, int32_t u) {
    if (c.kernel == 0) {
        if (c.node_b && c.rep_coupled) {
            const float b_u = c.node_b[u];
            const float pw = powf(dd, b_u);
            return 2.0f * b_u * c.repulsion_strength / ((0.001f + dd) * (c.a * pw + 1.0f));
        }
        const float pw = c.rep_b_is_one ? dd : powf(dd, c.rep_b);
        return c.two_b / ((0.001f + dd) * (c.rep_a * pw + 1.0f));
    }
    if (c.kernel == 1) {
        const float q = expf(-c.a * dd);
        return c.repulsion_strength * 2.0f * c.a * q / fmaxf(1.0f - q, 1e-3f);
    }
    if (c.kernel == 2) {
        const float r = sqrtf(dd); const float q = 1.0f / coshf(c.a * r);
        return c.repulsion_strength * c.a * q * tanhf(c.a * r) / (r * fmaxf(1.0f - q, 1e-3f));
    }
    const float th = fmaxf(tanhf(c.a * dd), 1e-3f);
    return c.repulsion_strength * 2.0f * c.a * (1.0f - th * th) / th;
}

// attraction coefficient at squared distance d2 > 0 (src/layout.cpp:149-157); pw_v = d2^b_uv
__device__ __forceinline__ float attraction_coeff(const SgdDev& c, float d2, float b_uv, float pw_v) {
    const float s = -c.exaggeration;
    if (c.kernel == 0) return s * 2.0f * c.a * b_uv * pw_v / (d2 * (c.a * pw_v + 1.0f));
    if (c.kernel == 1) return s * 2.0f * c.a;
    if (c.kernel == 2) { const float dd = sqrtf(d2); return s * c.a * tanhf(c.a * dd) / dd; }
    return s * 2.0f * c.a * (1.0f + tanhf(c.a * d2));
}

// ---------------------------------------------------------------------------------------------- one sample, in sequence
// One sampled edge of epoch_worker (src/layout.cpp:136-274), draws in the reference's order from `dr`, n_neg from
// the schedule. yu: the head's current position (updated in place when it moves); Y: where the other rows are read.
template <int D, class Sink, class Draws>
__device__ __forceinline__ void process_edge(const SgdDev& c, int64_t i, int n_neg, float alpha, float mid_w,
                                             Draws& dr, const Sink& sink, const Rec* rec, float* yu, const float* Y) {
    const int dim = D == 0 ? c.dim : D;
    constexpr int DM = D == 0 ? kMaxDim : D;
    const int32_t u = c.head[i], v = c.tail[i];
    float diff[DM], gu[DM], gk[DM];
    const bool move_u = u >= c.n_fixed, move_v = v >= c.n_fixed;
    float d2 = 0.0f;
    for (int d = 0; d < dim; ++d) {
        diff[d] = yu[d] - Y[(int64_t)v * dim + d];
        d2 = __fadd_rn(d2, __fmul_rn(diff[d], diff[d]));
        gu[d] = 0.0f;
    }
    const float b_uv = c.node_b ? 0.5f * (c.node_b[u] + c.node_b[v]) : c.b;
    const float pw_v = (c.b_is_one && !c.node_b) ? d2 : (d2 > 0.0f ? powf(d2, b_uv) : 0.0f);
    const float jit = 1e-3f / fmaxf(alpha, 1e-6f);
    int64_t rec_at = rec ? rec->neg_off[i] : 0;
    if (c.loss == 0) {
        if (d2 > 0.0f) {
            const float coeff = attraction_coeff(c, d2, b_uv, pw_v);
            for (int d = 0; d < dim; ++d) { const float g = coeff * diff[d]; gu[d] += g; gk[d] = -g; }
            if (move_v) sink.template apply<DM>(c, v, gk, alpha, dim);
        }
        for (int p = 0; p < n_neg; ++p) {
            const int32_t k = (int32_t)below_of(dr.neg(), (uint32_t)c.n);
            if (rec) { if (rec_at < rec->negs_cap) rec->negs[rec_at] = k; ++rec_at; }
            if (k == u) continue;
            float dd = 0.0f;
            for (int d = 0; d < dim; ++d) {
                diff[d] = yu[d] - Y[(int64_t)k * dim + d];
                dd = __fadd_rn(dd, __fmul_rn(diff[d], diff[d]));
            }
            if (dd > 0.0f) {
                const float coeff = repulsion_coeff(c, dd, u);
                for (int d = 0; d < dim; ++d) gu[d] += coeff * diff[d];
            } else {
                for (int d = 0; d < dim; ++d) gu[d] += (uniform_of(dr.jitter(p, d)) - 0.5f) * jit;
            }
        }
    } else {
        // InfoNCE (src/layout.cpp:185-223); the negatives are moved too
        int32_t negs[64]; float qk[64];
        const float q_v = 1.0f / (1.0f + c.a * pw_v);
        float Z = q_v;
        for (int p = 0; p < c.m_neg; ++p) {
            int32_t k = (int32_t)below_of(dr.neg(), (uint32_t)c.n);
            if (k == u) k = (int32_t)((k + 1) % c.n);
            negs[p] = k;
            if (rec) { if (rec_at < rec->negs_cap) rec->negs[rec_at] = k; ++rec_at; }
            float dd = 0.0f;
            for (int d = 0; d < dim; ++d) { const float t = yu[d] - Y[(int64_t)k * dim + d]; dd = __fadd_rn(dd, __fmul_rn(t, t)); }
            const float pw = c.b_is_one ? dd : (dd > 0.0f ? powf(dd, c.b) : 0.0f);
            qk[p] = 1.0f / (1.0f + c.a * pw);
            Z += qk[p];
        }
        const float w_v = q_v / Z;
        if (d2 > 0.0f) {
            const float coeff = -c.exaggeration * (1.0f - w_v) * c.two_ab * pw_v / (d2 * (c.a * pw_v + 1.0f));
            for (int d = 0; d < dim; ++d) { const float g = coeff * diff[d]; gu[d] += g; gk[d] = -g; }
            if (move_v) sink.template apply<DM>(c, v, gk, alpha, dim);
        }
        for (int p = 0; p < c.m_neg; ++p) {
            const int32_t k = negs[p];
            float dd = 0.0f;
            for (int d = 0; d < dim; ++d) { diff[d] = yu[d] - Y[(int64_t)k * dim + d]; dd = __fadd_rn(dd, __fmul_rn(diff[d], diff[d])); }
            if (dd <= 0.0f) {
                for (int d = 0; d < dim; ++d) gu[d] += (uniform_of(dr.jitter(p, d)) - 0.5f) * jit;
                continue;
            }
            const float pw = c.b_is_one ? dd : powf(dd, c.b);
            const float w_k = qk[p] / Z;
            const float coeff = c.repulsion_strength * w_k * c.two_ab * pw / (dd * (c.a * pw + 1.0f));
            for (int d = 0; d < dim; ++d) { const float g = coeff * diff[d]; gu[d] += g; gk[d] = -g; }
            if (k >= c.n_fixed) sink.template apply<DM>(c, k, gk, alpha, dim);
        }
    }
    // mid-range partner (src/layout.cpp:225-255)
    if (mid_w > 0.0f && uniform_of(dr.mid()) < c.mid_rate) {
        const int32_t w = mid_partner(c, u, v, dr);
        if (rec) rec->mid[i] = (w != u) ? w : -2;
        if (w != u) {
            for (int d = 0; d < dim; ++d) {
                const float g = -mid_w * (yu[d] - Y[(int64_t)w * dim + d]);
                gu[d] += g; gk[d] = -g;
            }
            if (w >= c.n_fixed) sink.template apply<DM>(c, w, gk, alpha, dim);
        }
    }
    if (move_u) local_step<DM>(c, yu, gu, alpha, u, dim);
}

// Schedule of one sample (src/layout.cpp:135, 160-163, 184; InfoNCE :221-222): n_neg, or -1 when the edge is not
// sampled this epoch; advances eons / eonns.
__device__ __forceinline__ int schedule_edge(const SgdDev& c, int64_t i, float fepoch) {
    const float eon = c.eons[i];
    if (eon > fepoch) return -1;
    const float eps = c.eps[i];
    c.eons[i] = __fadd_rn(eon, eps);
    if (c.loss == 0) {
        const float epn = eps / c.negative_sample_rate;
        const float eonn = c.eonns[i];
        const int n_neg = (int)((fepoch - eonn) / epn);
        c.eonns[i] = __fadd_rn(eonn, __fmul_rn((float)n_neg, epn));
        return n_neg > 0 ? n_neg : 0;
    }
    c.eonns[i] = fepoch;
    return c.m_neg;
}

template <int D>
__device__ __forceinline__ void load_row(const float* Y, int64_t u, int dim, float* yu) {
#pragma unroll
    for (int d = 0; d < (D == 0 ? kMaxDim : D); ++d)
        if (d < dim) yu[d] = Y[u * dim + d];
}

// the head's whole displacement of the row, on top of what the other rows added to it meanwhile
template <int D>
__device__ __forceinline__ void flush_head(const SgdDev& c, int64_t u, int dim, const float* yu, const float* y0) {
    if (D == 2) atomicAdd(reinterpret_cast<float2*>(c.Y) + u, make_float2(yu[0] - y0[0], yu[1] - y0[1]));
    else for (int d = 0; d < dim; ++d) atomicAdd(&c.Y[u * dim + d], yu[d] - y0[d]);
}

// ---------------------------------------------------------------------------------------------- counter mode kernels
// The counter mode's fast path (loss 0, dim 2 or 3, edges sorted by head) runs an epoch as three kernels (the split
// form below): the epoch's sampled edges as a bit set with per-chunk counts, the counts' prefix sums, and the sample
// pass, in which each thread walks an equal share of the samples in edge order. A sample first gathers what it
// reads (tail, draws, the positions of its tail and negatives), then computes.
constexpr int kNegBatch = 6;   // n_neg is 4-6 for almost every sample (its long-run mean is the rate, 5)

template <int D>
__device__ __forceinline__ void load_pos(const float* __restrict__ Y, int64_t k, float* out) {
    if constexpr (D == 2) {
        const float2 q = reinterpret_cast<const float2*>(Y)[k];
        out[0] = q.x; out[1] = q.y;
    } else {
#pragma unroll
        for (int d = 0; d < D; ++d) out[d] = Y[k * D + d];
    }
}

// what a sample reads before it computes
template <int D>
struct Fetched {
    int64_t i;
    int nn;
    int32_t v;
    uint32_t key;
    float yv[D];
    int32_t k[kNegBatch];
    float yk[kNegBatch][D];
};

// repulsion of negative k at position yk (dd = |yu - yk|^2): the common path (kernel 0, no per-node b) evaluates
// d^(2 rep_b) through log2 / exp2 (or directly when rep_b = 1) with a fast division (a few ulp)
template <int D, bool FAST, bool REP1>
__device__ __forceinline__ void add_negative(const SgdDev& c, int64_t u, const float* yu, const float* yk,
                                             uint32_t key, int p, float jit, float* gu) {
    float diff[D], dd = 0.0f;
#pragma unroll
    for (int d = 0; d < D; ++d) { diff[d] = yu[d] - yk[d]; dd = __fadd_rn(dd, __fmul_rn(diff[d], diff[d])); }
    if (dd > 0.0f) {
        float coeff;
        if constexpr (FAST) {
            const float pw = REP1 ? dd : exp2f(c.rep_b * __log2f(dd));
            coeff = __fdividef(c.two_b, (0.001f + dd) * (c.rep_a * pw + 1.0f));
        } else {
            coeff = repulsion_coeff(c, dd, (int32_t)u);
        }
#pragma unroll
        for (int d = 0; d < D; ++d) gu[d] += coeff * diff[d];
    } else {
#pragma unroll
        for (int d = 0; d < D; ++d) gu[d] += (uniform_of(counter_draw(key, kJitterDraw + 64 * p + d)) - 0.5f) * jit;
    }
}

// One sample: the steps of epoch_worker (src/layout.cpp:145-256) in the reference's order (attraction and the
// tail's step, negatives, mid-range partner, the head's step) with counter draws.
template <int D, bool FAST, bool REP1, bool B1>
__device__ __forceinline__ void compute_sample(const SgdDev& c, int64_t u, const Fetched<D>& f, float alpha,
                                               float mid_w, float jit, float* yu) {
    float gu[D];
#pragma unroll
    for (int d = 0; d < D; ++d) gu[d] = 0.0f;
    {
        float diff[D], d2 = 0.0f;
#pragma unroll
        for (int d = 0; d < D; ++d) { diff[d] = yu[d] - f.yv[d]; d2 = __fadd_rn(d2, __fmul_rn(diff[d], diff[d])); }
        if (d2 > 0.0f) {
            float coeff;
            if constexpr (FAST) {
                const float pw = B1 ? d2 : exp2f(c.b * __log2f(d2));
                coeff = __fdividef(-c.exaggeration * 2.0f * c.a * c.b * pw, d2 * (c.a * pw + 1.0f));
            } else {
                const float b_uv = c.node_b ? 0.5f * (c.node_b[u] + c.node_b[f.v]) : c.b;
                const float pw_v = (c.b_is_one && !c.node_b) ? d2 : powf(d2, b_uv);
                coeff = attraction_coeff(c, d2, b_uv, pw_v);
            }
            float gk[D];
#pragma unroll
            for (int d = 0; d < D; ++d) { const float g = coeff * diff[d]; gu[d] += g; gk[d] = -g; }
            if (f.v >= c.n_fixed) HogwildSink().template apply<D>(c, f.v, gk, alpha, D);
        }
    }
#pragma unroll
    for (int q = 0; q < kNegBatch; ++q)
        if (f.k[q] >= 0 && f.k[q] != (int32_t)u) add_negative<D, FAST, REP1>(c, u, yu, f.yk[q], f.key, q, jit, gu);
    for (int p = kNegBatch; p < f.nn; ++p) {   // rare: more negatives than one batch
        const int32_t k = (int32_t)below_of(counter_draw(f.key, p), (uint32_t)c.n);
        if (k == (int32_t)u) continue;
        float yk[D];
        load_pos<D>(c.Y, k, yk);
        add_negative<D, FAST, REP1>(c, u, yu, yk, f.key, p, jit, gu);
    }
    if (mid_w > 0.0f) {
        CounterDraws dr(f.key);
        if (uniform_of(dr.mid()) < c.mid_rate) {
            const int32_t w = mid_partner(c, (int32_t)u, f.v, dr);
            if (w != (int32_t)u) {
                float yw[D], gk[D];
                load_pos<D>(c.Y, w, yw);
#pragma unroll
                for (int d = 0; d < D; ++d) { const float g = -mid_w * (yu[d] - yw[d]); gu[d] += g; gk[d] = -g; }
                if (w >= c.n_fixed) HogwildSink().template apply<D>(c, w, gk, alpha, D);
            }
        }
    }
    if (u >= c.n_fixed) local_step<D>(c, yu, gu, alpha, u, D);
}

// One sample of the split form: the schedule update of its edge (eons / eonns as schedule_edge), then the sample's
// reads and its steps. The reads that do not depend on one another (the edge's schedule state and tail) are issued
// together, then the positions of the tail and the negatives.
template <int D, bool FAST, bool REP1, bool B1>
__device__ __forceinline__ void range_sample(const SgdDev& c, int64_t u, int64_t i, int epoch, float fepoch,
                                             float alpha, float mid_w, float jit, float* yu) {
    const float2 eo = c.eo[i];
    const EdgeRO te = c.te[i];
    const float eon = eo.x, eonn = eo.y, eps = te.eps;
    const int32_t v = te.tail;
    const uint32_t key = sample_key(stream_seed(c.seed, epoch, (uint64_t)i));
    const float epn = eps / c.negative_sample_rate;
    int nn = (int)((fepoch - eonn) / epn);
    c.eo[i] = make_float2(__fadd_rn(eon, eps), __fadd_rn(eonn, __fmul_rn((float)nn, epn)));
    nn = nn > 0 ? nn : 0;
    Fetched<D> f;
    f.i = i;
    f.nn = nn;
    f.v = v;
    f.key = key;
    load_pos<D>(c.Y, v, f.yv);
#pragma unroll
    for (int q = 0; q < kNegBatch; ++q) {
        f.k[q] = q < nn ? (int32_t)below_of(counter_draw(key, q), (uint32_t)c.n) : -1;
        if (f.k[q] >= 0) load_pos<D>(c.Y, f.k[q], f.yk[q]);
    }
    compute_sample<D, FAST, REP1, B1>(c, u, f, alpha, mid_w, jit, yu);
}

// ---------------------------------------------------------------------------------------------- split form
// The sample pass with the samples split evenly: thread t of T takes the samples of ranks [t S / T, (t + 1) S / T)
// of the epoch's S sampled edges, in edge order, one sample per trip of its loop (so a warp's lanes stay converged
// and carry equal counts). The edges are sorted by head, so a thread walks consecutive edges and a head's steps
// follow one another in its registers as in the reference's loop; the head's displacement lands with one atomic
// when the thread leaves the row (a row cut between two threads is held by both, and each lands its own). The
// schedule update of a sampled edge (eons / eonns) happens once, in the sample that consumes it. The sampled set is
// one bit per edge (eons <= epoch, the test of src/layout.cpp:135), counted per chunk of kChunkWords words, so a
// thread finds its first sample by a binary search of the chunks' prefix sums and a walk of one chunk.
constexpr int kChunkWords = 64;   // 2048 edges per chunk
constexpr int kSplitBlock = 128;  // threads per block of the sample pass

// the chunks' exclusive prefix sums and, in cpre[n], the total: one block, each thread a run of consecutive
// chunks (summed, then a block scan of the run sums, then the run written), so the scan waits on one round of loads
// instead of one per 1024 chunks
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) chunk_scan_kernel(const int32_t* __restrict__ count, int64_t n,
                                                                   int64_t* __restrict__ cpre) {
    __shared__ int64_t wsum[kScanThreads / 32];
    const int64_t per = (n + blockDim.x - 1) / blockDim.x;
    const int64_t b = (int64_t)threadIdx.x * per, e = b + per < n ? b + per : n;
    int64_t run = 0;
    for (int64_t i = b; i < e; ++i) run += count[i];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        wsum[lane] = w;
    }
    __syncthreads();
    int64_t acc = x - run + (warp > 0 ? wsum[warp - 1] : 0);
    for (int64_t i = b; i < e; ++i) { cpre[i] = acc; acc += count[i]; }
    if (threadIdx.x == blockDim.x - 1) cpre[n] = acc;
}

// the bit set (bit i of bits[i / 32] set when edge i is sampled), one warp ballot per 32 edges and one warp per
// chunk, and the chunk's count of sampled edges; words past the last edge are written as 0, so every chunk is whole
__global__ void __launch_bounds__(kThreads) chunk_bits_kernel(const float2* __restrict__ eo, int64_t E, float fepoch,
                                                              int64_t n_chunks, uint32_t* __restrict__ bits,
                                                              int32_t* __restrict__ count) {
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    for (int64_t ch = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; ch < n_chunks; ch += warps) {
        const int64_t base = ch * (kChunkWords * 32);
        int total = 0;
#pragma unroll 1
        for (int w0 = 0; w0 < kChunkWords; w0 += 8) {
            bool smp[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int64_t i = base + (int64_t)(w0 + q) * 32 + lane;
                smp[q] = i < E && !(eo[i].x > fepoch);
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const uint32_t m = __ballot_sync(0xffffffffu, smp[q]);
                total += __popc(m);
                if (lane == q) bits[ch * kChunkWords + w0 + q] = m;
            }
        }
        if (lane == 0) count[ch] = total;
    }
}

template <int D, bool FAST, bool REP1, bool B1>
__global__ void __launch_bounds__(kThreads, 4) hogwild_split_kernel(SgdDev c, const int64_t* __restrict__ eptr,
                                                                    const uint32_t* __restrict__ bits,
                                                                    const int64_t* __restrict__ cpre, int64_t n_chunks,
                                                                    int epoch, float alpha, float mid_w) {
    const float fepoch = (float)epoch;
    const float jit = 1e-3f / fmaxf(alpha, 1e-6f);
    const int64_t T = (int64_t)gridDim.x * blockDim.x;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t S = cpre[n_chunks];
    const int64_t r0 = t * S / T, r1 = (t + 1) * S / T;
    if (r0 >= r1) return;
    // the chunk holding the sample of rank r0: the last chunk whose prefix is <= r0 (it has a sample past r0)
    int64_t lo = 0, hi = n_chunks;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (cpre[mid] <= r0) lo = mid; else hi = mid;
    }
    int64_t k = r0 - cpre[lo];
    int64_t w = lo * kChunkWords;
    const int64_t w_end = n_chunks * kChunkWords;
    uint32_t m = bits[w];
    while (k >= __popc(m) && w + 1 < w_end) { k -= __popc(m); m = bits[++w]; }
    for (int j = 0; j < (int)k; ++j) m &= m - 1u;
    if (m == 0u) return;   // counts and bits disagree: cannot happen, both come from one ballot
    int64_t pos = w * 32 + __ffs(m) - 1;
    const int64_t end = c.n_edges;
    int64_t u = c.head[pos], row_end = eptr[u + 1];
    float yu[D], y0[D];
    bool have = false;
    for (int64_t left = r1 - r0; left > 0; --left) {
        int64_t i = -1;
        while (pos < end) {
            const uint32_t mm = bits[pos >> 5] & (0xffffffffu << (pos & 31));
            if (mm) { i = (pos & ~(int64_t)31) + __ffs(mm) - 1; pos = i + 1; break; }
            pos = (pos | 31) + 1;
        }
        if (i < 0 || i >= end) break;
        if (i >= row_end) {
            if (have && u >= c.n_fixed) flush_head<D>(c, u, D, yu, y0);
            have = false;
            do { ++u; row_end = eptr[u + 1]; } while (i >= row_end);
        }
        if (!have) {
            load_pos<D>(c.Y, u, yu);
#pragma unroll
            for (int d = 0; d < D; ++d) y0[d] = yu[d];
            have = true;
        }
        range_sample<D, FAST, REP1, B1>(c, u, i, epoch, fepoch, alpha, mid_w, jit, yu);
    }
    if (have && u >= c.n_fixed) flush_head<D>(c, u, D, yu, y0);
}

// The split form's packed copies of the edge fields, made at the start of a call and (eons, eonns) written back at
// its end; a sample then reads two records instead of four arrays and writes one.
__global__ void pack_edges_kernel(const float* __restrict__ eons, const float* __restrict__ eonns,
                                  const int32_t* __restrict__ tail, const float* __restrict__ eps, int64_t E,
                                  float2* __restrict__ eo, EdgeRO* __restrict__ te) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        eo[i] = make_float2(eons[i], eonns[i]);
        te[i] = EdgeRO{tail[i], eps[i]};
    }
}

__global__ void unpack_edges_kernel(const float2* __restrict__ eo, int64_t E, float* __restrict__ eons,
                                    float* __restrict__ eonns) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < E; i += (int64_t)gridDim.x * blockDim.x) {
        const float2 v = eo[i];
        eons[i] = v.x;
        eonns[i] = v.y;
    }
}

// Blocks of a kernel the device holds at once (the SM count times the blocks one SM holds), asked once per kernel.
// The split form's grid stays within it, so that no block waits for a second wave.
template <typename K>
int resident_blocks(K kernel) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> known;
    std::lock_guard<std::mutex> lock(mu);
    const auto it = known.find(reinterpret_cast<const void*>(kernel));
    if (it != known.end()) return it->second;
    int dev = 0, sms = 0, per_sm = 0;
    MGB_CUDA(cudaGetDevice(&dev));
    MGB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0));
    const int count = std::max(1, sms * per_sm);
    known.emplace(reinterpret_cast<const void*>(kernel), count);
    return count;
}

int env_int(const char* name, int dflt);

template <int D, bool FAST>
void launch_split(const SgdDev& c, int64_t threads, const int64_t* eptr, uint32_t* bits, int32_t* count, int64_t* cpre,
                  int64_t n_chunks, int epoch, float alpha, float mid_w, cudaStream_t s) {
    chunk_bits_kernel<<<blocks_for(n_chunks * 32, kThreads, 8), kThreads, 0, s>>>(c.eo, c.n_edges, (float)epoch,
                                                                                  n_chunks, bits, count);
    MGB_LAUNCH_CHECK();
    chunk_scan_kernel<<<1, kScanThreads, 0, s>>>(count, n_chunks, cpre);
    MGB_LAUNCH_CHECK();
    const bool rep1 = FAST && c.rep_b_is_one, b1 = FAST && c.b_is_one;
    auto kernel = rep1 && b1 ? hogwild_split_kernel<D, FAST, true, true>
                : rep1       ? hogwild_split_kernel<D, FAST, true, false>
                : b1         ? hogwild_split_kernel<D, FAST, false, true>
                             : hogwild_split_kernel<D, FAST, false, false>;
    // blocks of 128 threads (0.439 ms per epoch at 1M points against 0.449 with 256: 640 blocks spread more evenly
    // over the SMs than 320); few threads (small layouts): blocks of fewer threads, so that they reach every SM.
    // MGB_SGD_BLOCK sets another block size.
    int tpb = std::min(kThreads, std::max(32, env_int("MGB_SGD_BLOCK", kSplitBlock) / 32 * 32));
    if (threads < (int64_t)kNumSMs * tpb)
        tpb = (int)std::min<int64_t>(kThreads, std::max<int64_t>(32, ((threads + kNumSMs - 1) / kNumSMs + 31) / 32 * 32));
    int64_t blocks = std::max<int64_t>(1, (threads + tpb - 1) / tpb);
    if (tpb == kThreads) blocks = std::min<int64_t>(blocks, resident_blocks(kernel));
    else blocks = std::min<int64_t>(blocks, (int64_t)resident_blocks(kernel) * (kThreads / tpb));
    kernel<<<(int)blocks, tpb, 0, s>>>(c, eptr, bits, cpre, n_chunks, epoch, alpha, mid_w);
}

// Row kernel (any dim, any loss): one thread owns a head row and walks it in order with counter draws.
template <int D>
__global__ void __launch_bounds__(kThreads) hogwild_rows_kernel(SgdDev c, const int64_t* __restrict__ eptr, int epoch,
                                                                float alpha, float mid_w) {
    const int dim = D == 0 ? c.dim : D;
    constexpr int DM = D == 0 ? kMaxDim : D;
    const float fepoch = (float)epoch;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < c.n; u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e0 = eptr[u], e1 = eptr[u + 1];
        float yu[DM], y0[DM];
        bool any = false;
        for (int64_t i = e0; i < e1; ++i) {
            const int n_neg = schedule_edge(c, i, fepoch);
            if (n_neg < 0) continue;
            if (!any) { load_row<D>(c.Y, u, dim, yu); for (int d = 0; d < dim; ++d) y0[d] = yu[d]; any = true; }
            CounterDraws dr(sample_key(stream_seed(c.seed, epoch, (uint64_t)i)));
            process_edge<D>(c, i, n_neg, alpha, mid_w, dr, HogwildSink(), nullptr, yu, c.Y);
        }
        if (any && u >= c.n_fixed) flush_head<D>(c, u, dim, yu, y0);
    }
}

// Edge kernel (edges not sorted by head): one thread per edge; the head's step lands with an atomic.
template <int D>
__global__ void __launch_bounds__(kThreads) hogwild_edges_kernel(SgdDev c, int epoch, float alpha, float mid_w) {
    const int dim = D == 0 ? c.dim : D;
    constexpr int DM = D == 0 ? kMaxDim : D;
    const float fepoch = (float)epoch;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c.n_edges; i += (int64_t)gridDim.x * blockDim.x) {
        const int n_neg = schedule_edge(c, i, fepoch);
        if (n_neg < 0) continue;
        const int64_t u = c.head[i];
        float yu[DM], y0[DM];
        load_row<D>(c.Y, u, dim, yu);
        for (int d = 0; d < dim; ++d) y0[d] = yu[d];
        CounterDraws dr(sample_key(stream_seed(c.seed, epoch, (uint64_t)i)));
        process_edge<D>(c, i, n_neg, alpha, mid_w, dr, HogwildSink(), nullptr, yu, c.Y);
        if (u >= c.n_fixed) flush_head<D>(c, u, dim, yu, y0);
    }
}

// ---------------------------------------------------------------------------------------------- serial mode kernels
// phase 1: the schedule of the epoch (parallel); cnt[i] = n_neg or -1
__global__ void serial_schedule_kernel(SgdDev c, int epoch, int32_t* __restrict__ cnt) {
    const float fepoch = (float)epoch;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c.n_edges; i += (int64_t)gridDim.x * blockDim.x)
        cnt[i] = schedule_edge(c, i, fepoch);
}

// phase 2: one thread walks the sampled edges in order through the epoch's single stream (seed tid 0) and records
// the generator state at the start of each sampled edge, consuming the draws of each sample as the reference does:
// n_neg (or m_neg) below() calls, then with a mid-range weight one uniform() and, on success, the partner draws.
__global__ void serial_chain_kernel(SgdDev c, int epoch, float mid_w, const int32_t* __restrict__ cnt,
                                    uint64_t* __restrict__ state) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    SerialDraws dr{Rng(stream_seed(c.seed, epoch, 0))};
    for (int64_t i = 0; i < c.n_edges; ++i) {
        const int k = cnt[i];
        if (k < 0) continue;
        state[i] = dr.r.s;
        for (int p = 0; p < k; ++p) dr.r.next();
        if (mid_w > 0.0f && uniform_of(dr.mid()) < c.mid_rate) mid_partner(c, c.head[i], c.tail[i], dr);
    }
}

// phase 3 (rows), in kSerialPhases sub-steps: sub-step p processes the p-th sampled edge of every head row (the
// last sub-step the rest of the row, in order) from its recorded state, reading every position as committed after
// the previous sub-step; the sub-step's displacements are summed in fixed point and committed before the next.
// Each sub-step's result is a function of its inputs only, and the reads are never older than one sub-step.
constexpr int kSerialPhases = 8;

template <int D>
__global__ void __launch_bounds__(kThreads) serial_rows_kernel(SgdDev c, const int64_t* __restrict__ eptr, int phase,
                                                               float alpha, float mid_w,
                                                               const int32_t* __restrict__ cnt,
                                                               const uint64_t* __restrict__ state,
                                                               unsigned long long* __restrict__ delta) {
    const int dim = D == 0 ? c.dim : D;
    constexpr int DM = D == 0 ? kMaxDim : D;
    const FixedSink sink{delta};
    const bool last = phase == kSerialPhases - 1;
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u < c.n; u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t e0 = eptr[u], e1 = eptr[u + 1];
        float yu[DM], y0[DM];
        bool any = false;
        int seen = 0;
        for (int64_t i = e0; i < e1; ++i) {
            const int k = cnt[i];
            if (k < 0) continue;
            const int idx = seen++;
            if (idx < phase) continue;
            if (!any) { load_row<D>(c.Y, u, dim, yu); for (int d = 0; d < dim; ++d) y0[d] = yu[d]; any = true; }
            SerialDraws dr{Rng(0)};
            dr.r.s = state[i];
            process_edge<D>(c, i, k, alpha, mid_w, dr, sink, nullptr, yu, c.Y);
            if (!last) break;
        }
        if (!any || u < c.n_fixed) continue;
        for (int d = 0; d < dim; ++d)
            atomicAdd(&delta[u * dim + d], (unsigned long long)llrint((double)(yu[d] - y0[d]) * kFix));
    }
}

// phase 3 (edges not sorted by head): one thread per sampled edge against the epoch-start layout
template <int D>
__global__ void __launch_bounds__(kThreads) serial_edges_kernel(SgdDev c, float alpha, float mid_w,
                                                                const int32_t* __restrict__ cnt,
                                                                const uint64_t* __restrict__ state,
                                                                unsigned long long* __restrict__ delta) {
    const int dim = D == 0 ? c.dim : D;
    constexpr int DM = D == 0 ? kMaxDim : D;
    const FixedSink sink{delta};
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c.n_edges; i += (int64_t)gridDim.x * blockDim.x) {
        const int k = cnt[i];
        if (k < 0) continue;
        const int64_t u = c.head[i];
        float yu[DM], y0[DM];
        load_row<D>(c.Y, u, dim, yu);
        for (int d = 0; d < dim; ++d) y0[d] = yu[d];
        SerialDraws dr{Rng(0)};
        dr.r.s = state[i];
        process_edge<D>(c, i, k, alpha, mid_w, dr, sink, nullptr, yu, c.Y);
        if (u < c.n_fixed) continue;
        for (int d = 0; d < dim; ++d)
            atomicAdd(&delta[u * dim + d], (unsigned long long)llrint((double)(yu[d] - y0[d]) * kFix));
    }
}

// phase 4: y += delta * 2^-32, delta = 0
__global__ void commit_kernel(float* __restrict__ Y, unsigned long long* __restrict__ delta, int64_t total) {
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const long long q = (long long)delta[k];
        if (q != 0) {
            Y[k] = (float)((double)Y[k] + (double)q * (1.0 / kFix));
            delta[k] = 0ull;
        }
    }
}

// ---------------------------------------------------------------------------------------------- helpers
// row pointers of an edge list sorted by head: eptr[u] = first edge with head >= u
__global__ void row_ptr_kernel(const int32_t* __restrict__ head, int64_t E, int64_t n, int64_t* __restrict__ eptr) {
    for (int64_t u = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; u <= n; u += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = E;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (head[mid] < u) lo = mid + 1; else hi = mid;
        }
        eptr[u] = lo;
    }
}

__global__ void unsorted_kernel(const int32_t* __restrict__ head, int64_t E, int* __restrict__ flag) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; i < E; i += (int64_t)gridDim.x * blockDim.x)
        if (head[i] < head[i - 1]) { *flag = 1; return; }
}

// schedule hook: the draws of one epoch (no updates)
template <int D>
__global__ void record_kernel(SgdDev c, int epoch, float alpha, float mid_w, const int32_t* __restrict__ cnt,
                              const uint64_t* __restrict__ state, int per_edge, Rec rec) {
    const int dim = D == 0 ? c.dim : D;
    constexpr int DM = D == 0 ? kMaxDim : D;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c.n_edges; i += (int64_t)gridDim.x * blockDim.x) {
        rec.mid[i] = -1;
        const int k = cnt[i];
        if (k < 0) continue;
        float yu[DM];
        load_row<D>(c.Y, c.head[i], dim, yu);
        if (per_edge) {
            CounterDraws dr(sample_key(stream_seed(c.seed, epoch, (uint64_t)i)));
            process_edge<D>(c, i, k, alpha, mid_w, dr, NullSink(), &rec, yu, c.Y);
        } else {
            SerialDraws dr{Rng(0)};
            dr.r.s = state[i];
            process_edge<D>(c, i, k, alpha, mid_w, dr, NullSink(), &rec, yu, c.Y);
        }
    }
}

// exclusive prefix sum of max(cnt, 0) (single block; test hook sizes)
__global__ void offsets_kernel(const int32_t* __restrict__ cnt, int64_t n, int64_t* __restrict__ off, int64_t* total) {
    __shared__ int64_t carry;
    __shared__ int64_t wsum[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t base = 0; base < n; base += blockDim.x) {
        const int64_t i = base + threadIdx.x;
        int64_t v = (i < n && cnt[i] > 0) ? cnt[i] : 0;
        int64_t x = v;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) { const int64_t y = __shfl_up_sync(0xffffffffu, x, o); if (lane >= o) x += y; }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            int64_t w = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) { const int64_t y = __shfl_up_sync(0xffffffffu, w, o); if (lane >= o) w += y; }
            wsum[lane] = w;
        }
        __syncthreads();
        const int64_t incl = x + (warp > 0 ? wsum[warp - 1] : 0);
        if (i < n) off[i] = carry + incl - v;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

// Rows (or edges) in flight at once: at most n / 8 (and at least 64), so that at most about 12 % of the layout
// moves between a row's read of a position and its own write; small layouts otherwise update every row at once
// against stale positions. The reference bounds its hogwild threads for the same reason (one per 4096 edges,
// src/layout.cpp:421). At n = 1M the bound is close to what the device holds resident.
int env_int(const char* name, int dflt) {
    const char* v = std::getenv(name);
    return v && *v ? std::atoi(v) : dflt;
}
int64_t max_in_flight(const SgdDev& c) {
    const int div = std::max(1, env_int("MGB_SGD_INFLIGHT_DIV", 8));
    return std::max<int64_t>(64, c.n / div);
}

// Threads of the split form, each holding one head at a time: n / 4 (n / 8 with Adam, whose per-node moments take
// the concurrent steps of every thread that holds the node: at n / 4 a 600-point Adam layout lost 20 points of
// neighbourhood purity), at most 81,920 (2.2 blocks of 256 per SM).
// Measured on B200 (ms per epoch; 15-NN preservation of the finished layout unchanged within 0.002):
// 1M points 0.485 at 83k threads, 0.51 at 125k, 0.53 at 167k; the 10k-point umap pass 53 ms at
// n / 4, 94 ms at n / 8, 152 ms at n / 16 for 500 epochs. MGB_SGD_INFLIGHT_DIV = k sets n / k instead.
constexpr int64_t kSplitMaxThreads = 81920;
int64_t split_threads(const SgdDev& c) {
    const int div = env_int("MGB_SGD_INFLIGHT_DIV", 0);
    if (div > 0) return std::max<int64_t>(64, c.n / div);
    return std::max<int64_t>(64, std::min<int64_t>(c.n / (c.optimizer == 1 ? 8 : 4), kSplitMaxThreads));
}

template <int D>
void hogwild_epoch(const SgdDev& c, SgdWork& w, const int64_t* eptr, int epoch, float alpha, float mid_w,
                   cudaStream_t s) {
    const int64_t cap = max_in_flight(c);
    if (c.eo && eptr && c.loss == 0 && (D == 2 || D == 3)) {
        const int64_t n_chunks = std::max<int64_t>(1, (c.n_edges + kChunkWords * 32 - 1) / (kChunkWords * 32));
        uint32_t* bits = w.samp.as<uint32_t>();
        int64_t* cpre = reinterpret_cast<int64_t*>(bits + n_chunks * kChunkWords);
        int32_t* count = reinterpret_cast<int32_t*>(cpre + n_chunks + 1);
        constexpr int DD = D == 0 ? 2 : D;
        const int64_t threads = split_threads(c);
        if (c.kernel == 0 && !c.node_b) launch_split<DD, true>(c, threads, eptr, bits, count, cpre, n_chunks, epoch, alpha, mid_w, s);
        else launch_split<DD, false>(c, threads, eptr, bits, count, cpre, n_chunks, epoch, alpha, mid_w, s);
    } else if (eptr) {
        const int blocks = (int)std::min<int64_t>(blocks_for(c.n, kThreads), (cap + kThreads - 1) / kThreads);
        hogwild_rows_kernel<D><<<blocks, kThreads, 0, s>>>(c, eptr, epoch, alpha, mid_w);
    } else {
        const int blocks = (int)std::min<int64_t>(blocks_for(c.n_edges, kThreads), (cap + kThreads - 1) / kThreads);
        hogwild_edges_kernel<D><<<blocks, kThreads, 0, s>>>(c, epoch, alpha, mid_w);
    }
}

template <int D>
void serial_apply(const SgdDev& c, const int64_t* eptr, float alpha, float mid_w, const int32_t* cnt,
                  const uint64_t* st, unsigned long long* delta, cudaStream_t s) {
    const int64_t total = c.n * c.dim;
    if (!eptr) {
        serial_edges_kernel<D><<<blocks_for(c.n_edges, kThreads), kThreads, 0, s>>>(c, alpha, mid_w, cnt, st, delta);
        MGB_LAUNCH_CHECK();
        commit_kernel<<<blocks_for(total, kThreads), kThreads, 0, s>>>(c.Y, delta, total);
        return;
    }
    for (int p = 0; p < kSerialPhases; ++p) {
        serial_rows_kernel<D><<<blocks_for(c.n, kThreads), kThreads, 0, s>>>(c, eptr, p, alpha, mid_w, cnt, st, delta);
        MGB_LAUNCH_CHECK();
        commit_kernel<<<blocks_for(total, kThreads), kThreads, 0, s>>>(c.Y, delta, total);
        if (p + 1 < kSerialPhases) MGB_LAUNCH_CHECK();
    }
}

template <int D>
void record_launch(const SgdDev& c, int epoch, float alpha, float mid_w, const int32_t* cnt, const uint64_t* st,
                   int per_edge, Rec rec, cudaStream_t s) {
    record_kernel<D><<<blocks_for(c.n_edges, kThreads), kThreads, 0, s>>>(c, epoch, alpha, mid_w, cnt, st, per_edge, rec);
}

// row pointers when the edges are sorted by head, else nullptr (edge-parallel kernels)
const int64_t* row_pointers(const SgdDev& c, SgdWork& w, cudaStream_t s) {
    if (c.n_edges == 0) return nullptr;
    int* flag = static_cast<int*>(w.flag.ensure(sizeof(int)));
    MGB_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
    unsorted_kernel<<<blocks_for(c.n_edges, kThreads, 4), kThreads, 0, s>>>(c.head, c.n_edges, flag);
    MGB_LAUNCH_CHECK();
    int h = 0;
    MGB_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    MGB_CUDA(cudaStreamSynchronize(s));
    if (h) return nullptr;
    int64_t* eptr = static_cast<int64_t*>(w.eptr.ensure(sizeof(int64_t) * (c.n + 1)));
    row_ptr_kernel<<<blocks_for(c.n + 1, kThreads, 4), kThreads, 0, s>>>(c.head, c.n_edges, c.n, eptr);
    MGB_LAUNCH_CHECK();
    return eptr;
}

}  // namespace

void sgd_sched(const SgdDev& c, int epoch, int e0, int e1, float alpha0, float alpha1, float mid_w0, float mid_w1,
               float& alpha, float& mid_w) {
    // run_epochs' linear schedule inside a call (src/layout.cpp:284-289)
    const int n_span = std::max(1, e1 - e0);
    const float frac = (float)(epoch - e0) / (float)n_span;
    alpha = alpha0 + (alpha1 - alpha0) * frac;
    mid_w = c.use_mid ? mid_w0 + (mid_w1 - mid_w0) * frac : 0.0f;
}

void sgd_run(SgdDev& c, SgdWork& w, int stream_mode, int e0, int e1, float alpha0, float alpha1, float mid_w0,
             float mid_w1, cudaStream_t s) {
    const int64_t* eptr = row_pointers(c, w, s);
    if (stream_mode == 0) {
        SgdDev cc = c;
        const bool split = eptr && c.loss == 0 && (c.dim == 2 || c.dim == 3) && c.n_edges > 0 && e1 > e0;
        if (split) {
            // the split form's bit per edge (whole chunks of 2048 edges), the chunks' prefix sums and counts, and
            // the packed edge fields
            const size_t n_chunks = (size_t)std::max<int64_t>(1, (c.n_edges + kChunkWords * 32 - 1) / (kChunkWords * 32));
            w.samp.ensure(sizeof(uint32_t) * n_chunks * kChunkWords + sizeof(int64_t) * (n_chunks + 1) +
                          sizeof(int32_t) * n_chunks);
            char* pk = static_cast<char*>(w.pack.ensure((sizeof(float2) + sizeof(EdgeRO)) * (size_t)c.n_edges));
            cc.eo = reinterpret_cast<float2*>(pk);
            cc.te = reinterpret_cast<const EdgeRO*>(pk + sizeof(float2) * (size_t)c.n_edges);
            pack_edges_kernel<<<blocks_for(c.n_edges, kThreads), kThreads, 0, s>>>(
                c.eons, c.eonns, c.tail, c.eps, c.n_edges, cc.eo, const_cast<EdgeRO*>(cc.te));
            MGB_LAUNCH_CHECK();
        }
        for (int e = e0; e < e1; ++e) {
            float alpha, mid_w;
            sgd_sched(cc, e, e0, e1, alpha0, alpha1, mid_w0, mid_w1, alpha, mid_w);
            MGB_DIM_DISPATCH(cc.dim, hogwild_epoch, cc, w, eptr, e, alpha, mid_w, s);
            MGB_LAUNCH_CHECK();
        }
        if (split) {
            unpack_edges_kernel<<<blocks_for(c.n_edges, kThreads), kThreads, 0, s>>>(cc.eo, c.n_edges, c.eons, c.eonns);
            MGB_LAUNCH_CHECK();
        }
        return;
    }
    int32_t* cnt = static_cast<int32_t*>(w.cnt.ensure(sizeof(int32_t) * std::max<int64_t>(c.n_edges, 1)));
    uint64_t* st = static_cast<uint64_t*>(w.state.ensure(sizeof(uint64_t) * std::max<int64_t>(c.n_edges, 1)));
    const int64_t total = c.n * c.dim;
    unsigned long long* delta = static_cast<unsigned long long*>(w.delta.ensure(sizeof(unsigned long long) * total));
    MGB_CUDA(cudaMemsetAsync(delta, 0, sizeof(unsigned long long) * total, s));
    for (int e = e0; e < e1; ++e) {
        float alpha, mid_w;
        sgd_sched(c, e, e0, e1, alpha0, alpha1, mid_w0, mid_w1, alpha, mid_w);
        serial_schedule_kernel<<<blocks_for(c.n_edges, kThreads), kThreads, 0, s>>>(c, e, cnt);
        MGB_LAUNCH_CHECK();
        serial_chain_kernel<<<1, 32, 0, s>>>(c, e, mid_w, cnt, st);
        MGB_LAUNCH_CHECK();
        MGB_DIM_DISPATCH(c.dim, serial_apply, c, eptr, alpha, mid_w, cnt, st, delta, s);
        MGB_LAUNCH_CHECK();
    }
}

void sgd_record(SgdDev& c, SgdWork& w, int stream_mode, int epoch, float alpha, float mid_w, int32_t* n_neg_out,
                int64_t* off_out, int32_t* negs, int64_t negs_cap, int32_t* mid, int64_t* n_negs_dev,
                cudaStream_t s) {
    int32_t* cnt = static_cast<int32_t*>(w.cnt.ensure(sizeof(int32_t) * std::max<int64_t>(c.n_edges, 1)));
    uint64_t* st = static_cast<uint64_t*>(w.state.ensure(sizeof(uint64_t) * std::max<int64_t>(c.n_edges, 1)));
    serial_schedule_kernel<<<blocks_for(c.n_edges, kThreads), kThreads, 0, s>>>(c, epoch, cnt);
    MGB_LAUNCH_CHECK();
    if (stream_mode == 1) {
        serial_chain_kernel<<<1, 32, 0, s>>>(c, epoch, mid_w, cnt, st);
        MGB_LAUNCH_CHECK();
    }
    MGB_CUDA(cudaMemcpyAsync(n_neg_out, cnt, sizeof(int32_t) * c.n_edges, cudaMemcpyDeviceToDevice, s));
    offsets_kernel<<<1, 1024, 0, s>>>(cnt, c.n_edges, off_out, n_negs_dev);
    MGB_LAUNCH_CHECK();
    Rec rec{negs, off_out, negs_cap, mid};
    MGB_DIM_DISPATCH(c.dim, record_launch, c, epoch, alpha, mid_w, cnt, st, stream_mode == 0 ? 1 : 0, rec, s);
    MGB_LAUNCH_CHECK();
}

}  // namespace mgb
