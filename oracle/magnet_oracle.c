/*
 * TEST ORACLE — not part of the product. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load this library, and only as the checker (or the timed CPU baseline), never as the thing measured.
 *
 * A plain-C restatement of the reference's layout pass (kerighan/lib-magnet 3.0.2), written from its
 * behaviour, single-threaded, with the same float evaluation order so that it reproduces the reference
 * bit-exactly where the reference itself is deterministic (n_threads=1). Built with -ffp-contract=off and
 * without -ffast-math, like the reference's plain -O3 x86-64 build (no FMA contraction, IEEE single ops).
 *
 * Pieces and the reference code each one follows:
 *   orc_rng_*           src/rng.hpp:5-28            (splitmix64 seeding, xorshift64*, below, uniform)
 *   orc_sgd_serial      src/layout.cpp:90-116 (apply_step), :118-276 (epoch_worker, hogwild path),
 *                       :281-297 (run_epochs, single-thread path), :343-472 (optimize_layout argument rules)
 *   orc_sgd_owner       src/layout.cpp:118-276 (epoch_worker, OWNER = true), :300-330 (owner epochs), :441-463
 *                       (chunks at the edge quantiles), :31-40 (the owner attraction scale 1.5)
 *   orc_sgd_schedule    the draws epoch_worker makes (src/layout.cpp:123,135,160-166,184,226-249), recorded
 *                       instead of applied; one stream per epoch (tid 0, the n_threads=1 reference), or the
 *                       device fast mode's counter draws (each draw of a sample addressed by edge and index)
 *   orc_smooth_knn      src/graph.cpp:29-78 (one thread: the whole array's mean is one sequential FP64 sum)
 *   orc_fuzzy_union     magnet/knn.py:221-230 (scipy's csr construction, transpose, A + T - A o T, mix), float32
 *   orc_spread / orc_gather  src/fftconv.cpp:24-40 (lagrange_w), :83-123 (spread), :200-229 (gather)
 *   orc_tsne_attraction src/fftrep.cpp:129-177
 *   orc_tsne_step       src/fftrep.cpp:225-266 (one thread: nt = 1 partial sums, i.e. blocks of 1024 rows)
 *   orc_bbox_2d         src/fftrep.cpp:415-434
 *   orc_mid_near_pairs  src/nndescent.cpp:731-759 (mid_near_core, dense rows) with the distance kernels of :35-106
 *   orc_exact_repulsion FP64 all-pairs sumQ and F (the brute force of tests/test_magnet.py:221-231 and
 *                       benchmarks/theory/k16_fft_check.py:9-16), the precision oracle of the FFT pass
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define ORC_MAX_DIM 64

/* ------------------------------------------------------------------ RNG (src/rng.hpp:5-28) */
typedef struct { uint64_t s; } orc_rng;

static void orc_rng_seed(orc_rng* r, uint64_t seed) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    r->s = (z ^ (z >> 31)) | 1ULL;
}
static inline uint64_t orc_rng_next(orc_rng* r) {
    uint64_t s = r->s;
    s ^= s >> 12; s ^= s << 25; s ^= s >> 27;
    r->s = s;
    return s * 0x2545F4914F6CDD1DULL;
}
static inline uint32_t orc_rng_below(orc_rng* r, uint32_t n) {
    return (uint32_t)(((orc_rng_next(r) >> 32) * (uint64_t)n) >> 32);
}
static inline float orc_rng_uniform(orc_rng* r) {
    return (float)(orc_rng_next(r) >> 40) * (1.0f / 16777216.0f);
}
/* epoch stream seed of src/layout.cpp:123 */
static inline uint64_t orc_stream_seed(uint64_t seed, int epoch, uint64_t tid) {
    return seed * 0x9E3779B1ULL + (uint64_t)epoch * 0x85EBCA6BULL + tid * 0xC2B2AE35ULL;
}

/* Draw sources of one sample. Serial: the epoch's single stream, consumed in order (the reference).
 * Counter (the device's fast mode): the sample of edge i in epoch e has the 32-bit key
 * orc_hash32(lo ^ orc_hash32(hi)) of its stream seed orc_stream_seed(seed, e, i); its draw j is
 * orc_hash32(key + j * 0x9E3779B9) in the high 32 bits of a 64-bit draw. Negative p is draw p, the mid-range draws
 * are draws 1024, 1025, ..., and the distance-0 jitter of negative p in dimension q is draw 2048 + 64 p + q. */
typedef struct { orc_rng rng; int counter; uint32_t key; int p, t; } orc_draws;

/* 32-bit integer hash "lowbias32" (C. Wellons, hash-prospector): xorshift-multiply rounds */
static inline uint32_t orc_hash32(uint32_t x) {
    x ^= x >> 16; x *= 0x7feb352du;
    x ^= x >> 15; x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
static inline uint32_t orc_sample_key(uint64_t ss) {
    return orc_hash32((uint32_t)ss ^ orc_hash32((uint32_t)(ss >> 32)));
}
static inline uint64_t orc_counter_draw(uint32_t key, int j) {
    return (uint64_t)orc_hash32(key + (uint32_t)j * 0x9E3779B9u) << 32;
}
static inline uint32_t orc_below_of(uint64_t x, uint32_t n) { return (uint32_t)(((x >> 32) * (uint64_t)n) >> 32); }
static inline float orc_uniform_of(uint64_t x) { return (float)(x >> 40) * (1.0f / 16777216.0f); }
static inline uint64_t orc_draw_neg(orc_draws* d) {
    return d->counter ? orc_counter_draw(d->key, d->p++) : orc_rng_next(&d->rng);
}
static inline uint64_t orc_draw_mid(orc_draws* d) {
    return d->counter ? orc_counter_draw(d->key, 1024 + d->t++) : orc_rng_next(&d->rng);
}
static inline uint64_t orc_draw_jitter(orc_draws* d, int p, int q) {
    return d->counter ? orc_counter_draw(d->key, 2048 + 64 * p + q) : orc_rng_next(&d->rng);
}

/* exported for the RNG known-answer tests */
void orc_rng_stream(uint64_t seed, int64_t count, uint64_t* out) {
    orc_rng r; orc_rng_seed(&r, seed);
    for (int64_t i = 0; i < count; ++i) out[i] = orc_rng_next(&r);
}

/* ------------------------------------------------------------------ SGD (src/layout.cpp) */
typedef struct {
    /* layout and edges */
    float* Y; int64_t n; int dim;
    const int32_t* head; const int32_t* tail; const float* eps; float* eons; float* eonns; int64_t n_edges;
    /* mid-range partners */
    const int32_t* indptr; const int32_t* indices;         /* graph for walks (NULL if unused) */
    const int32_t* walk_lens;                                /* per node walk length or NULL */
    const int32_t* mid_pairs; int n_mid;                     /* (n, n_mid) or NULL */
    const int32_t* jump_indptr; const int32_t* jump_indices; float mid_jump;
    /* schedule */
    int epoch_start, epoch_end; float alpha0, alpha1, mid_w0, mid_w1;
    /* kernel */
    float a, b, rep_a, rep_b, negative_sample_rate; int loss; float exaggeration, repulsion_strength;
    int walk_len; float mid_rate; int optimizer, clip_mode; int64_t n_fixed;
    float* adam_m; float* adam_v; int32_t* adam_t; float beta1, beta2;
    int kernel; const float* node_b; uint64_t seed;
} orc_sgd_args;

typedef struct {
    float two_ab, two_b; int b_is_one, rep_b_is_one, rep_coupled, m_neg, use_mid;
} orc_derived;

static void orc_derive(orc_sgd_args* c, orc_derived* d) {
    /* src/layout.cpp:409-431: walks need the graph unless pairs are given; the coupled repulsion */
    const int has_pairs = c->mid_pairs != NULL && c->n_mid > 0;
    const int has_jumps = c->jump_indptr != NULL && c->mid_jump > 0.0f;
    d->use_mid = (c->mid_w0 > 0.0f || c->mid_w1 > 0.0f) && c->mid_rate > 0.0f && (has_pairs || c->walk_len > 0);
    if (has_jumps) c->mid_pairs = NULL;
    d->rep_coupled = c->rep_b <= 0.0f;
    if (c->rep_b <= 0.0f) { c->rep_a = c->a; c->rep_b = c->b; }
    d->two_ab = 2.0f * c->a * c->b;
    d->two_b = 2.0f * c->rep_b * c->repulsion_strength;
    d->b_is_one = fabsf(c->b - 1.0f) < 1e-6f;
    d->rep_b_is_one = fabsf(c->rep_b - 1.0f) < 1e-6f;
    long m = lroundf(c->negative_sample_rate);
    if (m < 1) m = 1;
    if (m > 64) m = 64;
    d->m_neg = (int)m;
}

static void orc_apply_step(const orc_sgd_args* c, float* yu, const float* g, float alpha, int64_t u) {
    const int dim = c->dim;
    float step[ORC_MAX_DIM];
    if (c->optimizer == 1) {
        const int32_t t = ++c->adam_t[u];
        const float c1 = 1.0f - powf(c->beta1, (float)t), c2 = 1.0f - powf(c->beta2, (float)t);
        float* m = c->adam_m + u * dim; float* v = c->adam_v + u * dim;
        for (int k = 0; k < dim; ++k) {
            m[k] = c->beta1 * m[k] + (1.0f - c->beta1) * g[k];
            v[k] = c->beta2 * v[k] + (1.0f - c->beta2) * g[k] * g[k];
            step[k] = alpha * (m[k] / c1) / (sqrtf(v[k] / c2) + 1e-7f);
        }
    } else {
        for (int k = 0; k < dim; ++k) step[k] = alpha * g[k];
    }
    const float cap = 4.0f * alpha;
    if (c->clip_mode == 1) {
        float n2 = 0.0f;
        for (int k = 0; k < dim; ++k) n2 += step[k] * step[k];
        if (n2 > cap * cap) { const float f = cap / sqrtf(n2); for (int k = 0; k < dim; ++k) step[k] *= f; }
    } else {
        for (int k = 0; k < dim; ++k) step[k] = step[k] > cap ? cap : (step[k] < -cap ? -cap : step[k]);
    }
    for (int k = 0; k < dim; ++k) yu[k] += step[k];
}

/* Recording of the draws of one epoch (for the schedule comparisons). Per edge: sampled flag, n_neg, the
 * offset of its negatives in `negs`, and the mid partner (-1 when no mid draw succeeded, -2 when the walk or
 * pair picked u itself). `negs` receives every drawn k, including the k == u ones the kernel skips. */
typedef struct {
    uint8_t* sampled; int32_t* n_neg; int64_t* neg_off; int32_t* negs; int64_t negs_cap; int32_t* mid;
    int64_t n_negs;
} orc_record;

/* One epoch, serial semantics of epoch_worker<DIM,false> with tid 0 (or the counter draws when
 * per_edge_stream). apply == 0: only the draws and the eons/eonns bookkeeping (schedule replay). */
static void orc_epoch(orc_sgd_args* c, const orc_derived* dv, int epoch, float alpha, float mid_w,
                      int per_edge_stream, int apply, orc_record* rec) {
    const int dim = c->dim;
    orc_draws dr; memset(&dr, 0, sizeof(dr));
    orc_rng_seed(&dr.rng, orc_stream_seed(c->seed, epoch, 0));
    dr.counter = per_edge_stream;
    const float fepoch = (float)epoch;
    float* Y = c->Y;
    float diff[ORC_MAX_DIM], gu[ORC_MAX_DIM], gk[ORC_MAX_DIM];
    int32_t negs[64]; float qk[64];
    for (int64_t i = 0; i < c->n_edges; ++i) {
        if (rec) { rec->sampled[i] = 0; rec->n_neg[i] = 0; rec->mid[i] = -1; rec->neg_off[i] = rec->n_negs; }
        if (c->eons[i] > fepoch) continue;
        dr.key = orc_sample_key(orc_stream_seed(c->seed, epoch, (uint64_t)i)); dr.p = 0; dr.t = 0;
        if (rec) rec->sampled[i] = 1;
        const int32_t u = c->head[i], v = c->tail[i];
        float* yu = Y + (int64_t)u * dim;
        float* yv = Y + (int64_t)v * dim;
        const int move_u = u >= c->n_fixed, move_v = v >= c->n_fixed;
        for (int k = 0; k < dim; ++k) gu[k] = 0.0f;
        float d2 = 0.0f;
        for (int k = 0; k < dim; ++k) { diff[k] = yu[k] - yv[k]; d2 += diff[k] * diff[k]; }
        const float b_u = c->node_b ? c->node_b[u] : c->b;
        const float b_uv = c->node_b ? 0.5f * (c->node_b[u] + c->node_b[v]) : c->b;
        const float pw_v = (dv->b_is_one && !c->node_b) ? d2 : (d2 > 0.0f ? powf(d2, b_uv) : 0.0f);
        if (c->loss == 0) {
            if (d2 > 0.0f) {
                float coeff;
                const float s = -1.0f * c->exaggeration;   /* -pair_scale * exaggeration, pair_scale = 1 */
                if (c->kernel == 0) coeff = s * 2.0f * c->a * b_uv * pw_v / (d2 * (c->a * pw_v + 1.0f));
                else if (c->kernel == 1) coeff = s * 2.0f * c->a;
                else if (c->kernel == 2) { const float dd = sqrtf(d2); coeff = s * c->a * tanhf(c->a * dd) / dd; }
                else coeff = s * 2.0f * c->a * (1.0f + tanhf(c->a * d2));
                for (int k = 0; k < dim; ++k) { const float g = coeff * diff[k]; gu[k] += g; gk[k] = -g; }
                if (apply && move_v) orc_apply_step(c, yv, gk, alpha, v);
            }
            c->eons[i] += c->eps[i];
            const float epn = c->eps[i] / c->negative_sample_rate;
            const int n_neg = (int)((fepoch - c->eonns[i]) / epn);
            if (rec) rec->n_neg[i] = n_neg > 0 ? n_neg : 0;
            for (int p = 0; p < n_neg; ++p) {
                const int32_t k = (int32_t)orc_below_of(orc_draw_neg(&dr), (uint32_t)c->n);
                if (rec && rec->n_negs < rec->negs_cap) rec->negs[rec->n_negs] = k;
                if (rec) rec->n_negs++;
                if (k == u) continue;
                const float* yk = Y + (int64_t)k * dim;
                float dd = 0.0f;
                for (int q = 0; q < dim; ++q) { diff[q] = yu[q] - yk[q]; dd += diff[q] * diff[q]; }
                if (dd > 0.0f) {
                    float coeff;
                    if (c->kernel == 0) {
                        if (c->node_b && dv->rep_coupled) { const float pw = powf(dd, b_u); coeff = 2.0f * b_u * c->repulsion_strength / ((0.001f + dd) * (c->a * pw + 1.0f)); }
                        else { const float pw = dv->rep_b_is_one ? dd : powf(dd, c->rep_b); coeff = dv->two_b / ((0.001f + dd) * (c->rep_a * pw + 1.0f)); }
                    } else if (c->kernel == 1) {
                        const float q = expf(-c->a * dd);
                        coeff = c->repulsion_strength * 2.0f * c->a * q / fmaxf(1.0f - q, 1e-3f);
                    } else if (c->kernel == 2) {
                        const float r = sqrtf(dd); const float q = 1.0f / coshf(c->a * r);
                        coeff = c->repulsion_strength * c->a * q * tanhf(c->a * r) / (r * fmaxf(1.0f - q, 1e-3f));
                    } else {
                        const float th = fmaxf(tanhf(c->a * dd), 1e-3f);
                        coeff = c->repulsion_strength * 2.0f * c->a * (1.0f - th * th) / th;
                    }
                    for (int q = 0; q < dim; ++q) gu[q] += coeff * diff[q];
                } else {
                    for (int q = 0; q < dim; ++q) gu[q] += (orc_uniform_of(orc_draw_jitter(&dr, p, q)) - 0.5f) * 1e-3f / fmaxf(alpha, 1e-6f);
                }
            }
            c->eonns[i] += (float)n_neg * epn;
        } else {
            /* InfoNCE (src/layout.cpp:185-223) */
            const float q_v = 1.0f / (1.0f + c->a * pw_v);
            float Z = q_v;
            for (int p = 0; p < dv->m_neg; ++p) {
                int32_t k = (int32_t)orc_below_of(orc_draw_neg(&dr), (uint32_t)c->n);
                if (k == u) k = (int32_t)((k + 1) % c->n);
                negs[p] = k;
                if (rec && rec->n_negs < rec->negs_cap) rec->negs[rec->n_negs] = k;
                if (rec) rec->n_negs++;
                const float* yk = Y + (int64_t)k * dim;
                float dd = 0.0f;
                for (int q = 0; q < dim; ++q) { const float t = yu[q] - yk[q]; dd += t * t; }
                const float pw = dv->b_is_one ? dd : (dd > 0.0f ? powf(dd, c->b) : 0.0f);
                qk[p] = 1.0f / (1.0f + c->a * pw);
                Z += qk[p];
            }
            if (rec) rec->n_neg[i] = dv->m_neg;
            const float w_v = q_v / Z;
            if (d2 > 0.0f) {
                const float coeff = -c->exaggeration * (1.0f - w_v) * dv->two_ab * pw_v / (d2 * (c->a * pw_v + 1.0f));
                for (int q = 0; q < dim; ++q) { const float g = coeff * diff[q]; gu[q] += g; gk[q] = -g; }
                if (apply && move_v) orc_apply_step(c, yv, gk, alpha, v);
            }
            for (int p = 0; p < dv->m_neg; ++p) {
                const int32_t k = negs[p];
                float* yk = Y + (int64_t)k * dim;
                float dd = 0.0f;
                for (int q = 0; q < dim; ++q) { diff[q] = yu[q] - yk[q]; dd += diff[q] * diff[q]; }
                if (dd <= 0.0f) {
                    for (int q = 0; q < dim; ++q) gu[q] += (orc_uniform_of(orc_draw_jitter(&dr, p, q)) - 0.5f) * 1e-3f / fmaxf(alpha, 1e-6f);
                    continue;
                }
                const float pw = dv->b_is_one ? dd : powf(dd, c->b);
                const float w_k = qk[p] / Z;
                const float coeff = c->repulsion_strength * w_k * dv->two_ab * pw / (dd * (c->a * pw + 1.0f));
                for (int q = 0; q < dim; ++q) { const float g = coeff * diff[q]; gu[q] += g; gk[q] = -g; }
                if (apply && k >= c->n_fixed) orc_apply_step(c, yk, gk, alpha, k);
            }
            c->eons[i] += c->eps[i];
            c->eonns[i] = fepoch;
        }
        /* mid-range partner (src/layout.cpp:225-255) */
        if (mid_w > 0.0f && orc_uniform_of(orc_draw_mid(&dr)) < c->mid_rate) {
            int32_t w = v;
            if (c->jump_indptr && c->mid_jump > 0.0f) {
                const int L = c->walk_lens ? c->walk_lens[v] : c->walk_len;
                for (int h = 0; h < L; ++h) {
                    const int32_t js = c->jump_indptr[w], je = c->jump_indptr[w + 1];
                    if (je > js && orc_uniform_of(orc_draw_mid(&dr)) < c->mid_jump) {
                        w = c->jump_indices[js + (int32_t)orc_below_of(orc_draw_mid(&dr), (uint32_t)(je - js))];
                    } else {
                        const int32_t s0 = c->indptr[w], e0 = c->indptr[w + 1];
                        if (e0 <= s0) break;
                        w = c->indices[s0 + (int32_t)orc_below_of(orc_draw_mid(&dr), (uint32_t)(e0 - s0))];
                    }
                }
            } else if (c->mid_pairs) {
                w = c->mid_pairs[(int64_t)u * c->n_mid + orc_below_of(orc_draw_mid(&dr), (uint32_t)c->n_mid)];
            } else {
                const int L = c->walk_lens ? c->walk_lens[v] : c->walk_len;
                for (int h = 0; h < L; ++h) {
                    const int32_t s0 = c->indptr[w], e0 = c->indptr[w + 1];
                    if (e0 <= s0) break;
                    w = c->indices[s0 + (int32_t)orc_below_of(orc_draw_mid(&dr), (uint32_t)(e0 - s0))];
                }
            }
            if (rec) rec->mid[i] = (w != u) ? w : -2;
            if (w != u) {
                float* yw = Y + (int64_t)w * dim;
                for (int q = 0; q < dim; ++q) { const float g = -mid_w * (yu[q] - yw[q]); gu[q] += g; gk[q] = -g; }
                if (apply && w >= c->n_fixed) orc_apply_step(c, yw, gk, alpha, w);
            }
        }
        if (apply && move_u) orc_apply_step(c, yu, gu, alpha, u);
    }
}

static void orc_sched(const orc_sgd_args* c, const orc_derived* dv, int epoch, float* alpha, float* mid_w) {
    const int n_span = (c->epoch_end - c->epoch_start) > 1 ? (c->epoch_end - c->epoch_start) : 1;
    const float frac = (float)(epoch - c->epoch_start) / (float)n_span;
    *alpha = c->alpha0 + (c->alpha1 - c->alpha0) * frac;
    *mid_w = dv->use_mid ? c->mid_w0 + (c->mid_w1 - c->mid_w0) * frac : 0.0f;
}

/* optimize_layout with n_threads = 1, parallel = 0 (hogwild path run on one thread): Y, eons, eonns and the
 * Adam state are updated in place. per_edge_stream = 1 runs the same updates with the GPU fast mode's
 * counter draws. Returns 0. */
int orc_sgd_serial(orc_sgd_args* c, int per_edge_stream) {
    orc_derived dv; orc_derive(c, &dv);
    for (int e = c->epoch_start; e < c->epoch_end; ++e) {
        float alpha, mid_w; orc_sched(c, &dv, e, &alpha, &mid_w);
        orc_epoch(c, &dv, e, alpha, mid_w, per_edge_stream, 1, NULL);
    }
    return 0;
}

/* Schedule of one epoch (the draws only, Y read-only). eons/eonns are advanced in place as the epoch would
 * advance them. Returns the number of negatives drawn (may exceed negs_cap; only negs_cap are stored). */
int64_t orc_sgd_schedule(orc_sgd_args* c, int epoch, int per_edge_stream,
                         uint8_t* sampled, int32_t* n_neg, int64_t* neg_off, int32_t* negs, int64_t negs_cap,
                         int32_t* mid) {
    orc_derived dv; orc_derive(c, &dv);
    float alpha, mid_w; orc_sched(c, &dv, epoch, &alpha, &mid_w);
    orc_record rec = {sampled, n_neg, neg_off, negs, negs_cap, mid, 0};
    orc_epoch(c, &dv, epoch, alpha, mid_w, per_edge_stream, 0, &rec);
    return rec.n_negs;
}

/* Owner mode (parallel = 1; src/layout.cpp:118-276 with OWNER = true, :300-330, :441-463), UMAP loss only.
 * Nodes are split at the edge quantiles into n_chunks = min(4096, max(1, E / 4096)) chunks (edges sorted by head);
 * chunk k of epoch e draws from its own stream (tid = k) over its edges in order, moves only its own heads u
 * (the attraction scaled by 1.5), and reads every other position from the layout as it was at the start of the
 * epoch. The reference's two alternating snapshot buffers hold exactly that layout, so one copy per epoch
 * restates them. With the reverse mid pairs (rev_indptr / rev_indices), u also receives, after each edge, the
 * mid-range pulls of the nodes that chose it. The result does not depend on the order the chunks run in. */
static void orc_owner_chunk(orc_sgd_args* c, const orc_derived* dv, int epoch, float alpha, float mid_w, int k,
                            int64_t e0, int64_t e1, const float* Yr, const int32_t* rev_indptr,
                            const int32_t* rev_indices) {
    const int dim = c->dim;
    orc_rng rng; orc_rng_seed(&rng, orc_stream_seed(c->seed, epoch, (uint64_t)k));
    /* n_mid stays set when a jump graph replaces the pairs (src/layout.cpp:397-407) */
    const float inv_n_mid = c->n_mid > 0 ? 1.0f / (float)c->n_mid : 0.0f;
    const float pair_scale = 1.5f;
    const float fepoch = (float)epoch;
    float diff[ORC_MAX_DIM], gu[ORC_MAX_DIM], gk[ORC_MAX_DIM];
    for (int64_t i = e0; i < e1; ++i) {
        if (c->eons[i] > fepoch) continue;
        const int32_t u = c->head[i], v = c->tail[i];
        float* yu = c->Y + (int64_t)u * dim;
        const float* yv = Yr + (int64_t)v * dim;
        const int move_u = u >= c->n_fixed;
        for (int q = 0; q < dim; ++q) gu[q] = 0.0f;
        float d2 = 0.0f;
        for (int q = 0; q < dim; ++q) { diff[q] = yu[q] - yv[q]; d2 += diff[q] * diff[q]; }
        const float b_u = c->node_b ? c->node_b[u] : c->b;
        const float b_uv = c->node_b ? 0.5f * (c->node_b[u] + c->node_b[v]) : c->b;
        const float pw_v = (dv->b_is_one && !c->node_b) ? d2 : (d2 > 0.0f ? powf(d2, b_uv) : 0.0f);
        if (d2 > 0.0f) {
            float coeff;
            if (c->kernel == 0) coeff = -pair_scale * c->exaggeration * 2.0f * c->a * b_uv * pw_v / (d2 * (c->a * pw_v + 1.0f));
            else if (c->kernel == 1) coeff = -pair_scale * c->exaggeration * 2.0f * c->a;
            else if (c->kernel == 2) { const float dd = sqrtf(d2); coeff = -pair_scale * c->exaggeration * c->a * tanhf(c->a * dd) / dd; }
            else coeff = -pair_scale * c->exaggeration * 2.0f * c->a * (1.0f + tanhf(c->a * d2));
            for (int q = 0; q < dim; ++q) gu[q] += coeff * diff[q];
        }
        c->eons[i] += c->eps[i];
        const float epn = c->eps[i] / c->negative_sample_rate;
        const int n_neg = (int)((fepoch - c->eonns[i]) / epn);
        for (int p = 0; p < n_neg; ++p) {
            const int32_t kk = (int32_t)orc_rng_below(&rng, (uint32_t)c->n);
            if (kk == u) continue;
            const float* yk = Yr + (int64_t)kk * dim;
            float dd = 0.0f;
            for (int q = 0; q < dim; ++q) { diff[q] = yu[q] - yk[q]; dd += diff[q] * diff[q]; }
            if (dd > 0.0f) {
                float coeff;
                if (c->kernel == 0) {
                    if (c->node_b && dv->rep_coupled) { const float pw = powf(dd, b_u); coeff = 2.0f * b_u * c->repulsion_strength / ((0.001f + dd) * (c->a * pw + 1.0f)); }
                    else { const float pw = dv->rep_b_is_one ? dd : powf(dd, c->rep_b); coeff = dv->two_b / ((0.001f + dd) * (c->rep_a * pw + 1.0f)); }
                } else if (c->kernel == 1) {
                    const float qq = expf(-c->a * dd);
                    coeff = c->repulsion_strength * 2.0f * c->a * qq / fmaxf(1.0f - qq, 1e-3f);
                } else if (c->kernel == 2) {
                    const float r = sqrtf(dd); const float qq = 1.0f / coshf(c->a * r);
                    coeff = c->repulsion_strength * c->a * qq * tanhf(c->a * r) / (r * fmaxf(1.0f - qq, 1e-3f));
                } else {
                    const float th = fmaxf(tanhf(c->a * dd), 1e-3f);
                    coeff = c->repulsion_strength * 2.0f * c->a * (1.0f - th * th) / th;
                }
                for (int q = 0; q < dim; ++q) gu[q] += coeff * diff[q];
            } else {
                for (int q = 0; q < dim; ++q) gu[q] += (orc_rng_uniform(&rng) - 0.5f) * 1e-3f / fmaxf(alpha, 1e-6f);
            }
        }
        c->eonns[i] += (float)n_neg * epn;
        if (mid_w > 0.0f && orc_rng_uniform(&rng) < c->mid_rate) {
            int32_t w = v;
            if (c->jump_indptr && c->mid_jump > 0.0f) {
                const int L = c->walk_lens ? c->walk_lens[v] : c->walk_len;
                for (int h = 0; h < L; ++h) {
                    const int32_t js = c->jump_indptr[w], je = c->jump_indptr[w + 1];
                    if (je > js && orc_rng_uniform(&rng) < c->mid_jump) {
                        w = c->jump_indices[js + (int32_t)orc_rng_below(&rng, (uint32_t)(je - js))];
                    } else {
                        const int32_t s0 = c->indptr[w], ee = c->indptr[w + 1];
                        if (ee <= s0) break;
                        w = c->indices[s0 + (int32_t)orc_rng_below(&rng, (uint32_t)(ee - s0))];
                    }
                }
            } else if (c->mid_pairs) {
                w = c->mid_pairs[(int64_t)u * c->n_mid + orc_rng_below(&rng, (uint32_t)c->n_mid)];
            } else {
                const int L = c->walk_lens ? c->walk_lens[v] : c->walk_len;
                for (int h = 0; h < L; ++h) {
                    const int32_t s0 = c->indptr[w], ee = c->indptr[w + 1];
                    if (ee <= s0) break;
                    w = c->indices[s0 + (int32_t)orc_rng_below(&rng, (uint32_t)(ee - s0))];
                }
            }
            if (w != u) {
                const float* yw = Yr + (int64_t)w * dim;
                for (int q = 0; q < dim; ++q) gu[q] += -mid_w * (yu[q] - yw[q]);
            }
        }
        if (move_u) orc_apply_step(c, yu, gu, alpha, u);
        if (move_u && mid_w > 0.0f && rev_indptr) {
            const int32_t rs = rev_indptr[u], re = rev_indptr[u + 1];
            float p = c->mid_rate * (float)(re - rs) * inv_n_mid;
            while (p > 0.0f && re > rs) {
                if (orc_rng_uniform(&rng) < p) {
                    const int32_t x = rev_indices[rs + (int32_t)orc_rng_below(&rng, (uint32_t)(re - rs))];
                    if (x != u) {
                        const float* yx = Yr + (int64_t)x * dim;
                        for (int q = 0; q < dim; ++q) gk[q] = -mid_w * (yu[q] - yx[q]);
                        orc_apply_step(c, yu, gk, alpha, u);
                    }
                }
                p -= 1.0f;
            }
        }
    }
}

/* chunk boundaries of owner mode (src/layout.cpp:441-463): own[k] the first node, eown[k] the first edge of chunk
 * k; both arrays hold n_chunks + 1 entries. Returns n_chunks (own / eown NULL: only the count). */
int orc_owner_chunks(const int32_t* head, int64_t n_edges, int64_t n, int64_t* own, int64_t* eown) {
    int64_t nc = n_edges / 4096;
    if (nc < 1) nc = 1;
    if (nc > 4096) nc = 4096;
    if (!own || !eown) return (int)nc;
    for (int64_t t = 0; t <= nc; ++t) { own[t] = 0; eown[t] = 0; }
    own[nc] = n; eown[nc] = n_edges;
    for (int64_t t = 1; t < nc; ++t) {
        const int64_t e = n_edges * t / nc;
        int64_t node = head[e] > own[t - 1] ? head[e] : own[t - 1];
        own[t] = node;
        int64_t k = eown[t - 1];
        while (k < n_edges && head[k] < node) ++k;
        eown[t] = k;
    }
    return (int)nc;
}

/* optimize_layout with parallel = 1 (owner mode); rev_indptr / rev_indices may be NULL. Returns 0, or -1 when the
 * edges are not sorted by head or the loss is InfoNCE (the reference's argument errors). */
int orc_sgd_owner(orc_sgd_args* c, const int32_t* rev_indptr, const int32_t* rev_indices) {
    if (c->loss != 0) return -1;
    for (int64_t i = 1; i < c->n_edges; ++i) if (c->head[i - 1] > c->head[i]) return -1;
    orc_derived dv; orc_derive(c, &dv);
    const int nc = orc_owner_chunks(c->head, c->n_edges, c->n, NULL, NULL);
    int64_t* own = (int64_t*)malloc(sizeof(int64_t) * (nc + 1));
    int64_t* eown = (int64_t*)malloc(sizeof(int64_t) * (nc + 1));
    orc_owner_chunks(c->head, c->n_edges, c->n, own, eown);
    const size_t bytes = sizeof(float) * (size_t)c->n * (size_t)c->dim;
    float* Yr = (float*)malloc(bytes > 0 ? bytes : 1);
    for (int e = c->epoch_start; e < c->epoch_end; ++e) {
        float alpha, mid_w; orc_sched(c, &dv, e, &alpha, &mid_w);
        memcpy(Yr, c->Y, bytes);
        for (int k = 0; k < nc; ++k)
            orc_owner_chunk(c, &dv, e, alpha, mid_w, k, eown[k], eown[k + 1], Yr, rev_indptr, rev_indices);
    }
    free(Yr); free(own); free(eown);
    return 0;
}

/* ------------------------------------------------------------------ fuzzy neighbour graph */
/* smooth_knn (src/graph.cpp:29-78) on one thread: the row's FP64 distance sum and rho (first positive
 * distance), the bisection of sigma (at most n_iter steps, stop within 1e-5 of log2(n_neighbors) * bandwidth),
 * the floor 1e-3 x the row's mean distance (the whole array's when rho = 0), then the memberships. */
void orc_smooth_knn(const float* D, int64_t n, int k, int n_neighbors, float bandwidth, int n_iter, float* out) {
    const float target = log2f((float)n_neighbors) * bandwidth;
    float* sigma = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    float* rho = (float*)malloc(sizeof(float) * (size_t)(n > 0 ? n : 1));
    double tot = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const float* d = D + i * k;
        double rowsum = 0.0; float r = 0.f; int has = 0;
        for (int j = 0; j < k; ++j) { rowsum += d[j]; if (!has && d[j] > 0.f) { r = d[j]; has = 1; } }
        tot += rowsum;
        rho[i] = r;
        float lo = 0.f, hi = INFINITY, mid = 1.f, sg = 1.f; int done = 0;
        for (int it = 0; it < n_iter; ++it) {
            float psum = 0.f;
            for (int j = 0; j < k; ++j) { const float dmr = d[j] - r; psum += dmr > 0.f ? expf(-dmr / mid) : 1.f; }
            if (fabsf(psum - target) < 1e-5f) { sg = mid; done = 1; break; }
            if (psum > target) { hi = mid; mid = (lo + hi) * 0.5f; }
            else { lo = mid; mid = isinf(hi) ? mid * 2.f : (lo + hi) * 0.5f; }
        }
        if (!done) sg = mid;
        const float mean_row = (float)(rowsum / k);
        if (r > 0.f) sg = fmaxf(sg, 1e-3f * mean_row);
        sigma[i] = sg;
    }
    const float mean_all = (float)(tot / (double)(n * k));
    for (int64_t i = 0; i < n; ++i) {
        const float* d = D + i * k; float* o = out + i * k;
        float sg = sigma[i];
        if (!(rho[i] > 0.f)) sg = fmaxf(sg, 1e-3f * mean_all);
        for (int j = 0; j < k; ++j) { const float dmr = d[j] - rho[i]; o[j] = dmr > 0.f ? expf(-dmr / sg) : 1.f; }
    }
    free(sigma); free(rho);
}

/* The fuzzy union of magnet/knn.py:221-230 with scipy's float32 arithmetic: A = csr((vals, (rows, ind))) with
 * duplicate columns summed (in row order) and zeros dropped; T = A^T; per entry (a, t):
 * both: d = (a + t) - a t, P = d mix + (a t) (1 - mix); one: P = x mix; zeros dropped, columns sorted.
 * mix and 1 - mix are the float32 roundings of the python floats. Returns nnz (entries beyond cap are not
 * written), or -1 for an index outside [0, n). */
int64_t orc_fuzzy_union(const int32_t* ind, const float* vals, int64_t n_rows, int k, int64_t n, double mix_d,
                        int32_t* indptr, int32_t* indices, float* data, int64_t cap) {
    const float mix = (float)mix_d, omm = (float)(1.0 - mix_d);
    const size_t ek = (size_t)(n_rows * k > 0 ? n_rows * k : 1);
    int32_t* ac = (int32_t*)malloc(sizeof(int32_t) * ek); float* av = (float*)malloc(sizeof(float) * ek);
    int32_t* al = (int32_t*)calloc((size_t)(n_rows > 0 ? n_rows : 1), sizeof(int32_t));
    int64_t* tp = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    int32_t* tr = (int32_t*)malloc(sizeof(int32_t) * ek); float* tv = (float*)malloc(sizeof(float) * ek);
    int64_t nnz = 0;
    for (int64_t i = 0; i < n_rows; ++i) {
        int32_t* c = ac + i * k; float* v = av + i * k;
        for (int j = 0; j < k; ++j) {
            const int32_t col = ind[i * k + j];
            if (col < 0 || col >= n) { nnz = -1; goto done; }
            int p = j;
            while (p > 0 && c[p - 1] > col) { c[p] = c[p - 1]; v[p] = v[p - 1]; --p; }
            c[p] = col; v[p] = vals[i * k + j];
        }
        int m = 0;
        for (int j = 0; j < k;) {
            const int32_t col = c[j]; float x = v[j]; int e = j + 1;
            for (; e < k && c[e] == col; ++e) x += v[e];
            if (x != 0.f) { c[m] = col; v[m] = x; ++m; }
            j = e;
        }
        al[i] = m;
    }
    /* T by a stable counting sort on the column: rows come out in increasing order */
    for (int64_t i = 0; i < n_rows; ++i) for (int j = 0; j < al[i]; ++j) tp[ac[i * k + j] + 1]++;
    for (int64_t r = 0; r < n; ++r) tp[r + 1] += tp[r];
    {
        int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
        for (int64_t r = 0; r < n; ++r) cur[r] = tp[r];
        for (int64_t i = 0; i < n_rows; ++i)
            for (int j = 0; j < al[i]; ++j) { const int32_t col = ac[i * k + j]; tr[cur[col]] = (int32_t)i; tv[cur[col]] = av[i * k + j]; cur[col]++; }
        free(cur);
    }
    indptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) {
        const int la = i < n_rows ? al[i] : 0;
        const int32_t* c = ac + i * k; const float* v = av + i * k;
        int ja = 0; int64_t ta = tp[i];
        while (ja < la || ta < tp[i + 1]) {
            const int32_t ca = ja < la ? c[ja] : INT32_MAX, ct = ta < tp[i + 1] ? tr[ta] : INT32_MAX;
            const int32_t col = ca < ct ? ca : ct;
            float x;
            if (ca == col && ct == col) {
                const float a = v[ja], t = tv[ta], prod = a * t, d = (a + t) - prod;
                x = d * mix + prod * omm;
                ++ja; ++ta;
            } else if (ca == col) { x = v[ja] * mix; ++ja; }
            else { x = tv[ta] * mix; ++ta; }
            if (x != 0.f) { if (nnz < cap) { indices[nnz] = col; data[nnz] = x; } ++nnz; }
        }
        indptr[i + 1] = (int32_t)nnz;
    }
done:
    free(ac); free(av); free(al); free(tp); free(tr); free(tv);
    return nnz;
}

/* ------------------------------------------------------------------ FFT repulsion pieces (src/fftconv.cpp) */
static void orc_lagrange(float u, int ni, float* w) {
    if (ni == 3) {
        const float a = u - 1.f / 6.f, b = u - 0.5f, c = u - 5.f / 6.f;
        w[0] = b * c * 4.5f; w[1] = -a * c * 9.f; w[2] = a * b * 4.5f;
        return;
    }
    for (int k = 0; k < ni; ++k) {
        const float uk = (k + 0.5f) / ni;
        float num = 1.f, den = 1.f;
        for (int m = 0; m < ni; ++m) {
            if (m == k) continue;
            const float um = (m + 0.5f) / ni;
            num *= (u - um); den *= (uk - um);
        }
        w[k] = num / den;
    }
}

static inline int orc_clampi(int x, int lo, int hi) { return x < lo ? lo : (x > hi ? hi : x); }

/* Box of a point as FFTConv2D::compute finds it: the x-box with the reciprocal (the sort, :88), the y-box
 * and both local coordinates with the division (:106-111). */
static void orc_locate(float x, float y, float xmin, float ymin, float width, int n_boxes, int ni,
                       int* bx, int* by, float* wx, float* wy) {
    const float inv_w = 1.f / width;
    *bx = orc_clampi((int)((x - xmin) * inv_w), 0, n_boxes - 1);
    const float ux = (x - xmin) / width, uy = (y - ymin) / width;
    *by = orc_clampi((int)uy, 0, n_boxes - 1);
    float tx = ux - (float)*bx, ty = uy - (float)*by;
    tx = tx < 0.f ? 0.f : (tx > 1.f ? 1.f : tx);
    ty = ty < 0.f ? 0.f : (ty > 1.f ? 1.f : ty);
    orc_lagrange(tx, ni, wx); orc_lagrange(ty, ni, wy);
}

/* charges (1, x, y) spread on the live N x N grid, W (3, N, N) float64 (exact sums of the float weights) */
void orc_spread(const float* Y, int64_t n, float xmin, float ymin, float width, int n_boxes, int ni, double* W) {
    const int64_t N = (int64_t)n_boxes * ni;
    memset(W, 0, sizeof(double) * 3 * N * N);
    float wx[8], wy[8]; int bx, by;
    for (int64_t i = 0; i < n; ++i) {
        const float x = Y[2 * i], y = Y[2 * i + 1];
        orc_locate(x, y, xmin, ymin, width, n_boxes, ni, &bx, &by, wx, wy);
        for (int a = 0; a < ni; ++a) {
            const int64_t gx = (int64_t)bx * ni + a;
            for (int b = 0; b < ni; ++b) {
                const int64_t gy = (int64_t)by * ni + b;
                const double w = (double)(wx[a] * wy[b]);
                W[(0 * N + gx) * N + gy] += w;
                W[(1 * N + gx) * N + gy] += w * (double)x;
                W[(2 * N + gx) * N + gy] += w * (double)y;
            }
        }
    }
}

/* potentials phi (4, N, N) float64 -> sumQ (float64, self terms removed) and F (n, 2) */
double orc_gather(const float* Y, int64_t n, float xmin, float ymin, float width, int n_boxes, int ni,
                  const double* phi, double* F) {
    const int64_t N = (int64_t)n_boxes * ni;
    float wx[8], wy[8]; int bx, by; double s = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const float x = Y[2 * i], y = Y[2 * i + 1];
        orc_locate(x, y, xmin, ymin, width, n_boxes, ni, &bx, &by, wx, wy);
        double pot[4] = {0, 0, 0, 0};
        for (int a = 0; a < ni; ++a) {
            const int64_t gx = (int64_t)bx * ni + a;
            for (int b = 0; b < ni; ++b) {
                const int64_t gy = (int64_t)by * ni + b;
                const double w = (double)(wx[a] * wy[b]);
                for (int c = 0; c < 4; ++c) pot[c] += w * phi[((int64_t)c * N + gx) * N + gy];
            }
        }
        s += pot[0];
        F[2 * i] = pot[1] * (double)x - pot[2];
        F[2 * i + 1] = pot[1] * (double)y - pot[3];
    }
    return s - (double)n;
}

/* FP64 all-pairs: sumQ = sum_{i != j} q_ij, F_i = sum_j q_ij^2 (y_i - y_j), q = 1/(1 + d^2) (dof = 1), or the
 * Student-t kernel of dof degrees of freedom: q = (1 + d^2/dof)^-dof, weight (1 + d^2/dof)^(-dof-1).
 * rows [r0, r1) only (for sub-samples); F has (r1 - r0) rows. */
double orc_exact_repulsion(const float* Y, int64_t n, int64_t r0, int64_t r1, double dof, double* F) {
    double s = 0.0;
    for (int64_t i = r0; i < r1; ++i) {
        const double xi = Y[2 * i], yi = Y[2 * i + 1];
        double fx = 0.0, fy = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == i) continue;
            const double dx = xi - (double)Y[2 * j], dy = yi - (double)Y[2 * j + 1];
            const double base = 1.0 + (dx * dx + dy * dy) / dof;
            double q, w;
            if (dof == 1.0) { q = 1.0 / base; w = q * q; }
            else { q = pow(base, -dof); w = pow(base, -dof - 1.0); }
            s += q; fx += w * dx; fy += w * dy;
        }
        F[2 * (i - r0)] = fx; F[2 * (i - r0) + 1] = fy;
    }
    return s;
}

/* ------------------------------------------------------------------ t-SNE kernels (src/fftrep.cpp) */
void orc_tsne_attraction(const int32_t* ip, const int32_t* ix, const float* P, const float* Y, int64_t n, int dim,
                         float dof, float* out) {
    const float inv_dof = 1.f / dof;
    if (dim == 2) {
        for (int64_t i = 0; i < n; ++i) {
            const float xi = Y[2 * i], yi = Y[2 * i + 1];
            float ax = 0.f, ay = 0.f;
            for (int32_t e = ip[i]; e < ip[i + 1]; ++e) {
                const int64_t j = ix[e];
                const float dx = xi - Y[2 * j], dy = yi - Y[2 * j + 1];
                const float w = P[e] / (1.f + (dx * dx + dy * dy) * inv_dof);
                ax += w * dx; ay += w * dy;
            }
            out[2 * i] = ax; out[2 * i + 1] = ay;
        }
        return;
    }
    float acc[ORC_MAX_DIM], diff[ORC_MAX_DIM];
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < dim; ++d) acc[d] = 0.f;
        const float* yi = Y + i * dim;
        for (int32_t e = ip[i]; e < ip[i + 1]; ++e) {
            const float* yj = Y + (int64_t)ix[e] * dim;
            float d2 = 0.f;
            for (int d = 0; d < dim; ++d) { diff[d] = yi[d] - yj[d]; d2 += diff[d] * diff[d]; }
            const float w = P[e] / (1.f + d2 * inv_dof);
            for (int d = 0; d < dim; ++d) acc[d] += w * diff[d];
        }
        for (int d = 0; d < dim; ++d) out[i * dim + d] = acc[d];
    }
}

/* tsne_step with one worker (nt = 1): the running float sums are flushed into the double every 1024 rows */
void orc_tsne_step(float* Y, float* U, float* G, const float* A, const float* F, int64_t n, int dim,
                   float rho, float inv_sumQ, float lr, float momentum) {
    double s[ORC_MAX_DIM]; float sl[ORC_MAX_DIM];
    for (int d = 0; d < dim; ++d) { s[d] = 0.0; sl[d] = 0.f; }
    for (int64_t i = 0; i < n; ++i) {
        for (int d = 0; d < dim; ++d) {
            const int64_t k = i * dim + d;
            const float g_ = rho * A[k] - F[k] * inv_sumQ;
            const int same = (g_ > 0.f) == (U[k] > 0.f);
            float g = same ? G[k] * 0.8f : G[k] + 0.2f;
            if (g < 0.01f) g = 0.01f;
            G[k] = g;
            const float u = momentum * U[k] - lr * g * g_;
            U[k] = u;
            const float y = Y[k] + u;
            Y[k] = y;
            sl[d] += y;
        }
        if ((i & 1023) == 1023) { for (int d = 0; d < dim; ++d) { s[d] += sl[d]; sl[d] = 0.f; } }
    }
    for (int d = 0; d < dim; ++d) s[d] += sl[d];
    float mean[ORC_MAX_DIM];
    for (int d = 0; d < dim; ++d) mean[d] = (float)(s[d] / (double)n);
    for (int64_t i = 0; i < n; ++i) for (int d = 0; d < dim; ++d) Y[i * dim + d] -= mean[d];
}

void orc_bbox_2d(const float* Y, int64_t n, float* out4) {
    float x0 = Y[0], x1 = x0, y0 = Y[1], y1 = y0;
    for (int64_t i = 0; i < n; ++i) {
        x0 = fminf(x0, Y[2 * i]); x1 = fmaxf(x1, Y[2 * i]);
        y0 = fminf(y0, Y[2 * i + 1]); y1 = fmaxf(y1, Y[2 * i + 1]);
    }
    out4[0] = x0; out4[1] = y0; out4[2] = x1; out4[3] = y1;
}

/* ---------------------------------------------------------------------------------------------------------------
 * Mid-near partners, src/nndescent.cpp:731-759 (mid_near_core over dense rows): nt = min(n_threads, max(1, n / 2048))
 * streams, stream t = Rng(seed + 48271 (t + 1)) over rows [n t / nt, n (t + 1) / nt); per row and pair, n_cand draws
 * j = below(n) (j == i -> (j + 1) % n) with their squared distances, the second smallest (distance, index) is kept.
 * The squared distance follows the reference's kernel for the host's instruction set (src/nndescent.cpp:35-116,
 * chosen at :101-106): order 0 the AVX-512 kernel (16 lanes of fused multiply-adds, the lanes summed high half
 * onto low half down to one, then the tail with fused multiply-adds), order 1 the AVX2 kernel (8 lanes, the lanes
 * summed ((0+1)+(2+3))+((4+5)+(6+7)), then the tail), order 2 the plain loop (4 interleaved sums, no fusion).
 * Order 0 equals the reference's distances bit for bit (checked against its nn_descent output). */
static float orc_sqdist(const float* a, const float* b, int d, int order) {
    if (order == 2) {
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
        int i = 0;
        for (; i + 4 <= d; i += 4) {
            const float d0 = a[i] - b[i], d1 = a[i + 1] - b[i + 1], d2 = a[i + 2] - b[i + 2], d3 = a[i + 3] - b[i + 3];
            s0 += d0 * d0; s1 += d1 * d1; s2 += d2 * d2; s3 += d3 * d3;
        }
        for (; i < d; ++i) { const float df = a[i] - b[i]; s0 += df * df; }
        return (s0 + s1) + (s2 + s3);
    }
    const int L = order == 0 ? 16 : 8;
    float acc[16] = {0};
    int i = 0;
    for (; i + L <= d; i += L)
        for (int l = 0; l < L; ++l) { const float df = a[i + l] - b[i + l]; acc[l] = fmaf(df, df, acc[l]); }
    float s;
    if (order == 0) {
        float t3[8], t6[4];
        for (int k = 0; k < 8; ++k) t3[k] = acc[8 + k] + acc[k];
        for (int k = 0; k < 4; ++k) t6[k] = t3[4 + k] + t3[k];
        s = (t6[0] + t6[2]) + (t6[1] + t6[3]);
    } else {
        s = ((acc[0] + acc[1]) + (acc[2] + acc[3])) + ((acc[4] + acc[5]) + (acc[6] + acc[7]));
    }
    for (; i < d; ++i) { const float df = a[i] - b[i]; s = fmaf(df, df, s); }
    return s;
}

int orc_mid_near_pairs(const float* X, int64_t n, int d, int n_pairs, int n_cand, uint64_t seed, int n_threads,
                       int order, int32_t* out) {
    if (!(n_pairs >= 1 && n_cand >= 2 && n >= n_cand + 1)) return 1;
    int64_t nt = n / 2048 > 1 ? n / 2048 : 1;
    if (n_threads < nt) nt = n_threads;
    float* dist = (float*)malloc(sizeof(float) * n_cand);
    int32_t* idx = (int32_t*)malloc(sizeof(int32_t) * n_cand);
    for (int64_t t = 0; t < nt; ++t) {
        orc_rng rng;
        orc_rng_seed(&rng, seed + 48271ULL * (uint64_t)(t + 1));
        const int64_t r0 = n * t / nt, r1 = n * (t + 1) / nt;
        for (int64_t i = r0; i < r1; ++i)
            for (int p = 0; p < n_pairs; ++p) {
                for (int c = 0; c < n_cand; ++c) {
                    int32_t j = (int32_t)orc_rng_below(&rng, (uint32_t)n);
                    if (j == i) j = (int32_t)((j + 1) % n);
                    idx[c] = j;
                    dist[c] = orc_sqdist(X + i * d, X + (int64_t)j * d, d, order);
                }
                /* the two smallest (distance, index) pairs in order; the second is kept */
                int b0 = -1, b1 = -1;
                for (int c = 0; c < n_cand; ++c) {
                    if (b0 < 0 || dist[c] < dist[b0] || (dist[c] == dist[b0] && idx[c] < idx[b0])) { b1 = b0; b0 = c; }
                    else if (b1 < 0 || dist[c] < dist[b1] || (dist[c] == dist[b1] && idx[c] < idx[b1])) b1 = c;
                }
                out[i * n_pairs + p] = idx[b1];
            }
    }
    free(dist); free(idx);
    return 0;
}
