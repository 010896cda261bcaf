// Register-tiled FFT engine of the repulsion pass: Stockham stages of large radices.
//
// A transform of length L = R1 R2 ... (at most five factors) runs as that many Stockham stages. Each stage is a
// radix-R DFT (R <= 16: 2, 3, 4, 5, 6, 8, 9, 10, 12, 15, 16, products of the base radices 2/3/4/5/8) held in the
// registers of one thread: R loads, inter-stage
// twiddles, the DFT, R stores. Against the one-base-radix-per-stage engine this halves the number of passes
// over shared memory; the first stage may read its input directly from global memory and the last may write
// its output directly to global memory, which removes the staging passes too.
//
// Stage s (radix R, Ns = product of the radices before it, j in [0, L/R)):
//   v[r] = src[j + r L/R] * w^(r (j mod Ns) L/(Ns R)),  v = DFT_R(v),
//   dst[(j / Ns) Ns R + (j mod Ns) + r Ns] = v[r]
// Internal DFT twiddles come from the same table: w_R^m = tw[m L / R], tw[m] = exp(-2 pi i m / L) (FP64 rounded).
//
// Shared-memory element i lives at pad(i) = i + i/16: large power-of-two radices write with stride R, and the
// padding spreads those writes over the banks.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "fft.cuh"

namespace mgb {
namespace fft2 {

constexpr int kMaxStages = 5;
constexpr int kMaxRadix = 16;
constexpr int kMaxLen = 13500;

__host__ __device__ __forceinline__ int pad(int i) { return i + (i >> 4); }
__host__ __device__ __forceinline__ int padded_len(int L) { return pad(L - 1) + 1; }

// the radices a stage may use
__host__ __device__ inline bool is_radix(int r) {
    switch (r) {
        case 2: case 3: case 4: case 5: case 6: case 8: case 9: case 10: case 12: case 15: case 16: return true;
        default: return false;
    }
}

struct Plan {
    int L;
    int n;
    int R[kMaxStages];
};

// Fewest stages; among equal counts, the most balanced radices (smallest largest radix). Host side; the device
// reads plans from a table built here.
inline bool plan_search(int L, int depth, int* cur, int* best, int& best_n, int& best_max, int mx) {
    static const int rad[] = {16, 15, 12, 10, 9, 8, 6, 5, 4, 3, 2};
    if (L == 1) {
        if (depth < best_n || (depth == best_n && mx < best_max)) {
            best_n = depth; best_max = mx;
            for (int s = 0; s < depth; ++s) best[s] = cur[s];
        }
        return true;
    }
    if (depth >= kMaxStages || depth + 1 > best_n) return false;
    bool any = false;
    for (int r : rad) {
        if (L % r) continue;
        cur[depth] = r;
        any |= plan_search(L / r, depth + 1, cur, best, best_n, best_max, mx > r ? mx : r);
    }
    return any;
}

inline bool make_plan(int L, Plan& p) {
    p.L = L; p.n = 0;
    if (L < 2 || L > kMaxLen || !fft::is_5smooth(L)) return false;
    int cur[kMaxStages], best[kMaxStages];
    int best_n = kMaxStages + 1, best_max = 1 << 30;
    plan_search(L, 0, cur, best, best_n, best_max, 0);
    if (best_n > kMaxStages) return false;
    p.n = best_n;
    for (int s = 0; s < best_n; ++s) p.R[s] = best[s];
    return true;
}

// ---------------------------------------------------------------------------------------------- DFT in registers
template <int R> struct Split { static constexpr int A = (R % 8 == 0) ? 8 : (R % 5 == 0) ? 5 : (R % 4 == 0) ? 4 : (R % 3 == 0) ? 3 : 2; };

template <int R>
__device__ __forceinline__ void dftr(float2* v, const float2* __restrict__ tw, int step) {
    if constexpr (R == 2) { fft::dft2(v); }
    else if constexpr (R == 3) { fft::dft3(v); }
    else if constexpr (R == 4) { fft::dft4(v); }
    else if constexpr (R == 5) { fft::dft5(v); }
    else if constexpr (R == 8) { fft::dft8(v); }
    else {
        // R = A B, n = B n1 + n2, k = k1 + A k2 (decimation in time)
        constexpr int A = Split<R>::A, B = R / A;
        float2 y[R];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) {
            float2 t[A];
#pragma unroll
            for (int n1 = 0; n1 < A; ++n1) t[n1] = v[B * n1 + n2];
            dftr<A>(t, tw, step * B);
#pragma unroll
            for (int k1 = 0; k1 < A; ++k1)
                y[n2 * A + k1] = (n2 * k1 == 0) ? t[k1] : fft::cmul(t[k1], __ldg(&tw[(n2 * k1) * step]));
        }
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            float2 t[B];
#pragma unroll
            for (int n2 = 0; n2 < B; ++n2) t[n2] = y[n2 * A + k1];
            dftr<B>(t, tw, step * A);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = t[k2];
        }
    }
}

// ---------------------------------------------------------------------------------------------- one stage
// Load / store policies: Load(idx) -> float2 for idx in [0, L); Store(idx, float2).
struct SmemLoad {
    const float2* p;
    __device__ __forceinline__ float2 operator()(int i) const { return p[pad(i)]; }
};
struct SmemStore {
    float2* p;
    __device__ __forceinline__ void operator()(int i, float2 v) const { p[pad(i)] = v; }
};

template <int R, class Load, class Store>
__device__ __forceinline__ void stage(const Load& ld, const Store& st, int L, int Ns, const float2* __restrict__ tw,
                                      int t0, int nt) {
    const int nb = L / R;
    const int tstep = L / (Ns * R);
    const int istep = L / R;
    for (int j = t0; j < nb; j += nt) {
        const int jm = j % Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = ld(j + r * nb);
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = fft::cmul(v[r], __ldg(&tw[r * jm * tstep]));
        }
        dftr<R>(v, tw, istep);
        const int base = (j / Ns) * Ns * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) st(base + r * Ns, v[r]);
    }
}

template <class Load, class Store>
__device__ __forceinline__ void stage_dispatch(int R, const Load& ld, const Store& st, int L, int Ns,
                                               const float2* __restrict__ tw, int t0, int nt) {
    switch (R) {
        case 2: stage<2>(ld, st, L, Ns, tw, t0, nt); break;
        case 3: stage<3>(ld, st, L, Ns, tw, t0, nt); break;
        case 4: stage<4>(ld, st, L, Ns, tw, t0, nt); break;
        case 5: stage<5>(ld, st, L, Ns, tw, t0, nt); break;
        case 6: stage<6>(ld, st, L, Ns, tw, t0, nt); break;
        case 8: stage<8>(ld, st, L, Ns, tw, t0, nt); break;
        case 9: stage<9>(ld, st, L, Ns, tw, t0, nt); break;
        case 10: stage<10>(ld, st, L, Ns, tw, t0, nt); break;
        case 12: stage<12>(ld, st, L, Ns, tw, t0, nt); break;
        case 15: stage<15>(ld, st, L, Ns, tw, t0, nt); break;
        default: stage<16>(ld, st, L, Ns, tw, t0, nt); break;
    }
}

// Whole forward transform: first stage reads with `first`, last stage writes with `last`, intermediate stages
// ping-pong between the padded shared buffers a and b. `sync` synchronises the participating threads.
// Returns nothing: the result is wherever `last` put it. Inverse transforms conjugate in `first` and `last`.
template <class First, class Last, class Sync>
__device__ __forceinline__ void transform(const Plan& p, const First& first, const Last& last, float2* a, float2* b,
                                          const float2* __restrict__ tw, int t0, int nt, Sync sync) {
    int Ns = 1;
    if (p.n == 1) {
        stage_dispatch(p.R[0], first, last, p.L, 1, tw, t0, nt);
        return;
    }
    stage_dispatch(p.R[0], first, SmemStore{a}, p.L, Ns, tw, t0, nt);
    sync();
    Ns *= p.R[0];
    float2* src = a;
    float2* dst = b;
    for (int s = 1; s < p.n - 1; ++s) {
        stage_dispatch(p.R[s], SmemLoad{src}, SmemStore{dst}, p.L, Ns, tw, t0, nt);
        sync();
        Ns *= p.R[s];
        float2* t = src; src = dst; dst = t;
    }
    stage_dispatch(p.R[p.n - 1], SmemLoad{src}, last, p.L, Ns, tw, t0, nt);
}

}  // namespace fft2
}  // namespace mgb
