// In-place mixed-radix FFT engine of the repulsion pass: decimation in frequency forward, decimation in time
// inverse, so that a convolution never reorders its spectrum.
//
// A transform of length M = R_1 R_2 ... R_S (2 <= S <= 4, every R_s in {2, 3, 4, 5, 6, 8, 9, 10, 12, 15, 16,
// 18, 20}) runs as S stages over one shared-memory buffer. Stage s splits every block of length Lp = R_s ... R_S
// into Ls = Lp / R_s butterflies; butterfly j of a block at u = blk Lp + j takes the R_s elements at u + Ls r,
// applies a DFT_{R_s} in registers, multiplies output q by exp(-2 pi i j q / Lp) and writes it back to u + Ls q.
// After the last stage the element at position p = sum_s q_s (R_{s+1} ... R_S) is the spectrum at the
// digit-reversed frequency f = sum_s q_s (R_1 ... R_{s-1}). The inverse runs the stages backwards (conjugate
// twiddles, then the inverse DFT), so a convolution is: forward stages 1..S-1, the last forward stage, the
// product with the kernel spectrum and the first inverse stage in the same registers, inverse stages S-1..1.
// The first forward stage can read global memory directly (zero padding past the live length) and the last
// inverse stage can write global memory directly, which leaves 2 (S - 1) shared-memory round trips per
// convolution.
//
// Twiddles between stages come from one table read per butterfly (powers by products). Bank conflicts: stages
// before the last read consecutive positions across threads; the last stage reads R_S
// consecutive positions per thread. When R_S is even the buffer inserts one slot every R_S elements
// (pad(i) = i + i / R_S), which makes that stride odd.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <utility>
#include <type_traits>
#include "fft.cuh"

namespace mgb {
namespace fft3 {

constexpr int kMaxStages = 4;
constexpr int kMaxRadix = 20;

struct Stage {
    int R;          // radix
    int Lp;         // block length before the stage
    int Ls;         // butterflies per block (block length after the stage)
    int nb;         // butterflies over the whole sequence, M / R
    int tws;        // twiddle table step, M / Lp
    int ps;         // padded distance between the R elements of a butterfly
    unsigned mLs;   // floor(x / Ls) = umulhi(x, mLs) (Ls >= 2)
};

struct Plan {
    int M;
    int S;          // number of stages (0: no plan)
    int padR;       // last radix when it is even (padding on), else 0
    unsigned mpad;  // floor(x / padR) = umulhi(x, mpad)
    int Mp;         // padded buffer length
    unsigned mR[kMaxStages];   // floor(x / R_s) = umulhi(x, mR[s])
    Stage st[kMaxStages];
};

// floor(x / d) = umulhi(x, magic_div(d)) for 2 <= d and x d < 2^32
__host__ __device__ inline unsigned magic_div(int d) {
    return d >= 2 ? (unsigned)((0x100000000ULL + (unsigned long long)d - 1) / (unsigned long long)d) : 0u;
}

// Host side: fewest stages; then the last radix odd (no padding); then the smallest largest radix; then the
// largest last radix (least padding).
inline bool plan_search(int L, int depth, int* cur, int* best, int& best_n, int& best_key) {
    static const int rad[] = {20, 18, 16, 15, 12, 10, 9, 8, 6, 5, 4, 3, 2};
    if (L == 1) {
        if (depth < 2) return false;
        int mx = 0;
        for (int s = 0; s < depth; ++s) mx = cur[s] > mx ? cur[s] : mx;
        const int last = cur[depth - 1];
        const int key = ((last & 1) ? 0 : 10000) + 100 * mx + (100 - last);
        if (depth < best_n || (depth == best_n && key < best_key)) {
            best_n = depth; best_key = key;
            for (int s = 0; s < depth; ++s) best[s] = cur[s];
        }
        return true;
    }
    if (depth >= kMaxStages) return false;
    bool any = false;
    for (int r : rad) {
        if (L % r) continue;
        cur[depth] = r;
        any |= plan_search(L / r, depth + 1, cur, best, best_n, best_key);
    }
    return any;
}

inline bool make_plan(int M, Plan& p) {
    p = Plan{};
    p.M = M;
    if (M < 4 || M > fft::kMaxLen || !fft::is_5smooth(M)) return false;
    int cur[kMaxStages], best[kMaxStages];
    int best_n = kMaxStages + 1, best_key = 1 << 30;
    plan_search(M, 0, cur, best, best_n, best_key);
    if (best_n > kMaxStages) return false;
    p.S = best_n;
    const int RS = best[best_n - 1];
    p.padR = (RS & 1) ? 0 : RS;
    p.mpad = magic_div(p.padR);
    p.Mp = p.padR ? M + (M - 1) / p.padR + 1 : M;
    int Lp = M;
    for (int s = 0; s < best_n; ++s) {
        Stage& st = p.st[s];
        st.R = best[s];
        st.Lp = Lp;
        st.Ls = Lp / st.R;
        st.nb = M / st.R;
        st.tws = M / Lp;
        st.ps = p.padR ? st.Ls + st.Ls / p.padR : st.Ls;
        st.mLs = magic_div(st.Ls);
        p.mR[s] = magic_div(st.R);
        Lp = st.Ls;
    }
    return true;
}

__device__ __forceinline__ int udiv(int x, unsigned m) { return (int)__umulhi((unsigned)x, m); }

// ---------------------------------------------------------------------------------------------- codelets
// exp(-2 pi i m / R) as compile-time constants: a Taylor series in double, evaluated by the compiler
constexpr double kPi = 3.14159265358979323846;
constexpr double cx_sin_series(double x) {
    double term = x, sum = x;
    for (int k = 1; k < 30; ++k) {
        term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
        sum += term;
    }
    return sum;
}
constexpr double cx_cos_series(double x) {
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 30; ++k) {
        term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
        sum += term;
    }
    return sum;
}
// cos(2 pi m / R), sin(2 pi m / R), exact at multiples of pi / 2, the angle reduced to (-pi, pi]
constexpr double cx_cos(int m, int R) {
    m %= R;
    if (4 * m == R || 4 * m == 3 * R) return 0.0;
    if (2 * m == R) return -1.0;
    if (m == 0) return 1.0;
    return cx_cos_series(2.0 * kPi * (double)(2 * m > R ? m - R : m) / (double)R);
}
constexpr double cx_sin(int m, int R) {
    m %= R;
    if (m == 0 || 2 * m == R) return 0.0;
    if (4 * m == R) return 1.0;
    if (4 * m == 3 * R) return -1.0;
    return cx_sin_series(2.0 * kPi * (double)(2 * m > R ? m - R : m) / (double)R);
}

template <class F, int... I>
__device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
__device__ __forceinline__ void static_for(F&& f) {
    static_for_impl(f, std::make_integer_sequence<int, N>{});
}

template <int R> struct Split {
    static constexpr int A = (R % 8 == 0 && R != 8) ? (R == 16 ? 4 : 8)
                           : (R % 5 == 0 && R != 5) ? 5 : (R % 4 == 0 && R != 4) ? 4 : (R % 3 == 0 && R != 3) ? 3 : 2;
};

// forward DFT_R in registers: base radices directly, composites R = A B by one Cooley-Tukey split
// (n = B n1 + n2, k = k1 + A k2)
template <int R>
__device__ __forceinline__ void dft_fwd(float2* v) {
    if constexpr (R == 2) fft::dft2(v);
    else if constexpr (R == 3) fft::dft3(v);
    else if constexpr (R == 4) fft::dft4(v);
    else if constexpr (R == 5) fft::dft5(v);
    else if constexpr (R == 8) fft::dft8(v);
    else {
        constexpr int A = Split<R>::A, B = R / A;
        float2 y[R];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) {
            float2 t[A];
#pragma unroll
            for (int n1 = 0; n1 < A; ++n1) t[n1] = v[B * n1 + n2];
            dft_fwd<A>(t);
#pragma unroll
            for (int k1 = 0; k1 < A; ++k1) y[n2 * A + k1] = t[k1];
        }
        // twiddles w_R^(n2 k1), folded at compile time
        static_for<B>([&](auto n2c) {
            constexpr int n2 = decltype(n2c)::value;
            static_for<A>([&](auto k1c) {
                constexpr int k1 = decltype(k1c)::value;
                if constexpr (n2 * k1 != 0) {
                    constexpr float c = (float)cx_cos(n2 * k1, R), s = -(float)cx_sin(n2 * k1, R);
                    const float2 a = y[n2 * A + k1];
                    y[n2 * A + k1] = make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
                }
            });
        });
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            float2 t[B];
#pragma unroll
            for (int n2 = 0; n2 < B; ++n2) t[n2] = y[n2 * A + k1];
            dft_fwd<B>(t);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = t[k2];
        }
    }
}

// inverse (unnormalised) DFT_R: conj(DFT(conj(v)))
template <int R>
__device__ __forceinline__ void dft_inv(float2* v) {
#pragma unroll
    for (int r = 0; r < R; ++r) v[r].y = -v[r].y;
    dft_fwd<R>(v);
#pragma unroll
    for (int r = 0; r < R; ++r) v[r].y = -v[r].y;
}

#define MGB_FFT3_RADIX_DISPATCH(R, F, ...)          \
    switch (R) {                                    \
        case 2: F<2>(__VA_ARGS__); break;           \
        case 3: F<3>(__VA_ARGS__); break;           \
        case 4: F<4>(__VA_ARGS__); break;           \
        case 5: F<5>(__VA_ARGS__); break;           \
        case 6: F<6>(__VA_ARGS__); break;           \
        case 8: F<8>(__VA_ARGS__); break;           \
        case 9: F<9>(__VA_ARGS__); break;           \
        case 10: F<10>(__VA_ARGS__); break;         \
        case 12: F<12>(__VA_ARGS__); break;         \
        case 15: F<15>(__VA_ARGS__); break;         \
        case 16: F<16>(__VA_ARGS__); break;         \
        case 18: F<18>(__VA_ARGS__); break;         \
        default: F<20>(__VA_ARGS__); break;         \
    }

// v[q] *= w^q for q >= 1 (CONJ: conj(w)^q), w = tw[step]: powers by successive products from one table read,
// re-read from the table every 8 powers so that the rounding of the recurrence stays within a few ulps
template <int R, bool CONJ>
__device__ __forceinline__ void twiddle(float2* v, const float2* __restrict__ tw, int step) {
    float2 w = __ldg(&tw[step]);
    if (CONJ) w.y = -w.y;
    float2 wq = w;
#pragma unroll
    for (int q = 1; q < R; ++q) {
        if (q > 1) {
            if (q % 8 == 0) {
                wq = __ldg(&tw[step * q]);
                if (CONJ) wq.y = -wq.y;
            } else {
                wq = fft::cmul(wq, w);
            }
        }
        v[q] = fft::cmul(v[q], wq);
    }
}

// ---------------------------------------------------------------------------------------------- stages
// Each stage function is compiled once per radix (not inlined), processes one or two buffers in one loop over
// nbuf * M / R butterflies, and is shared by every call site: a plan executes a handful of small functions, which
// keeps the instruction working set of a block inside the instruction cache.

// Butterfly geometry of stage st for butterfly b: its offset j in the block and its padded start.
__device__ __forceinline__ void bfly_at(int padR, unsigned mpad, const Stage& st, int b, int& j, int& base) {
    const int blk = st.Ls > 1 ? udiv(b, st.mLs) : b;
    j = b - blk * st.Ls;
    const int u = blk * st.Lp + j;
    base = padR ? u + udiv(u, mpad) : u;
}

// forward stage 1 from global memory: element n < n_live of transform t read as load(t, n), zero past it
template <int R, class Load>
__device__ __noinline__ void dif_first(const Plan& p, float2* __restrict__ A, float2* __restrict__ B, int nbuf,
                                       Load load, int n_live, const float2* __restrict__ tw) {
    const Stage st = p.st[0];
    const int padR = p.padR;
    const unsigned mpad = p.mpad;
    for (int i = threadIdx.x; i < st.nb * nbuf; i += blockDim.x) {
        const int t = i >= st.nb ? 1 : 0;
        const int b = i - t * st.nb;
        float2* buf = t ? B : A;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int n = b + st.Ls * r;
            v[r] = n < n_live ? load(t, n) : make_float2(0.f, 0.f);
        }
        dft_fwd<R>(v);
        if (b) twiddle<R, false>(v, tw, b);
        const int base = padR ? b + udiv(b, mpad) : b;
#pragma unroll
        for (int q = 0; q < R; ++q) buf[base + st.ps * q] = v[q];
    }
}

// forward stage s (1 <= s < S - 1) over shared memory, in place
template <int R>
__device__ __noinline__ void dif_mid(const Plan& p, int s, float2* __restrict__ A, float2* __restrict__ B, int nbuf,
                                     const float2* __restrict__ tw) {
    const Stage st = p.st[s];
    const int padR = p.padR;
    const unsigned mpad = p.mpad;
    for (int i = threadIdx.x; i < st.nb * nbuf; i += blockDim.x) {
        const int t = i >= st.nb ? 1 : 0;
        float2* buf = t ? B : A;
        int j, base;
        bfly_at(padR, mpad, st, i - t * st.nb, j, base);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = buf[base + st.ps * r];
        dft_fwd<R>(v);
        if (j) twiddle<R, false>(v, tw, st.tws * j);
#pragma unroll
        for (int q = 0; q < R; ++q) buf[base + st.ps * q] = v[q];
    }
}

// inverse stage s (1 <= s < S - 1) over shared memory, in place
template <int R>
__device__ __noinline__ void dit_mid(const Plan& p, int s, float2* __restrict__ A, float2* __restrict__ B, int nbuf,
                                     const float2* __restrict__ tw) {
    const Stage st = p.st[s];
    const int padR = p.padR;
    const unsigned mpad = p.mpad;
    for (int i = threadIdx.x; i < st.nb * nbuf; i += blockDim.x) {
        const int t = i >= st.nb ? 1 : 0;
        float2* buf = t ? B : A;
        int j, base;
        bfly_at(padR, mpad, st, i - t * st.nb, j, base);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = buf[base + st.ps * r];
        if (j) twiddle<R, true>(v, tw, st.tws * j);
        dft_inv<R>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) buf[base + st.ps * r] = v[r];
    }
}

// inverse stage 1 to global memory: element n < n_live of transform t written as store(t, n, value)
template <int R, class Store>
__device__ __noinline__ void dit_last(const Plan& p, const float2* __restrict__ A, const float2* __restrict__ B,
                                      int nbuf, Store store, int n_live, const float2* __restrict__ tw) {
    const Stage st = p.st[0];
    const int padR = p.padR;
    const unsigned mpad = p.mpad;
    for (int i = threadIdx.x; i < st.nb * nbuf; i += blockDim.x) {
        const int t = i >= st.nb ? 1 : 0;
        const int b = i - t * st.nb;
        const float2* buf = t ? B : A;
        const int base = padR ? b + udiv(b, mpad) : b;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = buf[base + st.ps * r];
        if (b) twiddle<R, true>(v, tw, b);
        dft_inv<R>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int n = b + st.Ls * r;
            if (n < n_live) store(t, n, v[r]);
        }
    }
}

// base frequency of last-stage butterfly b: the digits of b (R_1 .. R_{S-1}, last digit least significant)
// reversed into f = sum_s q_s R_1 ... R_{s-1}
__device__ __forceinline__ int base_freq(const Plan& p, int b) {
    int q[kMaxStages] = {0, 0, 0, 0};
    int x = b;
#pragma unroll
    for (int s = kMaxStages - 2; s >= 0; --s) {
        if (s < p.S - 1) {
            const int y = udiv(x, p.mR[s]);
            q[s] = x - y * p.st[s].R;
            x = y;
        }
    }
    int f = 0, w = 1;
#pragma unroll
    for (int s = 0; s < kMaxStages - 1; ++s) {
        if (s < p.S - 1) { f += q[s] * w; w *= p.st[s].R; }
    }
    return f;
}

// frequency held at (unpadded) position pos after the forward stages
__device__ __forceinline__ int freq_of_pos(const Plan& p, int pos) {
    const int RS = p.st[p.S - 1].R;
    const int b = udiv(pos, p.mR[p.S - 1]);
    return base_freq(p, b) + (p.M / RS) * (pos - b * RS);
}

// padded position of frequency f after the forward stages: the digits of f (R_1 least significant) read in
// the opposite order
__device__ __forceinline__ int pos_of_freq(const Plan& p, int f) {
    int q[kMaxStages] = {0, 0, 0, 0};
    int x = f;
#pragma unroll
    for (int s = 0; s < kMaxStages; ++s) {
        if (s < p.S) {
            const int y = udiv(x, p.mR[s]);
            q[s] = x - y * p.st[s].R;
            x = y;
        }
    }
    int pos = q[0];
#pragma unroll
    for (int s = 1; s < kMaxStages; ++s)
        if (s < p.S) pos = pos * p.st[s].R + q[s];
    return p.padR ? pos + udiv(pos, p.mpad) : pos;
}

}  // namespace fft3
}  // namespace mgb
