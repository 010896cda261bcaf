// Shared-memory FFT engine of the repulsion pass (replaces the vendored pocketfft of the reference,
// src/pocketfft_hdronly.h as used by src/fftconv.cpp:124-199).
//
// Complex float32 transforms of any 5-smooth length L (L = 2^a 3^b 5^c, as scipy's next_fast_len(real=True)
// returns them), executed by one thread block out of shared memory: Stockham auto-sort, one radix-R stage per
// pass over a ping-pong pair of buffers, radices 8/4/2/3/5 with butterflies held in registers. Twiddles come
// from a per-length table exp(-2 pi i m / L) computed in FP64 and rounded once (tw_table_kernel).
//
// Stage (radix R, Ns = product of the radices already applied, j in [0, L/R)):
//   v[r] = src[j + r L/R] * w^(r (j mod Ns) L/(Ns R)),  v = DFT_R(v),
//   dst[(j / Ns) Ns R + (j mod Ns) + r Ns] = v[r]
// which leaves the transform in natural order after the last stage.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace mgb {
namespace fft {

constexpr int kMaxStages = 24;
constexpr int kMaxLen = 13500;        // 2 x 108 KB ping-pong buffers per block

struct Plan {
    int L;
    int n;                 // number of stages
    uint8_t radix[kMaxStages];
};

// Factorisation into stages; returns false when L is not 5-smooth (or out of range).
__host__ __device__ inline bool make_plan(int L, Plan& p) {
    p.L = L; p.n = 0;
    if (L < 1 || L > kMaxLen) return false;
    int x = L, a = 0, b = 0, c = 0;
    while (x % 2 == 0) { x /= 2; ++a; }
    while (x % 3 == 0) { x /= 3; ++b; }
    while (x % 5 == 0) { x /= 5; ++c; }
    if (x != 1) return false;
    while (a >= 3) { p.radix[p.n++] = 8; a -= 3; }
    if (a == 2) p.radix[p.n++] = 4;
    if (a == 1) p.radix[p.n++] = 2;
    for (int i = 0; i < c; ++i) p.radix[p.n++] = 5;
    for (int i = 0; i < b; ++i) p.radix[p.n++] = 3;
    return true;
}

__host__ __device__ inline bool is_5smooth(int L) {
    if (L < 1) return false;
    while (L % 2 == 0) L /= 2;
    while (L % 3 == 0) L /= 3;
    while (L % 5 == 0) L /= 5;
    return L == 1;
}

// ----------------------------------------------------------------------------------------------- complex ops
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }   // -i * a
__device__ __forceinline__ float2 mul_pi(float2 a) { return make_float2(-a.y, a.x); }   // +i * a
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// ----------------------------------------------------------------------------------------------- butterflies
// forward DFTs, y_k = sum_n x_n exp(-2 pi i n k / R)
__device__ __forceinline__ void dft2(float2* v) {
    const float2 a = v[0], b = v[1];
    v[0] = cadd(a, b); v[1] = csub(a, b);
}
__device__ __forceinline__ void dft3(float2* v) {
    const float s3 = 0.86602540378443864676f;
    const float2 t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    const float2 m = make_float2(v[0].x - 0.5f * t1.x, v[0].y - 0.5f * t1.y);
    const float2 r = cscale(mul_mi(t2), s3);       // -i sqrt(3)/2 (x1 - x2)
    v[0] = cadd(v[0], t1);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
}
__device__ __forceinline__ void dft4(float2* v) {
    const float2 a = cadd(v[0], v[2]), b = csub(v[0], v[2]);
    const float2 c = cadd(v[1], v[3]), d = mul_mi(csub(v[1], v[3]));
    v[0] = cadd(a, c); v[2] = csub(a, c);
    v[1] = cadd(b, d); v[3] = csub(b, d);
}
__device__ __forceinline__ void dft5(float2* v) {
    const float c1 = 0.30901699437494742410f, c2 = -0.80901699437494742410f;
    const float s1 = 0.95105651629515357212f, s2 = 0.58778525229247312917f;
    const float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    const float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    const float2 x0 = v[0];
    const float2 a1 = make_float2(x0.x + c1 * t1.x + c2 * t2.x, x0.y + c1 * t1.y + c2 * t2.y);
    const float2 a2 = make_float2(x0.x + c2 * t1.x + c1 * t2.x, x0.y + c2 * t1.y + c1 * t2.y);
    const float2 b1 = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
    const float2 b2 = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
    v[0] = cadd(x0, cadd(t1, t2));
    v[1] = cadd(a1, mul_mi(b1)); v[4] = csub(a1, mul_mi(b1));
    v[2] = cadd(a2, mul_mi(b2)); v[3] = csub(a2, mul_mi(b2));
}
__device__ __forceinline__ void dft8(float2* v) {
    const float h = 0.70710678118654752440f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    dft4(e); dft4(o);
    // o_k *= w8^k, w8 = exp(-i pi/4)
    o[1] = make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    o[2] = mul_mi(o[2]);
    o[3] = make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
#pragma unroll
    for (int k = 0; k < 4; ++k) { v[k] = cadd(e[k], o[k]); v[k + 4] = csub(e[k], o[k]); }
}

template <int R> __device__ __forceinline__ void dft(float2* v);
template <> __device__ __forceinline__ void dft<2>(float2* v) { dft2(v); }
template <> __device__ __forceinline__ void dft<3>(float2* v) { dft3(v); }
template <> __device__ __forceinline__ void dft<4>(float2* v) { dft4(v); }
template <> __device__ __forceinline__ void dft<5>(float2* v) { dft5(v); }
template <> __device__ __forceinline__ void dft<8>(float2* v) { dft8(v); }

// One Stockham stage over the whole sequence by threads [t0, t0 + nt) of the block.
template <int R>
__device__ __forceinline__ void stage(const float2* __restrict__ src, float2* __restrict__ dst, int L, int Ns,
                                      const float2* __restrict__ tw, int t0, int nt) {
    const int nb = L / R;
    const int tstep = L / (Ns * R);
    for (int j = t0; j < nb; j += nt) {
        const int jm = j % Ns;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[j + r * nb];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = cmul(v[r], __ldg(&tw[r * jm * tstep]));
        }
        dft<R>(v);
        const int base = (j / Ns) * Ns * R + jm;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];
    }
}

// Forward transform of buf[0..L) using tmp[0..L) as the other ping-pong buffer, by threads [t0, t0+nt) of the
// calling block; `sync` must synchronise exactly those threads (the whole block when nt = blockDim.x).
// Returns the buffer that holds the result (buf or tmp).
template <class Sync>
__device__ float2* forward(float2* buf, float2* tmp, const Plan& p, const float2* __restrict__ tw, int t0, int nt,
                           Sync sync) {
    float2* src = buf;
    float2* dst = tmp;
    int Ns = 1;
    for (int s = 0; s < p.n; ++s) {
        const int R = p.radix[s];
        switch (R) {
            case 8: stage<8>(src, dst, p.L, Ns, tw, t0, nt); break;
            case 4: stage<4>(src, dst, p.L, Ns, tw, t0, nt); break;
            case 2: stage<2>(src, dst, p.L, Ns, tw, t0, nt); break;
            case 5: stage<5>(src, dst, p.L, Ns, tw, t0, nt); break;
            default: stage<3>(src, dst, p.L, Ns, tw, t0, nt); break;
        }
        Ns *= R;
        sync();
        float2* t = src; src = dst; dst = t;
    }
    return src;
}

}  // namespace fft
}  // namespace mgb
