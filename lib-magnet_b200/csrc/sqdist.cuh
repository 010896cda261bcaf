// Squared Euclidean distance in the evaluation order of the reference's host kernels (src/nndescent.cpp:35-116,
// chosen by CPUID at :101-106), so the device reproduces the reference's distances bit for bit on the same host:
//   ORDER 0, the AVX-512 kernel: 16 lanes of fused multiply-adds over whole 16-blocks, the lanes summed high half
//     onto low half down to one, then the tail with fused multiply-adds;
//   ORDER 1, the AVX2 kernel: 8 lanes, the lanes summed ((0+1)+(2+3))+((4+5)+(6+7)), then the tail fused;
//   ORDER 2, the plain loop: 4 interleaved sums without fusion, the tail into the first, (s0+s1)+(s2+s3).
// Every operation is an explicit rounding intrinsic, so the compiler neither fuses nor reorders them.
#pragma once
#include <cuda_runtime.h>

namespace mgb {

template <int ORDER>
__device__ __forceinline__ float sqdist(const float* __restrict__ a, const float* __restrict__ b, int d) {
    if constexpr (ORDER == 2) {
        float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f;
        int i = 0;
        for (; i + 4 <= d; i += 4) {
            const float d0 = __fsub_rn(a[i], b[i]), d1 = __fsub_rn(a[i + 1], b[i + 1]);
            const float d2 = __fsub_rn(a[i + 2], b[i + 2]), d3 = __fsub_rn(a[i + 3], b[i + 3]);
            s0 = __fadd_rn(s0, __fmul_rn(d0, d0)); s1 = __fadd_rn(s1, __fmul_rn(d1, d1));
            s2 = __fadd_rn(s2, __fmul_rn(d2, d2)); s3 = __fadd_rn(s3, __fmul_rn(d3, d3));
        }
        for (; i < d; ++i) { const float df = __fsub_rn(a[i], b[i]); s0 = __fadd_rn(s0, __fmul_rn(df, df)); }
        return __fadd_rn(__fadd_rn(s0, s1), __fadd_rn(s2, s3));
    } else {
        constexpr int L = ORDER == 0 ? 16 : 8;
        float acc[L];
#pragma unroll
        for (int l = 0; l < L; ++l) acc[l] = 0.f;
        int i = 0;
        for (; i + L <= d; i += L) {
#pragma unroll
            for (int l = 0; l < L; ++l) { const float df = __fsub_rn(a[i + l], b[i + l]); acc[l] = __fmaf_rn(df, df, acc[l]); }
        }
        float s;
        if constexpr (ORDER == 0) {
            float t3[8], t6[4];
#pragma unroll
            for (int k = 0; k < 8; ++k) t3[k] = __fadd_rn(acc[8 + k], acc[k]);
#pragma unroll
            for (int k = 0; k < 4; ++k) t6[k] = __fadd_rn(t3[4 + k], t3[k]);
            s = __fadd_rn(__fadd_rn(t6[0], t6[2]), __fadd_rn(t6[1], t6[3]));
        } else {
            s = __fadd_rn(__fadd_rn(__fadd_rn(acc[0], acc[1]), __fadd_rn(acc[2], acc[3])),
                          __fadd_rn(__fadd_rn(acc[4], acc[5]), __fadd_rn(acc[6], acc[7])));
        }
        for (; i < d; ++i) { const float df = __fsub_rn(a[i], b[i]); s = __fmaf_rn(df, df, s); }
        return s;
    }
}

}  // namespace mgb
