// Box location and Lagrange interpolation weights of the FFT repulsion, shared by the spread, the gather and
// the fused t-SNE iteration kernel.
#pragma once
#include <cuda_runtime.h>

namespace mgb {

// Lagrange weights of the n_interp equispaced nodes of a box (nodes at (k + 1/2) / n_interp), as
// lagrange_w, src/fftconv.cpp:24-40 (closed form with constant denominators for 3 nodes)
template <int NI>
__device__ __forceinline__ void lagrange_w(float u, float* w) {
    if (NI == 3) {
        const float a = u - 1.f / 6.f, b = u - 0.5f, c = u - 5.f / 6.f;
        w[0] = b * c * 4.5f; w[1] = -a * c * 9.f; w[2] = a * b * 4.5f;
        return;
    }
#pragma unroll
    for (int k = 0; k < NI; ++k) {
        const float uk = (k + 0.5f) / NI;
        float num = 1.f, den = 1.f;
#pragma unroll
        for (int m = 0; m < NI; ++m) {
            if (m == k) continue;
            const float um = (m + 0.5f) / NI;
            num = __fmul_rn(num, u - um); den = __fmul_rn(den, uk - um);
        }
        w[k] = num / den;
    }
}

// Box and weights of a point exactly as FFTConv2D::compute finds them: the x-box by the reciprocal of the
// width (the counting sort, src/fftconv.cpp:85-88), the y-box and both local coordinates by division (:106-111)
template <int NI>
__device__ __forceinline__ void locate(float x, float y, float xmin, float ymin, float width, float inv_w, int nb,
                                       int& bx, int& by, float* wx, float* wy) {
    bx = min(nb - 1, max(0, (int)(__fmul_rn(x - xmin, inv_w))));
    const float ux = (x - xmin) / width, uy = (y - ymin) / width;
    by = min(nb - 1, max(0, (int)uy));
    lagrange_w<NI>(fminf(1.f, fmaxf(0.f, ux - (float)bx)), wx);
    lagrange_w<NI>(fminf(1.f, fmaxf(0.f, uy - (float)by)), wy);
}

}  // namespace mgb
