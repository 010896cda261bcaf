// Column pass of the FFT repulsion on the in-place engine (fft3.cuh): src/fftconv.cpp:146-186 (forward column
// transforms, products with the real kernel spectra, inverse column transforms) and the FP64 Z of :226-229.
//
// One block per column k of the row half-spectra (persistent over columns). Two shared-memory buffers hold two
// transforms at once:
//   phase 1: channels 1 and 2 (x W, y W), each times K2, into outputs 2 and 3;
//   phase 2: channel 0 (W) once forward; its spectrum times K1 (output 0, and sum K1 |W0h|^2 for Z) and times K2
//            (output 1) leave the middle stage in the two buffers.
// The first forward stage reads the live rows (g < N) of WhT from global memory, the last inverse stage writes
// the live rows of PhT, so a column costs 2 (S - 1) shared-memory passes per transform and no reordering pass.
// Output convention as the one-radix engine: PhT = unnormalised inverse (M x the circular convolution).
#include "fftrep.cuh"
#include "fft3.cuh"
#include <vector>
#include <algorithm>

namespace mgb {

namespace {

constexpr int kColThreads = 256;

// transform t of a column pass reads / writes column k of channel a (t = 0) or b (t = 1)
struct ColLoad {
    const float2* a;
    const float2* b;
    __device__ __forceinline__ float2 operator()(int t, int n) const { return (t ? b : a)[n]; }
};
struct ColStore {
    float2* a;
    float2* b;
    __device__ __forceinline__ void operator()(int t, int n, float2 v) const { (t ? b : a)[n] = v; }
};

// last forward stage, product with one real kernel spectrum, first inverse stage (in place), on nbuf buffers
template <int R>
__device__ __noinline__ void middle1(const fft3::Plan& p, float2* __restrict__ A, float2* __restrict__ B, int nbuf,
                                     const float* __restrict__ K) {
    const int pb = p.padR ? R + 1 : R;
    const int nb = p.M / R;
    for (int i = threadIdx.x; i < nb * nbuf; i += blockDim.x) {
        const int t = i >= nb ? 1 : 0;
        const int b = i - t * nb;
        float2* buf = t ? B : A;
        const int base = b * pb;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = buf[base + r];
        fft3::dft_fwd<R>(v);
        const int fb = fft3::base_freq(p, b);
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = fft::cscale(v[q], __ldg(&K[fb + nb * q]));
        fft3::dft_inv<R>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) buf[base + r] = v[r];
    }
}

// channel 0: one spectrum (in A), two products (K1 into A, K2 into B); returns this thread's share of
// sum K1 |X|^2
template <int R>
__device__ __noinline__ double middle2(const fft3::Plan& p, float2* __restrict__ A, float2* __restrict__ B,
                                       const float* __restrict__ K1, const float* __restrict__ K2) {
    const int pb = p.padR ? R + 1 : R;
    const int nb = p.M / R;
    double zs = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        const int base = b * pb;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = A[base + r];
        fft3::dft_fwd<R>(v);
        const int fb = fft3::base_freq(p, b);
        // the K1 product waits in A (same positions, this thread only) while the K2 product is inverted, so that
        // one spectrum at a time is live in registers
        float zt = 0.f;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const float k1 = __ldg(&K1[fb + nb * q]);
            zt += k1 * (v[q].x * v[q].x + v[q].y * v[q].y);
            A[base + q] = fft::cscale(v[q], k1);
        }
        zs += (double)zt;
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = fft::cscale(v[q], __ldg(&K2[fb + nb * q]));
        fft3::dft_inv<R>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) B[base + r] = v[r];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = A[base + r];
        fft3::dft_inv<R>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) A[base + r] = v[r];
    }
    return zs;
}

__device__ __forceinline__ double middle2_dispatch(int R, const fft3::Plan& p, float2* A, float2* B, const float* K1,
                                                   const float* K2) {
    switch (R) {
        case 2: return middle2<2>(p, A, B, K1, K2);
        case 3: return middle2<3>(p, A, B, K1, K2);
        case 4: return middle2<4>(p, A, B, K1, K2);
        case 5: return middle2<5>(p, A, B, K1, K2);
        case 6: return middle2<6>(p, A, B, K1, K2);
        case 8: return middle2<8>(p, A, B, K1, K2);
        case 9: return middle2<9>(p, A, B, K1, K2);
        case 10: return middle2<10>(p, A, B, K1, K2);
        case 12: return middle2<12>(p, A, B, K1, K2);
        case 15: return middle2<15>(p, A, B, K1, K2);
        case 16: return middle2<16>(p, A, B, K1, K2);
        case 18: return middle2<18>(p, A, B, K1, K2);
        default: return middle2<20>(p, A, B, K1, K2);
    }
}

__global__ void __launch_bounds__(kColThreads, 2) col3_kernel(GridDesc* __restrict__ gd,
                                                              const fft3::Plan* __restrict__ plans,
                                                              const float2* __restrict__ WhT, float2* __restrict__ PhT,
                                                              int Np, int Mhmax, const float* __restrict__ Kt, int Mmax,
                                                              const float2* __restrict__ tw,
                                                              double* __restrict__ zpart, int64_t n_points) {
    extern __shared__ float2 sm[];
    __shared__ fft3::Plan p;
    __shared__ double red[kColThreads / 32];
    __shared__ int is_last;
    const int N = gd->N, M = gd->M, Mh = gd->Mh;
    if (threadIdx.x == 0) p = plans[M];
    __syncthreads();
    float2* A = sm;
    float2* B = sm + p.Mp;
    const int S = p.S;
    const int R0 = p.st[0].R, RS = p.st[S - 1].R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = blockIdx.x; k < Mh; k += gridDim.x) {
        const float2* src[3];
        float2* dst[4];
#pragma unroll
        for (int c = 0; c < 3; ++c) src[c] = WhT + ((size_t)c * Mhmax + k) * Np;
#pragma unroll
        for (int o = 0; o < 4; ++o) dst[o] = PhT + ((size_t)o * Mhmax + k) * Np;
        const float* K1 = Kt + (size_t)k * Mmax;
        const float* K2 = Kt + ((size_t)Mhmax + k) * Mmax;
        // ---- phase 1: channels 1 and 2, times K2, into outputs 2 and 3
        MGB_FFT3_RADIX_DISPATCH(R0, fft3::dif_first, p, A, B, 2, ColLoad{src[1], src[2]}, N, tw);
        __syncthreads();
        for (int s = 1; s < S - 1; ++s) {
            MGB_FFT3_RADIX_DISPATCH(p.st[s].R, fft3::dif_mid, p, s, A, B, 2, tw);
            __syncthreads();
        }
        MGB_FFT3_RADIX_DISPATCH(RS, middle1, p, A, B, 2, K2);
        __syncthreads();
        for (int s = S - 2; s >= 1; --s) {
            MGB_FFT3_RADIX_DISPATCH(p.st[s].R, fft3::dit_mid, p, s, A, B, 2, tw);
            __syncthreads();
        }
        MGB_FFT3_RADIX_DISPATCH(R0, fft3::dit_last, p, A, B, 2, ColStore{dst[2], dst[3]}, N, tw);
        __syncthreads();
        // ---- phase 2: channel 0, times K1 (and Z) into output 0, times K2 into output 1
        MGB_FFT3_RADIX_DISPATCH(R0, fft3::dif_first, p, A, B, 1, ColLoad{src[0], src[0]}, N, tw);
        __syncthreads();
        for (int s = 1; s < S - 1; ++s) {
            MGB_FFT3_RADIX_DISPATCH(p.st[s].R, fft3::dif_mid, p, s, A, B, 1, tw);
            __syncthreads();
        }
        double zs = middle2_dispatch(RS, p, A, B, K1, K2);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) zs += __shfl_xor_sync(0xffffffffu, zs, o);
        if (lane == 0) red[warp] = zs;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
            const bool single = (k == 0) || ((M & 1) == 0 && k == M / 2);
            zpart[k] = single ? t : 2.0 * t;
        }
        for (int s = S - 2; s >= 1; --s) {
            MGB_FFT3_RADIX_DISPATCH(p.st[s].R, fft3::dit_mid, p, s, A, B, 2, tw);
            __syncthreads();
        }
        MGB_FFT3_RADIX_DISPATCH(R0, fft3::dit_last, p, A, B, 2, ColStore{dst[0], dst[1]}, N, tw);
        __syncthreads();
    }
    // last block: Z = sum of the partials / M^2 - n
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = (atomicAdd(&gd->counter, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double t = 0.0;
    for (int k = threadIdx.x; k < Mh; k += blockDim.x) t += __ldcg(&zpart[k]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) red[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        const double sumQ = s / ((double)M * (double)M) - (double)n_points;
        gd->sumQ = sumQ;
        const float sf = (float)sumQ;
        gd->sumQ_f = sf;
        gd->inv_sumQ = (float)(1.0 / fmax((double)sf, 1e-12));
        gd->counter = 0u;
    }
}

size_t col3_smem(int Mp_max) { return (size_t)2 * Mp_max * sizeof(float2); }

}  // namespace

// Plans of every 5-smooth length up to Mmax (table indexed by M; S = 0 where there is none) and the largest
// padded length among them.
void fft3_build_plans(DevBuf& table, int Mmax, int& Mp_max) {
    std::vector<fft3::Plan> plans((size_t)Mmax + 1);
    Mp_max = 0;
    for (int M = 4; M <= Mmax; ++M) {
        if (!fft::is_5smooth(M)) continue;
        if (fft3::make_plan(M, plans[M])) Mp_max = std::max(Mp_max, plans[M].Mp);
    }
    table.ensure(plans.size() * sizeof(fft3::Plan));
    MGB_CUDA(cudaMemcpy(table.p, plans.data(), plans.size() * sizeof(fft3::Plan), cudaMemcpyHostToDevice));
}

// resident blocks of the column kernel for this buffer size (raises its shared-memory limit once per device)
int col3_blocks(int Mp_max) {
    static int cached_dev = -1, cached_mp = -1, cached_blocks = 0;
    int dev = 0, optin = 0;
    MGB_CUDA(cudaGetDevice(&dev));
    if (cached_dev == dev && cached_mp == Mp_max) return cached_blocks;
    const size_t smem = col3_smem(Mp_max);
    MGB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes a;
    MGB_CUDA(cudaFuncGetAttributes(&a, (const void*)col3_kernel));
    require(smem + a.sharedSizeBytes <= (size_t)optin, "FFT side too large for the column engine");
    MGB_CUDA(cudaFuncSetAttribute((const void*)col3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    MGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, col3_kernel, kColThreads, smem));
    cached_dev = dev;
    cached_mp = Mp_max;
    cached_blocks = std::max(1, per_sm) * kNumSMs;
    return cached_blocks;
}

void rep_col3(GridDesc* g, RepBuffers& b, int64_t n, cudaStream_t s) {
    const int blocks = std::min(col3_blocks(b.Mp3max), b.Mhmax);
    col3_kernel<<<blocks, kColThreads, col3_smem(b.Mp3max), s>>>(
        g, b.plans3.as<fft3::Plan>(), b.WhT.as<float2>(), b.PhT.as<float2>(), b.Npmax, b.Mhmax, b.Kt.as<float>(),
        b.Mmax, b.tw.as<float2>(), b.zpart.as<double>(), n);
    MGB_LAUNCH_CHECK();
}

}  // namespace mgb
