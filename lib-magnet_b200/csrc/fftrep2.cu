// FFT convolution of the repulsion pass on the register-tiled engine (fft2.cuh): the forward row transforms,
// the column pass (forward transform, product with the kernel spectra, inverse transform, Z by Parseval) and
// the inverse row transforms, plus the kernel spectra of the device loop. Same data layout and results as the
// kernels of fftrep.cu (which stay as the path for FFT sides the register-tiled engine cannot hold); the stages
// read their first input from global memory and write their last output to global memory directly.
//
// Reference: FFTConv2D::compute, src/fftconv.cpp:124-199 (r2c rows, c2c columns, products, inverse c2c, c2r).
#include "fftrep.cuh"
#include "fft2.cuh"
#include <vector>

namespace mgb {

namespace {

constexpr int kT = 256;

struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

__device__ __forceinline__ float chan(const float4& v, int c) { return c == 0 ? v.x : (c == 1 ? v.y : v.z); }

// -------------------------------------------------------------------------------------------- load / store
// two real W rows of channel c as one complex sequence, zero padded to M
struct RowPairLoad {
    const float4* r0; const float4* r1; int N; int c; bool has1;
    __device__ __forceinline__ float2 operator()(int i) const {
        if (i >= N) return make_float2(0.f, 0.f);
        return make_float2(chan(r0[i], c), has1 ? chan(r1[i], c) : 0.f);
    }
};
// a column of row spectra, zero padded
struct ColLoad {
    const float2* p; int N;
    __device__ __forceinline__ float2 operator()(int i) const { return i < N ? p[i] : make_float2(0.f, 0.f); }
};
// spectrum x real kernel, conjugated (inverse through the forward transform)
struct SpecKLoad {
    const float2* S; const float* K;
    __device__ __forceinline__ float2 operator()(int i) const {
        const float2 s = S[fft2::pad(i)];
        const float k = __ldg(&K[i]);
        return make_float2(s.x * k, -(s.y * k));
    }
};
// the first N outputs of an inverse transform, conjugated back
struct ColStoreConj {
    float2* p; int N;
    __device__ __forceinline__ void operator()(int i, float2 v) const { if (i < N) p[i] = make_float2(v.x, -v.y); }
};
// Hermitian rebuild of two real rows from their half spectra (transposed layout), conjugated for the inverse
struct RowPairSpecLoad {
    const float2* base; int Np; int Mhmax; int g0; int M; int Mh; bool even;
    __device__ __forceinline__ float2 operator()(int k) const {
        const int kk = k < Mh ? k : M - k;
        const float4 v = *reinterpret_cast<const float4*>(base + (size_t)kk * Np + g0);
        float2 a = make_float2(v.x, v.y), b = make_float2(v.z, v.w);
        if (kk == 0 || (even && kk == M / 2)) { a.y = 0.f; b.y = 0.f; }
        if (k >= Mh) { a.y = -a.y; b.y = -b.y; }
        return make_float2(a.x - b.y, -(a.y + b.x));
    }
};
// the N live outputs of the inverse row transform: row g0 = Re, row g1 = -Im, scaled
struct RowPairStore {
    float* r0; float* r1; int N; float scale; bool has1;
    __device__ __forceinline__ void operator()(int i, float2 v) const {
        if (i >= N) return;
        r0[i] = v.x * scale;
        if (has1) r1[i] = -v.y * scale;
    }
};
// K1 + i K2 on the wrapped offsets of row a (magnet/tsne.py:57-67)
struct KernelRowLoad {
    int M; double oa; double delta; double dof;
    __device__ __forceinline__ float2 operator()(int b) const {
        const double ob = (double)(b <= M / 2 ? b : b - M) * delta;
        const double base = 1.0 + (oa * oa + ob * ob) / dof;
        if (dof == 1.0) return make_float2((float)(1.0 / base), (float)pow(base, -2.0));
        return make_float2((float)pow(base, -dof), (float)pow(base, -dof - 1.0));
    }
};
struct MirrorColLoad {
    const float2* p; int M;
    __device__ __forceinline__ float2 operator()(int a) const { return p[a <= M / 2 ? a : M - a]; }
};
struct RealStore {
    float* p;
    __device__ __forceinline__ void operator()(int i, float2 v) const { p[i] = v.x; }
};

// -------------------------------------------------------------------------------------------- kernels
__global__ void __launch_bounds__(kT, 2) row_fwd2_kernel(const GridDesc* __restrict__ gd, float4* __restrict__ W,
                                                      int pitchW, float2* __restrict__ WhT, int Np, int Mhmax,
                                                      const float2* __restrict__ tw,
                                                      const fft2::Plan* __restrict__ plans) {
    extern __shared__ float2 sm[];
    const int N = gd->N, M = gd->M, Mh = gd->Mh;
    const fft2::Plan plan = plans[M];
    const int P = fft2::padded_len(M);
    float2* R = sm;
    float2* A = sm + P;
    float2* B = sm + 2 * P;
    const int npairs = (N + 1) / 2;
    for (int rp = blockIdx.x; rp < npairs; rp += gridDim.x) {
        const int g0 = 2 * rp, g1 = 2 * rp + 1;
        const bool has1 = g1 < N;
        for (int c = 0; c < 3; ++c) {
            fft2::transform(plan, RowPairLoad{W + (size_t)g0 * pitchW, W + (size_t)(has1 ? g1 : g0) * pitchW, N, c, has1},
                            fft2::SmemStore{R}, A, B, tw, threadIdx.x, blockDim.x, BlockSync());
            __syncthreads();
            for (int k = threadIdx.x; k < Mh; k += blockDim.x) {
                const float2 zk = R[fft2::pad(k)], zm = R[fft2::pad(k == 0 ? 0 : M - k)];
                const float4 v = make_float4(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y),
                                             0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
                *reinterpret_cast<float4*>(WhT + ((size_t)c * Mhmax + k) * Np + g0) = v;
            }
            __syncthreads();
        }
        const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int b = threadIdx.x; b < N; b += blockDim.x) {
            W[(size_t)g0 * pitchW + b] = z4;
            if (has1) W[(size_t)g1 * pitchW + b] = z4;
        }
    }
}

__global__ void __launch_bounds__(kT, 2) col2_kernel(GridDesc* __restrict__ gd, const float2* __restrict__ WhT,
                                                  float2* __restrict__ PhT, int Np, int Mhmax,
                                                  const float* __restrict__ Kt, int Mmax,
                                                  const float2* __restrict__ tw, double* __restrict__ zpart,
                                                  int64_t n_points, const fft2::Plan* __restrict__ plans) {
    extern __shared__ float2 sm[];
    __shared__ double red[kT / 32];
    __shared__ int is_last;
    const int N = gd->N, M = gd->M, Mh = gd->Mh;
    const fft2::Plan plan = plans[M];
    const int P = fft2::padded_len(M);
    float2* S = sm;
    float2* A = sm + P;
    float2* B = sm + 2 * P;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = blockIdx.x; k < Mh; k += gridDim.x) {
        const float* K1 = Kt + (size_t)k * Mmax;
        const float* K2 = Kt + ((size_t)Mhmax + k) * Mmax;
        for (int c = 0; c < 3; ++c) {
            fft2::transform(plan, ColLoad{WhT + ((size_t)c * Mhmax + k) * Np, N}, fft2::SmemStore{S}, A, B, tw,
                            threadIdx.x, blockDim.x, BlockSync());
            __syncthreads();
            if (c == 0) {
                double zs = 0.0;
                for (int a = threadIdx.x; a < M; a += blockDim.x) {
                    const float2 r = S[fft2::pad(a)];
                    zs += (double)__ldg(&K1[a]) * ((double)r.x * r.x + (double)r.y * r.y);
                }
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
            }
            // outputs of this channel: 0 -> (0: K1, 1: K2), 1 -> 2: K2, 2 -> 3: K2
            const int n_out = c == 0 ? 2 : 1;
            for (int o = 0; o < n_out; ++o) {
                const int out = c == 0 ? o : c + 1;
                const float* K = (c == 0 && o == 0) ? K1 : K2;
                fft2::transform(plan, SpecKLoad{S, K}, ColStoreConj{PhT + ((size_t)out * Mhmax + k) * Np, N}, A, B,
                                tw, threadIdx.x, blockDim.x, BlockSync());
                __syncthreads();
            }
        }
    }
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

__global__ void __launch_bounds__(kT, 2) row_inv2_kernel(const GridDesc* __restrict__ gd,
                                                      const float2* __restrict__ PhT, int Np, int Mhmax,
                                                      float* __restrict__ phi, int pitchP,
                                                      const float2* __restrict__ tw,
                                                      const fft2::Plan* __restrict__ plans) {
    extern __shared__ float2 sm[];
    const int N = gd->N, M = gd->M, Mh = gd->Mh;
    const fft2::Plan plan = plans[M];
    const int P = fft2::padded_len(M);
    float2* A = sm;
    float2* B = sm + P;
    const float scale = 1.f / ((float)M * (float)M);
    const bool even = (M & 1) == 0;
    const int npairs = (N + 1) / 2;
    const size_t plane = (size_t)pitchP * pitchP;
    for (int rp = blockIdx.x; rp < npairs; rp += gridDim.x) {
        const int g0 = 2 * rp, g1 = 2 * rp + 1;
        const bool has1 = g1 < N;
        for (int c = 0; c < 4; ++c) {
            fft2::transform(plan, RowPairSpecLoad{PhT + (size_t)c * Mhmax * Np, Np, Mhmax, g0, M, Mh, even},
                            RowPairStore{phi + c * plane + (size_t)g0 * pitchP, phi + c * plane + (size_t)(has1 ? g1 : g0) * pitchP,
                                         N, scale, has1},
                            A, B, tw, threadIdx.x, blockDim.x, BlockSync());
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(kT, 2) spec_rows2_kernel(const GridDesc* __restrict__ gd, float2* __restrict__ Rt,
                                                        int Pa, int Mhmax, const float2* __restrict__ tw, int ni,
                                                        double dof, const fft2::Plan* __restrict__ plans) {
    if (!gd->spec_dirty) return;
    extern __shared__ float2 sm[];
    const int M = gd->M, Mh = gd->Mh;
    const fft2::Plan plan = plans[M];
    const int P = fft2::padded_len(M);
    float2* R = sm;
    float2* A = sm + P;
    float2* B = sm + 2 * P;
    const double delta = gd->spec_width / (double)ni;
    const int nrows = M / 2 + 1;
    for (int a = blockIdx.x; a < nrows; a += gridDim.x) {
        const double oa = (double)(a <= M / 2 ? a : a - M) * delta;
        fft2::transform(plan, KernelRowLoad{M, oa, delta, dof}, fft2::SmemStore{R}, A, B, tw, threadIdx.x,
                        blockDim.x, BlockSync());
        __syncthreads();
        for (int k = threadIdx.x; k < Mh; k += blockDim.x) {
            const float2 zk = R[fft2::pad(k)], zm = R[fft2::pad(k == 0 ? 0 : M - k)];
            Rt[(size_t)k * Pa + a] = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
            Rt[((size_t)Mhmax + k) * Pa + a] = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kT, 2) spec_cols2_kernel(const GridDesc* __restrict__ gd,
                                                        const float2* __restrict__ Rt, int Pa, int Mhmax,
                                                        float* __restrict__ Kt, int Mmax,
                                                        const float2* __restrict__ tw,
                                                        const fft2::Plan* __restrict__ plans) {
    if (!gd->spec_dirty) return;
    extern __shared__ float2 sm[];
    const int M = gd->M, Mh = gd->Mh;
    const fft2::Plan plan = plans[M];
    const int P = fft2::padded_len(M);
    float2* A = sm;
    float2* B = sm + P;
    for (int w = blockIdx.x; w < 2 * Mh; w += gridDim.x) {
        const int kern = w / Mh, k = w % Mh;
        fft2::transform(plan, MirrorColLoad{Rt + ((size_t)kern * Mhmax + k) * Pa, M},
                        RealStore{Kt + ((size_t)kern * Mhmax + k) * Mmax}, A, B, tw, threadIdx.x, blockDim.x,
                        BlockSync());
        __syncthreads();
    }
}

int blocks2(int work) { return std::max(1, std::min(work, 2 * kNumSMs)); }

}  // namespace

// dynamic shared memory limit of a kernel: the device's opt-in maximum per block minus the kernel's static share
static void raise_smem(const void* fn, int optin) {
    cudaFuncAttributes a;
    MGB_CUDA(cudaFuncGetAttributes(&a, fn));
    MGB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)a.sharedSizeBytes));
}

void ensure_fft2_attrs() {
    static int done_dev = -1;
    int dev = 0;
    MGB_CUDA(cudaGetDevice(&dev));
    if (done_dev == dev) return;
    int optin = 0;
    MGB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    raise_smem((const void*)row_fwd2_kernel, optin);
    raise_smem((const void*)col2_kernel, optin);
    raise_smem((const void*)row_inv2_kernel, optin);
    raise_smem((const void*)spec_rows2_kernel, optin);
    raise_smem((const void*)spec_cols2_kernel, optin);
    done_dev = dev;
}

// the register-tiled engine holds 3 padded sequences of length Mmax per block (1 KB left for static shared data)
bool fft2_fits(int Mmax) { return (size_t)3 * fft2::padded_len(Mmax) * sizeof(float2) <= (size_t)226 * 1024; }

void fft2_build_plans(DevBuf& table, int Mmax) {
    std::vector<fft2::Plan> plans((size_t)Mmax + 1);
    for (int L = 0; L <= Mmax; ++L) {
        fft2::Plan p{};
        if (!fft2::make_plan(L, p)) { p.L = L; p.n = 0; }
        plans[L] = p;
    }
    table.ensure(plans.size() * sizeof(fft2::Plan));
    MGB_CUDA(cudaMemcpy(table.p, plans.data(), plans.size() * sizeof(fft2::Plan), cudaMemcpyHostToDevice));
}

void rep_convolve2(GridDesc* g, RepBuffers& b, int64_t n, cudaStream_t s, cudaEvent_t* ev) {
    const int P = fft2::padded_len(b.Mmax);
    const size_t smem3 = (size_t)3 * P * sizeof(float2), smem2 = (size_t)2 * P * sizeof(float2);
    const fft2::Plan* plans = b.plans.as<fft2::Plan>();
    const int pairs = (b.Nmax + 1) / 2;
    row_fwd2_kernel<<<blocks2(pairs), kT, smem3, s>>>(g, b.W.as<float4>(), b.Nmax, b.WhT.as<float2>(), b.Npmax,
                                                      b.Mhmax, b.tw.as<float2>(), plans);
    MGB_LAUNCH_CHECK();
    if (ev) MGB_CUDA(cudaEventRecord(ev[0], s));
    col2_kernel<<<blocks2(b.Mhmax), kT, smem3, s>>>(g, b.WhT.as<float2>(), b.PhT.as<float2>(), b.Npmax, b.Mhmax,
                                                    b.Kt.as<float>(), b.Mmax, b.tw.as<float2>(), b.zpart.as<double>(),
                                                    n, plans);
    MGB_LAUNCH_CHECK();
    if (ev) MGB_CUDA(cudaEventRecord(ev[1], s));
    row_inv2_kernel<<<blocks2(pairs), kT, smem2, s>>>(g, b.PhT.as<float2>(), b.Npmax, b.Mhmax, b.phi.as<float>(),
                                                      b.Nmax, b.tw.as<float2>(), plans);
    MGB_LAUNCH_CHECK();
    if (ev) MGB_CUDA(cudaEventRecord(ev[2], s));
}

void rep_update_spectra2(GridDesc* g, RepBuffers& b, float dof, cudaStream_t s) {
    const int Pa = b.Mmax / 2 + 1;
    const int P = fft2::padded_len(b.Mmax);
    const fft2::Plan* plans = b.plans.as<fft2::Plan>();
    spec_rows2_kernel<<<blocks2(Pa), kT, (size_t)3 * P * sizeof(float2), s>>>(g, b.Rt.as<float2>(), Pa, b.Mhmax,
                                                                             b.tw.as<float2>(), b.ni, (double)dof, plans);
    MGB_LAUNCH_CHECK();
    spec_cols2_kernel<<<blocks2(2 * b.Mhmax), kT, (size_t)2 * P * sizeof(float2), s>>>(
        g, b.Rt.as<float2>(), Pa, b.Mhmax, b.Kt.as<float>(), b.Mmax, b.tw.as<float2>(), plans);
    MGB_LAUNCH_CHECK();
}

}  // namespace mgb
