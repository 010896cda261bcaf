// Spectral initialisation on the device: chebyshev_eigenvectors (src/spectral.cpp:141-241), the Chebyshev-filtered
// subspace iteration with Rayleigh-Ritz of the reference, in FP64 as the reference computes it. The block X is
// n x p, row major (p <= 8 columns), as the reference holds it.
//
// Kernels: the SpMM of the lazy normalised adjacency (a group of lanes per row, one per column, each summing the
// row's entries in order, as src/spectral.cpp:34-48); the deflation of the trivial eigenvector per connected component (per-component sums by
// block reductions and FP64 atomics); block-partial sums of the p x p products X^T B (Gram matrix, Rayleigh
// quotient) and of the Ritz residuals, added on the host in block order; the filter's three-term recurrence, the
// rotation by the Ritz vectors and the Gram-Schmidt updates as elementwise kernels. The small symmetric
// eigenproblem runs on the host.
#include "spectral.cuh"
#include <algorithm>
#include <cmath>
#include <vector>

namespace mgb {
namespace {

constexpr int kSpecThreads = 256;

// blocks of the reductions (their partials go to the host) and of the row-parallel kernels (one row per thread)
int spec_blocks(int64_t rows) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((rows + kSpecThreads - 1) / kSpecThreads, 4 * kNumSMs));
}
int row_blocks(int64_t rows) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((rows + kSpecThreads - 1) / kSpecThreads, 64 * kNumSMs));
}

// the weight of node i on the trivial eigenvector: 1 / sd_i (0 for isolated nodes)
__device__ __forceinline__ double trivial_of(float sd) { return sd > 0.f ? 1.0 / (double)sd : 0.0; }

// out = M in, M = (I + D^-1/2 A D^-1/2) / 2 (src/spectral.cpp:34-48): a group of G lanes per row (G the power of
// two >= P), lane k summing column k over the row's entries in order, as the reference sums it; the group reads a
// neighbour's P values as one contiguous run
template <int P>
__global__ void __launch_bounds__(kSpecThreads) spmm_kernel(const int32_t* __restrict__ indptr,
                                                            const int32_t* __restrict__ indices,
                                                            const float* __restrict__ data,
                                                            const float* __restrict__ sd, int64_t n,
                                                            const double* __restrict__ in, double* __restrict__ out) {
    constexpr int G = P <= 2 ? 2 : (P <= 4 ? 4 : 8);
    const int k = threadIdx.x % G;
    const int64_t groups = (int64_t)gridDim.x * (blockDim.x / G);
    for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G; i < n; i += groups) {
        double acc = 0.0;
        const int32_t e1 = indptr[i + 1];
#pragma unroll 4
        for (int32_t j = indptr[i]; j < e1; ++j) {
            const int32_t col = indices[j];
            const double w = (double)data[j] * (double)sd[col];
            if (k < P) acc += w * in[(int64_t)col * P + k];
        }
        if (k < P) out[i * P + k] = 0.5 * (in[i * P + k] + (double)sd[i] * acc);
    }
}

// per-component sums proj[c][k] = sum over the component's nodes of t_i x_ik (with v == nullptr), or the
// component's sum of t_i^2 (tnorm, P = 1, v = nullptr and squares = true). A block whose rows all lie in one
// component reduces in shared memory and adds once per column; other blocks add per warp group.
template <int P>
__global__ void __launch_bounds__(kSpecThreads) component_sum_kernel(const float* __restrict__ sd,
                                                                     const int32_t* __restrict__ comp, int64_t n,
                                                                     const double* __restrict__ X, bool squares,
                                                                     double* __restrict__ proj) {
    __shared__ double red[kSpecThreads / 32][P];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = base + threadIdx.x;
        const bool act = i < n;
        const int c = act ? comp[i] : -1;
        double v[P];
        const double t = act ? trivial_of(sd[i]) : 0.0;
#pragma unroll
        for (int k = 0; k < P; ++k) v[k] = !act ? 0.0 : (squares ? t * t : t * X[i * P + k]);
        const int c0 = __shfl_sync(0xffffffffu, c, 0);
        const int block_c = comp[base];   // the block's first row (always in range)
        const bool one = __syncthreads_and(!act || c == block_c) != 0;
        if (one) {
#pragma unroll
            for (int k = 0; k < P; ++k) {
                double x = v[k];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                if (lane == 0) red[warp][k] = x;
            }
            __syncthreads();
            if (threadIdx.x < P) {
                double x = 0.0;
                for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += red[w][threadIdx.x];
                atomicAdd(&proj[(int64_t)block_c * P + threadIdx.x], x);
            }
            __syncthreads();
        } else if (__all_sync(0xffffffffu, !act || c == c0)) {
#pragma unroll
            for (int k = 0; k < P; ++k) {
                double x = v[k];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
                if (lane == 0 && c0 >= 0) atomicAdd(&proj[(int64_t)c0 * P + k], x);
            }
        } else if (act) {
#pragma unroll
            for (int k = 0; k < P; ++k) atomicAdd(&proj[(int64_t)c * P + k], v[k]);
        }
    }
}

// x_i -= t_i proj[c_i] / tnorm[c_i] (the per-component projection on the trivial eigenvector removed)
template <int P>
__global__ void __launch_bounds__(kSpecThreads) deflate_apply_kernel(const float* __restrict__ sd,
                                                                     const int32_t* __restrict__ comp, int64_t n,
                                                                     const double* __restrict__ proj,
                                                                     const double* __restrict__ tnorm,
                                                                     double* __restrict__ X) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double t = trivial_of(sd[i]);
        const int c = comp[i];
        const double tn = tnorm[c];
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const double pr = tn > 0.0 ? proj[(int64_t)c * P + k] / tn : 0.0;
            X[i * P + k] -= t * pr;
        }
    }
}

// per-block partial sums of the p x p products: part[b][a * P + c] = sum over the block's rows of A_ia B_ic
template <int P>
__global__ void __launch_bounds__(kSpecThreads) gram_kernel(const double* __restrict__ A,
                                                            const double* __restrict__ B, int64_t n,
                                                            double* __restrict__ part) {
    __shared__ double red[kSpecThreads / 32][P * P];
    double acc[P * P];
#pragma unroll
    for (int q = 0; q < P * P; ++q) acc[q] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double a[P], b[P];
#pragma unroll
        for (int k = 0; k < P; ++k) { a[k] = A[i * P + k]; b[k] = B[i * P + k]; }
#pragma unroll
        for (int r = 0; r < P; ++r)
#pragma unroll
            for (int c = 0; c < P; ++c) acc[r * P + c] += a[r] * b[c];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < P * P; ++q) {
        double x = acc[q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp][q] = x;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < P * P; q += blockDim.x) {
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += red[w][q];
        part[(int64_t)blockIdx.x * P * P + q] = x;
    }
}

// per-block partial sums of the Ritz residuals: part[b][c] = sum over the block's rows of (Z_ic - theta_c X_ic)^2
template <int P>
struct Coef {
    double v[P * P];
};

template <int P>
__global__ void __launch_bounds__(kSpecThreads) residual_kernel(const double* __restrict__ X,
                                                                const double* __restrict__ Z, int64_t n, Coef<P> th,
                                                                double* __restrict__ part) {
    __shared__ double red[kSpecThreads / 32][P];
    double acc[P];
#pragma unroll
    for (int k = 0; k < P; ++k) acc[k] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < P; ++k) {
            const double d = Z[i * P + k] - th.v[k] * X[i * P + k];
            acc[k] += d * d;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < P; ++k) {
        double x = acc[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[warp][k] = x;
    }
    __syncthreads();
    if (threadIdx.x < P) {
        double x = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += red[w][threadIdx.x];
        part[(int64_t)blockIdx.x * P + threadIdx.x] = x;
    }
}

// X <- X V (V p x p, row major: new column c = sum_k X_k V[k][c])
template <int P>
__global__ void __launch_bounds__(kSpecThreads) rotate_kernel(double* __restrict__ X, int64_t n, Coef<P> V) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double x[P];
#pragma unroll
        for (int k = 0; k < P; ++k) x[k] = X[i * P + k];
#pragma unroll
        for (int c = 0; c < P; ++c) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < P; ++k) s += x[k] * V.v[k * P + c];
            X[i * P + c] = s;
        }
    }
}

// column k of X: X_k <- (X_k - sum_{j < k} coef_j X_j) * scale
template <int P>
__global__ void __launch_bounds__(kSpecThreads) column_update_kernel(double* __restrict__ X, int64_t n, int k,
                                                                     Coef<P> coef, double scale) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        double x = X[i * P + k];
        for (int j = 0; j < k; ++j) x -= coef.v[j] * X[i * P + j];
        X[i * P + k] = x * scale;
    }
}

// the filter's recurrence, elementwise over the n p entries: first Y = (Y - c X) s1, then
// Ynew = (Ynew - c Y) s2 - ss X (src/spectral.cpp:215-229)
__global__ void cheb_first_kernel(double* __restrict__ Y, const double* __restrict__ X, int64_t count, double c,
                                  double s1) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        Y[i] = (Y[i] - c * X[i]) * s1;
}

__global__ void cheb_next_kernel(double* __restrict__ Ynew, const double* __restrict__ Y,
                                 const double* __restrict__ X, int64_t count, double c, double s2, double ss) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        Ynew[i] = (Ynew[i] - c * Y[i]) * s2 - ss * X[i];
}

__global__ void widen_kernel(const float* __restrict__ in, double* __restrict__ out, int64_t count) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

__global__ void narrow_kernel(const double* __restrict__ in, float* __restrict__ out, int64_t count) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}

// the solver for a block of P columns; the steps and the stopping rule of src/spectral.cpp:172-238
template <int P>
struct Solver {
    const int32_t* indptr; const int32_t* indices; const float* data; const float* sd; const int32_t* comp;
    int64_t n; int n_comp; int blocks; int rblocks; int sblocks; cudaStream_t s;
    double* proj; const double* tnorm; double* part;
    std::vector<double> host_part;

    void spmm(const double* in, double* out) {
        spmm_kernel<P><<<sblocks, kSpecThreads, 0, s>>>(indptr, indices, data, sd, n, in, out);
        MGB_LAUNCH_CHECK();
    }
    void deflate(double* X) {
        MGB_CUDA(cudaMemsetAsync(proj, 0, sizeof(double) * (size_t)n_comp * P, s));
        component_sum_kernel<P><<<rblocks, kSpecThreads, 0, s>>>(sd, comp, n, X, false, proj);
        MGB_LAUNCH_CHECK();
        deflate_apply_kernel<P><<<rblocks, kSpecThreads, 0, s>>>(sd, comp, n, proj, tnorm, X);
        MGB_LAUNCH_CHECK();
    }
    // the p x p matrix A^T B, its block partials added on the host in block order (the same bits every call)
    std::vector<double> gram(const double* A, const double* B) {
        gram_kernel<P><<<blocks, kSpecThreads, 0, s>>>(A, B, n, part);
        MGB_LAUNCH_CHECK();
        host_part.resize((size_t)blocks * P * P);
        MGB_CUDA(cudaMemcpyAsync(host_part.data(), part, sizeof(double) * host_part.size(), cudaMemcpyDeviceToHost, s));
        MGB_CUDA(cudaStreamSynchronize(s));
        std::vector<double> G((size_t)P * P, 0.0);
        for (int b = 0; b < blocks; ++b)
            for (int q = 0; q < P * P; ++q) G[q] += host_part[(size_t)b * P * P + q];
        return G;
    }
    // Gram-Schmidt of the P columns, each column against the ones before it, twice over (as the reference's two
    // passes of modified Gram-Schmidt): the projections of a column on the earlier ones are taken together
    // (classical Gram-Schmidt, the second pass restoring the orthogonality the first leaves), then its norm
    void orthonormalize(double* X) {
        for (int pass = 0; pass < 2; ++pass)
            for (int k = 0; k < P; ++k) {
                Coef<P> c{};
                if (k > 0) {
                    const std::vector<double> G = gram(X, X);
                    for (int j = 0; j < k; ++j) c.v[j] = G[(size_t)k * P + j];
                    column_update_kernel<P><<<rblocks, kSpecThreads, 0, s>>>(X, n, k, c, 1.0);
                    MGB_LAUNCH_CHECK();
                }
                const std::vector<double> G = gram(X, X);
                const double nrm = G[(size_t)k * P + k];
                const double inv = nrm > 1e-300 ? 1.0 / std::sqrt(nrm) : 0.0;
                column_update_kernel<P><<<rblocks, kSpecThreads, 0, s>>>(X, n, k, Coef<P>{}, inv);
                MGB_LAUNCH_CHECK();
            }
    }
    // Rayleigh-Ritz: Z = M X deflated, H = X^T Z (its upper triangle mirrored), H = V diag(theta) V^T, X and Z
    // rotated by V; returns the largest residual norm |Z_c - theta_c X_c| over the wanted columns
    double rayleigh_ritz(double* X, double* Z, int n_wanted, std::vector<double>& theta) {
        spmm(X, Z);
        deflate(Z);
        std::vector<double> H = gram(X, Z);
        for (int a = 0; a < P; ++a)
            for (int b = a + 1; b < P; ++b) H[(size_t)b * P + a] = H[(size_t)a * P + b];
        std::vector<double> V;
        symmetric_eigen(H, P, theta, V);
        Coef<P> v{};
        for (int q = 0; q < P * P; ++q) v.v[q] = V[q];
        rotate_kernel<P><<<rblocks, kSpecThreads, 0, s>>>(X, n, v);
        MGB_LAUNCH_CHECK();
        rotate_kernel<P><<<rblocks, kSpecThreads, 0, s>>>(Z, n, v);
        MGB_LAUNCH_CHECK();
        Coef<P> th{};
        for (int c = 0; c < P; ++c) th.v[c] = theta[c];
        residual_kernel<P><<<blocks, kSpecThreads, 0, s>>>(X, Z, n, th, part);
        MGB_LAUNCH_CHECK();
        host_part.resize((size_t)blocks * P);
        MGB_CUDA(cudaMemcpyAsync(host_part.data(), part, sizeof(double) * host_part.size(), cudaMemcpyDeviceToHost, s));
        MGB_CUDA(cudaStreamSynchronize(s));
        double worst = 0.0;
        for (int c = 0; c < n_wanted; ++c) {
            double r = 0.0;
            for (int b = 0; b < blocks; ++b) r += host_part[(size_t)b * P + c];
            worst = std::max(worst, std::sqrt(r));
        }
        return worst;
    }

    void run(float* Xout, int n_wanted, int degree, int max_iter, double tol, SpecWork& w) {
        const int64_t cnt = n * P;
        double* X = static_cast<double*>(w.X.ensure(sizeof(double) * (size_t)cnt));
        double* Z = static_cast<double*>(w.Z.ensure(sizeof(double) * (size_t)cnt));
        double* Y = static_cast<double*>(w.Y.ensure(sizeof(double) * (size_t)cnt));
        double* Yn = static_cast<double*>(w.Ynew.ensure(sizeof(double) * (size_t)cnt));
        const int eb = row_blocks(cnt);
        widen_kernel<<<eb, kSpecThreads, 0, s>>>(Xout, X, cnt);
        MGB_LAUNCH_CHECK();
        deflate(X);
        orthonormalize(X);
        std::vector<double> theta;
        double res = rayleigh_ritz(X, Z, n_wanted, theta);
        double prev_sum = -1.0;
        for (int it = 0; it < max_iter; ++it) {
            // stop when the residual is small against the gap after the wanted Ritz values (floored at 1e-3), or
            // when the wanted Ritz values no longer move (src/spectral.cpp:196-203)
            const double gap = std::max(theta[n_wanted - 1] - theta[n_wanted], 1e-3);
            double sum = 0.0;
            for (int c = 0; c < n_wanted; ++c) sum += theta[c];
            const bool stagnant = prev_sum >= 0 && std::fabs(sum - prev_sum) < 1e-9 * (double)n_wanted;
            if (res < tol * gap || res < 1e-9 || stagnant) break;
            prev_sum = sum;
            // the Chebyshev filter damping [0, alpha] (the scaled three-term recurrence of Zhou and Saad,
            // src/spectral.cpp:205-231)
            double alpha = theta[P - 1];
            alpha = std::min(alpha, theta[n_wanted - 1] - 0.5 * gap);
            alpha = std::max(alpha, 1e-3);
            const double a0 = std::min(1.0, theta[0] + 1e-9);
            const double e = 0.5 * alpha, cc = 0.5 * alpha;
            const double sigma1 = e / (a0 - cc);
            double sigma = sigma1;
            spmm(X, Y);
            deflate(Y);
            cheb_first_kernel<<<eb, kSpecThreads, 0, s>>>(Y, X, cnt, cc, sigma1 / e);
            MGB_LAUNCH_CHECK();
            for (int k = 2; k <= degree; ++k) {
                const double sigma_new = 1.0 / (2.0 / sigma1 - sigma);
                spmm(Y, Yn);
                deflate(Yn);
                cheb_next_kernel<<<eb, kSpecThreads, 0, s>>>(Yn, Y, X, cnt, cc, 2.0 * sigma_new / e, sigma * sigma_new);
                MGB_LAUNCH_CHECK();
                // X <- Y, Y <- Ynew: the previous iterate becomes the recurrence's X, as the reference copies it
                std::swap(X, Y);
                std::swap(Y, Yn);
                sigma = sigma_new;
            }
            MGB_CUDA(cudaMemcpyAsync(X, Y, sizeof(double) * (size_t)cnt, cudaMemcpyDeviceToDevice, s));
            deflate(X);
            orthonormalize(X);
            res = rayleigh_ritz(X, Z, n_wanted, theta);
        }
        narrow_kernel<<<eb, kSpecThreads, 0, s>>>(X, Xout, cnt);
        MGB_LAUNCH_CHECK();
        MGB_CUDA(cudaStreamSynchronize(s));
    }
};

template <int P>
void run_solver(const int32_t* indptr, const int32_t* indices, const float* data, int64_t n, const float* sd,
                const int32_t* comp, int n_comp, float* X, int n_wanted, int degree, int max_iter, double tol,
                SpecWork& w, cudaStream_t s) {
    Solver<P> sv;
    sv.indptr = indptr; sv.indices = indices; sv.data = data; sv.sd = sd; sv.comp = comp;
    sv.n = n; sv.n_comp = n_comp; sv.s = s;
    sv.blocks = spec_blocks(n);
    sv.rblocks = row_blocks(n);
    sv.sblocks = row_blocks(n * (P <= 2 ? 2 : (P <= 4 ? 4 : 8)));   // a group of lanes per row
    sv.proj = static_cast<double*>(w.proj.ensure(sizeof(double) * (size_t)n_comp * P));
    double* tn = static_cast<double*>(w.tnorm.ensure(sizeof(double) * (size_t)n_comp));
    sv.part = static_cast<double*>(w.part.ensure(sizeof(double) * (size_t)sv.blocks * P * P));
    // tnorm[c] = sum over the component of t_i^2
    MGB_CUDA(cudaMemsetAsync(tn, 0, sizeof(double) * (size_t)n_comp, s));
    component_sum_kernel<1><<<sv.rblocks, kSpecThreads, 0, s>>>(sd, comp, n, nullptr, true, tn);
    MGB_LAUNCH_CHECK();
    sv.tnorm = tn;
    sv.run(X, n_wanted, degree, max_iter, tol, w);
}

}  // namespace

// cyclic Jacobi rotations (Golub and Van Loan, Matrix Computations, section 8.5): each sweep zeroes the off-diagonal
// entries (i, j), i < j, in row order with the rotation whose tangent is the smaller root of
// t^2 + 2 theta t - 1 = 0, theta = (a_jj - a_ii) / (2 a_ij); sweeps stop once the squared off-diagonal sum is
// below 1e-22, as the reference's solver stops (src/spectral.cpp:87-123)
void symmetric_eigen(std::vector<double> A, int p, std::vector<double>& vals, std::vector<double>& V) {
    V.assign((size_t)p * p, 0.0);
    for (int i = 0; i < p; ++i) V[(size_t)i * p + i] = 1.0;
    auto at = [&](int r, int c) -> double& { return A[(size_t)r * p + c]; };
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < p; ++i)
            for (int j = i + 1; j < p; ++j) off += at(i, j) * at(i, j);
        if (off < 1e-22) break;
        for (int i = 0; i < p; ++i)
            for (int j = i + 1; j < p; ++j) {
                const double aij = at(i, j);
                if (std::fabs(aij) < 1e-300) continue;
                const double theta = (at(j, j) - at(i, i)) / (2.0 * aij);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
                for (int r = 0; r < p; ++r) {   // A <- A J (columns i and j)
                    const double x = at(r, i), y = at(r, j);
                    at(r, i) = c * x - sn * y;
                    at(r, j) = sn * x + c * y;
                }
                for (int r = 0; r < p; ++r) {   // A <- J^T A (rows i and j)
                    const double x = at(i, r), y = at(j, r);
                    at(i, r) = c * x - sn * y;
                    at(j, r) = sn * x + c * y;
                }
                for (int r = 0; r < p; ++r) {   // V <- V J
                    const double x = V[(size_t)r * p + i], y = V[(size_t)r * p + j];
                    V[(size_t)r * p + i] = c * x - sn * y;
                    V[(size_t)r * p + j] = sn * x + c * y;
                }
            }
    }
    std::vector<int> order(p);
    for (int i = 0; i < p; ++i) order[i] = i;
    std::vector<double> d(p);
    for (int i = 0; i < p; ++i) d[i] = at(i, i);
    std::sort(order.begin(), order.end(), [&](int a, int b) { return d[a] > d[b]; });
    vals.resize(p);
    std::vector<double> W((size_t)p * p);
    for (int c = 0; c < p; ++c) {
        vals[c] = d[order[c]];
        for (int r = 0; r < p; ++r) W[(size_t)r * p + c] = V[(size_t)r * p + order[c]];
    }
    V.swap(W);
}

void chebyshev_eigenvectors_dev(const int32_t* indptr, const int32_t* indices, const float* data, int64_t n,
                                const float* sd, const int32_t* comp, int n_comp, float* X, int p, int n_wanted,
                                int degree, int max_iter, double tol, SpecWork& w, cudaStream_t s) {
    switch (p) {
        case 2: run_solver<2>(indptr, indices, data, n, sd, comp, n_comp, X, n_wanted, degree, max_iter, tol, w, s); break;
        case 3: run_solver<3>(indptr, indices, data, n, sd, comp, n_comp, X, n_wanted, degree, max_iter, tol, w, s); break;
        case 4: run_solver<4>(indptr, indices, data, n, sd, comp, n_comp, X, n_wanted, degree, max_iter, tol, w, s); break;
        case 5: run_solver<5>(indptr, indices, data, n, sd, comp, n_comp, X, n_wanted, degree, max_iter, tol, w, s); break;
        case 6: run_solver<6>(indptr, indices, data, n, sd, comp, n_comp, X, n_wanted, degree, max_iter, tol, w, s); break;
        case 7: run_solver<7>(indptr, indices, data, n, sd, comp, n_comp, X, n_wanted, degree, max_iter, tol, w, s); break;
        case 8: run_solver<8>(indptr, indices, data, n, sd, comp, n_comp, X, n_wanted, degree, max_iter, tol, w, s); break;
        default: throw Error(MG_ERR_NOT_SUPPORTED, "the device solver takes 2 to 8 columns");
    }
}

}  // namespace mgb
