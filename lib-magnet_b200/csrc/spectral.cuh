// Spectral initialisation on the device: the Chebyshev-filtered subspace iteration of the reference's
// chebyshev_eigenvectors (src/spectral.cpp:141-241) for the leading non-trivial eigenvectors of the lazy normalised
// adjacency M = (I + D^-1/2 A D^-1/2) / 2, with the trivial eigenvector deflated per connected component.
#pragma once
#include "common.cuh"
#include <vector>

namespace mgb {

constexpr int kSpecMaxCols = 8;   // columns of the block (n_wanted + extra) the device solver takes

// device scratch of the solver: the block and its filter iterates (n x p FP64 each), per-component sums and
// per-block partial sums
struct SpecWork {
    DevBuf X, Z, Y, Ynew, proj, tnorm, part;
};

// X (n x p, device FP32, in and out): the start block in, the Ritz vectors out (columns by descending Ritz value).
// indptr / indices / data: the graph (device CSR); sd: 1 / sqrt(degree) per node (0 for isolated nodes); comp:
// connected-component labels in [0, n_comp). 2 <= p <= kSpecMaxCols, 1 <= n_wanted < p. Synchronises s.
void chebyshev_eigenvectors_dev(const int32_t* indptr, const int32_t* indices, const float* data, int64_t n,
                                const float* sd, const int32_t* comp, int n_comp, float* X, int p, int n_wanted,
                                int degree, int max_iter, double tol, SpecWork& w, cudaStream_t s);

// the small symmetric eigenproblem of the Rayleigh-Ritz step (host): A (p x p, row major) -> eigenvalues in
// descending order and the eigenvectors as the columns of V (row major)
void symmetric_eigen(std::vector<double> A, int p, std::vector<double>& vals, std::vector<double>& V);

}  // namespace mgb
