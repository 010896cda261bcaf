// FFT-interpolated repulsion on the device (the pass of src/fftconv.cpp:58-230 and magnet/tsne.py:30-90).
//
// HBM layout (N = live grid side = n_boxes * n_interp, M = padded FFT side, Mh = M/2 + 1, Np = N rounded up
// to even):
//   W    float4 [N][N]        spread charges (1, x, y, -) per node, interleaved; zeroed by the forward rows
//   WhT  float2 [3][Mh][Np]   row spectra, transposed (node row index contiguous) for the column pass
//   PhT  float2 [4][Mh][Np]   products after the inverse column transforms, same layout
//   phi  float  [4][N][N]     potentials per channel (planar)
//   Kt   float  [2][Mh][M]    kernel spectra K1h, K2h transposed (k1 contiguous)
//   Rt   float2 [2][Mh][M/2+1] row spectra of the two kernels (spectrum generation only)
//   tw   float2 [M]           exp(-2 pi i m / M), FP64-rounded
// GridDesc is device-resident: the grid choice is made on the device each iteration, so a captured
// iteration needs no host round trip; every pass kernel reads the live sizes from it.
#pragma once
#include "common.cuh"

namespace mgb {

struct GridDesc {
    float xmin, ymin, width, inv_width;
    int n_boxes, N, M, Mh;
    int spec_dirty;           // kernel spectra must be recomputed before the convolution
    double spec_width;        // FP64 box width the spectra are computed for (magnet/tsne.py:57)
    int tw_M;                 // length of the current twiddle table (0 = none)
    int tw_dirty;             // the twiddle table must be recomputed (M changed)
    int key_nb; long long key_w;   // spectrum cache key: (n_boxes, round(width * 1e6)) as magnet/tsne.py:51
    double sumQ;              // FP64 sum of the kernel over all pairs (self terms removed)
    float sumQ_f, inv_sumQ;   // (float)sumQ, (float)(1 / max((double)sumQ_f, 1e-12)) as magnet/tsne.py:177
    float mean[2];            // pending recentring of the layout (t-SNE loop)
    int recentre;             // 1: subtract mean at the next bbox pass
    int iter;                 // iteration counter of the device loop
    unsigned counter;         // last-block counters (reset by the last block)
    unsigned counter2;
};

struct RepBuffers {
    int Nmax = 0, Mmax = 0, Mhmax = 0, Npmax = 0, ni = 3;
    DevBuf W, WhT, PhT, phi, Kt, Rt, tw, zpart, fft_len_table, bbox_part, mean_part;
    int max_bbox_blocks = 0;
    DevBuf plans3;            // in-place engine (fft3.cuh) plans, indexed by M
    int Mp3max = 0;           // its largest padded length up to Mmax
    bool use3 = false;        // the in-place column pass (fftrep3.cu) runs every length these buffers see
    void alloc(int Nmax_, int Mmax_, int ni_);
};

// host-side next_fast_len(target, real=True) of scipy: smallest 5-smooth integer >= target
int next_5smooth(int target);
// smallest 5-smooth length >= target that the in-place engine has a plan for
int next_fft_len(int target);

// kernel launches (all asynchronous on stream s; sizes read from the device GridDesc g)
void rep_set_grid_host(GridDesc* g_dev, float xmin, float ymin, float width, int n_boxes, int ni, int M,
                       cudaStream_t s);
void rep_spread(const float2* Y, int64_t n, GridDesc* g, RepBuffers& b, cudaStream_t s);
void rep_prepare_device_spectra(RepBuffers& b);   // before capture: scratch of the spectrum generation
void rep_update_spectra(GridDesc* g, RepBuffers& b, float dof, cudaStream_t s);
void rep_convolve(GridDesc* g, RepBuffers& b, int64_t n, cudaStream_t s, cudaEvent_t* ev = nullptr);
void rep_gather_forces(const float2* Y, int64_t n, GridDesc* g, RepBuffers& b, float2* F, cudaStream_t s);
void rep_set_spectra_from_host_layout(RepBuffers& b, const float* K1h_dev, const float* K2h_dev, int M,
                                      cudaStream_t s);
void rep_twiddles(GridDesc* g, RepBuffers& b, cudaStream_t s, bool force);   // recompute tw if g->tw_dirty

// allocation-free FFTConv2D.compute on a static scratch (noalloc.cu); device arrays only
int noalloc_max_fft_side();
void fftconv_compute_noalloc(const float* K1h, const float* K2h, int M, int n_interp, const float* Y, int64_t n,
                             float xmin, float ymin, float width, int n_boxes, float* sumQ, float* F);

// in-place engine (fftrep3.cu)
void fft3_build_plans(DevBuf& table, int Mmax, int& Mp_max);
int col3_blocks(int Mp_max);
void fft3_prepare(int Mp_max);
void rep_col3(GridDesc* g, RepBuffers& b, int64_t n, cudaStream_t s);
void rep_row_fwd3(GridDesc* g, RepBuffers& b, cudaStream_t s);
void rep_row_inv3(GridDesc* g, RepBuffers& b, cudaStream_t s);


// the whole t-SNE iteration pieces (tsne.cu)
struct TsneDev;

}  // namespace mgb
