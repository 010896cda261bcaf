// FFT-interpolated repulsion without any device allocation: mg_fftconv_compute_noalloc.
//
// The same kernels as FFTConv2D.compute (spread, row FFTs, column FFTs with the kernel products and the FP64 Z,
// inverse row FFTs, gather), run on scratch carved out of one file-scope device array instead of the buffers of
// an mg_fftconv object. The array is sized for FFT sides up to kNoallocMaxM; larger grids are rejected. Its
// address is taken once per device with cudaGetSymbolAddress, by the first call on that device. Nothing here
// calls cudaMalloc, cudaFree or any other allocating routine, and no host array is staged: every array argument
// must already be device memory. There is one scratch per device, so calls whose work overlaps on the device
// (two streams, or two host threads) race on it.
#include "common.cuh"
#include "fftrep.cuh"
#include "fft.cuh"
#include <mutex>
#include <string>

namespace mgb {

namespace {

constexpr int kNoallocMaxM = 512;                           // largest FFT side (so N = n_boxes * n_interp <= 512)
constexpr int kMh = kNoallocMaxM / 2 + 1;                   // half-spectrum columns
constexpr int kNp = (kNoallocMaxM + 3) & ~3;                // rows rounded up to 4, as RepBuffers::alloc rounds
static_assert(kNp % 4 == 0, "the transposed spectra are written in 32-byte groups of 4 rows");
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// scratch layout (byte offsets), the same buffers RepBuffers holds for Nmax = Mmax = kNoallocMaxM
constexpr size_t kGridOff = 0;
constexpr size_t kWOff = kGridOff + align256(sizeof(GridDesc));
constexpr size_t kWBytes = (size_t)kNoallocMaxM * kNoallocMaxM * sizeof(float4);
constexpr size_t kWhOff = kWOff + align256(kWBytes);
constexpr size_t kWhBytes = (size_t)3 * kMh * kNp * sizeof(float2);
constexpr size_t kPhOff = kWhOff + align256(kWhBytes);
constexpr size_t kPhBytes = (size_t)4 * kMh * kNp * sizeof(float2);
constexpr size_t kPhiOff = kPhOff + align256(kPhBytes);
constexpr size_t kPhiBytes = (size_t)4 * kNoallocMaxM * kNoallocMaxM * sizeof(float);
constexpr size_t kKtOff = kPhiOff + align256(kPhiBytes);
constexpr size_t kKtBytes = (size_t)2 * kMh * kNoallocMaxM * sizeof(float);
constexpr size_t kTwOff = kKtOff + align256(kKtBytes);
constexpr size_t kTwBytes = (size_t)kNoallocMaxM * sizeof(float2);
constexpr size_t kZOff = kTwOff + align256(kTwBytes);
constexpr size_t kZBytes = (size_t)kMh * sizeof(double);
constexpr size_t kScratchBytes = kZOff + align256(kZBytes);   // 16.8 MB

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// once per device: the device address of the scratch array
unsigned char* scratch_for_current_device() {
    int dev = 0;
    MGB_CUDA(cudaGetDevice(&dev));
    require(dev >= 0 && dev < kMaxDevices, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            throw Error(MG_ERR_DEVICE, std::string("cudaGetSymbolAddress of the scratch failed: ") +
                                           cudaGetErrorString(e));
        }
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    return g_scratch_addr[dev];
}

// RepBuffers over the scratch: it borrows the memory and gives it back untouched (never frees it)
struct ScratchView {
    RepBuffers rb;
    explicit ScratchView(unsigned char* base, int ni) {
        rb.Nmax = kNoallocMaxM; rb.Mmax = kNoallocMaxM; rb.Mhmax = kMh; rb.Npmax = kNp; rb.ni = ni;
        lend(rb.W, base + kWOff, kWBytes);
        lend(rb.WhT, base + kWhOff, kWhBytes);
        lend(rb.PhT, base + kPhOff, kPhBytes);
        lend(rb.phi, base + kPhiOff, kPhiBytes);
        lend(rb.Kt, base + kKtOff, kKtBytes);
        lend(rb.tw, base + kTwOff, kTwBytes);
        lend(rb.zpart, base + kZOff, kZBytes);
    }
    ~ScratchView() {
        for (DevBuf* d : {&rb.W, &rb.WhT, &rb.PhT, &rb.phi, &rb.Kt, &rb.tw, &rb.zpart}) { d->p = nullptr; d->bytes = 0; }
    }
    static void lend(DevBuf& d, unsigned char* p, size_t bytes) { d.p = p; d.bytes = bytes; }
};

__global__ void noalloc_read_sumq_kernel(const GridDesc* g, float* out) { *out = g->sumQ_f; }

// device memory of the current device: a pointer into another GPU's memory would be read by this device's
// kernels through peer access, or fault without it
void require_device(const void* p, const char* what) {
    require(is_device_ptr(p), std::string(what) + " must be device memory (this entry point stages nothing)");
    cudaPointerAttributes a;
    int dev = 0;
    MGB_CUDA(cudaGetDevice(&dev));
    MGB_CUDA(cudaPointerGetAttributes(&a, p));
    require(a.type == cudaMemoryTypeManaged || a.device == dev,
            std::string(what) + " is memory of device " + std::to_string(a.device) + ", not of the current device " +
                std::to_string(dev));
}

}  // namespace

int noalloc_max_fft_side() { return kNoallocMaxM; }

void fftconv_compute_noalloc(const float* K1h, const float* K2h, int M, int n_interp, const float* Y, int64_t n,
                             float xmin, float ymin, float width, int n_boxes, float* sumQ, float* F) {
    require(M >= 2 && fft::is_5smooth(M), "M must be a 5-smooth FFT size >= 2 (2^a 3^b 5^c)");
    require(M <= kNoallocMaxM, "M = " + std::to_string(M) + " exceeds the maximum FFT side " +
                                   std::to_string(kNoallocMaxM) + " of the allocation-free scratch");
    require(n_interp >= 1 && n_interp <= 8, "n_interp must be between 1 and 8");
    require(n >= 0, "Y must be (n, 2)");
    require(n_boxes >= 1 && (int64_t)n_boxes * n_interp <= M && width > 0, "grid larger than the buffer");
    require(K1h && K2h && sumQ && (n == 0 || (Y && F)), "arrays must not be NULL");
    require_device(K1h, "K1h");
    require_device(K2h, "K2h");
    require_device(sumQ, "sumQ");
    if (n > 0) {
        require_device(Y, "Y");
        require_device(F, "F");
        require(((uintptr_t)Y & 7) == 0 && ((uintptr_t)F & 7) == 0, "Y and F must be 8-byte aligned");
    }
    unsigned char* base = scratch_for_current_device();
    cudaStream_t s = current_stream();
    ScratchView v(base, n_interp);
    GridDesc* g = reinterpret_cast<GridDesc*>(base + kGridOff);
    // what must start at zero: the grid descriptor (last-block counter, flags) and the rows of W the spread uses.
    // The forward row pass clears every W row it reads, so after a completed call these rows are zero already;
    // they are cleared here all the same, so that a call that stopped part-way (an error between two launches)
    // leaves nothing behind for the next one, at the price of one pass over N x 512 float4 per call.
    const int N = n_boxes * n_interp;
    MGB_CUDA(cudaMemsetAsync(g, 0, sizeof(GridDesc), s));
    MGB_CUDA(cudaMemsetAsync(base + kWOff, 0, (size_t)N * kNoallocMaxM * sizeof(float4), s));
    rep_set_grid_host(g, xmin, ymin, width, n_boxes, n_interp, M, s);
    rep_twiddles(g, v.rb, s, true);
    rep_set_spectra_from_host_layout(v.rb, K1h, K2h, M, s);
    const float2* Yd = reinterpret_cast<const float2*>(Y);
    if (n > 0) rep_spread(Yd, n, g, v.rb, s);
    rep_convolve(g, v.rb, n, s);
    if (n > 0) rep_gather_forces(Yd, n, g, v.rb, reinterpret_cast<float2*>(F), s);
    noalloc_read_sumq_kernel<<<1, 1, 0, s>>>(g, sumQ);
    MGB_LAUNCH_CHECK();
}

}  // namespace mgb
