// Shared definitions of the B200 layout-pass library: status codes and the thread-local error message, CUDA
// error checks, the device RNG, small device helpers and a grow-only device workspace.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <stdexcept>
#include <functional>

#include "../../include/magnet_b200.h"

namespace mgb {

// ------------------------------------------------------------------------------------------------ errors
// Internal code throws mgb::Error; the C-ABI layer converts it into a status code and a thread-local message
// (the reference raises std::runtime_error from `require`, src/layout.hpp:34; the pybind11 shim rethrows the
// message as RuntimeError so callers see the same exception type and text).
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void require(bool ok, const std::string& msg) {
    if (!ok) throw Error(MG_ERR_ARGUMENT, msg);
}
// the message is built only on failure (the host-side checks run once per edge on host arrays)
inline void require(bool ok, const char* msg) {
    if (!ok) throw Error(MG_ERR_ARGUMENT, msg);
}

#define MGB_CUDA(call)                                                                                    \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) {                                                                          \
            cudaGetLastError(); /* a non-sticky error must not surface again at the next check */        \
            throw ::mgb::Error(e_ == cudaErrorMemoryAllocation ? MG_ERR_OUT_OF_MEMORY : MG_ERR_DEVICE,    \
                               std::string(#call) + ": " + cudaGetErrorString(e_));                      \
        }                                                                                                 \
    } while (0)

// every kernel launch of the library is followed by MGB_LAUNCH_CHECK, which also counts it (mg_launch_count)
void count_launch(uint64_t k = 1);
uint64_t launch_count();
#define MGB_LAUNCH_CHECK()                  \
    do {                                    \
        MGB_CUDA(cudaGetLastError());       \
        ::mgb::count_launch();              \
    } while (0)

constexpr int kMaxDim = 64;      // same bound as the reference's MAX_DIM (src/layout.hpp:17)
constexpr int kNumSMs = 148;     // B200

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

// ------------------------------------------------------------------------------------------------ RNG
// xorshift64* with splitmix64 seeding: the generator of the reference (src/rng.hpp:5-28), kept bit-identical
// because the sampled negatives must match it.
struct Rng {
    uint64_t s;
    __host__ __device__ __forceinline__ explicit Rng(uint64_t seed) {
        uint64_t z = seed + 0x9E3779B97F4A7C15ULL;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        s = (z ^ (z >> 31)) | 1ULL;
    }
    __host__ __device__ __forceinline__ uint64_t next() {
        s ^= s >> 12;
        s ^= s << 25;
        s ^= s >> 27;
        return s * 0x2545F4914F6CDD1DULL;
    }
    __host__ __device__ __forceinline__ uint32_t below(uint32_t n) {
        return (uint32_t)(((next() >> 32) * (uint64_t)n) >> 32);
    }
    __host__ __device__ __forceinline__ float uniform() {
        return (float)(next() >> 40) * (1.0f / 16777216.0f);
    }
};

// Per-stream seed of an epoch (src/layout.cpp:123). The reference's hogwild threads use tid = thread index;
// the counter-based streams of this library use tid = edge index (one independent stream per edge and epoch).
__host__ __device__ __forceinline__ uint64_t stream_seed(uint64_t seed, int epoch, uint64_t tid) {
    return seed * 0x9E3779B1ULL + (uint64_t)epoch * 0x85EBCA6BULL + tid * 0xC2B2AE35ULL;
}

// ------------------------------------------------------------------------------------------------ workspace
// Grow-only device buffer (the reference's FFTConv2D keeps persistent buffers for the same reason: no
// allocation per call).
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void* ensure(size_t n) {
        if (n <= bytes && p) return p;
        release();
        size_t want = n < 256 ? 256 : n;
        MGB_CUDA(cudaMalloc(&p, want));
        bytes = want;
        return p;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// True when ptr is device (or managed) memory this process can use directly in kernels.
inline bool is_device_ptr(const void* ptr) {
    if (!ptr) return false;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, ptr);
    if (e != cudaSuccess) { cudaGetLastError(); return false; }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Current stream of the calling host thread (mg_set_stream).
cudaStream_t current_stream();

// Runs f with the C ABI's error convention: MG_OK, or the error's code with its message kept for mg_last_error().
int guard_call(const std::function<void()>& f);

}  // namespace mgb
