// Shared helpers for the lamino_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <stdexcept>
#include <string>

namespace lamino {

// Status codes of the C ABI (mirrored in include/lamino.h).
enum Status : int {
    OK = 0,
    ERR_ARG = 1,
    ERR_OOM = 2,
    ERR_CUDA = 3,
    ERR_CUFFT = 4,
    ERR_TIMEOUT = 5,
    ERR_NONFINITE = 6,
    ERR_STATE = 7,
};

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        int code = (e == cudaErrorMemoryAllocation) ? ERR_OOM : ERR_CUDA;
        throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}
inline void check_cufft(cufftResult r, const char *what) {
    if (r != CUFFT_SUCCESS) {
        int code = (r == CUFFT_ALLOC_FAILED) ? ERR_OOM : ERR_CUFFT;
        throw Error(code, std::string(what) + ": cufft error " + std::to_string((int)r));
    }
}
#define LAMINO_CUDA(x) ::lamino::check_cuda((x), #x)
#define LAMINO_CUFFT(x) ::lamino::check_cufft((x), #x)
#define LAMINO_LAUNCH(what) ::lamino::check_cuda(cudaGetLastError(), what)

inline unsigned grid_for(int64_t n, int block, int64_t cap = 148LL * 64) {
    int64_t g = (n + block - 1) / block;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (unsigned)g;
}

// Owning device buffer (no copy, movable).
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    void alloc(size_t count) {
        release();
        n = count;
        if (count) LAMINO_CUDA(cudaMalloc((void **)&p, count * sizeof(T)));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// cuFFT plan holder.
struct FftPlan {
    cufftHandle h = 0;
    bool valid = false;
    FftPlan() = default;
    ~FftPlan() { if (valid) cufftDestroy(h); }
    FftPlan(const FftPlan &) = delete;
    FftPlan &operator=(const FftPlan &) = delete;
};

struct Dims3 {
    int64_t n1, n2, n3;  // n3 fastest
    int64_t size() const { return n1 * n2 * n3; }
};

}  // namespace lamino
