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

// Raise a kernel's dynamic shared-memory limit to at least `bytes` (never
// lowers it; safe from several host threads).
void raise_smem_limit(const void *kernel, int bytes);

// Allocation stream of the calling host thread.  When it is set (a server
// worker sets its own stream), DevBuf memory comes from the device's
// stream-ordered pool on that stream and goes back with cudaFreeAsync, so a
// request that starts or finishes never stalls the requests running beside it
// (cudaFree waits for the whole device); small table uploads then go through
// upload()/zero_bytes(), which order them on the same stream.
inline cudaStream_t &alloc_stream() {
    static thread_local cudaStream_t s = nullptr;
    return s;
}
struct AllocStreamScope {
    cudaStream_t prev;
    explicit AllocStreamScope(cudaStream_t s) : prev(alloc_stream()) { alloc_stream() = s; }
    ~AllocStreamScope() { alloc_stream() = prev; }
    AllocStreamScope(const AllocStreamScope &) = delete;
    AllocStreamScope &operator=(const AllocStreamScope &) = delete;
};

template <typename T>
void upload(T *dst, const T *src, size_t count) {
    cudaStream_t s = alloc_stream();
    if (s) {
        LAMINO_CUDA(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, s));
        LAMINO_CUDA(cudaStreamSynchronize(s));  // the host source may go out of scope
    } else {
        LAMINO_CUDA(cudaMemcpy(dst, src, count * sizeof(T), cudaMemcpyHostToDevice));
    }
}
inline void zero_bytes(void *p, size_t bytes) {
    cudaStream_t s = alloc_stream();
    if (s) LAMINO_CUDA(cudaMemsetAsync(p, 0, bytes, s));
    else LAMINO_CUDA(cudaMemset(p, 0, bytes));
}

// Owning device buffer (no copy, movable).
template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    cudaStream_t as = nullptr;  // stream-ordered allocation on this stream, if set
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    void alloc(size_t count) {
        release();
        if (!count) return;
        as = alloc_stream();
        if (as) LAMINO_CUDA(cudaMallocAsync((void **)&p, count * sizeof(T), as));
        else LAMINO_CUDA(cudaMalloc((void **)&p, count * sizeof(T)));
        n = count;
    }
    void release() {
        if (p) {
            if (as) cudaFreeAsync(p, as);
            else cudaFree(p);
        }
        p = nullptr;
        n = 0;
        as = nullptr;
    }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n), as(o.as) { o.p = nullptr; o.n = 0; o.as = nullptr; }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            p = o.p; n = o.n; as = o.as;
            o.p = nullptr; o.n = 0; o.as = nullptr;
        }
        return *this;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// cuFFT plan holder; the work area is a DevBuf (stream-ordered under a worker).
struct FftPlan {
    cufftHandle h = 0;
    bool valid = false;
    DevBuf<char> work;
    FftPlan() = default;
    ~FftPlan() { reset(); }
    FftPlan(const FftPlan &) = delete;
    FftPlan &operator=(const FftPlan &) = delete;
    void reset() {
        if (valid) cufftDestroy(h);
        valid = false;
        work.release();
    }
    // contiguous batched transform of rank 1-3 (cufftPlanMany with default layouts)
    void make(int rank, int *n, cufftType type, int batch) {
        reset();
        LAMINO_CUFFT(cufftCreate(&h));
        valid = true;
        LAMINO_CUFFT(cufftSetAutoAllocation(h, 0));
        size_t ws = 0;
        LAMINO_CUFFT(cufftMakePlanMany(h, rank, n, nullptr, 1, 0, nullptr, 1, 0, type, batch, &ws));
        work.alloc(ws > 0 ? ws : 16);
        LAMINO_CUFFT(cufftSetWorkArea(h, work.p));
    }
};

struct Dims3 {
    int64_t n1, n2, n3;  // n3 fastest
    int64_t size() const { return n1 * n2 * n3; }
};

}  // namespace lamino
