// Host-side helpers: CUDA error handling and grow-only device buffers.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <algorithm>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace tmb {

// Raised inside the engine; the C ABI turns it into a status code and a
// message (tm_last_error), so no CUDA failure ends the process.
struct Error : std::runtime_error {
    int status;
    Error(int st, const std::string &msg) : std::runtime_error(msg), status(st) {}
};

inline std::string cuda_msg(cudaError_t e, const char *what, const char *file, int line) {
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
    return buf;
}

#define TM_CUDA(x)                                                                       \
    do {                                                                                 \
        cudaError_t e_ = (x);                                                            \
        if (e_ != cudaSuccess) throw ::tmb::Error(-2, ::tmb::cuda_msg(e_, #x, __FILE__, __LINE__)); \
    } while (0)

#define TM_CHECK_LAUNCH() TM_CUDA(cudaGetLastError())

// Grow-only device buffer.  reserve() keeps the old contents only when it
// does not reallocate; callers treat a grown buffer as uninitialised.
template <class T>
struct DevBuf {
    T *p = nullptr;
    size_t cap = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), cap(o.cap) { o.p = nullptr; o.cap = 0; }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            p = o.p;
            cap = o.cap;
            o.p = nullptr;
            o.cap = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    // Grows by at least half the current capacity, so a slowly growing
    // demand reallocates (and frees, which synchronises the device) rarely.
    void reserve(size_t n) {
        if (n <= cap && p) return;
        if (p) n = std::max(n, cap + cap / 2);
        release();
        size_t bytes = (n ? n : 1) * sizeof(T);
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) {
            p = nullptr;
            cap = 0;
            cudaGetLastError();
            throw Error(-5, cuda_msg(e, "cudaMalloc", __FILE__, __LINE__) + " bytes=" + std::to_string(bytes));
        }
        cap = n ? n : 1;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    T *get() const { return p; }
};

// Pinned host buffer (grow-only).
template <class T>
struct HostBuf {
    T *p = nullptr;
    size_t cap = 0;
    HostBuf() = default;
    HostBuf(const HostBuf &) = delete;
    HostBuf &operator=(const HostBuf &) = delete;
    HostBuf(HostBuf &&o) noexcept : p(o.p), cap(o.cap) { o.p = nullptr; o.cap = 0; }
    ~HostBuf() { release(); }
    void reserve(size_t n) {
        if (n <= cap && p) return;
        if (p) n = std::max(n, cap + cap / 2);
        release();
        size_t bytes = (n ? n : 1) * sizeof(T);
        cudaError_t e = cudaMallocHost(&p, bytes);
        if (e != cudaSuccess) {
            p = nullptr;
            cap = 0;
            cudaGetLastError();
            throw Error(-5, cuda_msg(e, "cudaMallocHost", __FILE__, __LINE__));
        }
        cap = n ? n : 1;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
};

// Pinned host buffer mapped into the device address space (grow-only).
// Kernels store small results into it (d); the host reads them (h) after a
// stream synchronisation.  Such stores leave the SMs over PCIe directly, so
// unlike a cudaMemcpyAsync they do not queue on a copy engine behind large
// copies that other streams have issued.
template <class T>
struct MappedBuf {
    T *h = nullptr;
    T *d = nullptr;
    size_t cap = 0;
    MappedBuf() = default;
    MappedBuf(const MappedBuf &) = delete;
    MappedBuf &operator=(const MappedBuf &) = delete;
    MappedBuf(MappedBuf &&o) noexcept : h(o.h), d(o.d), cap(o.cap) {
        o.h = o.d = nullptr;
        o.cap = 0;
    }
    MappedBuf &operator=(MappedBuf &&o) noexcept {
        if (this != &o) {
            release();
            h = o.h;
            d = o.d;
            cap = o.cap;
            o.h = o.d = nullptr;
            o.cap = 0;
        }
        return *this;
    }
    ~MappedBuf() { release(); }
    void reserve(size_t n) {
        if (n <= cap && h) return;
        if (h) n = std::max(n, cap + cap / 2);
        release();
        const size_t bytes = (n ? n : 1) * sizeof(T);
        cudaError_t e = cudaHostAlloc(reinterpret_cast<void **>(&h), bytes, cudaHostAllocMapped);
        if (e == cudaSuccess) e = cudaHostGetDevicePointer(reinterpret_cast<void **>(&d), h, 0);
        if (e != cudaSuccess) {
            if (h) cudaFreeHost(h);
            h = d = nullptr;
            cap = 0;
            cudaGetLastError();
            throw Error(-5, cuda_msg(e, "cudaHostAlloc(mapped)", __FILE__, __LINE__));
        }
        cap = n ? n : 1;
    }
    void release() {
        if (h) cudaFreeHost(h);
        h = d = nullptr;
        cap = 0;
    }
};

}  // namespace tmb
