// common.cuh -- status handling and device-memory ownership for the simulator runtime.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <utility>
#include <cstddef>
#include <vector>

#include "../../include/astrosim.h"

namespace astrosim {

// A failed call carries a status code and a message; nothing in the library aborts.
struct Status {
    int code = ASTROSIM_OK;
    std::string msg;
    bool ok() const { return code == ASTROSIM_OK; }
    static Status Ok() { return Status{}; }
};

inline Status make_error(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    Status s;
    s.code = code;
    s.msg = buf;
    return s;
}

inline Status cuda_status(cudaError_t e, const char* what, const char* file, int line) {
    if (e == cudaSuccess) return Status::Ok();
    const int code = (e == cudaErrorMemoryAllocation) ? ASTROSIM_ERR_OUT_OF_MEMORY : ASTROSIM_ERR_CUDA;
    return make_error(code, "%s failed at %s:%d: %s", what, file, line, cudaGetErrorString(e));
}

#define AS_CUDA(call)                                                                   \
    do {                                                                                \
        ::astrosim::Status _s = ::astrosim::cuda_status((call), #call, __FILE__, __LINE__); \
        if (!_s.ok()) return _s;                                                        \
    } while (0)

#define AS_TRY(expr)                       \
    do {                                   \
        ::astrosim::Status _s = (expr);    \
        if (!_s.ok()) return _s;           \
    } while (0)

// Stream for the device allocations made on this host thread (see AllocStream).
inline cudaStream_t& alloc_stream() {
    thread_local cudaStream_t s = nullptr;
    return s;
}

// While alive, DevBuf allocations on this thread are stream-ordered on `s`
// (cudaMallocAsync / cudaFreeAsync from the device's memory pool).  Plain
// cudaFree synchronizes the whole device, which would serialize concurrent
// network builds on different streams behind each other's kernels.
struct AllocStream {
    cudaStream_t prev;
    explicit AllocStream(cudaStream_t s) : prev(alloc_stream()) { alloc_stream() = s; }
    ~AllocStream() { alloc_stream() = prev; }
    AllocStream(const AllocStream&) = delete;
    AllocStream& operator=(const AllocStream&) = delete;
};

constexpr size_t kPoolMaxBytes = size_t(256) << 20;

// Owning device allocation, movable, never copied.  It is freed on the stream it was
// allocated on; the owner keeps that stream alive until its buffers are released.
template <typename T>
class DevBuf {
public:
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_), st_(o.st_) {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) {
            release();
            p_ = o.p_;
            n_ = o.n_;
            st_ = o.st_;
            o.p_ = nullptr;
            o.n_ = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }

    Status alloc(size_t n) {
        release();
        if (n == 0) n = 1;  // keep a valid pointer for empty arrays
        void* p = nullptr;
        // Buffers of kPoolMaxBytes or more come straight from cudaMalloc: growing the
        // stream-ordered pool by gigabytes the first time costs seconds (measured:
        // a first N = 1e7 build took 4.0 s from the pool, 0.6 s without it), and the
        // few multi-gigabyte frees of a large build, which synchronize the device,
        // are harmless.  Everything a network of up to a few 1e5 cells allocates
        // stays stream-ordered, so concurrent builds never wait for each other.
        st_ = n * sizeof(T) < kPoolMaxBytes ? alloc_stream() : nullptr;
        cudaError_t e = st_ ? cudaMallocAsync(&p, n * sizeof(T), st_) : cudaMalloc(&p, n * sizeof(T));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return make_error(ASTROSIM_ERR_OUT_OF_MEMORY, "device allocation of %zu bytes failed: %s", n * sizeof(T),
                              cudaGetErrorString(e));
        }
        p_ = static_cast<T*>(p);
        n_ = n;
        return Status::Ok();
    }
    Status alloc_zero(size_t n, cudaStream_t st) {
        AS_TRY(alloc(n));
        AS_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), st));
        return Status::Ok();
    }
    void release() {
        if (p_) {
            if (st_) cudaFreeAsync(p_, st_); else cudaFree(p_);
        }
        p_ = nullptr;
        n_ = 0;
    }
    T* get() const { return p_; }
    size_t size() const { return n_; }
    size_t bytes() const { return n_ * sizeof(T); }

private:
    T* p_ = nullptr;
    size_t n_ = 0;
    cudaStream_t st_ = nullptr;
};

// Keeps freed stream-ordered memory in the device pool (up to `bytes`) for reuse;
// set once per device (the first call wins).
inline void keep_pool_memory(int device, unsigned long long bytes) {
    static std::once_flag once[64];
    if (device < 0 || device >= 64) return;
    std::call_once(once[device], [&] {
        cudaMemPool_t pool = nullptr;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess && pool)
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &bytes);
        cudaGetLastError();
    });
}

// Streams handed from one simulation to the next: making and destroying a stream per
// network is driver work that serialises concurrent builds.  A stream goes back idle
// (its owner synchronises it first); the pool holds at most the peak number of
// simulations alive at once and lives until the process exits.
struct StreamPool {
    std::mutex mu;
    std::vector<std::pair<int, cudaStream_t>> idle;  // (device, stream)
};

inline StreamPool& stream_pool() {
    static StreamPool* p = new StreamPool();  // never destroyed: streams outlive static destruction order
    return *p;
}

// An idle non-blocking stream on `device` (the current device).
inline cudaError_t take_stream(int device, cudaStream_t* out) {
    {
        StreamPool& p = stream_pool();
        std::lock_guard<std::mutex> lock(p.mu);
        for (size_t i = 0; i < p.idle.size(); ++i)
            if (p.idle[i].first == device) {
                *out = p.idle[i].second;
                p.idle.erase(p.idle.begin() + static_cast<std::ptrdiff_t>(i));
                return cudaSuccess;
            }
    }
    return cudaStreamCreateWithFlags(out, cudaStreamNonBlocking);
}

// Returns a stream with no work pending to the pool.
inline void give_stream(int device, cudaStream_t s) {
    StreamPool& p = stream_pool();
    std::lock_guard<std::mutex> lock(p.mu);
    p.idle.emplace_back(device, s);
}

inline unsigned ceil_div(uint64_t a, uint64_t b) { return static_cast<unsigned>((a + b - 1) / b); }

// Streaming multiprocessors of the current device (cudaDevAttrMultiProcessorCount),
// read once per device; grids of persistent and grid-stride kernels are sized by it.
inline unsigned sm_count() {
    static unsigned cached[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        cudaGetLastError();
        return 148;
    }
    if (dev < 64 && cached[dev]) return cached[dev];
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
        cudaGetLastError();
        n = 148;  // B200
    }
    if (dev < 64) cached[dev] = static_cast<unsigned>(n);  // idempotent: every writer stores the same value
    return static_cast<unsigned>(n);
}

}  // namespace astrosim
