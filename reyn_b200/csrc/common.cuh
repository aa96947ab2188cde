// Shared host/device utilities of the reyn_b200 engine: error handling across
// the C ABI, RAII device buffers, launch geometry and block reductions.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <utility>

#include "reyn_b200.h"

namespace reyn {

// An engine error: a C-ABI status code and a message. Thrown inside the
// engine, caught at the ABI boundary by `guard`.
struct Error {
    int code;
    std::string msg;
};

void set_last_error(const std::string& msg);

[[noreturn]] inline void fail(int code, const std::string& msg)
{
    throw Error { code, msg };
}

inline void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
        fail(e == cudaErrorMemoryAllocation ? REYN_ERR_ALLOC : REYN_ERR_CUDA,
            std::string(what) + ": " + cudaGetErrorString(e));
}

#define REYN_CUDA(expr) ::reyn::cuda_check((expr), #expr)
#define REYN_LAUNCHED(name) ::reyn::cuda_check(cudaGetLastError(), name)

// Launch accounting: every kernel launch of the engine goes through
// REYN_KERNEL, which counts it per kernel name and, while timing is enabled
// (reyn_profile_enable), brackets it with a pair of CUDA events recorded on
// the launching stream.
class ProfScope {
public:
    ProfScope(const char* name, cudaStream_t s);
    ~ProfScope();
    ProfScope(const ProfScope&) = delete;
    ProfScope& operator=(const ProfScope&) = delete;

private:
    int slot_ = -1;
    cudaStream_t s_ = nullptr;
};

#define REYN_KERNEL(name, stream, ...)                                         \
    do {                                                                       \
        ::reyn::ProfScope reyn_prof_scope_(name, stream);                      \
        __VA_ARGS__;                                                           \
        ::reyn::cuda_check(cudaGetLastError(), name);                          \
    } while (0)

// Runs `f`, translating engine errors to status codes for the C ABI.
template <class F> int guard(F&& f) noexcept
{
    try {
        f();
        return REYN_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return REYN_ERR_ALLOC;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return REYN_ERR_INVALID;
    } catch (...) {
        set_last_error("unknown exception");
        return REYN_ERR_INVALID;
    }
}

inline void require(bool ok, const char* msg)
{
    if (!ok)
        fail(REYN_ERR_INVALID, msg);
}

// Owning device allocation of `n` elements of T (cudaMalloc'ed once, resized
// only when a larger size is requested).
template <class T> class DevArray {
public:
    DevArray() = default;
    explicit DevArray(size_t n) { resize(n); }
    ~DevArray() { release(); }
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    DevArray(DevArray&& o) noexcept
        : p_(std::exchange(o.p_, nullptr))
        , n_(std::exchange(o.n_, 0))
        , cap_(std::exchange(o.cap_, 0))
    {
    }
    DevArray& operator=(DevArray&& o) noexcept
    {
        if (this != &o) {
            release();
            p_ = std::exchange(o.p_, nullptr);
            n_ = std::exchange(o.n_, 0);
            cap_ = std::exchange(o.cap_, 0);
        }
        return *this;
    }
    void resize(size_t n)
    {
        if (n > cap_) {
            release();
            void* q = nullptr;
            REYN_CUDA(cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)));
            p_ = static_cast<T*>(q);
            cap_ = n;
        }
        n_ = n;
    }
    void zero(cudaStream_t s)
    {
        if (n_)
            REYN_CUDA(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
    }
    T* get() const { return p_; }
    size_t size() const { return n_; }
    void swap(DevArray& o) noexcept
    {
        std::swap(p_, o.p_);
        std::swap(n_, o.n_);
        std::swap(cap_, o.cap_);
    }

private:
    void release() noexcept
    {
        if (p_)
            cudaFree(p_);
        p_ = nullptr;
        n_ = cap_ = 0;
    }
    T* p_ = nullptr;
    size_t n_ = 0;
    size_t cap_ = 0;
};

// Pinned host scratch for small device->host readbacks.
template <class T> class PinnedArray {
public:
    explicit PinnedArray(size_t n)
    {
        void* q = nullptr;
        REYN_CUDA(cudaMallocHost(&q, std::max<size_t>(n, 1) * sizeof(T)));
        p_ = static_cast<T*>(q);
    }
    ~PinnedArray()
    {
        if (p_)
            cudaFreeHost(p_);
    }
    PinnedArray(const PinnedArray&) = delete;
    PinnedArray& operator=(const PinnedArray&) = delete;
    T* get() const { return p_; }
    T& operator[](size_t i) const { return p_[i]; }

private:
    T* p_ = nullptr;
};

// device status bits written by kernels, read back by the host
enum StatusBits : uint32_t {
    STATUS_OUT_OF_GRID = 1u, // a particle lay outside its grid (clamped)
    STATUS_NONFINITE = 2u    // a NaN/Inf position was met
};

constexpr int THREADS = 256; // threads per block of the streaming kernels
constexpr int NBR_THREADS = 128; // default threads per block of the neighbour loops
constexpr int NBR_MAX_THREADS = 512; // largest block size they are compiled for

inline unsigned blocks_for(size_t n, int threads)
{
    return static_cast<unsigned>((n + threads - 1) / threads);
}

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

} // namespace reyn
