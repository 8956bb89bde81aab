// Device-side plumbing shared by all culipx objects: the handle (device,
// stream, memory budget) and a budgeted device buffer.
#pragma once

#include "common.h"

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <utility>

namespace culipx {
struct Sqmr;
}

struct culipx_handle_t {
    culipx::Sqmr* sqmr = nullptr;       // SQMR workspace, grown on demand
    int device = 0;
    cudaStream_t stream = nullptr;
    long long budget = 0;               // <= 0: unlimited
    std::atomic<long long> used{0};     // bytes held by this handle's buffers
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    long long launches = 0;             // kernels launched through this handle
    double* vec_scratch = nullptr;      // reduction partials of the vector operations (vecops.cu)
    // the creator's reference plus one per object the C ABI created on this
    // handle (patterns, operators, plans, ...): culipx_handle_destroy and
    // those objects' destroy calls may come in any order, the last one frees
    std::atomic<int> refs{1};
};

namespace culipx {

#define CULIPX_CUDA(expr)                                                                  \
    do {                                                                                   \
        cudaError_t e_ = (expr);                                                           \
        if (e_ != cudaSuccess)                                                             \
            return ::culipx::fail(CULIPX_CUDA_ERROR, "%s failed: %s (%s:%d)", #expr,      \
                                  cudaGetErrorString(e_), __FILE__, __LINE__);             \
    } while (0)

#define CULIPX_TRY(expr)            \
    do {                            \
        int s_ = (expr);            \
        if (s_ != CULIPX_OK) return s_; \
    } while (0)

// References on a handle (see culipx_handle_t::refs); the last release frees it.
void handle_retain(culipx_handle_t* h);
void handle_release(culipx_handle_t* h);

// A process-wide serial number for objects whose device addresses a captured
// CUDA graph holds: a new object never repeats an old one's number, even when
// it reuses the old one's host address.
unsigned long long next_serial();

// Checks the last launch error on this thread.
int launch_check(const char* what);

// Device memory charged against the owning handle's budget.
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept { swap(o); }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept { release(); swap(o); return *this; }
    ~DeviceBuffer() { release(); }

    int alloc(culipx_handle_t* h, size_t bytes);
    int upload(culipx_handle_t* h, const void* src, size_t bytes);  // alloc + synchronous copy
    void release();

    template <class T> T* as() const { return static_cast<T*>(ptr_); }
    void* get() const { return ptr_; }
    size_t bytes() const { return bytes_; }

private:
    void swap(DeviceBuffer& o) noexcept
    {
        std::swap(ptr_, o.ptr_);
        std::swap(bytes_, o.bytes_);
        std::swap(h_, o.h_);
    }
    void* ptr_ = nullptr;
    size_t bytes_ = 0;
    culipx_handle_t* h_ = nullptr;
};

}  // namespace culipx
