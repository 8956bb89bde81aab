// Error reporting and budgeted device memory for the culipx library.
#include "device.h"

#include <cstdarg>
#include <cstring>

namespace culipx {

unsigned long long next_serial()
{
    static std::atomic<unsigned long long> n{0};
    return ++n;
}

namespace {
thread_local char g_last_error[1024] = "";
}

int fail(int status, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

void clear_error() { g_last_error[0] = 0; }

const char* last_error() { return g_last_error; }

int launch_check(const char* what)
{
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CULIPX_CUDA_ERROR, "%s: launch failed: %s", what, cudaGetErrorString(e));
    return CULIPX_OK;
}

int DeviceBuffer::alloc(culipx_handle_t* h, size_t bytes)
{
    release();
    if (bytes == 0) bytes = 16;
    if (h && h->budget > 0 && h->used.load() + (long long)bytes > h->budget)
        return fail(CULIPX_OOM, "device-memory budget exceeded: %lld + %zu > %lld bytes", h->used.load(), bytes,
                    h->budget);
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(CULIPX_OOM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    ptr_ = p;
    bytes_ = bytes;
    h_ = h;
    if (h) h->used += (long long)bytes;
    return CULIPX_OK;
}

int DeviceBuffer::upload(culipx_handle_t* h, const void* src, size_t bytes)
{
    CULIPX_TRY(alloc(h, bytes));
    if (bytes) CULIPX_CUDA(cudaMemcpy(ptr_, src, bytes, cudaMemcpyHostToDevice));
    return CULIPX_OK;
}

void DeviceBuffer::release()
{
    if (ptr_) {
        cudaFree(ptr_);
        if (h_) h_->used -= (long long)bytes_;
    }
    ptr_ = nullptr;
    bytes_ = 0;
    h_ = nullptr;
}

}  // namespace culipx
