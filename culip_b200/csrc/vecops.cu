// Vector operations on device vectors for the C++ class facade
// (include/culip_la.hpp): the BLAS-1 calls of libs/la/dense_la.cuh:35-85
// (T_nrm2, T_doti, T_scal, T_axpy, which call cuBLAS there) and precision
// conversion.  Reductions are deterministic: a fixed grid of kRedBlocks CTAs
// writes FP64 partials (fixed shuffle tree per CTA), one CTA sums them in
// index order; FP32 vectors are accumulated in FP64.
#include "device.h"

#include <cmath>

namespace culipx {
namespace {

constexpr int kRedBlocks = 256;
constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double warp_part[kRedThreads / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) warp_part[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kRedThreads / 32; ++w) s += warp_part[w];
    return s;  // valid in thread 0
}

template <class T>
__global__ void __launch_bounds__(kRedThreads) k_dot_part(long long n, const T* x, const T* y, double* part)
{
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * kRedThreads + threadIdx.x; i < n; i += (long long)kRedBlocks * kRedThreads)
        acc = fma((double)x[i], (double)y[i], acc);
    const double s = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void __launch_bounds__(kRedThreads) k_sum_parts(const double* part, double* out, int take_sqrt)
{
    double acc = 0.0;
    for (int i = threadIdx.x; i < kRedBlocks; i += kRedThreads) acc += part[i];
    const double s = block_sum(acc);
    if (threadIdx.x == 0) out[0] = take_sqrt ? sqrt(s) : s;
}

template <class T>
__global__ void k_axpy(long long n, double alpha, const T* x, T* y)
{
    const T a = (T)alpha;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = fma(a, x[i], y[i]);
}

template <class T>
__global__ void k_scal(long long n, double alpha, T* x)
{
    const T a = (T)alpha;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = a * x[i];
}

template <class S, class D>
__global__ void k_convert(long long n, const S* src, D* dst)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (D)src[i];
}

int grid_for(long long n)
{
    const long long g = (n + 255) / 256;
    return (int)(g < 1 ? 1 : (g > 4096 ? 4096 : g));
}

int prepare(culipx_handle_t* h, int precision, long long n)
{
    if (!h || h->device < 0) return fail(CULIPX_INVALID_ARG, "vector operation: null or host-only handle");
    if (precision != CULIPX_F64 && precision != CULIPX_F32)
        return fail(CULIPX_INVALID_ARG, "vector operation: bad precision %d", precision);
    if (n < 0) return fail(CULIPX_INVALID_ARG, "vector operation: negative length");
    CULIPX_CUDA(cudaSetDevice(h->device));
    return CULIPX_OK;
}

// dot product (or norm) into *result (host), synchronizing the handle's stream
int reduce(culipx_handle_t* h, int precision, long long n, const void* x, const void* y, bool norm, double* result)
{
    CULIPX_TRY(prepare(h, precision, n));
    if (!result) return fail(CULIPX_INVALID_ARG, "vector reduction: null result");
    if (!h->vec_scratch) CULIPX_CUDA(cudaMalloc(&h->vec_scratch, (kRedBlocks + 8) * sizeof(double)));
    double* part = h->vec_scratch;
    double* out = part + kRedBlocks;
    if (precision == CULIPX_F64)
        k_dot_part<double><<<kRedBlocks, kRedThreads, 0, h->stream>>>(n, static_cast<const double*>(x),
                                                                        static_cast<const double*>(y), part);
    else
        k_dot_part<float><<<kRedBlocks, kRedThreads, 0, h->stream>>>(n, static_cast<const float*>(x),
                                                                       static_cast<const float*>(y), part);
    k_sum_parts<<<1, kRedThreads, 0, h->stream>>>(part, out, norm ? 1 : 0);
    h->launches += 2;
    CULIPX_TRY(launch_check("vector reduction"));
    CULIPX_CUDA(cudaMemcpyAsync(result, out, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CULIPX_CUDA(cudaStreamSynchronize(h->stream));
    return CULIPX_OK;
}

}  // namespace
}  // namespace culipx

using namespace culipx;

CULIPX_API int culipx_vec_dot(culipx_handle h, int precision, long long n, const void* d_x, const void* d_y,
                              double* result)
{
    if (n > 0 && (!d_x || !d_y)) return fail(CULIPX_INVALID_ARG, "culipx_vec_dot: null vector");
    return reduce(h, precision, n, d_x, d_y, false, result);
}

CULIPX_API int culipx_vec_nrm2(culipx_handle h, int precision, long long n, const void* d_x, double* result)
{
    if (n > 0 && !d_x) return fail(CULIPX_INVALID_ARG, "culipx_vec_nrm2: null vector");
    return reduce(h, precision, n, d_x, d_x, true, result);
}

CULIPX_API int culipx_vec_axpy(culipx_handle h, int precision, long long n, double alpha, const void* d_x, void* d_y)
{
    CULIPX_TRY(prepare(h, precision, n));
    if (n == 0) return CULIPX_OK;
    if (!d_x || !d_y) return fail(CULIPX_INVALID_ARG, "culipx_vec_axpy: null vector");
    if (precision == CULIPX_F64)
        k_axpy<double><<<grid_for(n), 256, 0, h->stream>>>(n, alpha, static_cast<const double*>(d_x),
                                                           static_cast<double*>(d_y));
    else
        k_axpy<float><<<grid_for(n), 256, 0, h->stream>>>(n, alpha, static_cast<const float*>(d_x),
                                                          static_cast<float*>(d_y));
    h->launches += 1;
    return launch_check("culipx_vec_axpy");
}

CULIPX_API int culipx_vec_scal(culipx_handle h, int precision, long long n, double alpha, void* d_x)
{
    CULIPX_TRY(prepare(h, precision, n));
    if (n == 0) return CULIPX_OK;
    if (!d_x) return fail(CULIPX_INVALID_ARG, "culipx_vec_scal: null vector");
    if (precision == CULIPX_F64)
        k_scal<double><<<grid_for(n), 256, 0, h->stream>>>(n, alpha, static_cast<double*>(d_x));
    else
        k_scal<float><<<grid_for(n), 256, 0, h->stream>>>(n, alpha, static_cast<float*>(d_x));
    h->launches += 1;
    return launch_check("culipx_vec_scal");
}

CULIPX_API int culipx_vec_convert(culipx_handle h, long long n, int src_precision, const void* d_src,
                                  int dst_precision, void* d_dst)
{
    CULIPX_TRY(prepare(h, src_precision, n));
    CULIPX_TRY(prepare(h, dst_precision, n));
    if (n == 0) return CULIPX_OK;
    if (!d_src || !d_dst) return fail(CULIPX_INVALID_ARG, "culipx_vec_convert: null vector");
    const int g = grid_for(n);
    if (src_precision == dst_precision) {
        const size_t bytes = (size_t)n * (src_precision == CULIPX_F64 ? 8 : 4);
        if (d_src != d_dst) CULIPX_CUDA(cudaMemcpyAsync(d_dst, d_src, bytes, cudaMemcpyDeviceToDevice, h->stream));
        return CULIPX_OK;
    }
    if (src_precision == CULIPX_F64)
        k_convert<double, float><<<g, 256, 0, h->stream>>>(n, static_cast<const double*>(d_src),
                                                           static_cast<float*>(d_dst));
    else
        k_convert<float, double><<<g, 256, 0, h->stream>>>(n, static_cast<const float*>(d_src),
                                                           static_cast<double*>(d_dst));
    h->launches += 1;
    return launch_check("culipx_vec_convert");
}
