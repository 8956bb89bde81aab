// Device helpers shared by the culipx kernels.
#pragma once

#include "common.h"

#include <cuda_runtime.h>
#include <cstdint>

namespace culipx {

constexpr int kTileStride = 33;          // padded row stride of a 32x32 shared tile
constexpr int kTileElems = 32 * kTileStride;
constexpr double kNzEps = 1e-10;         // NZ_EPS, block_ildlt_kernels.impl.cuh:17

__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

template <class T>
__device__ __forceinline__ T shfl(T v, int src) { return __shfl_sync(0xffffffffu, v, src); }

// true when an FP32 factor inverts this 2x2 pivot in FP64 (kPivotFp64Default);
// the products of two floats are exact in double, so host and device decide
// alike
template <class T>
__device__ __forceinline__ bool wide_2x2(T d11, T d12, T d22, double bound)
{
    if (sizeof(T) != 4) return false;
    const double p = (double)d11 * (double)d22, q = (double)d12 * (double)d12;
    return fabs(p - q) < bound * (fabs(p) + q);
}

// per-block descriptor, mirror of BlockDesc (pattern.h)
struct DevBlock {
    int row, col, val_off, cap;
};

}  // namespace culipx
