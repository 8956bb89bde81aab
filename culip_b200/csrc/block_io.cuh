// Warp-level load / unload of one factor block into a padded shared tile
// (the role of d_load_block, block_ildlt_kernels.impl.cuh:22-81).
#pragma once

#include "kernels_common.cuh"

namespace culipx {

// place an h x w block stored at `off` (dense: row-major h*w values; sparse:
// cnt entries of (local index, value)) into the tile; returns the mask of
// columns holding a non-zero
template <class T>
__device__ __forceinline__ unsigned load_block_at(T* tile, int h, int w, bool dense, long long off, int cnt,
                                                  const T* val, const int* idx, bool zero_first)
{
    const int lane = lane_id();
    if (zero_first) {
        for (int e = lane; e < kTileElems; e += 32) tile[e] = T(0);
        __syncwarp();
    }
    unsigned colmask = 0;
    if (dense) {
        for (int i = 0; i < h; ++i) {
            const T v = (lane < w) ? val[off + (long long)i * w + lane] : T(0);
            if (lane < w) tile[i * kTileStride + lane] = v;
            colmask |= __ballot_sync(0xffffffffu, v != T(0));
        }
    } else {
        for (int e = lane; e < cnt; e += 32) {
            const int li = idx[off + e];
            const int r = li / w, c = li - r * w;
            const T v = val[off + e];
            tile[r * kTileStride + c] = v;
            if (v != T(0)) colmask |= 1u << c;
        }
        for (int o = 16; o > 0; o >>= 1) colmask |= __shfl_xor_sync(0xffffffffu, colmask, o);
    }
    __syncwarp();
    return colmask;
}

// load block b from its current storage (boff[b], nnz[b])
template <class T>
__device__ __forceinline__ unsigned load_block(T* tile, int b, const DevBlock* desc, const int* bs,
                                               const long long* boff, const int* nnz, const int* fmt, const T* val,
                                               const int* idx, bool zero_first)
{
    const DevBlock d = desc[b];
    const int h = bs[d.row + 1] - bs[d.row];
    const int w = bs[d.col + 1] - bs[d.col];
    const bool dense = fmt[b] == 1;
    return load_block_at(tile, h, w, dense, boff[b], dense ? 0 : nnz[b], val, idx, zero_first);
}

// zero what load_block_at placed (sparse) or the h x w region (dense)
template <class T>
__device__ __forceinline__ void unload_block_at(T* tile, int h, int w, bool dense, long long off, int cnt,
                                                const int* idx)
{
    const int lane = lane_id();
    __syncwarp();
    if (dense) {
        if (lane < w)
            for (int i = 0; i < h; ++i) tile[i * kTileStride + lane] = T(0);
    } else {
        for (int e = lane; e < cnt; e += 32) {
            const int li = idx[off + e];
            const int r = li / w, c = li - r * w;
            tile[r * kTileStride + c] = T(0);
        }
    }
    __syncwarp();
}

// zero what load_block placed
template <class T>
__device__ __forceinline__ void unload_block(T* tile, int b, const DevBlock* desc, const int* bs,
                                             const long long* boff, const int* nnz, const int* fmt, const int* idx)
{
    const DevBlock d = desc[b];
    const int h = bs[d.row + 1] - bs[d.row];
    const int w = bs[d.col + 1] - bs[d.col];
    const bool dense = fmt[b] == 1;
    unload_block_at(tile, h, w, dense, boff[b], dense ? 0 : nnz[b], idx);
}

}  // namespace culipx
