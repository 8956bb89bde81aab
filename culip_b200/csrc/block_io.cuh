// Warp-level load / unload of one factor block into a padded shared tile.
#pragma once

#include "kernels_common.cuh"

namespace culipx {

// load block b (h x w) into a zeroed tile; returns the column mask
template <class T>
__device__ __forceinline__ unsigned load_block(T* tile, int b, const DevBlock* desc, const int* bs,
                               const long long* boff, const int* nnz, const int* fmt,
                               const T* val, const int* idx, bool zero_first)
{
    const int lane = lane_id();
    if (zero_first) {
        for (int e = lane; e < kTileElems; e += 32) tile[e] = T(0);
        __syncwarp();
    }
    const DevBlock d = desc[b];
    const int h = bs[d.row + 1] - bs[d.row];
    const int w = bs[d.col + 1] - bs[d.col];
    const long long off = boff[b];
    unsigned colmask = 0;
    if (fmt[b] == 1) {
        for (int i = 0; i < h; ++i) {
            const T v = (lane < w) ? val[off + (long long)i * w + lane] : T(0);
            if (lane < w) tile[i * kTileStride + lane] = v;
            colmask |= __ballot_sync(0xffffffffu, v != T(0));
        }
    } else {
        const int cnt = nnz[b];
        for (int e = lane; e < cnt; e += 32) {
            const int li = idx[off + e];
            const int r = li / w, c = li - (li / w) * w;
            const T v = val[off + e];
            tile[r * kTileStride + c] = v;
            if (v != T(0)) colmask |= 1u << c;
        }
        for (int o = 16; o > 0; o >>= 1) colmask |= __shfl_xor_sync(0xffffffffu, colmask, o);
    }
    __syncwarp();
    return colmask;
}

// zero what load_block placed (sparse) or the h x w region (dense)
template <class T>
__device__ __forceinline__ void unload_block(T* tile, int b, const DevBlock* desc, const int* bs,
                             const long long* boff, const int* nnz, const int* fmt, const int* idx)
{
    const int lane = lane_id();
    const DevBlock d = desc[b];
    const int h = bs[d.row + 1] - bs[d.row];
    const int w = bs[d.col + 1] - bs[d.col];
    __syncwarp();
    if (fmt[b] == 1) {
        if (lane < w)
            for (int i = 0; i < h; ++i) tile[i * kTileStride + lane] = T(0);
    } else {
        const long long off = boff[b];
        const int cnt = nnz[b];
        for (int e = lane; e < cnt; e += 32) {
            const int li = idx[off + e];
            const int r = li / w, c = li - (li / w) * w;
            tile[r * kTileStride + c] = T(0);
        }
    }
    __syncwarp();
}

}  // namespace culipx
