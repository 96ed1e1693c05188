// Warp-shuffle argmax / sum reductions shared by the pivoting kernels.
#pragma once

#include <cstdint>

namespace isdf {

// Pivot key: larger value wins; ties go to the smaller position.
struct ArgKey {
    double v;
    int64_t pos;
    int64_t col;
};

__device__ __forceinline__ bool key_better(const ArgKey& a, const ArgKey& b) {
    return a.v > b.v || (a.v == b.v && a.pos < b.pos);
}

__device__ __forceinline__ ArgKey key_none() { return ArgKey{-1.0, INT64_MAX, -1}; }

__device__ __forceinline__ ArgKey warp_best(ArgKey k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ArgKey t;
        t.v = __shfl_down_sync(0xffffffffu, k.v, o);
        t.pos = __shfl_down_sync(0xffffffffu, k.pos, o);
        t.col = __shfl_down_sync(0xffffffffu, k.col, o);
        if (key_better(t, k)) k = t;
    }
    return k;
}

// Result valid in every lane.
__device__ __forceinline__ double warp_allsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Result valid in thread 0.  `sh` needs NT/32 entries.
template <int NT>
__device__ __forceinline__ ArgKey block_best(ArgKey k, ArgKey* sh) {
    k = warp_best(k);
    const int lane = threadIdx.x % 32, wid = threadIdx.x / 32;
    if (lane == 0) sh[wid] = k;
    __syncthreads();
    if (wid == 0) {
        k = lane < NT / 32 ? sh[lane] : key_none();
        k = warp_best(k);
    }
    __syncthreads();
    return k;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Result valid in thread 0.  `sh` needs NT/32 entries.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
    v = warp_sum(v);
    const int lane = threadIdx.x % 32, wid = threadIdx.x / 32;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < NT / 32 ? sh[lane] : 0.0;
        v = warp_sum(v);
    }
    __syncthreads();
    return v;
}

}  // namespace isdf
