// reduce.cuh -- deterministic block reductions shared by the kernels: fixed
// shuffle trees, per-block partials, and a last-arriving block that sums the
// partials in block order (no floating-point atomics).
#pragma once

#include "gpair_internal.cuh"

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; i++)
        for (int off = 16; off > 0; off >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], off);
    if (lane == 0)
        for (int i = 0; i < NV; i++) smem[i * 32 + warp] = v[i];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int i = 0; i < NV; i++) {
            v[i] = lane < nw ? smem[i * 32 + lane] : 0.0;
            for (int off = 16; off > 0; off >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], off);
        }
    }
    __syncthreads();
}

__device__ __forceinline__ double block_max(double v, double *smem)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < nw ? smem[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, off));
    }
    __syncthreads();
    return v;
}

// True in exactly one block: the last to arrive. Partials written before the
// call are visible to it. The counter is reset by that block.
__device__ __forceinline__ bool last_block(unsigned int *counter)
{
    __shared__ bool am_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int prev = atomicAdd(counter, 1u);
        am_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    return am_last;
}

// last_block over an explicit number of participating blocks (2-D grids)
__device__ __forceinline__ bool last_block_of(unsigned int *counter, unsigned int nblocks)
{
    __shared__ bool am_last_of;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int prev = atomicAdd(counter, 1u);
        am_last_of = (prev == nblocks - 1);
    }
    __syncthreads();
    return am_last_of;
}

// Sum NV partial vectors (layout [block][NV]) in a fixed order.
template <int NV>
__device__ void finish_sum(const double *partials, int nblocks, double (&out)[NV], double *smem)
{
    double v[NV];
#pragma unroll
    for (int i = 0; i < NV; i++) v[i] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
#pragma unroll
        for (int i = 0; i < NV; i++) v[i] += __ldcg(&partials[(size_t)b * NV + i]);
    block_sum<NV>(v, smem);
#pragma unroll
    for (int i = 0; i < NV; i++) out[i] = v[i];
}

