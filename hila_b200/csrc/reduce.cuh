// Deterministic block and grid reductions in FP64.
//
// Every block reduces its values with a fixed xor-butterfly inside each warp
// and a fixed-order sum over warps, writes one partial per value, and the
// last block to arrive (atomic ticket) sums the partials in block order and
// hands the totals to a finisher functor.  The result depends only on the
// data and the grid size, never on scheduling, so a solve gives bitwise the
// same scalars on every run.
#pragma once

#include <cuda_runtime.h>

namespace hw {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum of one value over the block; the result is valid in thread 0.
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v, double *smem /* BLOCK/32 */) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    double s = 0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int w = 0; w < BLOCK / 32; w++) s += smem[w];
    }
    __syncthreads();
    return s;
}

// Reduce NRED values over the whole grid; the last block calls fin(totals).
// partials must hold NRED * gridDim.x doubles; *ticket must be 0 on entry and
// is 0 again on exit.  Must be called by all threads of every block.
template <int NRED, int BLOCK, class Fin>
__device__ __forceinline__ void grid_reduce(double (&v)[NRED], double *partials, unsigned *ticket, Fin &fin) {
    __shared__ double smem[BLOCK / 32];
    __shared__ bool is_last;
    const unsigned nb = gridDim.x;
#pragma unroll
    for (int k = 0; k < NRED; k++) {
        double s = block_sum<BLOCK>(v[k], smem);
        if (threadIdx.x == 0) partials[(size_t)k * nb + blockIdx.x] = s;
    }
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        is_last = (t == nb - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double tot[NRED];
#pragma unroll
    for (int k = 0; k < NRED; k++) {
        double s = 0;
        for (unsigned j = threadIdx.x; j < nb; j += BLOCK) s += __ldcg(partials + (size_t)k * nb + j);
        tot[k] = block_sum<BLOCK>(s, smem);
    }
    if (threadIdx.x == 0) {
        fin(tot);
        *ticket = 0u;
    }
}

}  // namespace hw
