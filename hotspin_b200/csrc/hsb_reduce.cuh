// Device-finished FP64 reductions: each block folds its threads' (Kahan-accumulated)
// values with warp shuffles and a compensated sum over its warps, stores one partial per
// quantity, and the last block to finish (atomic counter) sums the partials in block order
// -- deterministic, no host pass.  The counter must be 0 on entry; the last block resets
// it.  out[q] = scale * total[q].
#pragma once
#include "hsb_common.cuh"

template <int NQ>
__device__ void block_reduce_store(double (&v)[NQ], double* partial, unsigned int* counter,
                                   double* out, int nblocks, double scale = 1.0) {
    __shared__ double sh[NQ][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        double x = warp_sum_d(v[q]);
        if (lane == 0) sh[q][warp] = x;
    }
    __syncthreads();
    __shared__ bool last;
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int q = 0; q < NQ; q++) {
            double s = 0, c = 0;
            for (int w = 0; w < nw; w++) {
                double yv = sh[q][w] - c;
                double tv = s + yv;
                c = (tv - s) - yv;
                s = tv;
            }
            partial[(long)blockIdx.x * NQ + q] = s;
        }
        __threadfence();
        unsigned int done = atomicAdd(counter, 1u);
        last = (done == (unsigned int)nblocks - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        for (int q = 0; q < NQ; q++) {
            double s = 0, c = 0;
            for (int b = 0; b < nblocks; b++) {
                double yv = ((volatile double*)partial)[(long)b * NQ + q] - c;
                double tv = s + yv;
                c = (tv - s) - yv;
                s = tv;
            }
            out[q] = scale * s;
        }
        *counter = 0;
    }
}

