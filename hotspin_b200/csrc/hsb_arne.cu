// Kernel_Arne demag tensor on the GPU in FP64 (setup only).
//
// Restates src/hotspin-core/modules/kernel_magnetostatic.go:25-241 (arithmetic in
// hsb_arne.cuh): for every wrapped target cell of the folded octant and every source axis s,
// the field of the two faces of a source cell normal to s, carrying unit surface charge,
// integrated over the target cell with a density set by the distance (accuracy), summed over
// the periodic images in the reference's loop order (z, then y, then x).  This file is
// compiled without FMA contraction, so every product rounds as the reference's does; the
// quadrature sum is formed per lane in the reference's order and then across the warp.
#include <math.h>

#include "hsb_arne.cuh"
#include "hsb_common.cuh"
#include "hsb_demag.h"


// One warp per (folded target, source axis s): the lanes split the source-face points (the
// (i, j) pairs of the quadrature below) and each lane keeps the reference's nested order for its
// points; the lane sums meet in a warp reduction.  The near targets carry nearly all the work
// (31104 quadrature points for a cell on itself against 4 in the far field), so spreading
// their points over 32 lanes removes the serial tail that one thread per target had.
__global__ void __launch_bounds__(128) k_arne_kernel(ArneGeom g, double* __restrict__ Kc) {
    const long n0 = g.h[0] + 1, n1 = g.h[1] + 1, n2 = g.h[2] + 1;
    const long ncell = n0 * n1 * n2;
    const long tot = ncell * 3;
    const int lane = threadIdx.x & 31;
    const long warps = (long)gridDim.x * (blockDim.x >> 5);
    for (long q = blockIdx.x * (long)(blockDim.x >> 5) + (threadIdx.x >> 5); q < tot; q += warps) {
        const int s = (int)(q / ncell);
        const long c = q - s * ncell;
        const int t0 = (int)(c / (n1 * n2));
        const int t1 = (int)((c / n2) % n1);
        const int t2 = (int)(c % n2);
        double acc[3];
        arne_target_part(g, s, t0, t1, t2, lane, 32, acc);
        for (int d = s; d < 3; d++) acc[d] = warp_sum_d(acc[d]);
        if (lane == 0) {
            const int full[3][3] = {{KXX, KXY, KXZ}, {KXY, KYY, KYZ}, {KXZ, KYZ, KZZ}};
            for (int d = s; d < 3; d++) Kc[(long)full[s][d] * ncell + c] = acc[d];
        }
    }
}

// Full real component c from the folded octant with the tensor parities
// (kernel_magnetostatic.go:185-230).
__global__ void k_arne_expand(const double* __restrict__ Kc, int comp, int L0, int L1, int L2,
                              double* __restrict__ out) {
    const int h0 = L0 / 2, h1 = L1 / 2, h2 = L2 / 2;
    const long n1 = h1 + 1, n2 = h2 + 1, ncell = (long)(h0 + 1) * n1 * n2;
    const long tot = (long)L0 * L1 * L2;
    // parity per flipped axis: rows XX YY ZZ YZ XZ XY
    const int par[3][6] = {{1, 1, 1, 1, -1, -1}, {1, 1, 1, -1, 1, -1}, {1, 1, 1, -1, -1, 1}};
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < tot; q += (long)gridDim.x * blockDim.x) {
        int i = (int)(q / ((long)L1 * L2));
        int j = (int)((q / L2) % L1);
        int k = (int)(q % L2);
        int sg = 1;
        if (i > h0) { i = L0 - i; sg *= par[0][comp]; }
        if (j > h1) { j = L1 - j; sg *= par[1][comp]; }
        if (k > h2) { k = L2 - k; sg *= par[2][comp]; }
        out[q] = sg * Kc[(long)comp * ncell + ((long)i * n1 + j) * n2 + k];
    }
}


cudaError_t hsb_arne_launch(const ArneGeom* g, double* Kc, cudaStream_t st) {
    const long nfold = (long)(g->h[0] + 1) * (g->h[1] + 1) * (g->h[2] + 1);
    // 4 warps (targets) per block
    k_arne_kernel<<<hsb_grid_1d(nfold * 3, 4, 16), 128, 0, st>>>(*g, Kc);
    return cudaGetLastError();
}

cudaError_t hsb_arne_expand_launch(const double* Kc, int comp, int L0, int L1, int L2, double* out,
                                   cudaStream_t st) {
    const long vol = (long)L0 * L1 * L2;
    k_arne_expand<<<hsb_grid_1d(vol, 256), 256, 0, st>>>(Kc, comp, L0, L1, L2, out);
    return cudaGetLastError();
}
