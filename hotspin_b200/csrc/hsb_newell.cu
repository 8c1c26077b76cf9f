// FP64 Newell demag tensor on the GPU (setup only): one thread per (folded target, source
// axis s) computes K_sd = -N_sd, d = s..2, summed over the periodic images, in the folded
// layout Kernel_Arne writes (hsb_arne.cu), so the same expansion, FP64 transforms and
// extraction turn it into the kernel spectrum.  The arithmetic is hsb_newell.cuh.
#include "hsb_common.cuh"
#include "hsb_newell.cuh"

__global__ void __launch_bounds__(128) k_newell_kernel(ArneGeom g, double* __restrict__ Kc) {
    const long n0 = g.h[0] + 1, n1 = g.h[1] + 1, n2 = g.h[2] + 1;
    const long ncell = n0 * n1 * n2;
    const long tot = ncell * 3;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < tot; q += (long)gridDim.x * blockDim.x) {
        const int s = (int)(q / ncell);
        const long c = q - s * ncell;
        const int t0 = (int)(c / (n1 * n2));
        const int t1 = (int)((c / n2) % n1);
        const int t2 = (int)(c % n2);
        double acc[3];
        newell_target(g, s, t0, t1, t2, acc);
        const int full[3][3] = {{KXX, KXY, KXZ}, {KXY, KYY, KYZ}, {KXZ, KYZ, KZZ}};
        for (int d = s; d < 3; d++) Kc[(long)full[s][d] * ncell + c] = acc[d];
    }
}

cudaError_t hsb_newell_launch(const ArneGeom* g, double* Kc, cudaStream_t st) {
    const long nfold = (long)(g->h[0] + 1) * (g->h[1] + 1) * (g->h[2] + 1);
    k_newell_kernel<<<hsb_grid_1d(nfold * 3, 128, 16), 128, 0, st>>>(*g, Kc);
    return cudaGetLastError();
}
