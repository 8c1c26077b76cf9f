// Kernel_Arne demag tensor on the GPU in FP64 (setup only).
//
// Restates src/hotspin-core/modules/kernel_magnetostatic.go:25-241: for every wrapped
// target cell of the folded octant and every source axis s, the field of the two faces of
// a source cell normal to s, carrying unit surface charge, integrated over the target
// cell with a density set by the distance (accuracy), summed over the periodic images in
// the reference's loop order (z, then y, then x).  This file is compiled without FMA
// contraction so every product and sum rounds as the sequential reference does.
#include <math.h>

#include "hsb_common.cuh"
#include "hsb_demag.h"


__device__ __forceinline__ double arne_delta(long d) {
    if (d < 0) d = -d;
    if (d > 0) d -= 1;
    return (double)d;
}

// Field at integer offset (x,y,z) cells of a source cell whose faces normal to axis s carry
// unit surface charge; same quadrature and expression order as the reference.
__device__ void arne_point(int s, long x, long y, long z, const double* cs, double Lmin,
                           double accuracy, double* B) {
    const int u = s, v = (s + 1) % 3, w = (s + 2) % 3;
    double R[3], R2[3], pole[3];
    R[0] = (double)x * cs[0];
    R[1] = (double)y * cs[1];
    R[2] = (double)z * cs[2];
    double dx = arne_delta(x) * cs[0], dy = arne_delta(y) * cs[1], dz = arne_delta(z) * cs[2];
    double d = sqrt(dx * dx + dy * dy + dz * dz);
    if (d == 0) d = Lmin;
    double maxSize = d / accuracy;
    int nv = (int)(fmax(cs[v] / maxSize, 1.0) + 0.5);
    int nw = (int)(fmax(cs[w] / maxSize, 1.0) + 0.5);
    int nx = (int)(fmax(cs[0] / maxSize, 1.0) + 0.5);
    int ny = (int)(fmax(cs[1] / maxSize, 1.0) + 0.5);
    int nz = (int)(fmax(cs[2] / maxSize, 1.0) + 0.5);
    nv *= 2;
    nw *= 2;
    double scale = 1 / (double)(nv * nw * nx * ny * nz);
    double charge = cs[v] * cs[w] * scale;
    double pu1 = cs[u] / 2.;
    double pu2 = -pu1;
    double b0 = 0, b1 = 0, b2 = 0;
    for (int i = 0; i < nv; i++) {
        pole[v] = -(cs[v] / 2.) + cs[v] / (double)(2 * nv) + (double)i * (cs[v] / (double)nv);
        for (int j = 0; j < nw; j++) {
            pole[w] = -(cs[w] / 2.) + cs[w] / (double)(2 * nw) + (double)j * (cs[w] / (double)nw);
            for (int a = 0; a < nx; a++) {
                double rx = R[0] - cs[0] / 2 + cs[0] / (double)(2 * nx) + (cs[0] / (double)nx) * (double)a;
                for (int b = 0; b < ny; b++) {
                    double ry = R[1] - cs[1] / 2 + cs[1] / (double)(2 * ny) + (cs[1] / (double)ny) * (double)b;
                    for (int g = 0; g < nz; g++) {
                        double rz = R[2] - cs[2] / 2 + cs[2] / (double)(2 * nz) + (cs[2] / (double)nz) * (double)g;
                        pole[u] = pu1;
                        R2[0] = rx - pole[0];
                        R2[1] = ry - pole[1];
                        R2[2] = rz - pole[2];
                        double r = sqrt(R2[0] * R2[0] + R2[1] * R2[1] + R2[2] * R2[2]);
                        double qr = charge / (4 * M_PI * r * r * r);
                        double bx = R2[0] * qr, by = R2[1] * qr, bz = R2[2] * qr;
                        pole[u] = pu2;
                        R2[0] = rx - pole[0];
                        R2[1] = ry - pole[1];
                        R2[2] = rz - pole[2];
                        r = sqrt(R2[0] * R2[0] + R2[1] * R2[1] + R2[2] * R2[2]);
                        qr = -charge / (4 * M_PI * r * r * r);
                        b0 += (bx + R2[0] * qr);
                        b1 += (by + R2[1] * qr);
                        b2 += (bz + R2[2] * qr);
                    }
                }
            }
        }
    }
    B[0] = b0;
    B[1] = b1;
    B[2] = b2;
}



// One thread per (folded target, source axis s).  Kc[6][h0+1][h1+1][h2+1].
__global__ void k_arne_kernel(ArneGeom g, double* __restrict__ Kc) {
    const long n0 = g.h[0] + 1, n1 = g.h[1] + 1, n2 = g.h[2] + 1;
    const long ncell = n0 * n1 * n2;
    const long tot = ncell * 3;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < tot; q += (long)gridDim.x * blockDim.x) {
        const int s = (int)(q / ncell);
        const long c = q - s * ncell;
        const int t0 = (int)(c / (n1 * n2));
        const int t1 = (int)((c / n2) % n1);
        const int t2 = (int)(c % n2);
        double acc[3] = {0, 0, 0};
        if (t0 < g.size[0] && t1 < g.size[1] && t2 < g.size[2]) {
            // first image >= r1 of each wrapped index
            long f[3];
            const int t[3] = {t0, t1, t2};
            for (int a = 0; a < 3; a++) {
                long x = t[a];
                while (x - g.size[a] >= g.r1[a]) x -= g.size[a];
                while (x < g.r1[a]) x += g.size[a];
                f[a] = x;
            }
            for (long z = f[2]; z <= g.r2[2]; z += g.size[2])
                for (long y = f[1]; y <= g.r2[1]; y += g.size[1])
                    for (long x = f[0]; x <= g.r2[0]; x += g.size[0]) {
                        double B[3];
                        arne_point(s, x, y, z, g.cs, g.Lmin, g.accuracy, B);
                        for (int d = s; d < 3; d++) acc[d] += B[d];
                    }
        }
        const int full[3][3] = {{KXX, KXY, KXZ}, {KXY, KYY, KYZ}, {KXZ, KYZ, KZZ}};
        for (int d = s; d < 3; d++) Kc[(long)full[s][d] * ncell + c] = acc[d];
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
    k_arne_kernel<<<hsb_grid_1d(nfold * 3, 128, 16), 128, 0, st>>>(*g, Kc);
    return cudaGetLastError();
}

cudaError_t hsb_arne_expand_launch(const double* Kc, int comp, int L0, int L1, int L2, double* out,
                                   cudaStream_t st) {
    const long vol = (long)L0 * L1 * L2;
    k_arne_expand<<<hsb_grid_1d(vol, 256), 256, 0, st>>>(Kc, comp, L0, L1, L2, out);
    return cudaGetLastError();
}
