// Kernel_Arne quadrature (kernel_magnetostatic.go:25-241), shared by the device kernel
// (hsb_arne.cu, one warp per target) and host builds (tests/native/rule_check.cu).
#pragma once
#include <math.h>

#include "hsb_demag.h"

__host__ __device__ inline double arne_delta(long d) {
    if (d < 0) d = -d;
    if (d > 0) d -= 1;
    return (double)d;
}

// Field at integer offset (x, y, z) cells of a source cell whose faces normal to axis s carry
// unit surface charge, over the share part, part + nparts, ... of the (i, j) pairs of
// source-face points; the points of a share are visited in the reference's nested order and
// expression order.  The shares' B add up to the whole field.
__host__ __device__ inline void arne_point_part(int s, long x, long y, long z, const double* cs, double Lmin,
                                                double accuracy, int part, int nparts, double* B) {
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
    for (int ij = part; ij < nv * nw; ij += nparts) {
        const int i = ij / nw, j = ij - (ij / nw) * nw;
        pole[v] = -(cs[v] / 2.) + cs[v] / (double)(2 * nv) + (double)i * (cs[v] / (double)nv);
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
    B[0] = b0;
    B[1] = b1;
    B[2] = b2;
}

// A share of the tensor row s at folded target (t0, t1, t2), summed over the periodic images
// (z, then y, then x as the reference); out[d] for d >= s.
__host__ __device__ inline void arne_target_part(const ArneGeom& g, int s, int t0, int t1, int t2, int part,
                                                 int nparts, double* out) {
    out[0] = out[1] = out[2] = 0.0;
    if (!(t0 < g.size[0] && t1 < g.size[1] && t2 < g.size[2])) return;
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
                arne_point_part(s, x, y, z, g.cs, g.Lmin, g.accuracy, part, nparts, B);
                for (int d = s; d < 3; d++) out[d] += B[d];
            }
}
