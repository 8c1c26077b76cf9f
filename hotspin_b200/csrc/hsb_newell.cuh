// FP64 Newell demag tensor, shared by the device kernel (hsb_newell.cu) and host builds.
//
// hotspin computes only Kernel_Arne (modules/kernel_magnetostatic.go:25-241); the Newell
// tensor is the closed-form alternative for large grids.  N_ij(R) is the demag tensor
// averaged over a target cell at offset R from a uniformly magnetised source cell of the
// same size (H = -N M); the kernel spectrum stores K = -N, the convention of Kernel_Arne.
//
// * Near field: Newell, Williams and Dunlop, J. Geophys. Res. 98 (1993) 9551 -- the
//   27-point second difference over the three axes (weights 2, -1, -1 per axis) of their
//   auxiliary functions f (diagonal entries) and g (off-diagonal entries), / (4 pi V).
// * Far field: the differences cancel catastrophically as R grows (about (R/a)^5 of the FP64
//   digits), so beyond NEWELL_CUTOFF largest-cell-edges the tensor is the multipole expansion
//   N_ij = -(V / 4 pi) E[d_i d_j (1/|R + u|)] over the offset u of two uniformly distributed
//   points of the two cells (per axis <u^2> = a^2/6, <u^4> = a^4/15, <u^6> = a^6/28) through
//   sixth order in the cell size; the derivatives of 1/|x| come from the Taylor-coefficient
//   recurrence n |x|^2 c_k = (2n - 1) sum_i x_i c_{k-e_i} - (n - 1) sum_i c_{k-2e_i}, n = |k|,
//   d^k (1/|x|) = k! c_k.  At the cutoff both forms agree to about 5e-8 of the largest entry
//   (measured in extended precision), below the FP32 rounding of the stored spectrum.
#pragma once
#include <math.h>

#include "hsb_demag.h"

#define NEWELL_CUTOFF 11.0
#define NEWELL_NMAX 165      // multi-indices of total order <= 8 in three dimensions

__host__ __device__ inline double nw_asinh_ratio(double a, double b2) {
    return b2 > 0.0 ? asinh(a / sqrt(b2)) : 0.0;
}
__host__ __device__ inline double nw_atan_ratio(double num, double den) {
    return den != 0.0 ? atan(num / den) : 0.0;
}

__host__ __device__ inline double newell_f(double x, double y, double z) {
    const double x2 = x * x, y2 = y * y, z2 = z * z;
    const double R = sqrt(x2 + y2 + z2);
    return 0.5 * y * (z2 - x2) * nw_asinh_ratio(y, x2 + z2) + 0.5 * z * (y2 - x2) * nw_asinh_ratio(z, x2 + y2) -
           x * y * z * nw_atan_ratio(y * z, x * R) + (2.0 * x2 - y2 - z2) * R / 6.0;
}

__host__ __device__ inline double newell_g(double x, double y, double z) {
    const double x2 = x * x, y2 = y * y, z2 = z * z;
    const double R = sqrt(x2 + y2 + z2);
    return x * y * z * nw_asinh_ratio(z, x2 + y2) + y * (3.0 * z2 - y2) * nw_asinh_ratio(x, y2 + z2) / 6.0 +
           x * (3.0 * z2 - x2) * nw_asinh_ratio(y, x2 + z2) / 6.0 - z * z2 * nw_atan_ratio(x * y, z * R) / 6.0 -
           z * y2 * nw_atan_ratio(x * z, y * R) / 2.0 - z * x2 * nw_atan_ratio(y * z, x * R) / 2.0 - x * y * R / 3.0;
}

// Near-field N_ij at offset R (program order) between cells of size cs.
__host__ __device__ inline double newell_exact(int i, int j, const double* R, const double* cs) {
    int o[3];
    if (i == j) {
        o[0] = i;
        o[1] = (i + 1) % 3;
        o[2] = (i + 2) % 3;
    } else {
        o[0] = i;
        o[1] = j;
        o[2] = 3 - i - j;
    }
    const double w[3] = {-1.0, 2.0, -1.0};
    double acc = 0.0;
    for (int a = -1; a <= 1; a++)
        for (int b = -1; b <= 1; b++)
            for (int c = -1; c <= 1; c++) {
                const double x = R[o[0]] + a * cs[o[0]];
                const double y = R[o[1]] + b * cs[o[1]];
                const double z = R[o[2]] + c * cs[o[2]];
                const double v = (i == j) ? newell_f(x, y, z) : newell_g(x, y, z);
                acc += w[a + 1] * w[b + 1] * w[c + 1] * v;
            }
    return acc / (4.0 * M_PI * cs[0] * cs[1] * cs[2]);
}

// Position of the multi-index (a, b, c) among those of total order <= 8, ordered by total
// order, then a, then b.
__host__ __device__ inline int nw_idx(int a, int b, int c) {
    const int n = a + b + c;
    return n * (n + 1) * (n + 2) / 6 + a * (n + 1) - a * (a - 1) / 2 + b;
}

__host__ __device__ inline double nw_fact(int k) {
    double f = 1.0;
    for (int i = 2; i <= k; i++) f *= (double)i;
    return f;
}

// Taylor coefficients c_k of 1/|x| about the origin offset x, every |k| <= 8.
__host__ __device__ inline void nw_taylor(const double* x, double* c) {
    const double r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
    c[0] = 1.0 / sqrt(r2);
    for (int n = 1; n <= 8; n++)
        for (int a = 0; a <= n; a++)
            for (int b = 0; b <= n - a; b++) {
                const int k[3] = {a, b, n - a - b};
                double s1 = 0.0, s2 = 0.0;
                for (int d = 0; d < 3; d++) {
                    int km[3] = {k[0], k[1], k[2]};
                    if (k[d] >= 1) {
                        km[d] -= 1;
                        s1 += x[d] * c[nw_idx(km[0], km[1], km[2])];
                        km[d] += 1;
                    }
                    if (k[d] >= 2) {
                        km[d] -= 2;
                        s2 += c[nw_idx(km[0], km[1], km[2])];
                    }
                }
                c[nw_idx(a, b, n - a - b)] = ((2 * n - 1) * s1 - (n - 1) * s2) / (n * r2);
            }
}

// d^k (1/|x|) from the Taylor coefficients: k! c_k.
__host__ __device__ inline double nw_deriv(const double* c, int a, int b, int cc) {
    return nw_fact(a) * nw_fact(b) * nw_fact(cc) * c[nw_idx(a, b, cc)];
}

// Far-field N_ij at offset R through sixth order in the cell size.
__host__ __device__ inline double newell_asymptotic(int i, int j, const double* R, const double* cs) {
    double c[NEWELL_NMAX];
    nw_taylor(R, c);
    int e[3] = {0, 0, 0};
    e[i] += 1;
    e[j] += 1;
    double s2[3], m4[3], m6[3];
    for (int k = 0; k < 3; k++) {
        const double a2 = cs[k] * cs[k];
        s2[k] = a2 / 6.0;
        m4[k] = a2 * a2 / 15.0;
        m6[k] = a2 * a2 * a2 / 28.0;
    }
#define NW_D(p0, p1, p2) nw_deriv(c, e[0] + (p0), e[1] + (p1), e[2] + (p2))
    double t = NW_D(0, 0, 0);
    t += 0.5 * (s2[0] * NW_D(2, 0, 0) + s2[1] * NW_D(0, 2, 0) + s2[2] * NW_D(0, 0, 2));
    double t4 = m4[0] * NW_D(4, 0, 0) + m4[1] * NW_D(0, 4, 0) + m4[2] * NW_D(0, 0, 4);
    t4 += 6.0 * (s2[0] * s2[1] * NW_D(2, 2, 0) + s2[0] * s2[2] * NW_D(2, 0, 2) + s2[1] * s2[2] * NW_D(0, 2, 2));
    t += t4 / 24.0;
    double t6 = m6[0] * NW_D(6, 0, 0) + m6[1] * NW_D(0, 6, 0) + m6[2] * NW_D(0, 0, 6);
    t6 += 15.0 * (m4[0] * s2[1] * NW_D(4, 2, 0) + m4[0] * s2[2] * NW_D(4, 0, 2) + m4[1] * s2[0] * NW_D(2, 4, 0) +
                  m4[1] * s2[2] * NW_D(0, 4, 2) + m4[2] * s2[0] * NW_D(2, 0, 4) + m4[2] * s2[1] * NW_D(0, 2, 4));
    t6 += 90.0 * s2[0] * s2[1] * s2[2] * NW_D(2, 2, 2);
    t += t6 / 720.0;
#undef NW_D
    return -cs[0] * cs[1] * cs[2] / (4.0 * M_PI) * t;
}

// N_ij at offset R: near-field differences below the cutoff, the expansion beyond it.
__host__ __device__ inline double newell_N(int i, int j, const double* R, const double* cs) {
    const double mx = fmax(cs[0], fmax(cs[1], cs[2]));
    const double dist = sqrt(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]) / mx;
    return dist < NEWELL_CUTOFF ? newell_exact(i, j, R, cs) : newell_asymptotic(i, j, R, cs);
}

// K_sd = -N_sd (d = s..2) at folded target (t0, t1, t2), summed over the periodic images in
// Kernel_Arne's loop order (kernel_magnetostatic.go: z, then y, then x); out[d] for d >= s.
__host__ __device__ inline void newell_target(const ArneGeom& g, int s, int t0, int t1, int t2, double* out) {
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
                const double R[3] = {(double)x * g.cs[0], (double)y * g.cs[1], (double)z * g.cs[2]};
                for (int d = s; d < 3; d++) out[d] -= newell_N(s, d, R, g.cs);
            }
}
