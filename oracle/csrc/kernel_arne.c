/*
 * FP64 C restatement of hotspin's demag kernel "Kernel_Arne" -- TEST INFRASTRUCTURE ONLY.
 *
 * Follows src/hotspin-core/modules/kernel_magnetostatic.go:25-241 (integration of the
 * field of the two charged faces of a source cell over a destination cell, integration
 * density from the distance and `accuracy`, periodic images summed, then the upper halves
 * mirrored with the tensor's parities) and kernelRanges/delta/wrap (:243-283).
 *
 * The per-point arithmetic keeps the reference's expression order.  Each wrapped target
 * cell sums its periodic images in the reference's loop order (z, then y, then x), so the
 * result equals a sequential run of the Go code.  Threads own disjoint target cells.
 *
 * Output layout: K[6][L0][L1][L2] (program order), components XX YY ZZ YZ XZ XY
 * (common/index.go:23-28).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { XX = 0, YY = 1, ZZ = 2, YZ = 3, XZ = 4, XY = 5 };
static const int FULL[3][3] = {{XX, XY, XZ}, {XY, YY, YZ}, {XZ, YZ, ZZ}};

static double delta_(long d) {
    if (d < 0) d = -d;
    if (d > 0) d -= 1;
    return (double)d;
}

static void ranges(const int *size, const int *pbc, long *r1, long *r2) {
    for (int c = 0; c < 3; c++) {
        if (pbc[c] == 0) {
            r1[c] = -(long)((size[c] - 1) / 2);
            r2[c] = (long)((size[c] - 1) / 2);
        } else {
            r1[c] = -((long)size[c] * pbc[c] - 1);
            r2[c] = (long)size[c] * pbc[c] - 1;
        }
    }
    if (size[2] == 1 && pbc[2] == 0) r2[2] = 0;
}

/* Field (3 comps) at offset (x,y,z) cells from a source cell charged on the faces normal to s. */
static void point_field(int s, long x, long y, long z, const double *cs, double L,
                        double accuracy, double *B) {
    int u = s, v = (s + 1) % 3, w = (s + 2) % 3;
    double R[3], R2[3], pole[3];
    R[0] = (double)x * cs[0];
    R[1] = (double)y * cs[1];
    R[2] = (double)z * cs[2];
    double dx = delta_(x) * cs[0], dy = delta_(y) * cs[1], dz = delta_(z) * cs[2];
    double d = sqrt(dx * dx + dy * dy + dz * dz);
    if (d == 0) d = L;
    double maxSize = d / accuracy;
    int nv = (int)(fmax(cs[v] / maxSize, 1) + 0.5);
    int nw = (int)(fmax(cs[w] / maxSize, 1) + 0.5);
    int nx = (int)(fmax(cs[0] / maxSize, 1) + 0.5);
    int ny = (int)(fmax(cs[1] / maxSize, 1) + 0.5);
    int nz = (int)(fmax(cs[2] / maxSize, 1) + 0.5);
    nv *= 2;
    nw *= 2;
    double scale = 1 / (double)(nv * nw * nx * ny * nz);
    double surface = cs[v] * cs[w];
    double charge = surface * scale;
    double pu1 = cs[u] / 2.;
    double pu2 = -pu1;
    B[0] = B[1] = B[2] = 0;
    for (int i = 0; i < nv; i++) {
        double pv = -(cs[v] / 2.) + cs[v] / (double)(2 * nv) + (double)i * (cs[v] / (double)nv);
        pole[v] = pv;
        for (int j = 0; j < nw; j++) {
            double pw = -(cs[w] / 2.) + cs[w] / (double)(2 * nw) + (double)j * (cs[w] / (double)nw);
            pole[w] = pw;
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
                        B[0] += (bx + R2[0] * qr);
                        B[1] += (by + R2[1] * qr);
                        B[2] += (bz + R2[2] * qr);
                    }
                }
            }
        }
    }
}

/* Images of wrapped index w within [r1, r2], ascending. */
static int images(long w, int size, long r1, long r2, long *out, int cap) {
    int n = 0;
    long first = w;
    while (first - size >= r1) first -= size;
    while (first < r1) first += size;
    for (long x = first; x <= r2 && n < cap; x += size) out[n++] = x;
    return n;
}

int hsb_oracle_kernel_arne(const int *size, const double *cellsize, const int *pbc,
                           int accuracy_, double *K) {
    long r1[3], r2[3];
    ranges(size, pbc, r1, r2);
    double L = cellsize[0];
    if (cellsize[1] < L) L = cellsize[1];
    if (cellsize[2] < L) L = cellsize[2];
    double accuracy = (double)accuracy_;
    long n0 = size[0], n1 = size[1], n2 = size[2];
    long plane = n1 * n2, vol = n0 * plane;
    memset(K, 0, sizeof(double) * 6 * vol);
    int h0 = size[0] / 2, h1 = size[1] / 2, h2 = size[2] / 2;
    long cap0 = (r2[0] - r1[0]) / size[0] + 2, cap1 = (r2[1] - r1[1]) / size[1] + 2,
         cap2 = (r2[2] - r1[2]) / size[2] + 2;
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
    for (int xw = 0; xw <= h0; xw++) {
        for (int yw = 0; yw <= h1; yw++) {
            long *ix = (long *)malloc(sizeof(long) * (cap0 + cap1 + cap2));
            long *iy = ix + cap0, *iz = iy + cap1;
            int nx = images(xw, size[0], r1[0], r2[0], ix, (int)cap0);
            int ny = images(yw, size[1], r1[1], r2[1], iy, (int)cap1);
            for (int zw = 0; zw <= h2 && zw < size[2]; zw++) {
                if (xw >= size[0] || yw >= size[1]) continue;
                int nz = images(zw, size[2], r1[2], r2[2], iz, (int)cap2);
                double acc[6] = {0, 0, 0, 0, 0, 0};
                for (int s = 0; s < 3; s++) {
                    for (int c = 0; c < nz; c++)
                        for (int b = 0; b < ny; b++)
                            for (int a = 0; a < nx; a++) {
                                double B[3];
                                point_field(s, ix[a], iy[b], iz[c], cellsize, L, accuracy, B);
                                for (int d = s; d < 3; d++) acc[FULL[s][d]] += B[d];
                            }
                }
                long I = xw * plane + yw * n2 + zw;
                for (int c = 0; c < 6; c++) K[c * vol + I] = acc[c];
            }
            free(ix);
        }
    }
    /* mirror (kernel_magnetostatic.go:185-230) */
    for (long x = h0 + 1; x < n0; x++)
        for (long y = 0; y < n1; y++)
            for (long z = 0; z < n2; z++) {
                long I = x * plane + y * n2 + z, J = (n0 - x) * plane + y * n2 + z;
                K[XX * vol + I] = +K[XX * vol + J];
                K[XY * vol + I] = -K[XY * vol + J];
                K[XZ * vol + I] = -K[XZ * vol + J];
                K[YY * vol + I] = +K[YY * vol + J];
                K[YZ * vol + I] = +K[YZ * vol + J];
                K[ZZ * vol + I] = +K[ZZ * vol + J];
            }
    for (long x = 0; x < n0; x++)
        for (long y = h1 + 1; y < n1; y++)
            for (long z = 0; z < n2; z++) {
                long I = x * plane + y * n2 + z, J = x * plane + (n1 - y) * n2 + z;
                K[XX * vol + I] = +K[XX * vol + J];
                K[XY * vol + I] = -K[XY * vol + J];
                K[XZ * vol + I] = +K[XZ * vol + J];
                K[YY * vol + I] = +K[YY * vol + J];
                K[YZ * vol + I] = -K[YZ * vol + J];
                K[ZZ * vol + I] = +K[ZZ * vol + J];
            }
    for (long x = 0; x < n0; x++)
        for (long y = 0; y < n1; y++)
            for (long z = h2 + 1; z < n2; z++) {
                long I = x * plane + y * n2 + z, J = x * plane + y * n2 + (n2 - z);
                K[XX * vol + I] = +K[XX * vol + J];
                K[XY * vol + I] = +K[XY * vol + J];
                K[XZ * vol + I] = -K[XZ * vol + J];
                K[YY * vol + I] = +K[YY * vol + J];
                K[YZ * vol + I] = -K[YZ * vol + J];
                K[ZZ * vol + I] = +K[ZZ * vol + J];
            }
    return 0;
}
