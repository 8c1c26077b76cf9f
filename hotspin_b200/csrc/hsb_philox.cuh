// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, SC'11) and Box-Muller
// normals, evaluated in registers -- the thermal field costs no memory traffic.
//
// Stream layout: one call per (cell, step): counter = (cell, step_lo, step_hi, 0x48535442),
// key = (seed_lo, seed_hi); outputs (r0, r1) -> normals x, y, (r2, r3) -> normal z, with
// u = (bits + 1/2) 2^-32.
#pragma once
#include <math.h>
#include <stdint.h>

#define HSB_PHILOX_TAG 0x48535442u

__host__ __device__ __forceinline__ uint32_t philox_mulhi(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t lo0 = 0xD2511F53u * c[0];
        const uint32_t hi0 = philox_mulhi(0xD2511F53u, c[0]);
        const uint32_t lo1 = 0xCD9E8D57u * c[2];
        const uint32_t hi1 = philox_mulhi(0xCD9E8D57u, c[2]);
        const uint32_t n0 = hi1 ^ c[1] ^ k0;
        const uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

__host__ __device__ __forceinline__ float philox_u01(uint32_t b) {
    return fmaf((float)b, 2.3283064365386963e-10f, 1.1641532182693481e-10f);
}

// Host builds (checks of the shared per-cell code) take sin / cos of pi x in FP64, rounded.
__host__ __device__ __forceinline__ void philox_normals3(uint32_t cell, uint64_t step, uint32_t seed_lo,
                                                         uint32_t seed_hi, float g[3]) {
    uint32_t c[4] = {cell, (uint32_t)step, (uint32_t)(step >> 32), HSB_PHILOX_TAG};
    philox4x32_10(c, seed_lo, seed_hi);
    const float r0 = sqrtf(-2.0f * logf(philox_u01(c[0])));
    float s0, c0;
    const float a1 = 2.0f * philox_u01(c[1]);
    const float r1 = sqrtf(-2.0f * logf(philox_u01(c[2])));
    const float a3 = 2.0f * philox_u01(c[3]);
#ifdef __CUDA_ARCH__
    sincospif(a1, &s0, &c0);
    const float c1 = cospif(a3);
#else
    s0 = (float)sin(M_PI * (double)a1);
    c0 = (float)cos(M_PI * (double)a1);
    const float c1 = (float)cos(M_PI * (double)a3);
#endif
    g[0] = r0 * c0;
    g[1] = r0 * s0;
    g[2] = r1 * c1;
}
