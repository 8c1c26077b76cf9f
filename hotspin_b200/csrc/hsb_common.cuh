// Common device/host helpers for the hotspin_b200 sm_100a library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#define HSB_EXPORT extern "C" __attribute__((visibility("default")))

// Status codes returned by every entry point of the handle API (include/hotspin_b200.h).
enum {
    HSB_OK = 0,
    HSB_ERR_INVALID = 1,      // bad argument (size, pointer, unsupported option)
    HSB_ERR_CUDA = 2,         // a CUDA runtime call failed
    HSB_ERR_NOMEM = 3,        // device allocation failed
    HSB_ERR_UNSUPPORTED = 4,  // geometry outside what the kernels implement
    HSB_ERR_NONFINITE = 5,    // the state became NaN/Inf
    HSB_ERR_SOLVER = 6,       // adaptive solver could not meet its tolerance
};

void hsb_set_error(const char* fmt, ...);

#define HSB_CUDA_TRY(expr)                                                          \
    do {                                                                            \
        cudaError_t _e = (expr);                                                    \
        if (_e != cudaSuccess) {                                                    \
            hsb_set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr,               \
                          cudaGetErrorString(_e));                                  \
            return HSB_ERR_CUDA;                                                    \
        }                                                                           \
    } while (0)

static inline int hsb_div_up(long a, long b) { return (int)((a + b - 1) / b); }

// Number of SMs of the current device (148 on B200), cached per device.
int hsb_sm_count();

// 1-D grid for a grid-stride loop over n items: a multiple of the SM count, capped so
// each thread gets at least one item.
static inline int hsb_grid_1d(long n, int threads, int blocks_per_sm = 8) {
    long need = (n + threads - 1) / threads;
    long cap = (long)hsb_sm_count() * blocks_per_sm;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

// ------------------------------------------------------------------ device helpers
__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_min_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Read-only loads and fast FP32 division: the device intrinsics, plain forms in host builds
// of the shared per-cell code.
#ifdef __CUDA_ARCH__
#define HSB_LDG(p) __ldg(p)
#define HSB_FDIV(a, b) __fdividef(a, b)
#else
#define HSB_LDG(p) (*(p))
#define HSB_FDIV(a, b) ((a) / (b))
#endif

// Harmonic mean 2ab/(a+b), 0 when a+b == 0 (the reference's avgGeomZero).
template <typename T>
__host__ __device__ __forceinline__ T harm0(T a, T b) {
    T s = a + b;
    return (s == T(0)) ? T(0) : T(2) * a * b / s;
}

// Neighbour index along an axis: wrap when periodic, clamp otherwise.
__host__ __device__ __forceinline__ int nb_lo(int i, int n, int wrap) {
    int j = i - 1;
    if (j < 0) j = wrap ? n - 1 : 0;
    return j;
}
__host__ __device__ __forceinline__ int nb_hi(int i, int n, int wrap) {
    int j = i + 1;
    if (j >= n) j = wrap ? 0 : n - 1;
    return j;
}
