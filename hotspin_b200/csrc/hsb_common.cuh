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

// ------------------------------------------------------------------ programmatic dependent launch
// Kernels on the step path begin with hsb_pdl_enter(): it waits until the preceding kernel in
// the stream has completed and its writes are visible (a no-op when this launch was not
// programmatic), then lets the next kernel start launching, so that its blocks are resident
// and waiting when this grid finishes instead of being launched after it.  Every access to
// global memory comes after the wait.  hsb_launch sets the programmatic-serialization
// attribute while hsb_pdl_enabled() (hsb_set_pdl; off by default: measured slower in the
// step graphs).
__device__ __forceinline__ void hsb_pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
int hsb_pdl_enabled();
template <typename... KArgs, typename... Args>
static inline cudaError_t hsb_launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                                     Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = hsb_pdl_enabled() ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, args...);
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

// Harmonic mean 2ab/(a+b), 0 when a+b == 0 (the reference's avgGeomZero).
template <typename T>
__device__ __forceinline__ T harm0(T a, T b) {
    T s = a + b;
    return (s == T(0)) ? T(0) : T(2) * a * b / s;
}

// Neighbour index along an axis: wrap when periodic, clamp otherwise.
__device__ __forceinline__ int nb_lo(int i, int n, int wrap) {
    int j = i - 1;
    if (j < 0) j = wrap ? n - 1 : 0;
    return j;
}
__device__ __forceinline__ int nb_hi(int i, int n, int wrap) {
    int j = i + 1;
    if (j >= n) j = wrap ? 0 : n - 1;
    return j;
}
