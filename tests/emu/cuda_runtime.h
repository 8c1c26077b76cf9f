// CPU emulation of the CUDA execution model -- TEST INFRASTRUCTURE ONLY.
//
// tests/emu/build.py compiles the library's own CUDA sources (hotspin_b200/csrc/*.cu) as host
// C++ against this header instead of the CUDA toolkit's, so that the test suite can run the
// kernels themselves, unchanged, on a machine without a GPU: every CUDA thread is a fiber, a
// block runs its fibers until each reaches a barrier (__syncthreads, __syncwarp, a warp
// shuffle) and releases them together, and the runtime calls the library makes (memory,
// copies, streams, events, graph capture and replay, function attributes) are served from
// host memory in stream order.  The launch checks of the real runtime that the library's
// host code could trip (block size, grid size, dynamic shared memory above a kernel's
// attribute) are made here too.  The product never loads the emulated library: hotspin_b200/_lib.py
// loads only the nvcc-built libhsb200.so; tests swap the emulated library in explicitly.
#pragma once
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include <functional>
#include <type_traits>
#include <utility>

// ------------------------------------------------------------------ qualifiers
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __grid_constant__
#define __shared__ static
#define __align__(n) __attribute__((aligned(n)))
#define __export__

// ------------------------------------------------------------------ vector types
struct dim3 {
    unsigned x, y, z;
    constexpr dim3(unsigned x_ = 1, unsigned y_ = 1, unsigned z_ = 1) : x(x_), y(y_), z(z_) {}
};
struct uint3 {
    unsigned x, y, z;
};
struct __attribute__((aligned(8))) float2 {
    float x, y;
};
struct __attribute__((aligned(16))) float4 {
    float x, y, z, w;
};
struct __attribute__((aligned(16))) double2 {
    double x, y;
};
struct double3 {
    double x, y, z;
};
struct int3 {
    int x, y, z;
};
inline double3 make_double3(double x, double y, double z) { return double3{x, y, z}; }
inline int3 make_int3(int x, int y, int z) { return int3{x, y, z}; }
inline float2 make_float2(float x, float y) { return float2{x, y}; }
inline float4 make_float4(float x, float y, float z, float w) { return float4{x, y, z, w}; }
inline double2 make_double2(double x, double y) { return double2{x, y}; }

// ------------------------------------------------------------------ built-in variables
extern uint3 threadIdx, blockIdx;
extern dim3 blockDim, gridDim;

// ------------------------------------------------------------------ runtime types
enum cudaError {
    cudaSuccess = 0,
    cudaErrorInvalidValue = 1,
    cudaErrorMemoryAllocation = 2,
    cudaErrorInvalidConfiguration = 9,
    cudaErrorLaunchFailure = 719,
    cudaErrorNotReady = 600,
    cudaErrorStreamCaptureUnsupported = 900,
};
typedef enum cudaError cudaError_t;
typedef struct CUstream_st* cudaStream_t;
typedef struct CUevent_st* cudaEvent_t;
typedef struct CUgraph_st* cudaGraph_t;
typedef struct CUgraphExec_st* cudaGraphExec_t;
enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3,
    cudaMemcpyDefault = 4
};
enum cudaStreamCaptureMode {
    cudaStreamCaptureModeGlobal = 0,
    cudaStreamCaptureModeThreadLocal = 1,
    cudaStreamCaptureModeRelaxed = 2
};
enum cudaFuncAttribute {
    cudaFuncAttributeMaxDynamicSharedMemorySize = 8,
    cudaFuncAttributePreferredSharedMemoryCarveout = 9
};
enum cudaDeviceAttr { cudaDevAttrMultiProcessorCount = 16 };
#define cudaStreamNonBlocking 0x01
#define cudaEventDisableTiming 0x02

// ------------------------------------------------------------------ runtime API (emulated)
cudaError_t cudaMalloc(void** p, size_t n);
template <class T>
inline cudaError_t cudaMalloc(T** p, size_t n) {
    return cudaMalloc((void**)p, n);
}
cudaError_t cudaMallocHost(void** p, size_t n);
template <class T>
inline cudaError_t cudaMallocHost(T** p, size_t n) {
    return cudaMallocHost((void**)p, n);
}
cudaError_t cudaFree(void* p);
cudaError_t cudaFreeHost(void* p);
cudaError_t cudaMemcpy(void* dst, const void* src, size_t n, cudaMemcpyKind kind);
cudaError_t cudaMemcpyAsync(void* dst, const void* src, size_t n, cudaMemcpyKind kind, cudaStream_t st = 0);
cudaError_t cudaMemset(void* p, int v, size_t n);
cudaError_t cudaMemsetAsync(void* p, int v, size_t n, cudaStream_t st = 0);
cudaError_t cudaStreamCreateWithFlags(cudaStream_t* st, unsigned flags);
cudaError_t cudaStreamDestroy(cudaStream_t st);
cudaError_t cudaStreamSynchronize(cudaStream_t st);
cudaError_t cudaStreamBeginCapture(cudaStream_t st, cudaStreamCaptureMode mode);
cudaError_t cudaStreamEndCapture(cudaStream_t st, cudaGraph_t* g);
cudaError_t cudaGraphInstantiate(cudaGraphExec_t* e, cudaGraph_t g, unsigned long long flags = 0);
cudaError_t cudaGraphLaunch(cudaGraphExec_t e, cudaStream_t st);
cudaError_t cudaGraphDestroy(cudaGraph_t g);
cudaError_t cudaGraphExecDestroy(cudaGraphExec_t e);
cudaError_t cudaEventCreate(cudaEvent_t* e);
cudaError_t cudaEventCreateWithFlags(cudaEvent_t* e, unsigned flags);
cudaError_t cudaEventDestroy(cudaEvent_t e);
cudaError_t cudaEventRecord(cudaEvent_t e, cudaStream_t st = 0);
cudaError_t cudaEventQuery(cudaEvent_t e);
cudaError_t cudaEventSynchronize(cudaEvent_t e);
cudaError_t cudaEventElapsedTime(float* ms, cudaEvent_t a, cudaEvent_t b);
cudaError_t cudaGetLastError();
const char* cudaGetErrorString(cudaError_t e);
cudaError_t cudaGetDevice(int* dev);
struct cudaDeviceProp {
    char name[256];
    size_t totalGlobalMem, sharedMemPerBlock, totalConstMem, textureAlignment, memPitch;
    int regsPerBlock, warpSize, maxThreadsPerBlock, maxThreadsDim[3], maxGridSize[3], major, minor, clockRate,
        multiProcessorCount, kernelExecTimeoutEnabled, computeMode, deviceOverlap, concurrentKernels, integrated,
        canMapHostMemory;
};
cudaError_t cudaGetDeviceProperties(cudaDeviceProp* p, int dev);
cudaError_t cudaThreadSynchronize();
cudaError_t cudaDeviceSynchronize();
cudaError_t cudaDeviceGetAttribute(int* v, cudaDeviceAttr a, int dev);
template <class T>
inline cudaError_t cudaGetSymbolAddress(void** p, const T& symbol) {
    *p = (void*)&symbol;
    return cudaSuccess;
}

// ------------------------------------------------------------------ launches
namespace hsbemu {
struct Cfg {
    dim3 grid, block;
    size_t smem;
    cudaStream_t st;
};
void set_attribute(const void* fn, int attr, int value);
// Run (or, while the stream is being captured, record) one launch of `body` over the grid.
void submit(const void* fn, const Cfg& c, std::function<void()> body);
void* dyn_smem();

template <class F>
struct Launcher;
template <class... P>
struct Launcher<void (*)(P...)> {
    void (*f)(P...);
    Cfg c;
    // the arguments convert to the kernel's parameter types at the call, as in a launch
    void operator()(P... a) const {
        void (*fn)(P...) = f;
        submit((const void*)fn, c, [fn, a...]() { fn(a...); });
    }
};
template <class... P>
inline Launcher<void (*)(P...)> launch(void (*f)(P...), dim3 g, dim3 b, size_t smem = 0, cudaStream_t st = 0) {
    return Launcher<void (*)(P...)>{f, Cfg{g, b, smem, st}};
}
}  // namespace hsbemu

template <class T>
inline cudaError_t cudaFuncSetAttribute(T* fn, cudaFuncAttribute attr, int value) {
    hsbemu::set_attribute((const void*)fn, (int)attr, value);
    return cudaSuccess;
}

// ------------------------------------------------------------------ device built-ins
void __syncthreads();
void __syncwarp(unsigned mask = 0xffffffffu);
uint64_t hsbemu_shfl_xor(unsigned mask, uint64_t bits, int lane_mask);
template <class T>
inline T __shfl_xor_sync(unsigned mask, T v, int lane_mask, int width = 32) {
    static_assert(sizeof(T) <= 8, "shuffle of a scalar");
    (void)width;
    uint64_t b = 0;
    memcpy(&b, &v, sizeof(T));
    b = hsbemu_shfl_xor(mask, b, lane_mask);
    T r;
    memcpy(&r, &b, sizeof(T));
    return r;
}
inline void __threadfence() {}
template <class T>
inline T __ldg(const T* p) {
    return *p;
}
inline float __uint_as_float(unsigned u) {
    float f;
    memcpy(&f, &u, 4);
    return f;
}
inline unsigned __float_as_uint(float f) {
    unsigned u;
    memcpy(&u, &f, 4);
    return u;
}
inline long long __double_as_longlong(double d) {
    long long u;
    memcpy(&u, &d, 8);
    return u;
}
inline double __longlong_as_double(long long u) {
    double d;
    memcpy(&d, &u, 8);
    return d;
}
inline float __fdividef(float a, float b) { return a / b; }
inline float __expf(float x) { return expf(x); }
inline unsigned __umulhi(unsigned a, unsigned b) { return (unsigned)(((unsigned long long)a * b) >> 32); }
inline int __ffs(int x) { return __builtin_ffs(x); }
inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
inline void sincospif(float x, float* s, float* c) {
    *s = (float)sin(M_PI * (double)x);
    *c = (float)cos(M_PI * (double)x);
}
inline float cospif(float x) { return (float)cos(M_PI * (double)x); }
inline double sinpi(double x) { return sin(M_PI * x); }
inline double cospi(double x) { return cos(M_PI * x); }
// The device's integer and floating-point min / max overloads.
template <class A, class B>
inline typename std::common_type<A, B>::type min(A a, B b) {
    typedef typename std::common_type<A, B>::type T;
    return (T)a < (T)b ? (T)a : (T)b;
}
template <class A, class B>
inline typename std::common_type<A, B>::type max(A a, B b) {
    typedef typename std::common_type<A, B>::type T;
    return (T)a < (T)b ? (T)b : (T)a;
}
// Fibers run one at a time, so read-modify-write is atomic here.
template <class T, class U>
inline T atomicAdd(T* a, U v) {
    T o = *a;
    *a = (T)(o + v);
    return o;
}
template <class T, class U>
inline T atomicMax(T* a, U v) {
    T o = *a;
    if ((T)v > o) *a = (T)v;
    return o;
}
template <class T, class U>
inline T atomicOr(T* a, U v) {
    T o = *a;
    *a = (T)(o | v);
    return o;
}
