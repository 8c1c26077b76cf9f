// Average of m with no device allocation by the library.
//
// Some callers cannot let a library allocate device memory: hotspin's own Go layer owns
// every device buffer (gpu.Array, and the reductor's partial buffer that it passes to
// partialSumAsync), and hosts that manage GPU memory through their own pool or budget
// cannot accept a cudaMalloc behind their back.  hsb_average_m_noalloc gives them the
// device-finished, Kahan-compensated FP64 reduction that hsb_sim_average_m runs on the
// simulation handle's own scratch, with the scratch (block partials and the completion
// counter) in a file-scope __device__ array instead of a cudaMalloc'd buffer.  The caller
// passes the input (its FP32 SoA magnetization) and the output (its device memory).
//
// Properties of the static scratch:
//   * fixed size: HSB_NOALLOC_BLOCKS x 3 doubles of block partials + one counter word
//     (about 7 KB), held by every GPU that loads the library until the process exits;
//   * shared by every call: the counter is cleared on the stream at the start of each
//     call, partials are rewritten before they are read, and the array keeps the last
//     call's contents afterwards;
//   * calls that overlap on the GPU (two streams, or two host threads) race on it and give
//     wrong results: serialise them.
#include "hsb_common.cuh"
#include "hsb_reduce.cuh"

#define HSB_NOALLOC_BLOCKS 296
#define HSB_NOALLOC_THREADS 256
#define HSB_NOALLOC_MAX_CELLS (1L << 28)

// [0, 3 * HSB_NOALLOC_BLOCKS): block partials; next 32 doubles: the counter word (padded)
static __device__ __align__(256) double g_noalloc_scratch[3 * HSB_NOALLOC_BLOCKS + 32];

// Same per-thread accumulation and block finish as the handle's reduction kernel
// (k_energy's average-of-m terms), on caller-owned input.
__global__ void k_average_m_static(const float* __restrict__ m, long n, double* partial, unsigned int* counter,
                                   double* out, double scale) {
    double v[3] = {0, 0, 0}, comp[3] = {0, 0, 0};
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int q = 0; q < 3; q++) {
            const double yv = (double)m[q * n + i] - comp[q];
            const double tv = v[q] + yv;
            comp[q] = (tv - v[q]) - yv;
            v[q] = tv;
        }
    }
    block_reduce_store<3>(v, partial, counter, out, gridDim.x, scale);
}

// Device address of the scratch in the current device's context (host code cannot use the
// symbol itself as a device pointer).  Resolved on every call, with the caller's device
// current: it is a host-side runtime query that allocates nothing, and a cached address
// would go stale when the context is destroyed and recreated (cudaDeviceReset).
static int noalloc_scratch(double** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        hsb_set_error("hsb_average_m_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return HSB_ERR_CUDA;
    }
    *out = (double*)p;
    return HSB_OK;
}

// avg3[c] = (1/ncell) * sum_i m[c * ncell + i] for c = 0, 1, 2, into caller-owned device
// memory, enqueued on `stream` (a cudaStream_t; NULL = the legacy default stream).
// Allocates nothing.  Each call resolves the scratch address in the current context (a
// host-side runtime query, no allocation); the first call on a device also loads the
// library's device code there, so make that first call before any stream capture.
HSB_EXPORT int hsb_average_m_noalloc(const float* m, int64_t ncell, double* avg3, void* stream) {
    if (!m || !avg3) {
        hsb_set_error("hsb_average_m_noalloc: null pointer");
        return HSB_ERR_INVALID;
    }
    if (ncell < 1 || ncell > HSB_NOALLOC_MAX_CELLS) {
        hsb_set_error("hsb_average_m_noalloc: ncell = %lld outside [1, %ld] (the fixed scratch serves at most "
                      "2^28 cells)", (long long)ncell, HSB_NOALLOC_MAX_CELLS);
        return HSB_ERR_INVALID;
    }
    double* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc != HSB_OK) return rc;
    double* partial = scratch;
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + 3 * HSB_NOALLOC_BLOCKS);
    cudaStream_t st = (cudaStream_t)stream;
    HSB_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned int), st));
    long blocks = (ncell + HSB_NOALLOC_THREADS - 1) / HSB_NOALLOC_THREADS;
    if (blocks > HSB_NOALLOC_BLOCKS) blocks = HSB_NOALLOC_BLOCKS;
    k_average_m_static<<<(int)blocks, HSB_NOALLOC_THREADS, 0, st>>>(m, (long)ncell, partial, counter, avg3,
                                                                     1.0 / (double)ncell);
    HSB_CUDA_TRY(cudaGetLastError());
    return HSB_OK;
}
