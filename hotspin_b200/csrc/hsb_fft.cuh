// Block-level power-of-two FFT building blocks (hand-written; no cuFFT).
//
// Stockham autosort passes of radix 16/8/4/2 over shared memory.  Each pass: every thread
// takes butterflies q = tid, tid + nthreads, ..., loads R points at stride L/R, applies
// the twiddles W_{Ns R}^{r (j mod Ns)}, runs an in-register radix-R transform and stores the
// R results at stride Ns.  Shared-memory indices are padded by one element every 16 to
// keep the stride-R stores of the first passes free of bank conflicts.
//
// Templated on the real type so the same code builds the FP64 kernel spectrum and runs
// the FP32 convolution.  DIR = -1 is the forward transform exp(-2 pi i k n / L), DIR = +1
// the inverse; both are unnormalised.
#pragma once
#include <cuda_runtime.h>

template <typename R> struct cplx_t;
template <> struct cplx_t<float> { typedef float2 T; };
template <> struct cplx_t<double> { typedef double2 T; };

__device__ __forceinline__ float2 mkc(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mkc(double a, double b) { return make_double2(a, b); }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mkc(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mkc(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
    return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C> __device__ __forceinline__ C cconj(C a) { return mkc(a.x, -a.y); }
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) { return mkc(a.x * s, a.y * s); }

// Global -> shared fill with UB independent loads in flight per thread: load UB elements
// into registers, then store them (a load followed directly by its dependent store would
// expose the full memory latency once per element).
template <int UB, typename T, typename LD, typename ST>
__device__ __forceinline__ void batched_fill(int total, int tid, int nthr, LD ld, ST st) {
    for (int base = tid; base < total; base += nthr * UB) {
        T v[UB];
#pragma unroll
        for (int u = 0; u < UB; u++) {
            const int e = base + u * nthr;
            if (e < total) v[u] = ld(e);
        }
#pragma unroll
        for (int u = 0; u < UB; u++) {
            const int e = base + u * nthr;
            if (e < total) st(e, v[u]);
        }
    }
}

// shared-memory index padding: one spare slot every 16 complex elements
__host__ __device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }
__host__ __device__ __forceinline__ int fpad_len(int n) { return n + (n >> 4) + 1; }

__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }
// reverse the low `bits` (<= 6) bits of i; straight-line so it folds after unrolling
__host__ __device__ __forceinline__ constexpr int brevc(int i, int bits) {
    return ((((i >> 0) & 1) << 5) | (((i >> 1) & 1) << 4) | (((i >> 2) & 1) << 3) |
            (((i >> 3) & 1) << 2) | (((i >> 4) & 1) << 1) | ((i >> 5) & 1)) >> (6 - bits);
}

// cos / sin of 2 pi k / 16 for k = 0..15 (exact decimal expansions of the constants)
__device__ __forceinline__ constexpr double c16cos(int k) {
    return (k & 15) == 0 ? 1.0
         : (k & 15) == 1 ? 0.92387953251128674
         : (k & 15) == 2 ? 0.70710678118654752
         : (k & 15) == 3 ? 0.38268343236508977
         : (k & 15) == 4 ? 0.0
         : (k & 15) == 5 ? -0.38268343236508977
         : (k & 15) == 6 ? -0.70710678118654752
         : (k & 15) == 7 ? -0.92387953251128674
         : (k & 15) == 8 ? -1.0
         : (k & 15) == 9 ? -0.92387953251128674
         : (k & 15) == 10 ? -0.70710678118654752
         : (k & 15) == 11 ? -0.38268343236508977
         : (k & 15) == 12 ? 0.0
         : (k & 15) == 13 ? 0.38268343236508977
         : (k & 15) == 14 ? 0.70710678118654752
         : 0.92387953251128674;
}
__device__ __forceinline__ constexpr double c16sin(int k) { return c16cos(k - 4); }

// In-register radix-R transform (R = 1, 2, 4, 8, 16) on v[0..R), iterative radix-2 DIT on
// the bit-reversed order.  Fully unrolled: indices and twiddles are compile-time constants.
template <int R, int DIR, typename C>
__device__ __forceinline__ void fft_regp(C* v) {
    typedef decltype(v[0].x) Real;
    constexpr int B = ilog2c(R);
#pragma unroll
    for (int i = 0; i < R; i++) {
        const int j = brevc(i, B);
        if (j > i) { C t = v[i]; v[i] = v[j]; v[j] = t; }
    }
#pragma unroll
    for (int st = 1; st <= B; st++) {
        const int len = 1 << st;
#pragma unroll
        for (int i = 0; i < R; i += len) {
#pragma unroll
            for (int k = 0; k < len / 2; k++) {
                C a = v[i + k]; C b = v[i + k + len / 2];
                const int e = k * (16 / len);
                C bw;
                if (e == 0) bw = b;
                else if (e == 4) bw = (DIR < 0) ? mkc(b.y, -b.x) : mkc(-b.y, b.x);
                else { const Real wr = (Real)c16cos(e); const Real wi = (Real)(DIR * c16sin(e)); bw = mkc(b.x * wr - b.y * wi, b.x * wi + b.y * wr); }
                v[i + k] = cadd(a, bw); v[i + k + len / 2] = csub(a, bw);
            }
        }
    }
}

// One Stockham pass of radix R over `nbatch` transforms of length L stored in `src` with
// batch stride `bs` (padded indices), writing `dst`.  tw[i] = exp(-2 pi i / twL), twL >= L.
template <int R, int DIR, typename C>
__device__ __forceinline__ void stockham_pass(const C* __restrict__ src, C* __restrict__ dst,
                                              int L, int Ns, int nbatch, int bs,
                                              const C* __restrict__ tw, int twL, int tid,
                                              int nthr) {
    const int LR = L / R;
    const int nbf = nbatch * LR;
    const int tstep = twL / (Ns * R);
    for (int q = tid; q < nbf; q += nthr) {
        const int b = q / LR;
        const int j = q - b * LR;
        const C* s = src + b * bs;
        C v[R];
        const int k = j % Ns;
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = s[fpad(j + r * LR)];
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                C w = tw[(r * k) * tstep];
                if (DIR > 0) w = cconj(w);
                v[r] = cmul(v[r], w);
            }
        }
        fft_regp<R, DIR>(v);
        const int d0 = (j - k) * R + k;
        C* d = dst + b * bs;
#pragma unroll
        for (int r = 0; r < R; r++) d[fpad(d0 + r * Ns)] = v[r];
    }
}

// Full transform of `nbatch` length-L sequences (L power of two) held in shared memory
// `a` (padded, batch stride bs); `b` is scratch of the same size.  All threads of the
// block must call it.  Returns the buffer holding the result (a or b).
template <int DIR, typename C>
__device__ C* block_fft(C* a, C* b, int L, int nbatch, int bs, const C* __restrict__ tw, int twL) {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthr = blockDim.x * blockDim.y * blockDim.z;
    C* src = a;
    C* dst = b;
    for (int Ns = 1; Ns < L;) {
        int rem = L / Ns;
        // radix 8 at most: with all radices in one loop the radix-16 butterfly leaves registers
        const int R = rem >= 8 ? 8 : rem;
        __syncthreads();
        switch (R) {
            case 8: stockham_pass<8, DIR>(src, dst, L, Ns, nbatch, bs, tw, twL, tid, nthr); break;
            case 4: stockham_pass<4, DIR>(src, dst, L, Ns, nbatch, bs, tw, twL, tid, nthr); break;
            default: stockham_pass<2, DIR>(src, dst, L, Ns, nbatch, bs, tw, twL, tid, nthr); break;
        }
        Ns *= R;
        C* t = src;
        src = dst;
        dst = t;
    }
    __syncthreads();
    return src;
}
