// Zero-padded FFT demagnetising convolution for sm_100a (hand-written FFTs, no cuFFT).
//
// Replaces hotspin's MaxwellPlan (src/hotspin-core/modules/maxwell_convolution.go:103-131):
// memset + copyPad3D + cuFFT D2Z per component, tensSYMMVecMul, cuFFT Z2D + copyUnPad3D
// per component (gpu/fftplanX.go:76-104, copypad.cu, mul.cu:31-90).
//
// Axes: program order a0 (slowest, user z), a1 (user y), a2 (fastest, user x); logic size
// L = 2N for open non-unit axes, N otherwise (engine/zeropad.go:12-22).  The real-to-complex
// axis is a2, packed as a length L2/2 complex FFT; C2 = L2/2 + 1 frequencies are kept.
//
// Forward path (FP32):
//   x-pass   m (SoA, [c][a0][a1][a2]) * msat mask -> X1[c][a0<N0][kx<C2][a1<N1]   (transposed)
//   yz-pass  per kx column: y FFT (N1 -> L1), z FFT (N0 -> L0), symmetric tensor multiply,
//            inverse z (keep a0 < N0), inverse y (keep a1 < N1)        X1 -> X1 (in place)
//            (fused in one kernel when the column fits in shared memory, else three
//             kernels y / z-multiply / y-inverse through X2[c][a0<N0][kx][L1])
//   inv x    X1 -> H[c][a0][a1][a2<N2] * Ms0  (A/m; B = mu0 * H)
// Zero padding is never materialised: the transforms skip the known-zero inputs and
// outputs outside the data block are never stored.
//
// Kernel (FP64): Kernel_Arne (kernel_magnetostatic.go:25-241) evaluated on the GPU, one
// thread per (wrapped target cell in the folded octant, source axis), images summed in
// the reference's loop order; each component is transformed with the same FFT code in
// FP64, the real part of the folded octant kept and scaled by 1/(L0 L1 L2)
// (maxwell_convolution.go:135-223, 350-388), stored FP32 as kern[kx][k1f][k0f][6].
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "hsb_common.cuh"
#include "hsb_demag.h"
#include "hsb_fft.cuh"
#include "hsb_fft4.cuh"


static bool is_pow2(int n) { return n >= 1 && (n & (n - 1)) == 0; }

// ------------------------------------------------------------------------------ x pass
// Forward R2C along a2 for rows of `planes` x N1 rows.  Row (p, y) of the input starts at
// in + p * in_pstride + y * N2 (in_pstride = N1 * N2 for plain layouts).  For FP32 input the
// optional mask multiplies every value.  Output X[(p * C2 + kx) * ldo + y], ldo >= N1.
template <typename Real>
__global__ void k_fft_x_fwd(const Real* __restrict__ in0, const Real* __restrict__ in1, const int* __restrict__ isel,
                            int iinv, const float* __restrict__ mask,
                            long in_cstride, int ncomp_planes_per_comp,
                            int N1, int N2, int L2, int ldo,
                            typename cplx_t<Real>::T* __restrict__ out,
                            const typename cplx_t<Real>::T* __restrict__ tw, int twL, int TY, const int* __restrict__ active) {
    if (active && !*active) return;
    typedef typename cplx_t<Real>::T C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    const int M = L2 / 2;
    const int bs = fpad_len(M);
    C* scr = buf + TY * bs;
    const Real* in = (isel && ((*isel) ^ iinv)) ? in1 : in0;
    const int C2 = M + 1;
    const int p = blockIdx.y;                 // plane = comp * N0 + a0
    const int y0 = blockIdx.x * TY;
    const int ny = min(TY, N1 - y0);
    const int comp = p / ncomp_planes_per_comp;
    const int a0 = p - comp * ncomp_planes_per_comp;
    const Real* src = in + comp * in_cstride + ((long)a0 * N1 + y0) * N2;
    const float* msk = mask ? mask + ((long)a0 * N1 + y0) * N2 : nullptr;
    const int tid = threadIdx.x;
    const int nthr = blockDim.x;
    // load packed z[n] = x[2n] + i x[2n+1], zero beyond N2
    batched_fill<8, C>(
        TY * M, tid, nthr,
        [&](int e) {
            const int r = e / M;
            const int n = e - r * M;
            Real a = 0, b = 0;
            if (r < ny) {
                const int i0 = 2 * n, i1 = 2 * n + 1;
                if (i0 < N2) { a = src[(long)r * N2 + i0]; if (msk) a *= (Real)msk[(long)r * N2 + i0]; }
                if (i1 < N2) { b = src[(long)r * N2 + i1]; if (msk) b *= (Real)msk[(long)r * N2 + i1]; }
            }
            return mkc(a, b);
        },
        [&](int e, C v) {
            const int r = e / M;
            buf[r * bs + fpad(e - r * M)] = v;
        });
    buf = block_fft<-1>(buf, scr, M, TY, bs, tw, twL);
    // post-process: X[k] = E[k] + W^k O[k]; write transposed, y fastest
    const int tstep = twL / L2;
    for (int e = tid; e < C2 * TY; e += nthr) {
        const int k = e / TY;
        const int r = e - k * TY;
        if (r >= ny) continue;
        const C* z = buf + r * bs;
        const C zk = z[fpad(k == M ? 0 : k)];
        const C zc = cconj(z[fpad(k == 0 ? 0 : M - k)]);
        const C ev = mkc((Real)0.5 * (zk.x + zc.x), (Real)0.5 * (zk.y + zc.y));
        // O = (zk - zc) / (2i) = (-i/2)(zk - zc)
        const C df = csub(zk, zc);
        const C od = mkc((Real)0.5 * df.y, (Real)-0.5 * df.x);
        const C w = tw[k * tstep];
        const C xk = cadd(ev, cmul(w, od));
        out[((long)p * C2 + k) * ldo + y0 + r] = xk;
    }
}

// Inverse C2R along a2 with transposed input X[(p * C2 + kx) * ldi + y]; writes the first
// N2 reals of each row, times `scale`, to out + comp * out_cstride + (a0 * N1 + y) * N2.
__global__ void k_fft_x_inv(const float2* __restrict__ in, int ldi, int planes_per_comp, int N1,
                            int N2, int L2, float* __restrict__ out0, float* __restrict__ out1,
                            const int* __restrict__ osel, int oinv, long out_cstride, float scale,
                            const float2* __restrict__ tw, int twL, int TY, const int* __restrict__ active) {
    if (active && !*active) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* buf = reinterpret_cast<float2*>(smem_raw);
    const int M = L2 / 2;
    const int bs = fpad_len(M);
    float2* scr = buf + TY * bs;
    const int C2 = M + 1;
    const int p = blockIdx.y;
    const int y0 = blockIdx.x * TY;
    const int ny = min(TY, N1 - y0);
    const int comp = p / planes_per_comp;
    const int a0 = p - comp * planes_per_comp;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int tstep = twL / L2;
    // stage X[k] for k < M into smem rows as Z[k] = (X[k] + conj(X[M-k])) + i W^-k (X[k] - conj(X[M-k]))
    batched_fill<8, float2>(
        M * TY, tid, nthr,
        [&](int e) {
            const int k = e / TY;
            const int r = e - k * TY;
            float2 zk = make_float2(0.f, 0.f);
            if (r < ny) {
                const float2 xk = in[((long)p * C2 + k) * ldi + y0 + r];
                const float2 xc = cconj(in[((long)p * C2 + (M - k)) * ldi + y0 + r]);
                const float2 s = cadd(xk, xc);
                const float2 d = csub(xk, xc);
                const float2 w = cconj(tw[k * tstep]);
                const float2 wd = cmul(w, d);
                zk = make_float2(s.x - wd.y, s.y + wd.x);  // s + i * wd
            }
            return zk;
        },
        [&](int e, float2 v) {
            const int k = e / TY;
            buf[(e - k * TY) * bs + fpad(k)] = v;
        });
    buf = block_fft<+1>(buf, scr, M, TY, bs, tw, twL);
    float* out = (osel && ((*osel) ^ oinv)) ? out1 : out0;
    float* dst = out + comp * out_cstride + ((long)a0 * N1 + y0) * N2;
    for (int e = tid; e < TY * N2; e += nthr) {
        const int r = e / N2;
        const int x = e - r * N2;
        if (r >= ny) continue;
        const float2 z = buf[r * bs + fpad(x >> 1)];
        dst[(long)r * N2 + x] = scale * ((x & 1) ? z.y : z.x);
    }
}

// ------------------------------------------------------------------------------ y pass
// Columns col = 0..ncol-1, column c holds `nin` values at in + c * ldi (zero-padded to L)
// and `nout` values are stored at out + c * ldo.  May run in place when ldi == ldo.
template <typename Real, int DIR>
__global__ void k_fft_cols(const typename cplx_t<Real>::T* in, int ldi, int nin,
                           typename cplx_t<Real>::T* out, int ldo, int nout, int L, long ncol,
                           const typename cplx_t<Real>::T* __restrict__ tw, int twL, int TB, const int* __restrict__ active) {
    if (active && !*active) return;
    typedef typename cplx_t<Real>::T C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    const int bs = fpad_len(L);
    C* scr = buf + TB * bs;
    const long c0 = (long)blockIdx.x * TB;
    const int nb = (int)min((long)TB, ncol - c0);
    const int tid = threadIdx.x, nthr = blockDim.x;
    batched_fill<8, C>(
        TB * L, tid, nthr,
        [&](int e) {
            const int b = e / L;
            const int n = e - b * L;
            C v = mkc((Real)0, (Real)0);
            if (b < nb && n < nin) v = in[(c0 + b) * (long)ldi + n];
            return v;
        },
        [&](int e, C v) {
            const int b = e / L;
            buf[b * bs + fpad(e - b * L)] = v;
        });
    buf = block_fft<DIR>(buf, scr, L, TB, bs, tw, twL);
    for (int e = tid; e < TB * nout; e += nthr) {
        const int b = e / nout;
        const int n = e - b * nout;
        if (b < nb) out[(c0 + b) * (long)ldo + n] = buf[b * bs + fpad(n)];
    }
}

// ------------------------------------------------------------------------------ z pass
// Data X[((c * Nz + a0) * C2 + kx) * L1 + k1] for c < ncomp, a0 < Nz.  Block = (kx, tile of
// TK consecutive k1).  Forward z transform of the Nz stored rows (zero-padded to L0);
// with `conv`, the symmetric tensor multiply and the inverse transform follow and the
// first Nz rows are stored back.  Without `conv` (kernel setup) all L0 rows are stored
// (then Nz must equal L0).
template <typename Real>
__global__ void k_fft_z(typename cplx_t<Real>::T* X, int ncomp, int Nz, int L0, int C2, int L1,
                        const float* __restrict__ kern, int conv,
                        const typename cplx_t<Real>::T* __restrict__ tw, int twL, int TK, const int* __restrict__ active) {
    if (active && !*active) return;
    typedef typename cplx_t<Real>::T C;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    C* buf = reinterpret_cast<C*>(smem_raw);
    const int bs = fpad_len(L0);
    C* scr = buf + ncomp * TK * bs;
    const int kx = blockIdx.y;
    const int k10 = blockIdx.x * TK;
    const int nk = min(TK, L1 - k10);
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int nbatch = ncomp * TK;  // batch index = c * TK + t
    batched_fill<8, C>(
        ncomp * L0 * TK, tid, nthr,
        [&](int e) {
            const int t = e % TK;
            const int rest = e / TK;
            const int a0 = rest % L0;
            const int c = rest / L0;
            C v = mkc((Real)0, (Real)0);
            if (t < nk && a0 < Nz) v = X[(((long)c * Nz + a0) * C2 + kx) * L1 + k10 + t];
            return v;
        },
        [&](int e, C v) {
            const int t = e % TK;
            const int rest = e / TK;
            buf[((rest / L0) * TK + t) * bs + fpad(rest % L0)] = v;
        });
    buf = block_fft<-1>(buf, scr, L0, nbatch, bs, tw, twL);
    scr = (buf == reinterpret_cast<C*>(smem_raw)) ? buf + ncomp * TK * bs : reinterpret_cast<C*>(smem_raw);
    if (conv) {
        const int h0 = L0 / 2, h1 = L1 / 2;
        for (int e = tid; e < L0 * TK; e += nthr) {
            const int t = e % TK;
            const int k0 = e / TK;
            if (t >= nk) continue;
            const int k1 = k10 + t;
            const int f0 = k0 > h0 ? L0 - k0 : k0;
            const int f1 = k1 > h1 ? L1 - k1 : k1;
            const Real s0 = k0 > h0 ? (Real)-1 : (Real)1;
            const Real s1 = k1 > h1 ? (Real)-1 : (Real)1;
            const float* K = kern + (((long)kx * (h1 + 1) + f1) * (h0 + 1) + f0) * 6;
            const Real kxx = K[KXX], kyy = K[KYY], kzz = K[KZZ];
            const Real kyz = s1 * K[KYZ], kxz = s0 * K[KXZ], kxy = s0 * s1 * K[KXY];
            C* p0 = &buf[(0 * TK + t) * bs + fpad(k0)];
            C* p1 = &buf[(1 * TK + t) * bs + fpad(k0)];
            C* p2 = &buf[(2 * TK + t) * bs + fpad(k0)];
            const C m0 = *p0, m1 = *p1, m2 = *p2;
            *p0 = mkc(kxx * m0.x + kxy * m1.x + kxz * m2.x, kxx * m0.y + kxy * m1.y + kxz * m2.y);
            *p1 = mkc(kxy * m0.x + kyy * m1.x + kyz * m2.x, kxy * m0.y + kyy * m1.y + kyz * m2.y);
            *p2 = mkc(kxz * m0.x + kyz * m1.x + kzz * m2.x, kxz * m0.y + kyz * m1.y + kzz * m2.y);
        }
        buf = block_fft<+1>(buf, scr, L0, nbatch, bs, tw, twL);
    }
    const int nstore = conv ? Nz : L0;
    for (int e = tid; e < ncomp * nstore * TK; e += nthr) {
        const int t = e % TK;
        const int rest = e / TK;
        const int a0 = rest % nstore;
        const int c = rest / nstore;
        if (t < nk) X[(((long)c * Nz + a0) * C2 + kx) * L1 + k10 + t] = buf[(c * TK + t) * bs + fpad(a0)];
    }
}

// ------------------------------------------------------------------------------ fused y/z
// One block per kx column.  X1[((c * N0 + a0) * C2 + kx) * N1 + a1].  Shared memory holds
// the 3*N0 y-columns of length L1; the z transform (length L0 = LZ <= 16) runs in
// registers, one thread per k1.
// Threads per block of the fused kernel: the per-thread z transform holds 3 x LZ complex
// values, so long z axes trade threads for registers.
template <int LZ> struct yz_threads { static const int value = LZ >= 16 ? 256 : (LZ >= 8 ? 512 : 1024); };

template <int LZ>
__global__ void __launch_bounds__(yz_threads<LZ>::value) k_fft_yz_conv(float2* __restrict__ X1, int N0, int N1, int L1, int C2,
                                                     const float* __restrict__ kern,
                                                     const float2* __restrict__ tw, int twL, const int* __restrict__ active) {
    if (active && !*active) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* buf = reinterpret_cast<float2*>(smem_raw);
    const int bs = fpad_len(L1);
    const int kx = blockIdx.x;
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int ncol = 3 * N0;
    float2* scr = buf + ncol * bs;
    // load columns (N1 values each, zero-padded to L1)
    batched_fill<8, float2>(
        ncol * L1, tid, nthr,
        [&](int e) {
            const int col = e / L1;
            const int n = e - col * L1;
            float2 v = make_float2(0.f, 0.f);
            if (n < N1) v = X1[((long)col * C2 + kx) * N1 + n];
            return v;
        },
        [&](int e, float2 v) {
            const int col = e / L1;
            buf[col * bs + fpad(e - col * L1)] = v;
        });
    buf = block_fft<-1>(buf, scr, L1, ncol, bs, tw, twL);
    scr = (buf == reinterpret_cast<float2*>(smem_raw)) ? buf + ncol * bs : reinterpret_cast<float2*>(smem_raw);
    const int h0 = LZ / 2, h1 = L1 / 2;
    const int ztstep = twL / LZ;
    (void)ztstep;
    for (int k1 = tid; k1 < L1; k1 += nthr) {
        float2 v[3][LZ];
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int z = 0; z < LZ; z++)
                v[c][z] = (z < N0) ? buf[(c * N0 + z) * bs + fpad(k1)] : make_float2(0.f, 0.f);
#pragma unroll
        for (int c = 0; c < 3; c++) fft_regp<LZ, -1>(v[c]);
        const int f1 = k1 > h1 ? L1 - k1 : k1;
        const float s1 = k1 > h1 ? -1.f : 1.f;
        const float* Kb = kern + ((long)kx * (h1 + 1) + f1) * (h0 + 1) * 6;
#pragma unroll
        for (int k0 = 0; k0 < LZ; k0++) {
            const int f0 = k0 > h0 ? LZ - k0 : k0;
            const float s0 = k0 > h0 ? -1.f : 1.f;
            const float* K = Kb + f0 * 6;
            const float kxx = K[KXX], kyy = K[KYY], kzz = K[KZZ];
            const float kyz = s1 * K[KYZ], kxz = s0 * K[KXZ], kxy = s0 * s1 * K[KXY];
            const float2 m0 = v[0][k0], m1 = v[1][k0], m2 = v[2][k0];
            v[0][k0] = make_float2(kxx * m0.x + kxy * m1.x + kxz * m2.x, kxx * m0.y + kxy * m1.y + kxz * m2.y);
            v[1][k0] = make_float2(kxy * m0.x + kyy * m1.x + kyz * m2.x, kxy * m0.y + kyy * m1.y + kyz * m2.y);
            v[2][k0] = make_float2(kxz * m0.x + kyz * m1.x + kzz * m2.x, kxz * m0.y + kyz * m1.y + kzz * m2.y);
        }
#pragma unroll
        for (int c = 0; c < 3; c++) fft_regp<LZ, +1>(v[c]);
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int z = 0; z < LZ; z++)
                if (z < N0) buf[(c * N0 + z) * bs + fpad(k1)] = v[c][z];
    }
    buf = block_fft<+1>(buf, scr, L1, ncol, bs, tw, twL);
    for (int e = tid; e < ncol * N1; e += nthr) {
        const int col = e / N1;
        const int n = e - col * N1;
        X1[((long)col * C2 + kx) * N1 + n] = buf[col * bs + fpad(n)];
    }
}

// ------------------------------------------------------------------------------ fast path
// Compile-time-sized kernels on the four-step register FFT (hsb_fft4.cuh).  Same data
// layouts and results as the generic kernels above; selected when the lengths fit.

// Per-slot offsets of a batched launch (slot = blockIdx.z; all zero for a single convolution).
struct SlotStrides {
    long in;            // floats between slots' inputs
    long x1;            // complex elements between slots' spectra
    long out;           // floats between slots' outputs
    int sel;            // ints between slots' selector / active words
    const float* scale; // per-slot output scale (null: the launch's scale)
    int scale_stride;
    long kern;          // floats between slots' kernel spectra (0: one shared spectrum)
};

// R2C along a2 for TY rows per block, B lanes per row; M = L2/2 packed complex points.
// PR: the row is zero-padded to twice its length (open boundary), so the upper half of
// the packed input is zero.
template <int M, bool PR>
__global__ void __launch_bounds__(256, 3) k_xfwd4(const float* __restrict__ in0, const float* __restrict__ in1,
                                               const int* __restrict__ isel, int iinv,
                                               const float* __restrict__ mask, long in_cstride,
                                               int planes_per_comp, int N1, int N2, int ldo,
                                               float2* __restrict__ out, const float2* __restrict__ tw, int twL,
                                               const float2* __restrict__ tw4, int TY,
                                               const int* __restrict__ active, const SlotStrides ss) {
    const int sl = blockIdx.z;
    if (active && !active[sl * ss.sel]) return;
    in0 += sl * ss.in;
    in1 += sl * ss.in;
    if (isel) isel += sl * ss.sel;
    out += sl * ss.x1;
    constexpr int A = Split<M>::A, B = Split<M>::B, SS = Slot<M>::S, L2 = 2 * M, C2 = M + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int r = tid / B, lane = tid - r * B;
    const int p = blockIdx.y;
    const int y0 = blockIdx.x * TY;
    const int ny = min(TY, N1 - y0);
    const int comp = p / planes_per_comp;
    const int a0 = p - comp * planes_per_comp;
    const float* in = (isel && ((*isel) ^ iinv)) ? in1 : in0;
    float2* slot = sm + r * SS;
    float2 v[A];
    {
        const long row = ((long)a0 * N1 + y0 + r) * N2;
        const float* src = in + comp * in_cstride + row;
        const float* msk = mask ? mask + row : nullptr;
        const bool even = (N2 & 1) == 0;
        if (!msk && even) {
            // the common case as a straight run of independent loads, without the mask and
            // parity branches of the general loop (measured 17 % faster at 512x512x4)
#pragma unroll
            for (int n1 = 0; n1 < A; n1++) {
                const int n = B * n1 + lane;
                v[n1] = (!(PR && n1 >= A / 2) && r < ny && 2 * n < N2)
                            ? __ldg(reinterpret_cast<const float2*>(src) + n) : make_float2(0.f, 0.f);
            }
        } else
#pragma unroll
        for (int n1 = 0; n1 < A; n1++) {
            const int n = B * n1 + lane;
            float a = 0.f, b = 0.f;
            if (!(PR && n1 >= A / 2) && r < ny && 2 * n < N2) {
                if (even) {
                    const float2 t = __ldg(reinterpret_cast<const float2*>(src) + n);
                    a = t.x;
                    b = t.y;
                    if (msk) {
                        const float2 q = __ldg(reinterpret_cast<const float2*>(msk) + n);
                        a *= q.x;
                        b *= q.y;
                    }
                } else {
                    a = __ldg(src + 2 * n);
                    if (msk) a *= __ldg(msk + 2 * n);
                    if (2 * n + 1 < N2) {
                        b = __ldg(src + 2 * n + 1);
                        if (msk) b *= __ldg(msk + 2 * n + 1);
                    }
                }
            }
            v[n1] = make_float2(a, b);
        }
    }
    fft4<M, -1, PR, false>(v, slot, lane, tw4);
    // natural order Z[k] into the slot
#pragma unroll
    for (int j = 0; j < A; j++) slot[fft4_out_index<M>(lane, j)] = v[j];
    __syncwarp();
    // X[k] = E[k] + W^k O[k], k = lane + B j (and k = M on lane 0), with
    // W_L2^k = W_L2^lane (one table entry) x exp(-2 pi i j / 2A) (a constant per j)
    const float2 wl = __ldg(&tw[lane * (twL / L2)]);
#pragma unroll
    for (int j = 0; j < A; j++) {
        const int k = lane + B * j;
        const float2 zk = slot[k];
        const float2 zc0 = slot[(M - k) & (M - 1)];
        const float2 zc = make_float2(zc0.x, -zc0.y);
        const float2 ev = make_float2(0.5f * (zk.x + zc.x), 0.5f * (zk.y + zc.y));
        const float2 od = make_float2(0.5f * (zk.y - zc.y), -0.5f * (zk.x - zc.x));
        const float cr = (float)c64cos(j * (32 / A)), ci = (float)-c64sin(j * (32 / A));
        const float2 w = make_float2(wl.x * cr - wl.y * ci, wl.x * ci + wl.y * cr);
        v[j] = make_float2(ev.x + w.x * od.x - w.y * od.y, ev.y + w.x * od.y + w.y * od.x);
    }
    float2 xm = make_float2(0.f, 0.f);
    if (lane == 0) {
        const float2 z0 = slot[0];  // X[M] = E[0] - O[0]
        xm = make_float2(z0.x - z0.y, 0.f);
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < A; j++) slot[lane + B * j] = v[j];
    if (lane == 0) slot[M] = xm;
    __syncthreads();
    // transposed store: TY (a power of two, nthr = TY * B) consecutive rows per kx, so a
    // thread keeps its row and steps kx by B
    const int rr = tid & (TY - 1);
    if (rr < ny) {
        float2* o = out + (long)p * C2 * ldo + y0 + rr;
        const float2* srow = sm + rr * SS;
        for (int kx = tid >> (__ffs(TY) - 1); kx < C2; kx += B) o[(long)kx * ldo] = srow[kx];
    }
}

// C2R along a2 with transposed input; writes the first N2 reals times `scale`.
// PR: only the first half of the row is kept (open boundary).
template <int M, bool PR>
__global__ void __launch_bounds__(256, 3) k_xinv4(const float2* __restrict__ in, int ldi, int planes_per_comp, int N1,
                                               int N2, float* __restrict__ out0, float* __restrict__ out1,
                                               const int* __restrict__ osel, int oinv, long out_cstride,
                                               float scale, const float2* __restrict__ tw, int twL,
                                               const float2* __restrict__ tw4, int TY,
                                               const int* __restrict__ active, const SlotStrides ss) {
    const int sl = blockIdx.z;
    if (active && !active[sl * ss.sel]) return;
    in += sl * ss.x1;
    out0 += sl * ss.out;
    out1 += sl * ss.out;
    if (osel) osel += sl * ss.sel;
    if (ss.scale) scale = ss.scale[sl * ss.scale_stride];
    constexpr int A = Split<M>::A, B = Split<M>::B, SS = Slot<M>::S, L2 = 2 * M, C2 = M + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int r = tid / B, lane = tid - r * B;
    const int p = blockIdx.y;
    const int y0 = blockIdx.x * TY;
    const int ny = min(TY, N1 - y0);
    const int comp = p / planes_per_comp;
    const int a0 = p - comp * planes_per_comp;
    {
        // transposed load: TY (a power of two, nthr = TY * B) consecutive rows per kx; a
        // thread keeps its row and steps kx by B, eight loads in flight before the stores
        const int rr = tid & (TY - 1);
        const float2* src = in + (long)p * C2 * ldi + y0 + rr;
        float2* srow = sm + rr * SS;
        for (int k0 = tid >> (__ffs(TY) - 1); k0 < C2; k0 += 8 * B) {
            float2 t[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const int kx = k0 + u * B;
                t[u] = (kx < C2 && rr < ny) ? src[(long)kx * ldi] : make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < 8; u++)
                if (k0 + u * B < C2) srow[k0 + u * B] = t[u];
        }
    }
    __syncthreads();
    float2* slot = sm + r * SS;
    // W_L2^k = W_L2^lane x exp(-2 pi i n1 / 2A) for k = lane + B n1
    const float2 wl = __ldg(&tw[lane * (twL / L2)]);
    float2 v[A];
#pragma unroll
    for (int n1 = 0; n1 < A; n1++) {
        // Z[k] = (X[k] + conj X[M-k]) + i W^-k (X[k] - conj X[M-k]),  k = lane + B n1
        const int k = lane + B * n1;
        const float2 xk = slot[k];
        const float2 xc0 = slot[M - k];
        const float2 xc = make_float2(xc0.x, -xc0.y);
        const float2 sA = make_float2(xk.x + xc.x, xk.y + xc.y);
        const float2 d = make_float2(xk.x - xc.x, xk.y - xc.y);
        const float cr = (float)c64cos(n1 * (32 / A)), ci = (float)-c64sin(n1 * (32 / A));
        const float2 w0 = make_float2(wl.x * cr - wl.y * ci, wl.x * ci + wl.y * cr);
        const float2 w = make_float2(w0.x, -w0.y);
        const float2 wd = make_float2(w.x * d.x - w.y * d.y, w.x * d.y + w.y * d.x);
        v[n1] = make_float2(sA.x - wd.y, sA.y + wd.x);
    }
    __syncwarp();
    fft4<M, +1, false, PR>(v, slot, lane, tw4);
    float* out = (osel && ((*osel) ^ oinv)) ? out1 : out0;
    if (r < ny) {
        float* dst = out + comp * out_cstride + ((long)a0 * N1 + y0 + r) * N2;
        const bool even = (N2 & 1) == 0;
        if (even) {
#pragma unroll
            for (int j = 0; j < A; j++) {
                const int n = fft4_out_index<M>(lane, j);
                if (2 * n < N2) reinterpret_cast<float2*>(dst)[n] = make_float2(scale * v[j].x, scale * v[j].y);
            }
        } else {
#pragma unroll
            for (int j = 0; j < A; j++) {
                const int n = fft4_out_index<M>(lane, j);
                if (2 * n < N2) {
                    dst[2 * n] = scale * v[j].x;
                    if (2 * n + 1 < N2) dst[2 * n + 1] = scale * v[j].y;
                }
            }
        }
    }
}

// Fused y FFT + z FFT + symmetric tensor multiply + inverse z + inverse y for one kx column;
// 3*N0 sequences of length L1 (B lanes each), z in registers (LZ = L0 <= 16).
// PR: y and z are zero-padded to twice their lengths (open boundaries): the upper halves of
// the forward inputs are zero and only the lower halves of the inverse outputs are kept.
// Symmetric-tensor component of the pair (c, c2) of program components.
__host__ __device__ constexpr int kcomp(int c, int c2) {
    return c == c2 ? c : ((c + c2 == 3) ? KYZ : ((c + c2 == 2) ? KXZ : KXY));
}

// DZ: a zero-padded z axis of 2 or 4 cells is convolved directly (see k_zdirect).
template <int L1, int LZ, bool PR, bool DZ = PR && (LZ == 4 || LZ == 8)>
__global__ void __launch_bounds__(384, LZ >= 16 ? 1 : 2) k_yz4(float2* __restrict__ X1, int N0, int N1, int C2,
                                             const float* __restrict__ kern4, const float2* __restrict__ tw4,
                                             const int* __restrict__ active, const SlotStrides ss) {
    const int sl = blockIdx.z;
    if (active && !active[sl * ss.sel]) return;
    X1 += sl * ss.x1;
    kern4 += sl * ss.kern;
    constexpr int A = Split<L1>::A, B = Split<L1>::B, SS = Slot<L1>::S;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* sm = reinterpret_cast<float2*>(smem_raw);
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int col = tid / B, lane = tid - col * B;
    const int ncol = 3 * N0;
    const int kx = blockIdx.x;
    float2* slot = sm + col * SS;
    // lanes that exist in this thread's warp (the block may end with a partial warp)
    const int wbase = tid & ~31;
    const unsigned wmask = (nthr - wbase >= 32) ? 0xffffffffu : ((1u << (nthr - wbase)) - 1u);
    float2 v[A];
    const float2* src = X1 + ((long)col * C2 + kx) * N1;
#pragma unroll
    for (int n1 = 0; n1 < A; n1++) {
        const int n = B * n1 + lane;
        v[n1] = (!(PR && n1 >= A / 2) && n < N1) ? src[n] : make_float2(0.f, 0.f);
    }
    // the block's copy of the four-step twiddle matrix (after the column loads are issued)
    float2* tws = sm + ncol * SS;
    for (int i = tid; i < L1; i += nthr) tws[i] = __ldg(&tw4[i]);
    __syncthreads();
    fft4<L1, -1, PR, false, true>(v, slot, lane, tws, wmask);
#pragma unroll
    for (int j = 0; j < A; j++) slot[fft4_out_index<L1>(lane, j)] = v[j];
    __syncthreads();
    const int h0 = LZ / 2, h1 = L1 / 2;
    for (int k1 = tid; k1 < L1; k1 += nthr) {
        if constexpr (DZ) {
            // direct convolution along z with the kernel's z-space rows (k_zdirect):
            // H_c(a0) = sum_b0,c2 G_c,c2(a0 - b0) m_c2(b0), G real for the components even
            // in z, i x (the stored value) for KXZ, KXY, and G(-d) = conj G(d)
            constexpr int NZ = LZ / 2;
            float2 mz[3][NZ];
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int z = 0; z < NZ; z++) mz[c][z] = sm[(c * N0 + z) * SS + k1];
            const float s1 = k1 > h1 ? -1.f : 1.f;
            const long cs = h1 + 1;
            const float* Gb = kern4 + (long)kx * (h0 + 1) * 6 * cs + (k1 > h1 ? L1 - k1 : k1);
            float g[6][NZ];
#pragma unroll
            for (int d = 0; d < NZ; d++)
#pragma unroll
                for (int q = 0; q < 6; q++) g[q][d] = __ldg(Gb + ((long)d * 6 + q) * cs);
#pragma unroll
            for (int d = 0; d < NZ; d++) {
                g[KYZ][d] *= s1;
                g[KXY][d] *= s1;
            }
#pragma unroll
            for (int a0 = 0; a0 < NZ; a0++)
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    float ax = 0.f, ay = 0.f;
#pragma unroll
                    for (int b0 = 0; b0 < NZ; b0++)
#pragma unroll
                        for (int c2 = 0; c2 < 3; c2++) {
                            const int q = kcomp(c, c2);
                            const int d = a0 - b0;
                            const float2 m = mz[c2][b0];
                            if (q == KXZ || q == KXY) {
                                const float hv = d < 0 ? -g[q][-d] : g[q][d];
                                ax = fmaf(-hv, m.y, ax);
                                ay = fmaf(hv, m.x, ay);
                            } else {
                                const float gv = g[q][d < 0 ? -d : d];
                                ax = fmaf(gv, m.x, ax);
                                ay = fmaf(gv, m.y, ay);
                            }
                        }
                    sm[(c * N0 + a0) * SS + k1] = make_float2(ax, ay);
                }
        } else {
        float2 w[3][LZ];
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int z = 0; z < LZ; z++)
                w[c][z] = (!(PR && LZ > 1 && z >= LZ / 2) && z < N0) ? sm[(c * N0 + z) * SS + k1]
                                                                       : make_float2(0.f, 0.f);
#pragma unroll
        for (int c = 0; c < 3; c++) fft_reg64<LZ, -1, PR && (LZ > 1), false>(w[c]);
        const int f1 = k1 > h1 ? L1 - k1 : k1;
        const float s1 = k1 > h1 ? -1.f : 1.f;
        // kern4 layout [kx][f0][component][f1]: consecutive k1 read consecutive words
        const float* Kb = kern4 + (long)kx * (h0 + 1) * 6 * (h1 + 1) + f1;
#pragma unroll
        for (int k0 = 0; k0 < LZ; k0++) {
            const int f0 = k0 > h0 ? LZ - k0 : k0;
            const float s0 = k0 > h0 ? -1.f : 1.f;
            const float* K = Kb + (long)f0 * 6 * (h1 + 1);
            const long cs = h1 + 1;
            const float kxx = __ldg(K + KXX * cs), kyy = __ldg(K + KYY * cs), kzz = __ldg(K + KZZ * cs);
            const float kyz = s1 * __ldg(K + KYZ * cs), kxz = s0 * __ldg(K + KXZ * cs),
                        kxy = s0 * s1 * __ldg(K + KXY * cs);
            const float2 m0 = w[0][k0], m1 = w[1][k0], m2 = w[2][k0];
            w[0][k0] = make_float2(kxx * m0.x + kxy * m1.x + kxz * m2.x, kxx * m0.y + kxy * m1.y + kxz * m2.y);
            w[1][k0] = make_float2(kxy * m0.x + kyy * m1.x + kyz * m2.x, kxy * m0.y + kyy * m1.y + kyz * m2.y);
            w[2][k0] = make_float2(kxz * m0.x + kyz * m1.x + kzz * m2.x, kxz * m0.y + kyz * m1.y + kzz * m2.y);
        }
#pragma unroll
        for (int c = 0; c < 3; c++) fft_reg64<LZ, +1, false, PR && (LZ > 1)>(w[c]);
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int z = 0; z < LZ; z++)
                if (z < N0) sm[(c * N0 + z) * SS + k1] = w[c][z];
        }
    }
    __syncthreads();
#pragma unroll
    for (int n1 = 0; n1 < A; n1++) v[n1] = slot[B * n1 + lane];
    __syncwarp(wmask);
    fft4<L1, +1, false, PR, true>(v, slot, lane, tws, wmask);
    float2* dst = X1 + ((long)col * C2 + kx) * N1;
#pragma unroll
    for (int j = 0; j < A; j++) {
        const int n = fft4_out_index<L1>(lane, j);
        if (n < N1) dst[n] = v[j];
    }
}

// ------------------------------------------------------------------------------ multi-pass, four-step
// Register four-step kernels for the three-kernel y / z path (L0 > 16).  Same layouts as the
// generic k_fft_cols / k_fft_z: X1[col][a1 < N1], X2[col][k1 < L1] with col = (c * N0 + a0) * C2
// + kx.  Every lane of a block runs the transforms (fft4 synchronises whole warps); lanes
// past the last column only skip their loads and stores.

// Forward y transform of columns of `nin` values (zero-padded to L): one column per B lanes.
// PR: nin <= L/2 (open boundary), the upper half of the input is known zero.
template <int L, bool PR>
__global__ void __launch_bounds__(256) k_ycolf4(const float2* __restrict__ in, int nin, float2* __restrict__ out,
                                              long ncol, const float2* __restrict__ tw4,
                                              const int* __restrict__ active) {
    if (active && !*active) return;
    constexpr int A = Split<L>::A, B = Split<L>::B, SS = Slot<L>::S;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const int q = tid / B, lane = tid - q * B;
    const long col = (long)blockIdx.x * (blockDim.x / B) + q;
    const bool ok = col < ncol;
    float2* slot = reinterpret_cast<float2*>(smem_raw) + q * SS;
    const float2* src = in + (ok ? col : 0) * nin;
    float2 v[A];
#pragma unroll
    for (int n1 = 0; n1 < A; n1++) {
        const int n = B * n1 + lane;
        v[n1] = (ok && !(PR && n1 >= A / 2) && n < nin) ? __ldg(src + n) : make_float2(0.f, 0.f);
    }
    fft4<L, -1, PR, false>(v, slot, lane, tw4);
    if (ok) {
        float2* dst = out + col * L;
#pragma unroll
        for (int j = 0; j < A; j++) dst[fft4_out_index<L>(lane, j)] = v[j];
    }
}

// Inverse y transform of columns of L values, keeping the first `nout`.  PR: nout <= L/2.
template <int L, bool PR>
__global__ void __launch_bounds__(256) k_ycoli4(const float2* __restrict__ in, float2* __restrict__ out, int nout,
                                              long ncol, const float2* __restrict__ tw4,
                                              const int* __restrict__ active) {
    if (active && !*active) return;
    constexpr int A = Split<L>::A, B = Split<L>::B, SS = Slot<L>::S;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const int q = tid / B, lane = tid - q * B;
    const long col = (long)blockIdx.x * (blockDim.x / B) + q;
    const bool ok = col < ncol;
    float2* slot = reinterpret_cast<float2*>(smem_raw) + q * SS;
    const float2* src = in + (ok ? col : 0) * L;
    float2 v[A];
#pragma unroll
    for (int n1 = 0; n1 < A; n1++) v[n1] = ok ? __ldg(src + B * n1 + lane) : make_float2(0.f, 0.f);
    fft4<L, +1, false, PR>(v, slot, lane, tw4);
    if (ok) {
        float2* dst = out + col * nout;
#pragma unroll
        for (int j = 0; j < A; j++) {
            const int n = fft4_out_index<L>(lane, j);
            if (n < nout) dst[n] = v[j];
        }
    }
}

// L = 2048 with nin <= 1024 (open boundary) as two 1024-point transforms, one warp per
// column: X[2k] = FFT_1024(x)[k] and X[2k+1] = FFT_1024(x[n] W_2048^n)[k] (the zero upper
// half removes the second radix-2 input).  The column's inputs wait in a per-lane
// shared-memory stash (1024 complex per warp after the fft4 slots) for the odd pass.
// tw: the plan's table exp(-2 pi i j / twL).  (Measured: one warp per column at 12 warps
// per SM beats two warps per column, one per parity, at 24.)
__global__ void __launch_bounds__(128, 4) k_ycolf4_2k(const float2* __restrict__ in, int nin, float2* __restrict__ out,
                                                 long ncol, const float2* __restrict__ tw4, const float2* __restrict__ tw,
                                                 int twL, const int* __restrict__ active) {
    if (active && !*active) return;
    constexpr int L = 1024, A = Split<L>::A, B = Split<L>::B, SS = Slot<L>::S;
    static_assert(B == 32, "one warp per column");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const int q = tid >> 5, lane = tid & 31;
    const long col = (long)blockIdx.x * (blockDim.x >> 5) + q;
    const bool ok = col < ncol;
    float2* slot = reinterpret_cast<float2*>(smem_raw) + q * SS;
    const float2* src = in + (ok ? col : 0) * nin;
    float2* dst = out + (ok ? col : 0) * (2 * L);
    float2* stash = reinterpret_cast<float2*>(smem_raw) + (blockDim.x >> 5) * SS + q * (A * 32);
    const int ts = twL / (2 * L);
    {
        float2 v[A];
#pragma unroll
        for (int n1 = 0; n1 < A; n1++) {
            const int n = B * n1 + lane;
            v[n1] = (ok && n < nin) ? __ldg(src + n) : make_float2(0.f, 0.f);
            stash[n1 * 32 + lane] = v[n1];   // the odd pass re-reads its own lane's inputs
        }
        fft4<L, -1, false, false>(v, slot, lane, tw4);
        if (ok) {
#pragma unroll
            for (int j = 0; j < A; j++) dst[2 * fft4_out_index<L>(lane, j)] = v[j];
        }
    }
    {
        float2 v[A];
#pragma unroll
        for (int n1 = 0; n1 < A; n1++) {
            const int n = B * n1 + lane;
            const float2 x = stash[n1 * 32 + lane];
            const float2 w = __ldg(&tw[n * ts]);
            v[n1] = make_float2(x.x * w.x - x.y * w.y, x.x * w.y + x.y * w.x);
        }
        fft4<L, -1, false, false>(v, slot, lane, tw4);
        if (ok) {
#pragma unroll
            for (int j = 0; j < A; j++) dst[2 * fft4_out_index<L>(lane, j) + 1] = v[j];
        }
    }
}

// Inverse of k_ycolf4_2k keeping nout <= 1024 outputs: x[n] = E[n] + W_2048^-n O[n] with E, O
// the inverse 1024-point transforms of the even and odd spectrum entries.  E waits in a
// per-lane shared-memory stash (1024 complex per warp after the fft4 slots) while O is formed.
__global__ void __launch_bounds__(128, 4) k_ycoli4_2k(const float2* __restrict__ in, float2* __restrict__ out, int nout,
                                                 long ncol, const float2* __restrict__ tw4, const float2* __restrict__ tw,
                                                 int twL, const int* __restrict__ active) {
    if (active && !*active) return;
    constexpr int L = 1024, A = Split<L>::A, B = Split<L>::B, SS = Slot<L>::S;
    static_assert(B == 32, "one warp per column");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int tid = threadIdx.x;
    const int q = tid >> 5, lane = tid & 31;
    const long col = (long)blockIdx.x * (blockDim.x >> 5) + q;
    const bool ok = col < ncol;
    float2* slot = reinterpret_cast<float2*>(smem_raw) + q * SS;
    float2* stash = reinterpret_cast<float2*>(smem_raw) + (blockDim.x >> 5) * SS + q * (A * 32);
    const float2* src = in + (ok ? col : 0) * (2 * L);
    const int ts = twL / (2 * L);
    float2 v[A];
#pragma unroll
    for (int n1 = 0; n1 < A; n1++) v[n1] = ok ? __ldg(src + 2 * (B * n1 + lane)) : make_float2(0.f, 0.f);
    fft4<L, +1, false, false>(v, slot, lane, tw4);
#pragma unroll
    for (int j = 0; j < A; j++) stash[j * 32 + lane] = v[j];   // read back by the same lane
#pragma unroll
    for (int n1 = 0; n1 < A; n1++) v[n1] = ok ? __ldg(src + 2 * (B * n1 + lane) + 1) : make_float2(0.f, 0.f);
    fft4<L, +1, false, false>(v, slot, lane, tw4);
    if (ok) {
        float2* dst = out + col * nout;
#pragma unroll
        for (int j = 0; j < A; j++) {
            const int n = fft4_out_index<L>(lane, j);
            if (n < nout) {
                const float2 w = __ldg(&tw[n * ts]);   // conj(w) = W_2048^-n for the inverse
                const float2 o = v[j], e = stash[j * 32 + lane];
                dst[n] = make_float2(e.x + w.x * o.x + w.y * o.y, e.y + w.x * o.y - w.y * o.x);
            }
        }
    }
}

// z transform + symmetric tensor multiply + inverse z for one (kx, k1) per B lanes, all three
// components in registers (3 x A complex), so the multiply needs no exchange.  Lane l of a
// warp: sequence l % G (consecutive k1), member l / G (G = 32 / B sequences per warp).
// 256 threads = K1B consecutive k1 per block.  kern4: [kx][f0][6][f1]; the block's
// f1 range (always K1B consecutive values) is staged in shared memory with coalesced loads.
// PR: the z axis is zero-padded (N0 = LZ / 2).
// Slot stride ZS: a half-warp holds G sequences (G = 32 / B), so their slots must start on
// distinct 64-bit bank pairs: ZS = 16 / G (mod 16), and ZS holds the B x (A + 1) transpose and
// the L natural-order entries.
template <int LZ> struct ZConv {
    static constexpr int A = Split<LZ>::A, B = Split<LZ>::B, G = 32 / B, K1B = 256 / B, KS = K1B + 1;
    static constexpr int T = B * (A + 1) > LZ ? B * (A + 1) : LZ;
    static constexpr int ZS = ((T - 16 / G + 15) / 16) * 16 + 16 / G;
    static constexpr int smem = K1B * ZS * 8 + (LZ / 2 + 1) * 6 * KS * 4;
};
template <int LZ, bool PR>
__global__ void __launch_bounds__(256, LZ <= 64 ? 2 : 1) k_zconv4(float2* __restrict__ X2, int N0, int C2, int L1,
                                              const float* __restrict__ kern4, const float2* __restrict__ tw4,
                                              const int* __restrict__ active) {
    if (active && !*active) return;
    constexpr int A = Split<LZ>::A, B = Split<LZ>::B, SS = ZConv<LZ>::ZS, G = 32 / B;
    constexpr int K1B = ZConv<LZ>::K1B, KS = ZConv<LZ>::KS, h0 = LZ / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float* ks = reinterpret_cast<float*>(smem_raw + K1B * SS * sizeof(float2));   // [(h0 + 1) * 6][KS]
    const int tid = threadIdx.x;
    const int l = tid & 31, w = tid >> 5;
    const int q = l % G, lane = l / G;
    const int kx = blockIdx.y;
    const int k10 = blockIdx.x * K1B;
    const int k1 = k10 + w * G + q;
    const bool ok = k1 < L1;
    const int h1 = L1 / 2;
    // smallest f1 = min(k1, L1 - k1) over the block's k1 < L1
    const int flo = min(k10, L1 - (min(k10 + K1B, L1) - 1));
    float2* slot = reinterpret_cast<float2*>(smem_raw) + (w * G + q) * SS;
    const long pst = (long)C2 * L1;   // between a0 rows
    const long cst = (long)N0 * pst;  // between components
    float2* base = X2 + (long)kx * L1 + (ok ? k1 : 0);
    float2 v[3][A];
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
        for (int n1 = 0; n1 < A; n1++) {
            const int a0 = B * n1 + lane;
            v[c][n1] = (ok && !(PR && n1 >= A / 2) && a0 < N0) ? base[c * cst + a0 * pst] : make_float2(0.f, 0.f);
        }
    {
        const float* kb = kern4 + (long)kx * (h0 + 1) * 6 * (h1 + 1);
        for (int e = tid; e < (h0 + 1) * 6 * K1B; e += 256) {
            const int row = e / K1B, i = e - row * K1B;
            const int f1 = flo + i;
            if (f1 <= h1) ks[row * KS + i] = __ldg(kb + (long)row * (h1 + 1) + f1);
        }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) fft4<LZ, -1, PR, false>(v[c], slot, lane, tw4);
    __syncthreads();   // the staged spectrum is complete (the slots are per sequence)
    const int k1c = ok ? k1 : k10;
    const int f1 = k1c > h1 ? L1 - k1c : k1c;
    const float s1 = k1c > h1 ? -1.f : 1.f;
    const float* Kb = ks + (f1 - flo);
#pragma unroll
    for (int j = 0; j < A; j++) {
        const int k0 = fft4_out_index<LZ>(lane, j);
        const int f0 = k0 > h0 ? LZ - k0 : k0;
        const float s0 = k0 > h0 ? -1.f : 1.f;
        const float* K = Kb + f0 * 6 * KS;
        const float kxx = K[KXX * KS], kyy = K[KYY * KS], kzz = K[KZZ * KS];
        const float kyz = s1 * K[KYZ * KS], kxz = s0 * K[KXZ * KS], kxy = s0 * s1 * K[KXY * KS];
        const float2 m0 = v[0][j], m1 = v[1][j], m2 = v[2][j];
        v[0][j] = make_float2(kxx * m0.x + kxy * m1.x + kxz * m2.x, kxx * m0.y + kxy * m1.y + kxz * m2.y);
        v[1][j] = make_float2(kxy * m0.x + kyy * m1.x + kyz * m2.x, kxy * m0.y + kyy * m1.y + kyz * m2.y);
        v[2][j] = make_float2(kxz * m0.x + kyz * m1.x + kzz * m2.x, kxz * m0.y + kyz * m1.y + kzz * m2.y);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
        // back to the natural input distribution (lane n2 holds entries B n1 + n2)
#pragma unroll
        for (int j = 0; j < A; j++) slot[fft4_out_index<LZ>(lane, j)] = v[c][j];
        __syncwarp();
#pragma unroll
        for (int n1 = 0; n1 < A; n1++) v[c][n1] = slot[B * n1 + lane];
        __syncwarp();
        fft4<LZ, +1, false, PR>(v[c], slot, lane, tw4);
    }
    if (ok) {
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
            for (int j = 0; j < A; j++) {
                const int a0 = fft4_out_index<LZ>(lane, j);
                if (a0 < N0) base[c * cst + a0 * pst] = v[c][j];
            }
    }
}

// Dispatch tables for the fast kernels.
typedef void (*xfwd4_fn)(const float*, const float*, const int*, int, const float*, long, int, int, int, int,
                         float2*, const float2*, int, const float2*, int, const int*, const SlotStrides);
typedef void (*xinv4_fn)(const float2*, int, int, int, int, float*, float*, const int*, int, long, float,
                         const float2*, int, const float2*, int, const int*, const SlotStrides);
typedef void (*yz4_fn)(float2*, int, int, int, const float*, const float2*, const int*, const SlotStrides);

static xfwd4_fn xfwd4_for(int M, bool pr, int* B, int* S) {
    switch (M) {
#define XF(m) case m: *B = Split<m>::B; *S = Slot<m>::S; return pr ? k_xfwd4<m, true> : k_xfwd4<m, false>;
        XF(8) XF(16) XF(32) XF(64) XF(128) XF(256) XF(512) XF(1024)
#undef XF
    }
    return nullptr;
}
static xinv4_fn xinv4_for(int M, bool pr) {
    switch (M) {
#define XI(m) case m: return pr ? k_xinv4<m, true> : k_xinv4<m, false>;
        XI(8) XI(16) XI(32) XI(64) XI(128) XI(256) XI(512) XI(1024)
#undef XI
    }
    return nullptr;
}
template <int L1, bool PR>
static yz4_fn yz4_for_z(int LZ) {
    switch (LZ) {
        case 1: return k_yz4<L1, 1, PR>;
        case 2: return k_yz4<L1, 2, PR>;
        case 4: return k_yz4<L1, 4, PR>;
        case 8: return k_yz4<L1, 8, PR>;
        case 16: return k_yz4<L1, 16, PR>;
    }
    return nullptr;
}
typedef void (*ycf4_fn)(const float2*, int, float2*, long, const float2*, const int*);
typedef void (*yci4_fn)(const float2*, float2*, int, long, const float2*, const int*);
typedef void (*zc4_fn)(float2*, int, int, int, const float*, const float2*, const int*);

static ycf4_fn ycf4_for(int L, bool pr, int* B, int* S) {
    switch (L) {
#define YC(l) case l: *B = Split<l>::B; *S = Slot<l>::S; return pr ? k_ycolf4<l, true> : k_ycolf4<l, false>;
        YC(16) YC(32) YC(64) YC(128) YC(256) YC(512) YC(1024)
#undef YC
    }
    return nullptr;
}
static yci4_fn yci4_for(int L, bool pr) {
    switch (L) {
#define YC(l) case l: return pr ? k_ycoli4<l, true> : k_ycoli4<l, false>;
        YC(16) YC(32) YC(64) YC(128) YC(256) YC(512) YC(1024)
#undef YC
    }
    return nullptr;
}
static zc4_fn zc4_for(int LZ, bool pr, int* K1B, int* smem) {
    switch (LZ) {
#define ZC(l) case l: *K1B = ZConv<l>::K1B; *smem = ZConv<l>::smem; return pr ? k_zconv4<l, true> : k_zconv4<l, false>;
        ZC(32) ZC(64) ZC(128)
#undef ZC
    }
    return nullptr;
}

static yz4_fn yz4_for(int L1, int LZ, bool pr, int* B, int* S) {
    switch (L1) {
#define YZ(l) case l: *B = Split<l>::B; *S = Slot<l>::S; return pr ? yz4_for_z<l, true>(LZ) : yz4_for_z<l, false>(LZ);
        YZ(16) YZ(32) YZ(64) YZ(128) YZ(256) YZ(512) YZ(1024)
#undef YZ
    }
    return nullptr;
}

// ------------------------------------------------------------------------------ extract
// Real part of the folded octant of one transformed component, scaled, into kern.
__global__ void k_extract(const double2* __restrict__ X, int L0, int C2, int L1, int comp,
                          double scale, float* __restrict__ kern, float* __restrict__ kern4,
                          double* __restrict__ maximag) {
    const int h0 = L0 / 2, h1 = L1 / 2;
    const long tot = (long)C2 * (h1 + 1) * (h0 + 1);
    double mi = 0;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < tot; q += (long)gridDim.x * blockDim.x) {
        const int f0 = (int)(q % (h0 + 1));
        const int f1 = (int)((q / (h0 + 1)) % (h1 + 1));
        const int kx = (int)(q / ((long)(h0 + 1) * (h1 + 1)));
        const double2 v = X[((long)f0 * C2 + kx) * L1 + f1];
        const float kv = (float)(v.x * scale);
        if (kern) kern[q * 6 + comp] = kv;
        if (kern4) kern4[(((long)kx * (h0 + 1) + f0) * 6 + comp) * (h1 + 1) + f1] = kv;
        mi = fmax(mi, fabs(v.y * scale));
    }
    mi = warp_max_d(mi);
    if ((threadIdx.x & 31) == 0 && mi > 0) {
        unsigned long long* a = (unsigned long long*)maximag;
        atomicMax(a, __double_as_longlong(mi));  // positive doubles order like integers
    }
}

// Direct-z rows of the kernel for a zero-padded z axis of N0 = L0 / 2 <= 4 cells (the y/z
// kernel's DZ form): the inverse z transform of the folded spectrum of one component,
// G(d) = sum_k0 K(k0) exp(+2 pi i k0 d / L0), d < N0, in FP64 from the FP64 spectrum.  It is
// real for the components even in z and imaginary for KXZ and KXY (odd in z; stored: the
// imaginary part); its real or imaginary part replaces rows d of kern4 (row N0 = h0 keeps
// the spectrum's value, unused).  Run after k_extract of the same component.
__global__ void k_zdirect(const double2* __restrict__ X, int L0, int C2, int L1, int comp, double scale,
                          float* __restrict__ kern4) {
    const int h0 = L0 / 2, h1 = L1 / 2, N0 = L0 / 2;
    const bool odd = comp == KXZ || comp == KXY;
    const long tot = (long)C2 * (h1 + 1);
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < tot; q += (long)gridDim.x * blockDim.x) {
        const int f1 = (int)(q % (h1 + 1));
        const int kx = (int)(q / (h1 + 1));
        double V[5];
        for (int f0 = 0; f0 <= h0 && f0 < 5; f0++) V[f0] = X[((long)f0 * C2 + kx) * L1 + f1].x * scale;
        for (int d = 0; d < N0; d++) {
            double g = 0.0;
            for (int k0 = 0; k0 < L0; k0++) {
                const int f0 = k0 > h0 ? L0 - k0 : k0;
                const double a = 2.0 * (double)k0 * (double)d / (double)L0;   // angle / pi
                if (odd) g += (k0 > h0 ? -V[f0] : V[f0]) * sinpi(a);
                else g += V[f0] * cospi(a);
            }
            kern4[(((long)kx * (h0 + 1) + d) * 6 + comp) * (h1 + 1) + f1] = (float)g;
        }
    }
}

// ------------------------------------------------------------------------------ host plan
struct hsb_demag_plan_s {
    int N[3], L[3], pbc[3];
    double cs[3];
    int C2, twL;
    int fused;          // 1 = single yz kernel
    int lz;             // compile-time z length for the fused kernel
    float* kern;        // [C2][L1/2+1][L0/2+1][6]
    float* kern4;       // the same values as [C2][L0/2+1][6][L1/2+1] (fast y/z kernel)
    float2* tw4x;       // four-step twiddle matrices of the x (length L2/2) and y (L1) transforms
    float2* tw4y;
    float2* X1;         // [3][N0][C2][N1]
    float2* X2;         // multipass: [3][N0][C2][L1]
    float2* tw;
    double kern_max_imag;
    double kern_max_real;
    int smem_x, smem_xi, smem_yz, smem_y, smem_z;
    int TYx, TYxi, TBy, TKz;
    // four-step fast path (null when the lengths are outside its instantiations)
    xfwd4_fn xfwd4;
    xinv4_fn xinv4;
    yz4_fn yz4;
    int x4_rows, x4_threads, x4_smem, yz4_threads, yz4_smem;
    int x4_S;           // slot stride of the x kernels
    int x4i_rows, x4i_threads, x4i_smem;  // inverse x kernel (tuned separately)
    // four-step multi-pass kernels (L0 > 16): y columns (yc2k = the 2048-point split) and z
    ycf4_fn ycf4;
    yci4_fn yci4;
    zc4_fn zc4;
    int yc2k, yc_threads, yc_cols, yc_smem, zc_k1, zc_smem;
    float2* tw4c;       // four-step twiddles of the y columns (length L1, or 1024 for yc2k)
    int zdirect;        // the y/z kernel convolves z directly: kern4 rows d < N0 hold k_zdirect
    int tensor;         // HSB_DEMAG_ARNE (0) or HSB_DEMAG_NEWELL (1)
    // Grids whose open axes do not pad to a power of two run embedded in the next power-of-two
    // grid (vacuum around them): `inner` is that grid's plan, mpad / hpad its m and H.
    hsb_demag_plan_s* inner;
    float* mpad;
    float* hpad;
    float2* tw4z;       // and of the z transform (length L0)
};

// Largest power-of-two tile (<= cap) whose ping-pong buffers of `per_item` padded complex
// elements of `esize` bytes fit in `budget` bytes of shared memory.
static int pick_tile(int per_item, int esize, int budget, int cap) {
    long per = 2L * fpad_len(per_item) * esize;
    long t = budget / (per > 0 ? per : 1);
    if (t > cap) t = cap;
    if (t < 1) t = 1;
    int p = 1;
    while (p * 2 <= t) p *= 2;
    return p;
}

template <typename C>
static int make_twiddles(int twL, C** out) {
    std::vector<C> h(twL);
    for (int i = 0; i < twL; i++) {
        double a = -2.0 * M_PI * (double)i / (double)twL;
        h[i].x = cos(a);
        h[i].y = sin(a);
    }
    HSB_CUDA_TRY(cudaMalloc((void**)out, sizeof(C) * twL));
    HSB_CUDA_TRY(cudaMemcpy(*out, h.data(), sizeof(C) * twL, cudaMemcpyHostToDevice));
    return HSB_OK;
}

// Four-step twiddle matrix of length L: [k1 B + n2] = the table entry tw[(n2 k1 mod L) twL / L],
// computed by the same expression as make_twiddles so both give identical values.
static int make_tw4(int L, int B, int twL, float2** out) {
    const int A = L / B, ts = twL / L;
    std::vector<float2> h((size_t)A * B);
    for (int k1 = 0; k1 < A; k1++)
        for (int n2 = 0; n2 < B; n2++) {
            const int j = ((n2 * k1) & (L - 1)) * ts;
            const double a = -2.0 * M_PI * (double)j / (double)twL;
            h[(size_t)k1 * B + n2] = make_float2((float)cos(a), (float)sin(a));
        }
    HSB_CUDA_TRY(cudaMalloc((void**)out, sizeof(float2) * h.size()));
    HSB_CUDA_TRY(cudaMemcpy(*out, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice));
    return HSB_OK;
}

static const int XTHREADS = 256;
static const int SMEM_TILE_BUDGET = 72 * 1024;

// FP64 transform of the kernel and extraction (setup only).
// FP64 device scratch of one kernel-spectrum evaluation (Kernel_Arne octant, one expanded
// component, its transform, the imaginary-part maximum).
struct hsb_demag_spec_s {
    double* Kc;
    double* full;
    double2* X;
    double2* tw64;
    double* dmax;
};

static void spec_free(hsb_demag_spec_s* s) {
    if (!s) return;
    cudaFree(s->Kc);
    cudaFree(s->full);
    cudaFree(s->X);
    cudaFree(s->tw64);
    cudaFree(s->dmax);
    delete s;
}

static long spec_nfold(const hsb_demag_plan_s* P) {
    return (long)(P->L[0] / 2 + 1) * (P->L[1] / 2 + 1) * (P->L[2] / 2 + 1);
}

long hsb_demag_spectrum_scratch_bytes(hsb_demag_plan P) {
    const long vol = (long)P->L[0] * P->L[1] * P->L[2];
    return (long)sizeof(double) * 6 * spec_nfold(P) + (long)sizeof(double) * vol +
           (long)sizeof(double2) * (long)P->L[0] * P->C2 * P->L[1] + (long)sizeof(double2) * P->twL + 256;
}

int hsb_demag_spectrum_scratch_create(hsb_demag_plan P, hsb_demag_spec_s** out) {
    hsb_demag_spec_s* s = new hsb_demag_spec_s();
    const long vol = (long)P->L[0] * P->L[1] * P->L[2];
#define STRY2(x)                                                                        \
    do {                                                                                \
        cudaError_t e_ = (x);                                                           \
        if (e_ != cudaSuccess) {                                                        \
            hsb_set_error("demag spectrum scratch: %s: %s", #x, cudaGetErrorString(e_)); \
            spec_free(s);                                                               \
            return e_ == cudaErrorMemoryAllocation ? HSB_ERR_NOMEM : HSB_ERR_CUDA;      \
        }                                                                               \
    } while (0)
    STRY2(cudaMalloc(&s->Kc, sizeof(double) * 6 * spec_nfold(P)));
    STRY2(cudaMalloc(&s->full, sizeof(double) * vol));
    STRY2(cudaMalloc(&s->X, sizeof(double2) * (long)P->L[0] * P->C2 * P->L[1]));
    STRY2(cudaMalloc(&s->dmax, sizeof(double)));
#undef STRY2
    if (make_twiddles<double2>(P->twL, &s->tw64) != HSB_OK) {
        spec_free(s);
        return HSB_ERR_CUDA;
    }
    *out = s;
    return HSB_OK;
}

void hsb_demag_spectrum_scratch_destroy(hsb_demag_spec_s* s) { spec_free(s); }

long hsb_demag_kern_floats(hsb_demag_plan P) {
    return (long)P->C2 * (P->L[1] / 2 + 1) * (P->L[0] / 2 + 1) * 6;
}

// Enqueue the FP64 Kernel_Arne tensor of the plan's grid for cells of size `cs` and the
// extraction of its FP32 folded spectrum into `kern` and / or `kern4` (the fast y/z kernel's
// layout; either may be null; hsb_demag_kern_floats floats each).  The
// scratch's imaginary-part maximum is reset first and holds this evaluation's afterwards.
int hsb_demag_spectrum_enqueue(hsb_demag_plan P, const double* cs, int accuracy, hsb_demag_spec_s* s, float* kern,
                               float* kern4, cudaStream_t st) {
    const int L0 = P->L[0], L1 = P->L[1], L2 = P->L[2];
    const int h0 = L0 / 2, h1 = L1 / 2;
    const int C2 = P->C2;
    ArneGeom g;
    for (int a = 0; a < 3; a++) {
        g.size[a] = P->L[a];
        g.cs[a] = cs[a];
        g.h[a] = P->L[a] / 2;
        if (P->pbc[a] == 0) {
            g.r1[a] = -(long)((P->L[a] - 1) / 2);
            g.r2[a] = (long)((P->L[a] - 1) / 2);
        } else {
            g.r1[a] = -((long)P->L[a] * P->pbc[a] - 1);
            g.r2[a] = (long)P->L[a] * P->pbc[a] - 1;
        }
    }
    if (P->L[2] == 1 && P->pbc[2] == 0) g.r2[2] = 0;
    g.Lmin = fmin(cs[0], fmin(cs[1], cs[2]));
    g.accuracy = (double)accuracy;
    HSB_CUDA_TRY(cudaMemsetAsync(s->dmax, 0, sizeof(double), st));
    HSB_CUDA_TRY(P->tensor == 1 ? hsb_newell_launch(&g, s->Kc, st) : hsb_arne_launch(&g, s->Kc, st));
    const int M = L2 / 2;
    const int TY = pick_tile(M, sizeof(double2), SMEM_TILE_BUDGET, 16);
    const int smx = 2 * TY * fpad_len(M) * (int)sizeof(double2);
    HSB_CUDA_TRY(cudaFuncSetAttribute(k_fft_x_fwd<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smx));
    const int TB = pick_tile(L1, sizeof(double2), SMEM_TILE_BUDGET, 16);
    const int smy = 2 * TB * fpad_len(L1) * (int)sizeof(double2);
    HSB_CUDA_TRY(cudaFuncSetAttribute(k_fft_cols<double, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smy));
    const int TK = pick_tile(L0, sizeof(double2), SMEM_TILE_BUDGET, 16);
    const int smz = 2 * TK * fpad_len(L0) * (int)sizeof(double2);
    HSB_CUDA_TRY(cudaFuncSetAttribute(k_fft_z<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, smz));
    const double scale = 1.0 / ((double)L0 * L1 * L2);
    for (int comp = 0; comp < 6; comp++) {
        HSB_CUDA_TRY(hsb_arne_expand_launch(s->Kc, comp, L0, L1, L2, s->full, st));
        dim3 gx(hsb_div_up(L1, TY), L0);
        k_fft_x_fwd<double><<<gx, XTHREADS, smx, st>>>(s->full, s->full, nullptr, 0, nullptr, 0, L0, L1, L2, L2, L1,
                                                          s->X, s->tw64, P->twL, TY, nullptr);
        const long ncol = (long)L0 * C2;
        k_fft_cols<double, -1><<<hsb_div_up(ncol, TB), XTHREADS, smy, st>>>(s->X, L1, L1, s->X, L1, L1, L1, ncol,
                                                                              s->tw64, P->twL, TB, nullptr);
        dim3 gz(hsb_div_up(L1, TK), C2);
        k_fft_z<double><<<gz, XTHREADS, smz, st>>>(s->X, 1, L0, L0, C2, L1, nullptr, 0, s->tw64, P->twL, TK, nullptr);
        k_extract<<<hsb_grid_1d((long)C2 * (h1 + 1) * (h0 + 1), 256), 256, 0, st>>>(s->X, L0, C2, L1, comp, scale,
                                                                                     kern, kern4, s->dmax);
        if (kern4 && P->zdirect)
            k_zdirect<<<hsb_grid_1d((long)C2 * (h1 + 1), 256), 256, 0, st>>>(s->X, L0, C2, L1, comp, scale, kern4);
        HSB_CUDA_TRY(cudaGetLastError());
    }
    return HSB_OK;
}

// FP64 transform of the kernel and extraction (plan setup).
static int build_kernel_spectrum(hsb_demag_plan_s* P, int accuracy, cudaStream_t st) {
    hsb_demag_spec_s* s = nullptr;
    int rc = hsb_demag_spectrum_scratch_create(P, &s);
    if (rc != HSB_OK) return rc;
    rc = hsb_demag_spectrum_enqueue(P, P->cs, accuracy, s, P->kern, P->kern4, st);
    if (rc == HSB_OK) {
        cudaError_t e = cudaMemcpyAsync(&P->kern_max_imag, s->dmax, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) {
            hsb_set_error("demag setup: %s", cudaGetErrorString(e));
            rc = HSB_ERR_CUDA;
        }
    }
    spec_free(s);
    return rc;
}

// Launch-shape tuning of the fast x kernels: block sizes of 64, 128 and 256 threads (rows of
// the transform per block = threads / lanes per row) are timed on the plan's own buffers
// and the fastest kept, per kernel.  Every shape computes each row identically, so the
// choice changes timing only.  Results are cached per grid size for the process.
struct XTune {
    int f, i;
};
static std::mutex g_xtune_mu;
static std::map<std::tuple<int, int, int>, XTune> g_xtune;

static int tune_x(hsb_demag_plan_s* P, cudaStream_t st) {
    if (!P->xfwd4) return HSB_OK;
    const int N0 = P->N[0], N1 = P->N[1], N2 = P->N[2];
    const auto key = std::make_tuple(N0, N1, N2);
    const int B = 256 / P->x4_rows;
    XTune best = {256, 256};
    bool found = false;
    {
        std::lock_guard<std::mutex> lk(g_xtune_mu);
        auto it = g_xtune.find(key);
        if (it != g_xtune.end()) {
            best = it->second;
            found = true;
        }
    }
    if (!found) {
        const long ncell = (long)N0 * N1 * N2;
        float* m = nullptr;
        float* H = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        int rc = HSB_OK;
        SlotStrides ss = {0, 0, 0, 0, nullptr, 0, 0};
        float bf = 1e30f, bi = 1e30f;
        if (cudaMalloc(&m, sizeof(float) * 3 * ncell) != cudaSuccess ||
            cudaMalloc(&H, sizeof(float) * 3 * ncell) != cudaSuccess ||
            cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
            cudaMemsetAsync(m, 0, sizeof(float) * 3 * ncell, st) != cudaSuccess) {
            rc = HSB_ERR_CUDA;
        }
        for (int th = 64; th <= 256 && rc == HSB_OK; th *= 2) {
            const int rows = th / B;
            if (rows < 1) continue;
            const int smem = rows * P->x4_S * (int)sizeof(float2);
            dim3 g(hsb_div_up(N1, rows), 3 * N0);
            for (int which = 0; which < 2; which++) {
                float best_ms = 1e30f;
                // each timing covers 8 back-to-back launches: single ~20 us launches between
                // events were noisy enough to pick a slower shape on some runs
                for (int rep = 0; rep < 4; rep++) {
                    cudaEventRecord(e0, st);
                    for (int k = 0; k < 8; k++) {
                        if (which == 0)
                            P->xfwd4<<<g, th, smem, st>>>(m, m, nullptr, 0, nullptr, ncell, N0, N1, N2, N1, P->X1,
                                                          P->tw, P->twL, P->tw4x, rows, nullptr, ss);
                        else
                            P->xinv4<<<g, th, smem, st>>>(P->X1, N1, N0, N1, N2, H, H, nullptr, 0, ncell, 1.0f,
                                                          P->tw, P->twL, P->tw4x, rows, nullptr, ss);
                    }
                    cudaEventRecord(e1, st);
                    if (cudaEventSynchronize(e1) != cudaSuccess) {
                        rc = HSB_ERR_CUDA;
                        break;
                    }
                    float ms = 0;
                    cudaEventElapsedTime(&ms, e0, e1);
                    if (rep > 0 && ms < best_ms) best_ms = ms;   // the first rep is a warm-up
                }
                if (which == 0 && best_ms < bf) {
                    bf = best_ms;
                    best.f = th;
                }
                if (which == 1 && best_ms < bi) {
                    bi = best_ms;
                    best.i = th;
                }
            }
        }
        if (cudaGetLastError() != cudaSuccess) rc = HSB_ERR_CUDA;
        cudaFree(m);
        cudaFree(H);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (rc != HSB_OK) {
            hsb_set_error("hsb_demag_plan_create: x-kernel tuning failed");
            return rc;
        }
        std::lock_guard<std::mutex> lk(g_xtune_mu);
        g_xtune[key] = best;
    }
    P->x4_threads = best.f;
    P->x4_rows = best.f / B;
    P->x4_smem = P->x4_rows * P->x4_S * (int)sizeof(float2);
    P->x4i_threads = best.i;
    P->x4i_rows = best.i / B;
    P->x4i_smem = P->x4i_rows * P->x4_S * (int)sizeof(float2);
    return HSB_OK;
}

HSB_EXPORT int hsb_demag_plan_create(const int* size, const double* cellsize, const int* pbc,
                                     int accuracy, void* stream, hsb_demag_plan* out) {
    return hsb_demag_plan_create_tensor(size, cellsize, pbc, accuracy, 0, stream, out);
}

HSB_EXPORT int hsb_demag_plan_create_tensor(const int* size, const double* cellsize, const int* pbc, int accuracy,
                                            int tensor, void* stream, hsb_demag_plan* out) {
    if (!size || !cellsize || !pbc || !out) {
        hsb_set_error("hsb_demag_plan_create: null argument");
        return HSB_ERR_INVALID;
    }
    *out = nullptr;
    if (tensor != 0 && tensor != 1) {
        hsb_set_error("hsb_demag_plan_create: tensor %d is neither Kernel_Arne (0) nor Newell (1)", tensor);
        return HSB_ERR_INVALID;
    }
    hsb_demag_plan_s* P = (hsb_demag_plan_s*)calloc(1, sizeof(hsb_demag_plan_s));
    if (!P) return HSB_ERR_NOMEM;
    P->tensor = tensor;
    for (int a = 0; a < 3; a++) {
        P->N[a] = size[a];
        P->pbc[a] = pbc[a];
        P->cs[a] = cellsize[a];
        if (size[a] < 1 || cellsize[a] <= 0 || pbc[a] < 0) {
            hsb_set_error("hsb_demag_plan_create: bad size/cellsize/pbc on axis %d", a);
            free(P);
            return HSB_ERR_INVALID;
        }
        P->L[a] = (size[a] > 1 && pbc[a] == 0) ? 2 * size[a] : size[a];
        if (!is_pow2(P->L[a]) && pbc[a] != 0) {
            hsb_set_error("hsb_demag_plan_create: periodic axis %d of %d cells is not a power of two", a, size[a]);
            free(P);
            return HSB_ERR_UNSUPPORTED;
        }
    }
    if (!is_pow2(P->L[0]) || !is_pow2(P->L[1]) || !is_pow2(P->L[2])) {
        // Open axes whose padded size 2N is not a power of two: the convolution runs on the grid
        // of next_pow2(N) cells along them, the N cells at its origin and vacuum (m = 0)
        // beyond.  The reference pads to 2N (engine/zeropad.go:12-22); any padding of at
        // least 2N - 1 gives the same linear convolution, and Kernel_Arne's entries for the
        // offsets |d| <= N - 1 that reach the N cells do not depend on the padded size.
        int in[3];
        for (int a = 0; a < 3; a++) {
            in[a] = size[a];
            if (pbc[a] == 0 && size[a] > 1)
                while (!is_pow2(in[a])) in[a]++;
        }
        int rc = hsb_demag_plan_create_tensor(in, cellsize, pbc, accuracy, tensor, stream, &P->inner);
        if (rc != HSB_OK) {
            free(P);
            return rc;
        }
        const long ninner = 3L * in[0] * in[1] * in[2];
        if (cudaMalloc(&P->mpad, sizeof(float) * ninner) != cudaSuccess ||
            cudaMalloc(&P->hpad, sizeof(float) * ninner) != cudaSuccess) {
            hsb_set_error("hsb_demag_plan_create: cudaMalloc of the embedding buffers failed");
            hsb_demag_plan_destroy(P);
            return HSB_ERR_NOMEM;
        }
        // zero once: the vacuum cells of mpad are never written
        if (cudaMemset(P->mpad, 0, sizeof(float) * ninner) != cudaSuccess) {
            hsb_set_error("hsb_demag_plan_create: cudaMemset failed");
            hsb_demag_plan_destroy(P);
            return HSB_ERR_CUDA;
        }
        for (int a = 0; a < 3; a++) P->L[a] = P->inner->L[a];
        P->C2 = P->inner->C2;
        *out = P;
        return HSB_OK;
    }
    if (P->L[2] < 2 || P->L[0] > 4096 || P->L[1] > 4096 || P->L[2] > 8192) {
        hsb_set_error("hsb_demag_plan_create: padded size (%d,%d,%d) outside 2..4096 (a2 >= 2)", P->L[0], P->L[1], P->L[2]);
        free(P);
        return HSB_ERR_UNSUPPORTED;
    }
    const int N0 = P->N[0], N1 = P->N[1], L0 = P->L[0], L1 = P->L[1], L2 = P->L[2];
    P->C2 = L2 / 2 + 1;
    P->twL = L0 > L1 ? L0 : L1;
    if (L2 > P->twL) P->twL = L2;
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
#define PTRY(x)                                                                   \
    do {                                                                          \
        cudaError_t e_ = (x);                                                     \
        if (e_ != cudaSuccess) {                                                  \
            hsb_set_error("hsb_demag_plan_create: %s: %s", #x, cudaGetErrorString(e_)); \
            hsb_demag_plan_destroy(P);                                            \
            return HSB_ERR_CUDA;                                                  \
        }                                                                         \
    } while (0)
    const long kcount = (long)P->C2 * (L1 / 2 + 1) * (L0 / 2 + 1) * 6;
    PTRY(cudaMalloc(&P->kern, sizeof(float) * kcount));
    PTRY(cudaMalloc(&P->X1, sizeof(float2) * 3L * N0 * P->C2 * N1));
    rc = make_twiddles<float2>(P->twL, &P->tw);
    if (rc != HSB_OK) { hsb_demag_plan_destroy(P); return rc; }
    // launch geometry
    const int M = L2 / 2;
    P->TYx = pick_tile(M, sizeof(float2), SMEM_TILE_BUDGET, 16);
    P->smem_x = 2 * P->TYx * fpad_len(M) * (int)sizeof(float2);
    P->TYxi = P->TYx;
    P->smem_xi = P->smem_x;
    PTRY(cudaFuncSetAttribute(k_fft_x_fwd<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, P->smem_x));
    PTRY(cudaFuncSetAttribute(k_fft_x_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, P->smem_xi));
    const int yz_smem = 2 * 3 * N0 * fpad_len(L1) * (int)sizeof(float2);
    P->fused = (L0 <= 16 && yz_smem <= 220 * 1024);
    if (P->fused) {
        P->lz = L0;
        P->smem_yz = yz_smem;
        switch (L0) {
#define SETYZ(LZ) case LZ: PTRY(cudaFuncSetAttribute(k_fft_yz_conv<LZ>, cudaFuncAttributeMaxDynamicSharedMemorySize, yz_smem)); break;
            SETYZ(1) SETYZ(2) SETYZ(4) SETYZ(8) SETYZ(16)
#undef SETYZ
        }
    } else {
        PTRY(cudaMalloc(&P->X2, sizeof(float2) * 3L * N0 * P->C2 * L1));
        P->TBy = pick_tile(L1, sizeof(float2), SMEM_TILE_BUDGET, 16);
        P->smem_y = 2 * P->TBy * fpad_len(L1) * (int)sizeof(float2);
        PTRY(cudaFuncSetAttribute(k_fft_cols<float, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, P->smem_y));
        PTRY(cudaFuncSetAttribute(k_fft_cols<float, +1>, cudaFuncAttributeMaxDynamicSharedMemorySize, P->smem_y));
        P->TKz = pick_tile(L0, 3 * sizeof(float2), SMEM_TILE_BUDGET, 32);
        P->smem_z = 2 * 3 * P->TKz * fpad_len(L0) * (int)sizeof(float2);
        PTRY(cudaFuncSetAttribute(k_fft_z<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, P->smem_z));
        // four-step register kernels where the lengths fit; an axis is zero-padded exactly
        // when its logic size is twice the grid's
        const bool pry = L1 == 2 * N1, prz = L0 == 2 * N0;
        int Bc = 0, Sc = 0;
        P->ycf4 = ycf4_for(L1, pry, &Bc, &Sc);
        if (P->ycf4) {
            P->yci4 = yci4_for(L1, pry);
            P->yc_threads = 256;
            P->yc_cols = 256 / Bc;
            P->yc_smem = P->yc_cols * Sc * (int)sizeof(float2);
            rc = make_tw4(L1, Bc, P->twL, &P->tw4c);
            if (rc != HSB_OK) { hsb_demag_plan_destroy(P); return rc; }
            PTRY(cudaFuncSetAttribute(P->ycf4, cudaFuncAttributeMaxDynamicSharedMemorySize, P->yc_smem));
            PTRY(cudaFuncSetAttribute(P->yci4, cudaFuncAttributeMaxDynamicSharedMemorySize, P->yc_smem));
        } else if (L1 == 2048 && pry) {
            P->yc2k = 1;
            P->yc_threads = 128;
            P->yc_cols = 4;
            // fft4 slots, then the per-warp stash of 1024 complex
            P->yc_smem = P->yc_cols * (Slot<1024>::S + 1024) * (int)sizeof(float2);
            rc = make_tw4(1024, Split<1024>::B, P->twL, &P->tw4c);
            if (rc != HSB_OK) { hsb_demag_plan_destroy(P); return rc; }
            PTRY(cudaFuncSetAttribute(k_ycolf4_2k, cudaFuncAttributeMaxDynamicSharedMemorySize, P->yc_smem));
            PTRY(cudaFuncSetAttribute(k_ycoli4_2k, cudaFuncAttributeMaxDynamicSharedMemorySize, P->yc_smem));
        }
        P->zc4 = zc4_for(L0, prz, &P->zc_k1, &P->zc_smem);
        if (P->zc4) {
            rc = make_tw4(L0, 256 / P->zc_k1, P->twL, &P->tw4z);
            if (rc != HSB_OK) { hsb_demag_plan_destroy(P); return rc; }
            if (!P->kern4) PTRY(cudaMalloc(&P->kern4, sizeof(float) * kcount));
            PTRY(cudaFuncSetAttribute(P->zc4, cudaFuncAttributeMaxDynamicSharedMemorySize, P->zc_smem));
        }
    }
    {
        // four-step kernels for the FP32 convolution when the lengths fit
        int B = 0, S = 0;
        // zero-padding pruning where the padded length is twice the grid's
        const bool prx = P->pbc[2] == 0 && P->N[2] > 1;
        const bool pryz = P->pbc[1] == 0 && P->N[1] > 1 && (P->N[0] == 1 || P->pbc[0] == 0);
        xfwd4_fn xf = xfwd4_for(M, prx, &B, &S);
        if (xf && B > 0) {
            P->xfwd4 = xf;
            P->xinv4 = xinv4_for(M, prx);
            rc = make_tw4(M, B, P->twL, &P->tw4x);
            if (rc != HSB_OK) { hsb_demag_plan_destroy(P); return rc; }
            P->x4_rows = 256 / B;
            P->x4_threads = 256;
            P->x4_smem = P->x4_rows * S * (int)sizeof(float2);
            P->x4_S = S;
            P->x4i_rows = P->x4_rows;
            P->x4i_threads = P->x4_threads;
            P->x4i_smem = P->x4_smem;
            PTRY(cudaFuncSetAttribute(P->xfwd4, cudaFuncAttributeMaxDynamicSharedMemorySize, P->x4_smem));
            PTRY(cudaFuncSetAttribute(P->xinv4, cudaFuncAttributeMaxDynamicSharedMemorySize, P->x4_smem));
            // prefer shared memory over L1 so that several blocks fit per SM
            PTRY(cudaFuncSetAttribute(P->xfwd4, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
            PTRY(cudaFuncSetAttribute(P->xinv4, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        }
        int By = 0, Sy = 0;
        yz4_fn yf = (L0 <= 16) ? yz4_for(L1, L0, pryz, &By, &Sy) : nullptr;
        if (yf && 3 * N0 * By <= 384 && (3 * N0 * Sy + L1) * (int)sizeof(float2) <= 110 * 1024) {
            P->yz4 = yf;
            P->zdirect = pryz && (L0 == 4 || L0 == 8);   // the DZ instantiations of k_yz4
            if (!P->kern4) PTRY(cudaMalloc(&P->kern4, sizeof(float) * kcount));
            rc = make_tw4(L1, By, P->twL, &P->tw4y);
            if (rc != HSB_OK) { hsb_demag_plan_destroy(P); return rc; }
            P->yz4_threads = 3 * N0 * By;
            P->yz4_smem = (3 * N0 * Sy + L1) * (int)sizeof(float2);   // column slots + twiddle matrix
            PTRY(cudaFuncSetAttribute(P->yz4, cudaFuncAttributeMaxDynamicSharedMemorySize, P->yz4_smem));
            PTRY(cudaFuncSetAttribute(P->yz4, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        }
    }
#undef PTRY
    rc = build_kernel_spectrum(P, accuracy, st);
    if (rc == HSB_OK) rc = tune_x(P, st);
    if (rc != HSB_OK) {
        hsb_demag_plan_destroy(P);
        return rc;
    }
    *out = P;
    return HSB_OK;
}

HSB_EXPORT int hsb_demag_plan_destroy(hsb_demag_plan P) {
    if (!P) return HSB_OK;
    if (P->inner) hsb_demag_plan_destroy(P->inner);
    cudaFree(P->mpad);
    cudaFree(P->hpad);
    cudaFree(P->kern);
    cudaFree(P->kern4);
    cudaFree(P->tw4x);
    cudaFree(P->tw4y);
    cudaFree(P->tw4c);
    cudaFree(P->tw4z);
    cudaFree(P->X1);
    cudaFree(P->X2);
    cudaFree(P->tw);
    free(P);
    return HSB_OK;
}

int hsb_demag_nlaunch(hsb_demag_plan P) {
    if (P && P->inner) return hsb_demag_nlaunch(P->inner) + 2;
    return P ? ((P->yz4 || P->fused) ? 3 : 5) : 0;
}

HSB_EXPORT int hsb_demag_plan_info(hsb_demag_plan P, int* logic, int* fused, double* max_imag) {
    if (!P) return HSB_ERR_INVALID;
    if (logic) for (int a = 0; a < 3; a++) logic[a] = P->L[a];
    if (P->inner) P = P->inner;
    if (fused) *fused = P->fused;
    if (max_imag) *max_imag = P->kern_max_imag;
    return HSB_OK;
}

// Launch the convolution: H (A/m, FP32 SoA [3][N0][N1][N2]) = Ms0 * K (*) (m * mask).
long hsb_demag_x1_bytes(hsb_demag_plan P) {
    if (!P || P->inner || !P->xfwd4 || !P->yz4 || !P->xinv4) return 0;
    return 3L * P->N[0] * P->C2 * P->N[1] * (long)sizeof(float2);
}

// Embedding of an N-cell grid in the plan's power-of-two grid of M cells (M >= N per axis): m
// (times the optional Ms mask) into the first N cells of each axis; the other cells were zeroed
// at plan creation and stay zero.  Reads m[(*msel) ^ minv] as the x kernels do.
__global__ void k_demag_embed(const float* __restrict__ m0, const float* __restrict__ m1, const int* msel, int minv,
                              const float* __restrict__ mask, int N0, int N1, int N2, int M0, int M1, int M2,
                              float* __restrict__ mpad, const int* active) {
    if (active && !*active) return;
    const float* m = (msel && ((*msel) ^ minv)) ? m1 : m0;
    const long n = (long)N0 * N1 * N2, npad = (long)M0 * M1 * M2;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < 3 * n; q += (long)gridDim.x * blockDim.x) {
        const int c = (int)(q / n);
        const long i = q - c * n;
        const int i2 = (int)(i % N2);
        const long r = i / N2;
        const int i1 = (int)(r % N1);
        const int i0 = (int)(r / N1);
        const float v = m[q];
        mpad[c * npad + ((long)i0 * M1 + i1) * M2 + i2] = mask ? v * mask[i] : v;
    }
}

// The field of the N cells back out of the embedding grid, into h[(*hsel) ^ hinv].
__global__ void k_demag_extract(const float* __restrict__ hpad, float* h0, float* h1, const int* hsel, int hinv,
                                int N0, int N1, int N2, int M0, int M1, int M2, const int* active) {
    if (active && !*active) return;
    float* h = (hsel && ((*hsel) ^ hinv)) ? h1 : h0;
    const long n = (long)N0 * N1 * N2, npad = (long)M0 * M1 * M2;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < 3 * n; q += (long)gridDim.x * blockDim.x) {
        const int c = (int)(q / n);
        const long i = q - c * n;
        const int i2 = (int)(i % N2);
        const long r = i / N2;
        const int i1 = (int)(r % N1);
        const int i0 = (int)(r / N1);
        h[q] = hpad[c * npad + ((long)i0 * M1 + i1) * M2 + i2];
    }
}

int hsb_demag_launch(hsb_demag_plan P, const HsbDemagIO& io, const float* mask, float ms0,
                     cudaStream_t st, const int* active, const HsbDemagBatch* batch) {
    if (P->inner) {
        if (batch) {
            hsb_set_error("hsb_demag_launch: batches need padded sizes that are powers of two");
            return HSB_ERR_UNSUPPORTED;
        }
        const hsb_demag_plan_s* Q = P->inner;
        const long n3 = 3L * P->N[0] * P->N[1] * P->N[2];
        const int grid = hsb_grid_1d(n3, 256);
        k_demag_embed<<<grid, 256, 0, st>>>(io.m[0], io.m[1], io.msel, io.minv, mask, P->N[0], P->N[1], P->N[2],
                                            Q->N[0], Q->N[1], Q->N[2], P->mpad, active);
        HsbDemagIO inner = {};
        inner.m[0] = inner.m[1] = P->mpad;
        inner.h[0] = inner.h[1] = P->hpad;
        inner.ev = io.ev;
        int rc = hsb_demag_launch(P->inner, inner, nullptr, ms0, st, active, nullptr);
        if (rc != HSB_OK) return rc;
        k_demag_extract<<<grid, 256, 0, st>>>(P->hpad, io.h[0], io.h[1], io.hsel, io.hinv, P->N[0], P->N[1],
                                              P->N[2], Q->N[0], Q->N[1], Q->N[2], active);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            hsb_set_error("hsb_demag_launch: %s", cudaGetErrorString(e));
            return HSB_ERR_CUDA;
        }
        return HSB_OK;
    }
    const int N0 = P->N[0], N1 = P->N[1], N2 = P->N[2];
    const int L0 = P->L[0], L1 = P->L[1], L2 = P->L[2];
    const int C2 = P->C2;
    const long ncell = (long)N0 * N1 * N2;
    SlotStrides ss = {0, 0, 0, 0, nullptr, 0, 0};
    float2* X1 = P->X1;
    const float* kern = P->kern4;
    int nz = 1;
    if (batch) {
        if (!hsb_demag_x1_bytes(P) || mask || !batch->X1 || batch->nslot < 1) {
            hsb_set_error("hsb_demag_launch: batched convolutions need the fast kernels, no mask and a spectrum "
                          "arena");
            return HSB_ERR_UNSUPPORTED;
        }
        ss.in = batch->m_stride;
        ss.x1 = batch->x1_stride;
        ss.out = batch->h_stride;
        ss.sel = batch->sel_stride;
        ss.scale = batch->scale;
        ss.scale_stride = batch->scale_stride;
        X1 = (float2*)batch->X1;
        nz = batch->nslot;
        if (batch->kern) {
            kern = batch->kern;
            ss.kern = batch->kern_stride;
        }
    }
    if (io.ev) cudaEventRecord(io.ev[0], st);
    if (P->xfwd4) {
        dim3 gx(hsb_div_up(N1, P->x4_rows), 3 * N0, nz);
        P->xfwd4<<<gx, P->x4_threads, P->x4_smem, st>>>(io.m[0], io.m[1], io.msel, io.minv, mask, ncell, N0, N1, N2,
                                                        N1, X1, P->tw, P->twL, P->tw4x, P->x4_rows, active, ss);
    } else {
        dim3 gx(hsb_div_up(N1, P->TYx), 3 * N0);
        k_fft_x_fwd<float><<<gx, XTHREADS, P->smem_x, st>>>(io.m[0], io.m[1], io.msel, io.minv, mask, ncell, N0, N1,
                                                            N2, L2, N1, P->X1, P->tw, P->twL, P->TYx, active);
    }
    if (io.ev) cudaEventRecord(io.ev[1], st);
    if (P->yz4) {
        dim3 gyz(C2, 1, nz);
        P->yz4<<<gyz, P->yz4_threads, P->yz4_smem, st>>>(X1, N0, N1, C2, kern, P->tw4y, active, ss);
    } else if (P->fused) {
        switch (P->lz) {
#define RUNYZ(LZ) case LZ: k_fft_yz_conv<LZ><<<C2, yz_threads<LZ>::value, P->smem_yz, st>>>(P->X1, N0, N1, L1, C2, P->kern, P->tw, P->twL, active); break;
            RUNYZ(1) RUNYZ(2) RUNYZ(4) RUNYZ(8) RUNYZ(16)
#undef RUNYZ
        }
    } else {
        const long ncol = 3L * N0 * C2;
        const long gc = P->yc_cols ? hsb_div_up(ncol, P->yc_cols) : 0;
        if (P->ycf4)
            P->ycf4<<<gc, P->yc_threads, P->yc_smem, st>>>(P->X1, N1, P->X2, ncol, P->tw4c, active);
        else if (P->yc2k)
            k_ycolf4_2k<<<gc, P->yc_threads, P->yc_smem, st>>>(P->X1, N1, P->X2, ncol, P->tw4c, P->tw, P->twL, active);
        else
            k_fft_cols<float, -1><<<hsb_div_up(ncol, P->TBy), XTHREADS, P->smem_y, st>>>(
                P->X1, N1, N1, P->X2, L1, L1, L1, ncol, P->tw, P->twL, P->TBy, active);
        if (P->zc4) {
            dim3 gz(hsb_div_up(L1, P->zc_k1), C2);
            P->zc4<<<gz, 256, P->zc_smem, st>>>(P->X2, N0, C2, L1, P->kern4, P->tw4z, active);
        } else {
            dim3 gz(hsb_div_up(L1, P->TKz), C2);
            k_fft_z<float><<<gz, XTHREADS, P->smem_z, st>>>(P->X2, 3, N0, L0, C2, L1, P->kern, 1, P->tw, P->twL,
                                                                   P->TKz, active);
        }
        if (P->yci4)
            P->yci4<<<gc, P->yc_threads, P->yc_smem, st>>>(P->X2, P->X1, N1, ncol, P->tw4c, active);
        else if (P->yc2k)
            k_ycoli4_2k<<<gc, P->yc_threads, P->yc_smem, st>>>(P->X2, P->X1, N1, ncol, P->tw4c, P->tw, P->twL, active);
        else
            k_fft_cols<float, +1><<<hsb_div_up(ncol, P->TBy), XTHREADS, P->smem_y, st>>>(
                P->X2, L1, L1, P->X1, N1, N1, L1, ncol, P->tw, P->twL, P->TBy, active);
    }
    if (io.ev) cudaEventRecord(io.ev[2], st);
    if (P->xinv4) {
        dim3 gi(hsb_div_up(N1, P->x4i_rows), 3 * N0, nz);
        P->xinv4<<<gi, P->x4i_threads, P->x4i_smem, st>>>(X1, N1, N0, N1, N2, io.h[0], io.h[1], io.hsel, io.hinv,
                                                          ncell, ms0, P->tw, P->twL, P->tw4x, P->x4i_rows, active, ss);
    } else {
        dim3 gi(hsb_div_up(N1, P->TYxi), 3 * N0);
        k_fft_x_inv<<<gi, XTHREADS, P->smem_xi, st>>>(P->X1, N1, N0, N1, N2, L2, io.h[0], io.h[1], io.hsel, io.hinv,
                                                      ncell, ms0, P->tw, P->twL, P->TYxi, active);
    }
    if (io.ev) cudaEventRecord(io.ev[3], st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        hsb_set_error("hsb_demag_launch: %s", cudaGetErrorString(e));
        return HSB_ERR_CUDA;
    }
    return HSB_OK;
}

HSB_EXPORT int hsb_demag_field(hsb_demag_plan P, const float* m, const float* mask, double msat0T0,
                               float* H, void* stream) {
    if (!P || !m || !H) {
        hsb_set_error("hsb_demag_field: null argument");
        return HSB_ERR_INVALID;
    }
    HsbDemagIO io = {{m, m}, nullptr, 0, {H, H}, nullptr, 0, nullptr};
    return hsb_demag_launch(P, io, mask, (float)msat0T0, (cudaStream_t)stream, nullptr);
}

// Per-kernel device time of one convolution: ms[0] x-pass, ms[1] y/z pass(es), ms[2] inverse
// x-pass (CUDA events on `stream`, averaged over `reps` launches after one warm-up).
HSB_EXPORT int hsb_demag_profile(hsb_demag_plan P, const float* m, const float* mask, double msat0T0, float* H,
                                 void* stream, int reps, double* ms) {
    if (!P || !m || !H || !ms || reps < 1) return HSB_ERR_INVALID;
    cudaStream_t st = (cudaStream_t)stream;
    cudaEvent_t ev[4];
    for (int i = 0; i < 4; i++) HSB_CUDA_TRY(cudaEventCreate(&ev[i]));
    double acc[3] = {0, 0, 0};
    int rc = HSB_OK;
    for (int r = 0; r <= reps && rc == HSB_OK; r++) {
        HsbDemagIO io = {{m, m}, nullptr, 0, {H, H}, nullptr, 0, ev};
        rc = hsb_demag_launch(P, io, mask, (float)msat0T0, st, nullptr);
        if (rc != HSB_OK) break;
        if (cudaEventSynchronize(ev[3]) != cudaSuccess) { rc = HSB_ERR_CUDA; break; }
        if (r == 0) continue;
        for (int i = 0; i < 3; i++) {
            float t = 0;
            cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
            acc[i] += t;
        }
    }
    for (int i = 0; i < 4; i++) cudaEventDestroy(ev[i]);
    for (int i = 0; i < 3; i++) ms[i] = acc[i] / reps;
    return rc;
}

HSB_EXPORT int hsb_demag_kernel_copy(hsb_demag_plan P, float* host_out, long count) {
    if (!P || !host_out) return HSB_ERR_INVALID;
    if (P->inner) P = P->inner;
    const long kcount = (long)P->C2 * (P->L[1] / 2 + 1) * (P->L[0] / 2 + 1) * 6;
    if (count < kcount) {
        hsb_set_error("hsb_demag_kernel_copy: need %ld floats", kcount);
        return HSB_ERR_INVALID;
    }
    HSB_CUDA_TRY(cudaMemcpy(host_out, P->kern, sizeof(float) * kcount, cudaMemcpyDeviceToHost));
    return HSB_OK;
}

// ==================================================================================== FFT plan
// FP64 3-D real FFT with the semantics of hotspin's FFTPlanX (gpu/fftplanX.go:76-104), the
// FFTInterface a hotspin build selects with -fft (gpu/fftinterface.go:16-42):
//   forward: the data block (N0, N1, N2) zero-padded to the logic size (L0, L1, L2), then the
//            unnormalised real-to-complex transform, output (L0, L1, L2/2 + 1) complex
//            (cuFFT's packed layout: L2 + 2 doubles per row);
//   inverse: the unnormalised complex-to-real transform of such a spectrum, cropped to the
//            data block.
// Three passes of the column transform k_fft_cols (FP64 Stockham, any power of two up to
// 4096) with a transpose between them, each axis contiguous in turn; the real axis runs as a
// complex transform of the real row (forward) or of the row's Hermitian extension (inverse).
#define RC_OK(x)                  \
    do {                          \
        const int rc_ = (x);      \
        if (rc_ != HSB_OK) return rc_; \
    } while (0)

HSB_EXPORT int hsb_fft_plan_destroy(struct hsb_fft_plan_s* P);

struct hsb_fft_plan_s {
    int N[3], L[3], C2, twL;
    double2* tw;
    double2* s0;        // scratch, max(C2 L1 L0, N0 N1 L2) complex each
    double2* s1;
    cudaStream_t st;
};

// in (N0, N1, N2) real -> s (N0 N1 N2) complex
__global__ void k_fftp_complexify(const double* __restrict__ in, double2* __restrict__ s, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        s[i] = make_double2(in[i], 0.0);
}

// out[(a * B + b) * C + c] = in[(a * C + c) * B + b]: swap the two fastest axes (B <-> C) of
// `na` blocks
__global__ void k_fftp_swap(const double2* __restrict__ in, double2* __restrict__ out, long na, int B, int C) {
    const long n = na * B * C;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long r = i / C;
        const int b = (int)(r % B);
        const long a = r / B;
        out[i] = in[(a * C + c) * B + b];
    }
}

// out[(b * C + c) * A + a] = in[(a * B + b) * C + c]: the slowest axis (A) moved to the fastest
__global__ void k_fftp_rotate(const double2* __restrict__ in, double2* __restrict__ out, int A, int B, int C) {
    const long n = (long)A * B * C;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int a = (int)(i % A);
        const long r = i / A;
        const int c = (int)(r % C);
        const int b = (int)(r / C);
        out[i] = in[((long)a * B + b) * C + c];
    }
}

// out[(a * B + b) * C + c] = in[(b * C + c) * A + a]: the fastest axis (A) moved to the slowest
__global__ void k_fftp_unrotate(const double2* __restrict__ in, double2* __restrict__ out, int A, int B, int C) {
    const long n = (long)A * B * C;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        const long r = i / C;
        const int b = (int)(r % B);
        const int a = (int)(r / B);
        out[i] = in[((long)b * C + c) * A + a];
    }
}

// rows of C2 spectrum values -> rows of L2 values, X[L2 - k] = conj(X[k]) for k >= C2
__global__ void k_fftp_hermitian(const double2* __restrict__ in, double2* __restrict__ out, long nrow, int C2,
                                 int L2) {
    const long n = nrow * L2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int k = (int)(i % L2);
        const long r = i / L2;
        double2 v;
        if (k < C2) {
            v = in[r * C2 + k];
        } else {
            const double2 w = in[r * C2 + (L2 - k)];
            v = make_double2(w.x, -w.y);
        }
        out[i] = v;
    }
}

__global__ void k_fftp_real(const double2* __restrict__ s, double* __restrict__ out, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] = s[i].x;
}

// One column pass: ncol columns of nin values (stride ldi) transformed at length L, the first
// nout kept (stride ldo).  Sets the kernel's shared-memory limit before the launch: other plans
// set the same function's limit for their own lengths.
template <int DIR>
static int fftp_cols(hsb_fft_plan_s* P, const double2* in, int ldi, int nin, double2* out, int ldo, int nout,
                     int L, long ncol) {
    const int TB = pick_tile(L, sizeof(double2), SMEM_TILE_BUDGET, 16);
    const int smem = 2 * TB * fpad_len(L) * (int)sizeof(double2);
    HSB_CUDA_TRY(cudaFuncSetAttribute(k_fft_cols<double, DIR>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_fft_cols<double, DIR><<<hsb_div_up(ncol, TB), XTHREADS, smem, P->st>>>(in, ldi, nin, out, ldo, nout, L, ncol,
                                                                            P->tw, P->twL, TB, nullptr);
    HSB_CUDA_TRY(cudaGetLastError());
    return HSB_OK;
}

HSB_EXPORT int hsb_fft_plan_create(const int* data_size, const int* logic_size, void* stream, hsb_fft_plan_s** out) {
    if (!data_size || !logic_size || !out) {
        hsb_set_error("hsb_fft_plan_create: null argument");
        return HSB_ERR_INVALID;
    }
    *out = nullptr;
    for (int a = 0; a < 3; a++) {
        const int n = data_size[a], l = logic_size[a];
        if (n < 1 || l < n || !is_pow2(l) || l > 4096) {
            hsb_set_error("hsb_fft_plan_create: axis %d: data size %d, logic size %d (the logic size must be a power "
                          "of two in [data size, 4096])", a, n, l);
            return HSB_ERR_UNSUPPORTED;
        }
    }
    if (logic_size[2] < 2) {
        hsb_set_error("hsb_fft_plan_create: the real (last) axis needs a logic size of at least 2");
        return HSB_ERR_UNSUPPORTED;
    }
    hsb_fft_plan_s* P = new hsb_fft_plan_s();
    for (int a = 0; a < 3; a++) {
        P->N[a] = data_size[a];
        P->L[a] = logic_size[a];
    }
    P->C2 = P->L[2] / 2 + 1;
    P->twL = std::max(P->L[0], std::max(P->L[1], P->L[2]));
    P->st = (cudaStream_t)stream;
    const long nscr = std::max((long)P->C2 * P->L[1] * P->L[0], (long)P->N[0] * P->N[1] * P->L[2]);
    int rc = make_twiddles<double2>(P->twL, &P->tw);
    if (rc == HSB_OK && (cudaMalloc(&P->s0, sizeof(double2) * nscr) != cudaSuccess ||
                         cudaMalloc(&P->s1, sizeof(double2) * nscr) != cudaSuccess)) {
        hsb_set_error("hsb_fft_plan_create: cudaMalloc of %ld complex scratch values failed", 2 * nscr);
        rc = HSB_ERR_NOMEM;
    }
    if (rc != HSB_OK) {
        hsb_fft_plan_destroy(P);
        return rc;
    }
    *out = P;
    return HSB_OK;
}

HSB_EXPORT int hsb_fft_plan_destroy(hsb_fft_plan_s* P) {
    if (!P) return HSB_OK;
    cudaFree(P->tw);
    cudaFree(P->s0);
    cudaFree(P->s1);
    delete P;
    return HSB_OK;
}

HSB_EXPORT int hsb_fft_forward(hsb_fft_plan_s* P, const double* in, double* out) {
    if (!P || !in || !out) {
        hsb_set_error("hsb_fft_forward: null argument");
        return HSB_ERR_INVALID;
    }
    const int N0 = P->N[0], N1 = P->N[1], N2 = P->N[2], L0 = P->L[0], L1 = P->L[1], L2 = P->L[2], C2 = P->C2;
    const long nd = (long)N0 * N1 * N2;
    k_fftp_complexify<<<hsb_grid_1d(nd, 256), 256, 0, P->st>>>(in, P->s0, nd);
    // x: rows (z, y) of N2 values, zero-padded to L2, C2 kept -> s1 (N0, N1, C2)
    RC_OK(fftp_cols<-1>(P, P->s0, N2, N2, P->s1, C2, C2, L2, (long)N0 * N1));
    // (N0, N1, C2) -> (N0, C2, N1); y: N1 values zero-padded to L1 -> s1 (N0, C2, L1)
    k_fftp_swap<<<hsb_grid_1d((long)N0 * N1 * C2, 256), 256, 0, P->st>>>(P->s1, P->s0, N0, C2, N1);
    RC_OK(fftp_cols<-1>(P, P->s0, N1, N1, P->s1, L1, L1, L1, (long)N0 * C2));
    // (N0, C2, L1) -> (N0, L1, C2) -> (L1, C2, N0); z: N0 values zero-padded to L0 -> s0 (L1, C2, L0)
    k_fftp_swap<<<hsb_grid_1d((long)N0 * C2 * L1, 256), 256, 0, P->st>>>(P->s1, P->s0, N0, L1, C2);
    k_fftp_rotate<<<hsb_grid_1d((long)N0 * L1 * C2, 256), 256, 0, P->st>>>(P->s0, P->s1, N0, L1, C2);
    RC_OK(fftp_cols<-1>(P, P->s1, N0, N0, P->s0, L0, L0, L0, (long)L1 * C2));
    // (L1, C2, L0) -> (L0, L1, C2): cuFFT's packed R2C layout
    k_fftp_unrotate<<<hsb_grid_1d((long)L0 * L1 * C2, 256), 256, 0, P->st>>>(P->s0, (double2*)out, L0, L1, C2);
    HSB_CUDA_TRY(cudaGetLastError());
    HSB_CUDA_TRY(cudaStreamSynchronize(P->st));
    return HSB_OK;
}

HSB_EXPORT int hsb_fft_inverse(hsb_fft_plan_s* P, const double* in, double* out) {
    if (!P || !in || !out) {
        hsb_set_error("hsb_fft_inverse: null argument");
        return HSB_ERR_INVALID;
    }
    const int N0 = P->N[0], N1 = P->N[1], N2 = P->N[2], L0 = P->L[0], L1 = P->L[1], L2 = P->L[2], C2 = P->C2;
    // (L0, L1, C2) -> (L1, C2, L0); z: all L0 values, the first N0 kept -> s1 (L1, C2, N0)
    k_fftp_rotate<<<hsb_grid_1d((long)L0 * L1 * C2, 256), 256, 0, P->st>>>((const double2*)in, P->s0, L0, L1, C2);
    RC_OK(fftp_cols<+1>(P, P->s0, L0, L0, P->s1, N0, N0, L0, (long)L1 * C2));
    // (L1, C2, N0) -> (N0, L1, C2)
    k_fftp_unrotate<<<hsb_grid_1d((long)N0 * L1 * C2, 256), 256, 0, P->st>>>(P->s1, P->s0, N0, L1, C2);
    // s0 (N0, L1, C2) -> (N0, C2, L1); y: all L1 values, the first N1 kept -> s1 (N0, C2, N1)
    k_fftp_swap<<<hsb_grid_1d((long)N0 * L1 * C2, 256), 256, 0, P->st>>>(P->s0, P->s1, N0, C2, L1);
    RC_OK(fftp_cols<+1>(P, P->s1, L1, L1, P->s0, N1, N1, L1, (long)N0 * C2));
    // (N0, C2, N1) -> (N0, N1, C2); Hermitian rows of L2; x: complex inverse, N2 kept, real part
    k_fftp_swap<<<hsb_grid_1d((long)N0 * N1 * C2, 256), 256, 0, P->st>>>(P->s0, P->s1, N0, N1, C2);
    k_fftp_hermitian<<<hsb_grid_1d((long)N0 * N1 * L2, 256), 256, 0, P->st>>>(P->s1, P->s0, (long)N0 * N1, C2, L2);
    RC_OK(fftp_cols<+1>(P, P->s0, L2, L2, P->s1, N2, N2, L2, (long)N0 * N1));
    const long nd = (long)N0 * N1 * N2;
    k_fftp_real<<<hsb_grid_1d(nd, 256), 256, 0, P->st>>>(P->s1, out, nd);
    HSB_CUDA_TRY(cudaGetLastError());
    HSB_CUDA_TRY(cudaStreamSynchronize(P->st));
    return HSB_OK;
}
