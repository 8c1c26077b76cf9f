// Register-resident four-step FFT for power-of-two lengths L = A * B (A >= B, B <= 32).
//
// One sequence is handled by B consecutive lanes of a warp.  With x[n], n = B n1 + n2:
//   1. lane n2 holds x[B n1 + n2] for n1 < A and runs an A-point FFT in registers
//   2. multiplies by the twiddles W_L^(n2 k1)
//   3. writes the A x B intermediate to a padded shared slot, __syncwarp
//   4. lane t runs the B-point FFTs of the A/B columns k1 = t + B i  (in registers)
// giving X[k1 + A k2]; lane t ends with v[i B + k2] = X[(t + B i) + A k2].
// One shared-memory round trip per transform instead of log_R(L) Stockham passes, all
// indices compile-time.  The step-2 twiddles come from a per-plan matrix
// tw4[k1 B + n2] = exp(-2 pi i n2 k1 / L), so the B lanes of a sequence read B consecutive
// entries per k1 (one coalesced load instead of B scattered ones).
#pragma once
#include <cuda_runtime.h>

#include "hsb_fft.cuh"

// cos(2 pi k / 64) through quarter-wave symmetry of cos(2 pi k / 64), k = 0..16
// (mathematical constants).
__host__ __device__ __forceinline__ constexpr double c64q(int k) {
    return k == 0 ? 1.0
         : k == 1 ? 0.9951847266721969
         : k == 2 ? 0.9807852804032304
         : k == 3 ? 0.9569403357322088
         : k == 4 ? 0.9238795325112867
         : k == 5 ? 0.881921264348355
         : k == 6 ? 0.8314696123025452
         : k == 7 ? 0.773010453362737
         : k == 8 ? 0.7071067811865476
         : k == 9 ? 0.6343932841636455
         : k == 10 ? 0.5555702330196023
         : k == 11 ? 0.4713967368259978
         : k == 12 ? 0.38268343236508984
         : k == 13 ? 0.29028467725446233
         : k == 14 ? 0.19509032201612833
         : k == 15 ? 0.09801714032956077
         : 0.0;
}
__host__ __device__ __forceinline__ constexpr double c64cos(int k) {
    return (k & 63) <= 16 ? c64q(k & 63)
         : (k & 63) <= 32 ? -c64q(32 - (k & 63))
         : (k & 63) <= 48 ? -c64q((k & 63) - 32)
         : c64q(64 - (k & 63));
}
__host__ __device__ __forceinline__ constexpr double c64sin(int k) { return c64cos(k - 16); }

// In-register radix-2 DIT FFT of R = 1..64 points on v[0..R), bit-reversed input order
// handled by the unrolled permutation; every twiddle is a compile-time constant.
// ZIN: the upper half of the input is zero (zero padding) — the first stage reduces to
// copies.  HOUT: only the lower half of the output is wanted — the last stage skips the
// upper outputs (left unspecified).
template <int R, int DIR, bool ZIN = false, bool HOUT = false>
__host__ __device__ __forceinline__ void fft_reg64(float2* v) {
    constexpr int B = ilog2c(R);
#pragma unroll
    for (int i = 0; i < R; i++) {
        const int j = brevc(i, B);
        if (j > i) {
            float2 t = v[i];
            v[i] = v[j];
            v[j] = t;
        }
    }
#pragma unroll
    for (int st = 1; st <= B; st++) {
        const int len = 1 << st;
        if (ZIN && R > 1 && st == 1) {
            // after the bit reversal, v[i + 1] holds input brev(i) + R/2, which is zero
#pragma unroll
            for (int i = 0; i < R; i += 2) v[i + 1] = v[i];
            continue;
        }
#pragma unroll
        for (int i = 0; i < R; i += len) {
#pragma unroll
            for (int k = 0; k < len / 2; k++) {
                const float2 a = v[i + k];
                const float2 b = v[i + k + len / 2];
                const int e = k * (64 / len);  // angle 2 pi e / 64
                float2 bw;
                if (e == 0) {
                    bw = b;
                } else if (e == 16) {
                    bw = (DIR < 0) ? make_float2(b.y, -b.x) : make_float2(-b.y, b.x);
                } else {
                    const float wr = (float)c64cos(e);
                    const float wi = (float)(DIR * c64sin(e));
                    bw = make_float2(b.x * wr - b.y * wi, b.x * wi + b.y * wr);
                }
                v[i + k] = make_float2(a.x + bw.x, a.y + bw.y);
                if (!(HOUT && st == B)) v[i + k + len / 2] = make_float2(a.x - bw.x, a.y - bw.y);
            }
        }
    }
}

// Split L into A * B with A >= B, both powers of two.
template <int L> struct Split {
    static constexpr int LOG = ilog2c(L);
    static constexpr int A = 1 << ((LOG + 1) / 2);
    static constexpr int B = L / A;
};

// Padded slot stride (complex elements) for one sequence: holds the B x (A+1) transpose
// and, in natural order, L entries plus the R2C Nyquist term; odd so that consecutive
// slots start on different banks.
template <int L> struct Slot {
    static constexpr int A = Split<L>::A, B = Split<L>::B;
    static constexpr int T = B * (A + 1) > L + 1 ? B * (A + 1) : L + 1;
    static constexpr int S = (T % 2 == 0) ? T + 1 : T;
};

// The two halves of the four-step transform of one sequence, split at its shared-memory
// exchange (host builds run every lane's first half, then every lane's second half).
// First: the A-point FFT in registers, the twiddles, the A x B intermediate to the slot.
template <int L, int DIR, bool ZIN = false, bool SMTW = false>
__host__ __device__ __forceinline__ void fft4_first(float2 (&v)[Split<L>::A], float2* slot, int lane,
                                                    const float2* __restrict__ tw4) {
    constexpr int A = Split<L>::A, B = Split<L>::B;
    // n = B n1 + n2 >= L/2 exactly when n1 >= A/2
    fft_reg64<A, DIR, ZIN>(v);
    if (B > 1) {
#pragma unroll
        for (int k1 = 1; k1 < A; k1++) {
#ifdef __CUDA_ARCH__
            float2 w = SMTW ? tw4[k1 * B + lane] : __ldg(&tw4[k1 * B + lane]);
#else
            float2 w = tw4[k1 * B + lane];
#endif
            if (DIR > 0) w.y = -w.y;
            const float2 a = v[k1];
            v[k1] = make_float2(a.x * w.x - a.y * w.y, a.x * w.y + a.y * w.x);
        }
#pragma unroll
        for (int k1 = 0; k1 < A; k1++) slot[lane * (A + 1) + k1] = v[k1];
    }
}

// Second: lane t reads the A/B columns k1 = t + B i back and runs their B-point FFTs.
template <int L, int DIR, bool HOUT = false>
__host__ __device__ __forceinline__ void fft4_second(float2 (&v)[Split<L>::A], const float2* slot, int lane) {
    constexpr int A = Split<L>::A, B = Split<L>::B;
    if (B > 1) {
#pragma unroll
        for (int i = 0; i < A / B; i++) {
#pragma unroll
            for (int n2 = 0; n2 < B; n2++) v[i * B + n2] = slot[n2 * (A + 1) + lane + B * i];
            // X index (lane + B i) + A k2 >= L/2 exactly when k2 >= B/2
            fft_reg64<B, DIR, false, HOUT>(v + i * B);
        }
    }
}

// Four-step transform of one sequence (see header).  `lane` in [0, B); all B lanes of
// the sequence, and every existing lane of the warp (`wmask`), must call it.
// `tw4`: the A x B twiddle matrix of length L, in global memory, or in shared memory
// when SMTW (a block-staged copy).
// ZIN: inputs L/2..L-1 are zero; HOUT: only outputs 0..L/2-1 are wanted.
template <int L, int DIR, bool ZIN = false, bool HOUT = false, bool SMTW = false>
__device__ __forceinline__ void fft4(float2 (&v)[Split<L>::A], float2* slot, int lane,
                                     const float2* __restrict__ tw4, unsigned wmask = 0xffffffffu) {
    fft4_first<L, DIR, ZIN, SMTW>(v, slot, lane, tw4);
    if (Split<L>::B > 1) {
        __syncwarp(wmask);
        fft4_second<L, DIR, HOUT>(v, slot, lane);
        __syncwarp(wmask);
    }
}

// Index of output element j of lane `lane`: X index (lane + B i) + A k2 with j = i B + k2.
template <int L>
__host__ __device__ __forceinline__ constexpr int fft4_out_index(int lane, int j) {
    return (lane + Split<L>::B * (j / Split<L>::B)) + Split<L>::A * (j % Split<L>::B);
}
