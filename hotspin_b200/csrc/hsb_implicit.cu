// Fixed-point iterations of hotspin's implicit solvers on the device.
//
// solver/am12 (solve_am01.go:45-318): explicit Euler start, implicit Euler predictor and
// trapezoidal corrector, each solved by fixed-point sweeps; solver/bdf-euler
// (solve_euler_backward.go:29-91): fixed-step backward Euler, one equation after the other.
// The reference runs every sweep from the host with a stream synchronisation and four
// reductions (MaxDiff / MaxAbs / MaxSum through gpu.Reductor) per equation.  Here a sweep is
// one kernel that forms the new iterate, renormalises m where the reference's update would,
// and folds the per-channel maxima into the solver word; a one-thread-per-slot kernel applies
// the reference's decision (hsb_am_* / hsb_bdf_* rules in hsb_llg.cuh, shared with the host);
// the right-hand sides between sweeps are the fused stage kernels.  Every launch is gated on
// words of the solver word, so an attempt with all its possible sweeps is one fixed kernel
// sequence that a CUDA graph replays.
#include "hsb_common.cuh"
#include "hsb_llg.cuh"

__device__ __forceinline__ float* imp_resolve(const PtrSel& s, const HsbSolverDev* sd, long off) {
    float* p;
    switch (s.sel) {
        case SEL_CUR: p = s.p[sd->cur]; break;
        case SEL_NEXT: p = s.p[1 - sd->cur]; break;
        default: p = s.p[0];
    }
    return p ? p + off : nullptr;
}

__device__ __forceinline__ double* imp_slot64(double* p, long off) {
    return p ? (double*)((float*)p + off) : nullptr;
}

__device__ __forceinline__ void imp_fold_max(float v, unsigned int* word) {
    v = warp_max_f(v);
    if ((threadIdx.x & 31) == 0 && v > 0.f) atomicMax(word, __float_as_uint(v));
}

// One sweep (or the explicit step / the am12 step error) over every cell of a slot.
template <int CH, bool BATCH>
__global__ void __launch_bounds__(256) k_imp_sweep(const __grid_constant__ HsbPhys P0, const ImpArgs A,
                                                   HsbSolverDev* sd0, const BatchArgs Bt) {
    const int slot = BATCH ? (int)blockIdx.z : 0;
    HsbSolverDev* sd = sd0 + slot;
    const int mode = A.mode;
    bool run;
    if (mode == IMP_AM_ERR) run = sd->active && !(sd->it_flags & 4);
    else if (mode == IMP_BDF_EULER || mode == IMP_AM_EULER) run = sd->active != 0;
    else run = sd->active && sd->it_active;
    if (!run) return;
    const HsbPhys& P = BATCH ? Bt.phys[slot] : P0;
    const long off = BATCH ? (long)slot * Bt.stride : 0;
    const int normalize = BATCH ? (A.normalize && P.normalize) : A.normalize;
    const long n = P.ncell;
    const double dt = sd->dt;
    const float* y0 = imp_resolve(A.y0, sd, off);
    float* w = imp_resolve(A.w, sd, off);
    const float* k0 = A.k0 ? A.k0 + off : nullptr;
    const float* dy = (sd->dysel ? A.k2 : A.k1);
    if (dy) dy += off;
    // the FP64 iterates lie in the slot's arena (the slot stride, in floats, keeps 256-byte alignment)
    double* w64 = imp_slot64(A.w64, off);
    double* up64 = imp_slot64(A.up64, off);
    double* uc64 = imp_slot64(A.uc64, off);
    const double* prev64 = (mode == IMP_AM_CORR && sd->prevsel) ? up64 : w64;
    double* u64 = (mode == IMP_AM_PRED) ? up64 : (mode == IMP_AM_CORR ? uc64 : nullptr);
    // channels this launch touches
    int c0 = 0, c1 = CH;
    if (mode == IMP_BDF_EULER || mode == IMP_BDF_SWEEP) {
        c0 = hsb_eq_first(A.eq);
        c1 = c0 + hsb_eq_count(A.eq);
    }
    float dmax[CH], smax[CH];
#pragma unroll
    for (int c = 0; c < CH; c++) dmax[c] = smax[c] = 0.f;
    bool bad = false;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        hsb_imp_sweep_cell<CH>(mode, i, n, dt, c0, c1, normalize, y0, w, w, dy, k0, w64, prev64, u64, up64, uc64,
                               dmax, smax, bad);
    if (mode != IMP_BDF_EULER && mode != IMP_AM_EULER) {
#pragma unroll
        for (int c = 0; c < CH; c++) {
            imp_fold_max(dmax[c], &sd->red[c]);
            imp_fold_max(smax[c], &sd->red[5 + c]);
        }
    }
    if (bad) atomicOr(&sd->nonfinite, 1u);
}

// Decisions, one thread per slot (hsb_imp_rule in hsb_llg.cuh).
__global__ void k_imp_rule(HsbSolverDev* sd0, int nslot, const ImpLimits L, int which) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nslot) return;
    hsb_imp_rule(sd0[slot], L, which);
}

int hsb_launch_imp_sweep(const HsbPhys& P, const ImpArgs& A, HsbSolverDev* sd, const BatchArgs& Bt, int nslot,
                         bool batched, cudaStream_t st) {
    const int threads = 256;
    long g = (P.ncell + threads - 1) / threads;
    const long cap = (long)hsb_sm_count() * 4;
    dim3 grid((unsigned)(g < cap ? g : cap), 1, (unsigned)nslot);
    if (batched) {
        if (P.nch == 5) k_imp_sweep<5, true><<<grid, threads, 0, st>>>(P, A, sd, Bt);
        else k_imp_sweep<3, true><<<grid, threads, 0, st>>>(P, A, sd, Bt);
    } else {
        if (P.nch == 5) k_imp_sweep<5, false><<<grid, threads, 0, st>>>(P, A, sd, Bt);
        else k_imp_sweep<3, false><<<grid, threads, 0, st>>>(P, A, sd, Bt);
    }
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}

int hsb_launch_imp_rule(HsbSolverDev* sd, int nslot, const ImpLimits& L, int which, cudaStream_t st) {
    k_imp_rule<<<(nslot + 31) / 32, 32, 0, st>>>(sd, nslot, L, which);
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}
