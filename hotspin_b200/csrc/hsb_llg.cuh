// Fused right-hand side + Runge-Kutta stage kernel: shared declarations.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

// Maximum number of stored stages any integrator reads (Dormand-Prince: 7).
#define HSB_MAXK 7

// Uniform physics parameters of one simulation, FP32 where used in the bulk arithmetic.
struct HsbPhys {
    int N0, N1, N2;      // program order, N2 fastest (user x)
    int pbc0, pbc1, pbc2;
    int nch;             // state channels: 3 (m) or 5 (m, Te, Tl)
    long ncell;
    float ex_c[3];       // Ms0 * lex^2 / cs_d^2 (A/m)
    const float* lex_mask;   // optional per-cell lex mask (harmonic lex^2 weights)
    const float* msat_mask;  // optional per-cell Ms0 mask (0 = vacuum)
    float gamma;         // gamma_LL (m/As)
    float lam[3];        // relativistic damping diagonal (program components)
    float bext[3];       // B_ext / mu0 (A/m)
    float ku_pre;        // 2 Ku / (mu0 Ms0) (A/m)
    float u[3];          // anisotropy axis as given
    float uhat[3];       // normalised axis
    int demag;
    // MFA longitudinal field
    int llb;
    float lf_pre;        // n kB / (mu0 Ms0)  (A/m per K)
    float lf_b;          // 3 S/(S+1) Tc   (K)   (S = J; 3 Tc for the Langevin case)
    float lf_gpre, lf_lpre, lf_lim;  // Brillouin constants (2J+1)/2J, 1/2J, series limit
    int lf_langevin;
    float T_uniform;     // bath temperature when there is no two-temperature model
    // thermal field
    int thermal;
    uint32_t seed_lo, seed_hi;
    double th_pre;       // 2 kB / (mu0 V gamma Ms0) (multiplied by T / dt_eff)
    double cutoff_dt;
    // two-temperature model
    int ttm;
    float ke_c[3], kl_c[3];  // k / cs_d^2 (W/m^3/K)
    float g_ep, gamma_e, c_l;
    float laser_p0, laser_t0, laser_c;  // c = 4 ln2 / fwhm^2
    float laser_inv2s2;                 // 1/(2 sigma^2), 0 = uniform spot
    const double2* laser_tab;           // pointwise time profile (t, factor), laser_npts >= 2
    int laser_npts;                     // 0: Gaussian pulse in time
    const double* bext_tab;             // pointwise applied field: rows (t, Bx, By, Bz) in tesla
    int bext_npts;                      // 0: the constant bext
    float cs1, cs2;
    int normalize;       // renormalise m at stage formation (LLG mode); used by batched launches
    float ms0;           // Ms0 (A/m), the demag scale of this simulation
    // division of a cell index (< 2^31) by N2 and by N1 as a multiply-high and shift
    // (round-up reciprocal, Granlund & Montgomery 1994): q = umulhi(x, mul) >> shr
    unsigned div2_mul, div2_shr, div1_mul, div1_shr;
};

// Absorbed laser power density (W/m^3, before the lateral spot) at time t: laser_p0 times a
// Gaussian of the given FWHM around laser_t0, or times the piecewise-linear interpolation of
// a (time, factor) table as hotspin's pointwise quantities evaluate theirs
// (engine/update_pointwiseof.go:31-98); zero outside the table's time range.  Uniform over a
// launch: every thread finds the same table interval.
__device__ __forceinline__ float hsb_laser_power(const HsbPhys& P, double t) {
    if (P.laser_p0 == 0.f) return 0.f;
    if (P.laser_npts >= 2) {
        const double2* tab = P.laser_tab;
        int lo = 0, hi = P.laser_npts - 1;
        if (t < tab[0].x || t > tab[hi].x) return 0.f;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (tab[mid].x <= t) lo = mid;
            else hi = mid;
        }
        const double2 a = tab[lo], b = tab[hi];
        const double f = a.y + (t - a.x) / (b.x - a.x) * (b.y - a.y);
        return (float)((double)P.laser_p0 * f);
    }
    const float tt = (float)(t - (double)P.laser_t0);
    return P.laser_p0 * expf(-P.laser_c * tt * tt);
}

// Applied field H_ext (A/m) at time t: the constant bext, or the piecewise-linear interpolation
// of the (time, B) table divided by mu0 (a pointwise quantity as in
// engine/update_pointwiseof.go:31-98), zero outside the table's time range.
__device__ __forceinline__ void hsb_bext(const HsbPhys& P, double t, float* h) {
    if (P.bext_npts >= 2) {
        const double* tab = P.bext_tab;
        int lo = 0, hi = P.bext_npts - 1;
        if (t < tab[0] || t > tab[4 * hi]) {
            h[0] = h[1] = h[2] = 0.f;
            return;
        }
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (tab[4 * mid] <= t) lo = mid;
            else hi = mid;
        }
        const double f = (t - tab[4 * lo]) / (tab[4 * hi] - tab[4 * lo]);
        const double inv_mu0 = 1.0 / (4e-7 * 3.14159265358979323846);
        for (int c = 0; c < 3; c++) {
            const double a = tab[4 * lo + 1 + c], b = tab[4 * hi + 1 + c];
            h[c] = (float)((a + f * (b - a)) * inv_mu0);
        }
        return;
    }
    h[0] = P.bext[0];
    h[1] = P.bext[1];
    h[2] = P.bext[2];
}

// Quotient by the divisor encoded in (mul, shr); mul == 0 encodes a divisor of 1.
__host__ __device__ __forceinline__ unsigned hsb_fastdiv(unsigned x, unsigned mul, unsigned shr) {
#ifdef __CUDA_ARCH__
    return mul ? (__umulhi(x, mul) >> shr) : x;
#else
    return mul ? (unsigned)(((unsigned long long)x * mul) >> 32) >> shr : x;
#endif
}

// Multiplier and shift for dividing indices below 2^31 by d >= 1: with l = ceil(log2 d),
// mul = ceil(2^(31 + l) / d) and shr = l - 1, so that q = floor(x mul / 2^(32 + shr)).
inline void hsb_fastdiv_init(unsigned d, unsigned* mul, unsigned* shr) {
    if (d <= 1) {
        *mul = 0;
        *shr = 0;
        return;
    }
    unsigned l = 0;
    while ((1ull << l) < d) l++;
    const unsigned long long p = 31 + l;
    *mul = (unsigned)(((1ull << p) + d - 1) / d);
    *shr = (unsigned)(p - 32);
}

// Batched launches: slot = blockIdx.z; every per-slot buffer of slot s lives at the slot-0
// address + s * stride (one arena per slot), physics and solver state per slot.
struct BatchArgs {
    long stride;               // floats between slots' arenas (0 = not batched)
    const HsbPhys* phys;       // device array [nslot]
    int nslot;
};

// Device-resident solver state (read by every kernel of an attempt, written by the
// controller).  Lives in device memory so whole steps can be captured in a CUDA graph.
struct HsbSolverDev {
    double t, dt;
    long long step;        // accepted steps
    long long attempts, rejects;
    int cur;               // state buffer holding y0 (0/1)
    int kslot;             // which of the two first/last stage slots holds k1 (DP45)
    int active;            // 0 once the target is reached: kernels of later attempts return
    int status;            // bit 0: non-finite state seen; bit 1: dt hit mindt
    double err;            // last error norm
    double mindt, maxdt;
    double t_stop;         // > 0: do not step past this time
    long long step_stop;   // >= 0: stop after this many accepted steps
    unsigned int err_acc;  // float bits of the running max error of the attempt
    unsigned int nonfinite;
    int prep;              // batched slots: 1 while the slot's first-stage data is being prepared
    int pad_;
    unsigned int err_eq[3];  // rk12: float bits of the attempt's per-equation errors (m, Te, Tl)
    int tries;             // rk12: rejected attempts of the current step
};

// Step-size rule of hotspin's adaptive Heun solver (solve_rk12.go:91-214), applied to one
// solver word after an attempt.  err[q] = dt max_i |k1_i - k0_i| over the cells and
// components of equation q (m, Te, Tl in this order; neq of them), maxerr[q] its
// per-step limit (<m>_maxError; +inf leaves an equation uncontrolled), nonfinite the
// attempt's non-finite flag.  The equations are visited in order with the reference's
// running bad-step flag: a bad equation and every one after it take the cube-root factor,
// the others the square root; factor x 0.8 clamped to [0.1, 1.5], the smallest over the
// equations; dt_new = dt factor clamped to [mindt, maxdt].  The attempt is kept when no
// equation was bad or dt_new is at mindt (status bit 2 if it was bad).  A step that still
// fails after 10 retries sets status bit 4 and stops, where the reference panics.  A
// non-finite attempt is rejected with the smallest factor; at mindt it sets status bit 1.
// Host and device share this code.
__host__ __device__ inline void hsb_rk12_rule(HsbSolverDev& sd, const float* err, const double* maxerr, int neq,
                                             bool nonfinite) {
    const double h = sd.dt;
    bool finite = !nonfinite;
    for (int q = 0; q < neq; q++) finite = finite && isfinite((double)err[q]);
    bool bad = false;
    double fmin = 2.0;
    double emax = 0.0;
    if (finite) {
        for (int q = 0; q < neq; q++) {
            const double e = (double)err[q];
            const double r = maxerr[q] / e;            // inf when e == 0 or uncontrolled
            if (e > maxerr[q]) bad = true;
            double f = bad ? cbrt(r) : sqrt(r);
            f *= 0.8;
            if (f > 1.5) f = 1.5;
            if (f < 0.1) f = 0.1;
            if (f < fmin) fmin = f;
            const double en = e / maxerr[q];
            if (en > emax) emax = en;
        }
    } else {
        fmin = 0.1;
    }
    double nd = h * fmin;
    if (nd < sd.mindt) nd = sd.mindt;
    if (nd > sd.maxdt) nd = sd.maxdt;
    const bool accept = finite && (!bad || nd == sd.mindt);
    sd.err = finite ? emax : INFINITY;
    sd.attempts += 1;
    if (!finite && h <= sd.mindt) sd.status |= 1;
    if (accept) {
        if (bad) sd.status |= 2;
        sd.t += h;
        sd.step += 1;
        sd.cur = 1 - sd.cur;
        sd.tries = 0;
    } else {
        sd.rejects += 1;
        if (sd.tries > 10) {
            sd.status |= 4;
            sd.active = 0;
        } else {
            sd.tries += 1;
        }
    }
    if (sd.t_stop > 0.0) {
        const double rem = sd.t_stop - sd.t;
        if (rem <= 1e-6 * nd || rem <= 0.0) sd.active = 0;
        else if (nd > rem) nd = rem;
    }
    if (sd.step_stop >= 0 && sd.step >= sd.step_stop) sd.active = 0;
    if (sd.status & 1) sd.active = 0;
    sd.dt = nd;
}

// Pointer selectors resolved on the device against HsbSolverDev.
enum { SEL_FIXED = 0, SEL_CUR = 1, SEL_NEXT = 2, SEL_K1 = 3, SEL_K7 = 4 };

struct PtrSel {
    float* p[2];
    int sel;
};

struct StageArgs {
    PtrSel ys;               // right-hand-side input state [nch][ncell]
    PtrSel hd;               // demag field of ys (3 x ncell) or null
    PtrSel ytherm;           // state whose Te sets the thermal amplitude (step start)
    float tfrac;             // stage time = t + tfrac * dt
    // k_s storage: kout = kacc_w * kacc + kself_w * k_s
    PtrSel kout;
    PtrSel kacc;
    float kacc_w, kself_w;
    // next state: ynext = ybase + dt * (sum_j ck[j] kin[j] + cself k_s)
    PtrSel ynext;
    PtrSel ybase;
    int nk;
    PtrSel kin[HSB_MAXK];
    float ck[HSB_MAXK];
    float cself;
    int normalize;           // renormalise m of ynext
    // error estimate: e = dt * (sum_j ce[j] kin[j] + ceself k_s), max-norm per equation
    int err;
    float ce[HSB_MAXK];
    float ceself;
    PtrSel yerr0;            // y0 (for the relative temperature norm)
    float rtol;
    int ungated;             // run even when the solver is inactive (state queries)
    int prep_gated;          // gate on HsbSolverDev.prep instead of .active (batched slot preparation)
    // thermal field of the step (the same in every stage of an attempt): 0 = generate it,
    // 1 = generate it and store it to hth, 2 = read it from hth (load-first kernel only)
    int hth_mode;
    PtrSel hth;              // [3][ncell]
    int torque_only;         // generic kernel only: k = gamma (m x H), without the relaxation term
    // error mode: 0 = the DP45 norm (m: |e| / rtol, T: |e| / (rtol max(|T0|, |T|)), one
    // maximum); 1 = per-equation absolute errors dt |e| into HsbSolverDev.err_eq (rk12)
    int err_abs;
};
