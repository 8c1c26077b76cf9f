// Fused right-hand side + Runge-Kutta stage kernel: shared declarations.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

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
    // second-order local relaxation terms of the LLBar equation (0 = not loaded):
    // llbar/damping/nonconservative/02/local (mu_par) and conservative/02/local (mu_perp)
    int llbar02;
    float mu_par[3], mu_perp[3];
    // zero-order non-local relaxation (llbar/damping/nonconservative/00/nonlocal, alpha_e):
    // -gamma diag(alpha_e) lap(H_eff); the effective field of every cell is stored in hbuf by
    // a first pass of the generic stage kernel so the second can take the neighbours' values
    int nonlocal;
    float lam_e[3];
    float inv_cs2[3];    // 1 / cs_d^2 (1/m^2)
    float* hbuf;         // [3][ncell]
    // division of a cell index (< 2^31) by N2 and by N1 as a multiply-high and shift
    // (round-up reciprocal, Granlund & Montgomery 1994): q = umulhi(x, mul) >> shr
    unsigned div2_mul, div2_shr, div1_mul, div1_shr;
};

// Absorbed laser power density (W/m^3, before the lateral spot) at time t: laser_p0 times a
// Gaussian of the given FWHM around laser_t0, or times the piecewise-linear interpolation of
// a (time, factor) table as hotspin's pointwise quantities evaluate theirs
// (engine/update_pointwiseof.go:31-98); zero outside the table's time range.  Uniform over a
// launch: every thread finds the same table interval.
__host__ __device__ __forceinline__ float hsb_laser_power(const HsbPhys& P, double t) {
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
__host__ __device__ __forceinline__ void hsb_bext(const HsbPhys& P, double t, float* h) {
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
    int tries;             // rk12 / am12: rejected attempts of the current step
    // am12 / bdf-euler fixed-point iterations
    int it_active;         // 1 while the current iteration continues (gates its kernels)
    int it_count;          // sweeps of the current iteration
    int it_flags;          // bit 0: the iteration failed; bit 1: limit the next dt by the
                           // predictor's alpha; bit 2: the attempt was abandoned
    int aborts;            // abandoned attempts of the current step
    int dysel;             // derivative a sweep uses: 0 = at the explicit Euler point, 1 = latest
    int prevsel;           // previous iterate a sweep compares with: 0 = renormalised, 1 = raw predictor
    int eq;                // bdf-euler: the equation being iterated (0 m, 1 Te, 2 Tl)
    int rhs_due;           // bdf-euler: 1 when the last sweep ran (its result's derivative is due)
    double er[3];          // am12: the previous sweep's errors, sorted ascending
    double alpha[3];       // am12: the predictor's last per-equation convergence ratios
    double alpha_max;      // am12: the last sweep's largest ratio
    unsigned int red[10];  // float bits of a sweep's maxima: |prev - new| per channel (0..4), the
                           // scale per channel (5..9: |new|, |predictor| or |prev + new|)
};

// Dormand-Prince step-size rule (the controller described in include/hotspin_b200.h), applied
// to one solver word after an attempt: err = the attempt's error norm (max over the cells of
// |e| / (rtol scale)), nonfinite its non-finite flag.  Accept at err <= 1 or at the dt floor;
// factor 0.9 err^(-1/5) clamped to [0.2, 5] (to [0.2, 1] after a rejection), 0.2 for a
// non-finite attempt (status bit 1 at the floor), 5 for err = 0; dt_new clamped to
// [mindt, maxdt] and to the time left before t_stop.  Status bit 2: an attempt at the floor
// that did not meet the tolerance.
__host__ __device__ inline void hsb_dp45_rule(HsbSolverDev& sd, float ef, bool nonfinite) {
    const double h = sd.dt;
    const double err = (double)ef;
    const bool finite = !nonfinite && isfinite(err);
    const bool accept = finite && (err <= 1.0 || h <= sd.mindt);
    double fac;
    if (!finite) fac = 0.2;
    else if (err == 0.0) fac = 5.0;
    else fac = 0.9 * pow(err, -0.2);
    fac = fmin(fmax(fac, 0.2), accept ? 5.0 : 1.0);
    double nd = fmin(fmax(h * fac, sd.mindt), sd.maxdt);
    sd.err = finite ? err : INFINITY;
    sd.attempts += 1;
    if (!finite && h <= sd.mindt) sd.status |= 1;
    // a step taken at the floor without meeting the tolerance (accepted because dt cannot
    // shrink further; hotspin's rk12 accepts such steps the same way, solve_rk12.go:196-198)
    if (finite && err > 1.0 && h <= sd.mindt) sd.status |= 2;
    if (accept) {
        sd.t += h;
        sd.step += 1;
        sd.cur = 1 - sd.cur;
        sd.kslot = 1 - sd.kslot;
    } else {
        sd.rejects += 1;
        if (h <= sd.mindt) sd.status |= 2;
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
    float* heff_out;         // generic kernel only: store H_eff of ys here and compute nothing else
    // error mode: 0 = the DP45 norm (m: |e| / rtol, T: |e| / (rtol max(|T0|, |T|)), one
    // maximum); 1 = per-equation absolute errors dt |e| into HsbSolverDev.err_eq (rk12)
    int err_abs;
    // gate word: 0 = HsbSolverDev.active; else the byte offset of an int word of the solver
    // word that must also be nonzero (the fixed-point iterations of am12 / bdf-euler)
    int gate_word;
};

// Whether a launch gated on `gate_word` (see StageArgs) runs for this solver word.
__host__ __device__ inline bool hsb_gate(const HsbSolverDev* sd, int gate_word) {
    if (!sd->active) return false;
    return gate_word == 0 || *(const int*)((const char*)sd + gate_word) != 0;
}

// ------------------------------------------------------------------ am12 / bdf-euler sweeps
enum { IMP_AM_PRED = 0, IMP_AM_CORR = 1, IMP_AM_ERR = 2, IMP_BDF_EULER = 3, IMP_BDF_SWEEP = 4, IMP_AM_EULER = 5 };
enum {
    IMP_RULE_AM_BEGIN = 0, IMP_RULE_AM_ITER_PRED = 1, IMP_RULE_AM_ITER_CORR = 2, IMP_RULE_AM_PRED_END = 3,
    IMP_RULE_AM_CORR_END = 4, IMP_RULE_AM_FINAL = 5, IMP_RULE_BDF_BEGIN = 6, IMP_RULE_BDF_ITER = 7,
    IMP_RULE_BDF_CLEAR = 8
};

// Buffers of a sweep (k_imp_sweep): new iterates are formed from y0 and a derivative, compared
// with the previous iterate, and written (m renormalised in LLG mode) to w.
struct ImpArgs {
    PtrSel y0;         // state at the start of the step (y[cur])
    PtrSel w;          // renormalised iterate / working state (y[next])
    float* k0;         // am12: f(y0); bdf-euler: the latest derivative
    float* k1;         // am12: derivative at the explicit Euler point
    float* k2;         // am12: derivative of the latest iterate
    // am12: FP64 renormalised iterate and raw predictor / corrector iterates, which the sweeps
    // compare (the FP32 w, rounded from w64, feeds the right-hand side); slot 0's, the others
    // one slot stride of floats further
    double* w64;
    double* up64;
    double* uc64;
    int mode;          // IMP_AM_* / IMP_BDF_*
    int normalize;     // renormalise m where it is written to w (LLG mode)
    int eq;            // bdf-euler: equation (0 m, 1 Te, 2 Tl)
};

// Tolerances of the implicit solvers.
struct ImpLimits {
    double abs_err[3], rel_err[3];   // am12: per-equation absolute / relative errors
    double max_iter_err;             // bdf-euler: iterator error
    int max_iter;                    // bdf-euler: sweeps
    int neq;
    int eq;                          // bdf-euler: the equation a BEGIN starts
};

// ------------------------------------------------------------------ am12 / bdf-euler rules
// hotspin's adaptive Adams-Moulton 1-2 solver (solver/am12, solve_am01.go:45-318) and fixed-step
// backward Euler (solver/bdf-euler, solve_euler_backward.go:29-91) iterate their implicit
// stages by fixed point; the sweeps run on the device (k_am_sweep) and leave per-channel maxima
// in HsbSolverDev.red; these rules, shared by host and device, turn them into the decisions.

// Channels of equation q: m = 0..2, Te = 3, Tl = 4.
__host__ __device__ inline int hsb_eq_first(int q) { return q == 0 ? 0 : q + 2; }
__host__ __device__ inline int hsb_eq_count(int q) { return q == 0 ? 3 : 1; }

// am12 error norm of equation q from the sweep maxima: per channel d / (abs + scale rel), root
// mean square over the equation's channels (solve_am01.go:120-131).
__host__ __device__ inline double hsb_am_norm(const unsigned int* red, int q, double abs_err, double rel_err) {
    const int c0 = hsb_eq_first(q), nc = hsb_eq_count(q);
    double t = 0.0;
    for (int c = c0; c < c0 + nc; c++) {
        float d, m;
#ifdef __CUDA_ARCH__
        d = __uint_as_float(red[c]);
        m = __uint_as_float(red[5 + c]);
#else
        memcpy(&d, &red[c], 4);
        memcpy(&m, &red[5 + c], 4);
#endif
        const double v = (double)d / (abs_err + (double)m * rel_err);
        t += v * v;
    }
    return sqrt(t) / sqrt((double)nc);
}

// One sweep of an am12 iteration (phase 0 predictor, 1 corrector): alpha_q = tErr_q / er_q
// against the previous sweep's list, er = the new errors sorted ascending (the reference sorts
// its list in place, so the next sweep pairs each equation with a rank, not with itself), err
// and alpha their maxima; converged when err <= 0.1, failed when alpha >= 1 or after the 6th
// sweep, else another sweep with the latest derivative (solve_am01.go:105-158, 176-223).
__host__ __device__ inline void hsb_am_iter_rule(HsbSolverDev& sd, const double* abs_err, const double* rel_err,
                                                 int neq, int phase) {
    double terr[3], alp[3];
    for (int q = 0; q < neq; q++) {
        terr[q] = hsb_am_norm(sd.red, q, abs_err[q], rel_err[q]);
        alp[q] = terr[q] / sd.er[q];
    }
    for (int i = 1; i < neq; i++)       // insertion sort, ascending, NaN last
        for (int j = i; j > 0 && (terr[j - 1] > terr[j] || (terr[j - 1] != terr[j - 1] && terr[j] == terr[j])); j--) {
            const double t = terr[j - 1];
            terr[j - 1] = terr[j];
            terr[j] = t;
        }
    double amax = alp[0];
    for (int q = 0; q < neq; q++) {
        sd.er[q] = terr[q];
        if (phase == 0) sd.alpha[q] = alp[q];
        if (!(alp[q] <= amax)) amax = alp[q];
    }
    const double err = terr[neq - 1];
    sd.alpha_max = amax;
    sd.it_count += 1;
    for (int c = 0; c < 10; c++) sd.red[c] = 0u;
    if (err <= 0.1) {
        sd.it_active = 0;
    } else if (amax >= 1.0 || sd.it_count > 5 || !(err == err)) {
        sd.it_active = 0;
        sd.it_flags |= 1;
    } else {
        sd.dysel = 1;
        sd.prevsel = 0;
    }
}

// End of an am12 iteration phase.  A failed iteration abandons the attempt: dt is halved, or
// scaled by sqrt(0.6 / alpha) when alpha > 0.6; after a failed predictor the next step size is
// limited by the predictor's alphas (solve_am01.go:160-172, 225-236).  The reference panics when
// this happens on its 10th try (status 4 here) and otherwise retries without counting a bad
// step; 64 abandoned attempts in one step also stop the run here (the reference keeps halving).
// A finished predictor starts the corrector with the explicit-Euler-point derivative.
__host__ __device__ inline void hsb_am_phase_rule(HsbSolverDev& sd, int phase, int neq) {
    if (sd.it_flags & 1) {
        sd.it_flags &= ~1;
        sd.it_flags |= 4;
        if (phase == 0) sd.it_flags |= 2;
        if (sd.tries == 9) {
            sd.status |= 4;
            sd.active = 0;
            return;
        }
        double h = 0.5 * sd.dt;
        if (sd.alpha_max > 0.6) h = sd.dt * sqrt(0.6 / sd.alpha_max);
        sd.dt = h;
        sd.aborts += 1;
        sd.attempts += 1;
        if (sd.aborts > 64) {
            sd.status |= 4;
            sd.active = 0;
        }
        return;
    }
    if (phase == 0) {
        sd.it_active = 1;
        sd.it_count = 0;
        for (int q = 0; q < neq; q++) sd.er[q] = 0.1;
        sd.dysel = 0;
        sd.prevsel = 1;
    }
}

// End of an am12 attempt: per equation the step error (corrector vs predictor, scale: the
// predictor), bad when above 1; dt_new = dt sqrt(0.8 / err), limited by dt sqrt(0.6 / alpha_q)
// for the first equation when the flag is set (the reference clears it inside its loop), clamped
// to [mindt, maxdt], the smallest over the equations; kept when no equation was bad or dt_new is
// mindt; the 12th bad attempt stops the run, where the reference panics (solve_am01.go:238-306).
__host__ __device__ inline void hsb_am_final_rule(HsbSolverDev& sd, const double* abs_err, const double* rel_err,
                                                  int neq, bool nonfinite) {
    if (sd.it_flags & 4) {        // abandoned attempt: dt was set by the phase rule
        sd.it_flags &= ~4;
        for (int c = 0; c < 10; c++) sd.red[c] = 0u;
        return;
    }
    const double h = sd.dt;
    bool bad = false;
    bool finite = !nonfinite;
    double nd = INFINITY, emax = 0.0;
    for (int q = 0; q < neq; q++) {
        const double te = hsb_am_norm(sd.red, q, abs_err[q], rel_err[q]);
        if (!(te == te)) finite = false;
        if (te > 1.0) bad = true;
        const double hr = h * sqrt(0.8 / te);
        double n = hr;
        if (sd.it_flags & 2) {
            const double ha = h * sqrt(0.6 / sd.alpha[q]);
            n = hr < ha ? hr : ha;
            sd.it_flags &= ~2;
        }
        if (n < sd.mindt) n = sd.mindt;
        if (n > sd.maxdt) n = sd.maxdt;
        if (n < nd) nd = n;
        if (te > emax) emax = te;
    }
    for (int c = 0; c < 10; c++) sd.red[c] = 0u;
    if (!finite) {
        nd = h * 0.1;
        if (nd < sd.mindt) nd = sd.mindt;
        bad = true;
    }
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
        sd.aborts = 0;
        sd.it_flags = 0;
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

// Start of an am12 attempt: the predictor iteration begins with the explicit-Euler-point
// derivative and the renormalised Euler point as its previous iterate.
__host__ __device__ inline void hsb_am_begin_rule(HsbSolverDev& sd, int neq) {
    sd.it_active = 1;
    sd.it_count = 0;
    sd.dysel = 0;
    sd.prevsel = 0;
    sd.it_flags &= 2;
    for (int q = 0; q < neq; q++) sd.er[q] = 0.1;
    for (int c = 0; c < 10; c++) sd.red[c] = 0u;
}

// One backward-Euler sweep of equation sd.eq: err = MaxDiff / MaxSum over the equation's
// channels (relative when the sum is positive), converged at err <= max_iter_err; more than
// max_iter sweeps stop the run (status 4), where the reference panics
// (solve_euler_backward.go:64-84).
__host__ __device__ inline void hsb_bdf_iter_rule(HsbSolverDev& sd, double max_iter_err, int max_iter) {
    const int c0 = hsb_eq_first(sd.eq), nc = hsb_eq_count(sd.eq);
    float d = 0.f, m = 0.f;
    for (int c = c0; c < c0 + nc; c++) {
        float dc, mc;
#ifdef __CUDA_ARCH__
        dc = __uint_as_float(sd.red[c]);
        mc = __uint_as_float(sd.red[5 + c]);
#else
        memcpy(&dc, &sd.red[c], 4);
        memcpy(&mc, &sd.red[5 + c], 4);
#endif
        if (!(dc <= d)) d = dc;
        if (!(mc <= m)) m = mc;
    }
    double err = (double)d;
    if (m > 0.f) err = err / (double)m;
    sd.err = err;
    sd.it_count += 1;
    sd.rhs_due = 1;               // the sweep ran: the derivative of its result is due
    for (int c = 0; c < 10; c++) sd.red[c] = 0u;
    // the reference checks the sweep count after every sweep, converged or not
    if (sd.it_count > max_iter || !(err == err)) {
        sd.it_active = 0;
        sd.status |= (err == err) ? 4 : 1;
        sd.active = 0;
    } else if (err <= max_iter_err) {
        sd.it_active = 0;
    }
}

// The decision kernel's dispatch (k_imp_rule, one thread per slot): which rule a launch applies
// to the slot's solver word.  A stopped slot is left alone, except that the due flag of
// bdf-euler is always cleared.
__host__ __device__ inline void hsb_imp_rule(HsbSolverDev& sd, const ImpLimits& L, int which) {
    if (which == IMP_RULE_BDF_CLEAR) {
        sd.rhs_due = 0;
        return;
    }
    if (!sd.active) return;
    switch (which) {
        case IMP_RULE_AM_BEGIN: hsb_am_begin_rule(sd, L.neq); break;
        case IMP_RULE_AM_ITER_PRED:
        case IMP_RULE_AM_ITER_CORR:
            if (sd.it_active) hsb_am_iter_rule(sd, L.abs_err, L.rel_err, L.neq, which == IMP_RULE_AM_ITER_PRED ? 0 : 1);
            break;
        case IMP_RULE_AM_PRED_END:
        case IMP_RULE_AM_CORR_END:
            if (!(sd.it_flags & 4)) hsb_am_phase_rule(sd, which == IMP_RULE_AM_PRED_END ? 0 : 1, L.neq);
            break;
        case IMP_RULE_AM_FINAL: {
            const bool nf = sd.nonfinite != 0u;
            sd.nonfinite = 0u;
            hsb_am_final_rule(sd, L.abs_err, L.rel_err, L.neq, nf);
            break;
        }
        case IMP_RULE_BDF_BEGIN:
            sd.eq = L.eq;
            sd.it_active = 1;
            sd.it_count = 0;
            sd.rhs_due = 0;
            for (int c = 0; c < 10; c++) sd.red[c] = 0u;
            break;
        case IMP_RULE_BDF_ITER:
            if (sd.it_active) hsb_bdf_iter_rule(sd, L.max_iter_err, L.max_iter);
            break;
        default: break;
    }
}

// The LLBar equation's second-order local relaxation terms at one cell, added to k (the
// torque and zero-order relaxation already in it), for m and the cell's effective field H:
//   llbar-local02nc.cu:11-73:  gamma diag(mu_par) (m . H) m
//   llbar-local02c.cu:11-69:   gamma cross(diag(mu_perp) cross(m, H), m) with the reference's
//                              cross(a, b) = b x a (common_func.h:52-55): gamma m x (mu_perp (H x m))
// Host and device share this code.
__host__ __device__ inline void hsb_llbar02(const float* m, const float* H, float g, const float* mu_par,
                                            const float* mu_perp, float* k) {
    const float mH = m[0] * H[0] + m[1] * H[1] + m[2] * H[2];
    // a = mu_perp (H x m)
    const float a0 = mu_perp[0] * (H[1] * m[2] - H[2] * m[1]);
    const float a1 = mu_perp[1] * (H[2] * m[0] - H[0] * m[2]);
    const float a2 = mu_perp[2] * (H[0] * m[1] - H[1] * m[0]);
    k[0] += g * (mu_par[0] * mH * m[0] + (m[1] * a2 - m[2] * a1));
    k[1] += g * (mu_par[1] * mH * m[1] + (m[2] * a0 - m[0] * a2));
    k[2] += g * (mu_par[2] * mH * m[2] + (m[0] * a1 - m[1] * a0));
}

// One cell of a fixed-point sweep (k_imp_sweep; host builds drive it cell by cell).
// am12 (modes IMP_AM_*): the iterate is formed in FP64 from the FP32 state y0 and derivatives,
// compared in FP64 with the previous iterate's FP64 copy (w64, or the raw predictor up64 in the
// corrector's first sweep), so the sweep errors carry no FP32 rounding of the iterates; the raw
// iterate goes to up64 / uc64, the renormalised one (m, when `normalize`) to w64 and, rounded,
// to w for the next right-hand side.  IMP_AM_EULER forms the explicit Euler point that way; the
// step-error mode compares uc64 with up64 (scale |up64|) and writes nothing.  bdf-euler
// (IMP_BDF_*): FP32 throughout on the channels [c0, c1) of one equation, scale |prev + new|.
// dmax / smax fold max|prev - new| and the error scale per channel.
template <int CH>
__host__ __device__ inline void hsb_imp_sweep_cell(int mode, long i, long n, double dt, int c0, int c1,
                                                   int normalize, const float* y0, float* w, const float* prev,
                                                   const float* dy, const float* k0, double* w64,
                                                   const double* prev64, double* u64, const double* up64,
                                                   const double* uc64, float* dmax, float* smax, bool& bad) {
    if (mode == IMP_AM_ERR) {
        for (int c = 0; c < CH; c++) {
            const double a = uc64[c * n + i], b = up64[c * n + i];
            dmax[c] = fmaxf(dmax[c], (float)fabs(a - b));
            smax[c] = fmaxf(smax[c], (float)fabs(b));
            bad |= !isfinite(a - b);
        }
        return;
    }
    if (mode == IMP_AM_PRED || mode == IMP_AM_CORR || mode == IMP_AM_EULER) {
        double nv[CH];
        for (int c = 0; c < CH; c++) {
            const double b = (double)y0[c * n + i];
            if (mode == IMP_AM_CORR)
                nv[c] = b + (0.5 * dt) * ((double)dy[c * n + i] + (double)k0[c * n + i]);
            else if (mode == IMP_AM_PRED)
                nv[c] = b + dt * (double)dy[c * n + i];
            else
                nv[c] = b + dt * (double)k0[c * n + i];
            bad |= !isfinite(nv[c]);
        }
        if (mode != IMP_AM_EULER) {
            for (int c = 0; c < CH; c++) {
                const double pv = prev64[c * n + i];
                dmax[c] = fmaxf(dmax[c], (float)fabs(pv - nv[c]));
                smax[c] = fmaxf(smax[c], (float)fabs(nv[c]));
            }
            for (int c = 0; c < CH; c++) u64[c * n + i] = nv[c];
        }
        // the reference renormalises m when it next updates it (before the next right-hand side)
        if (normalize) {
            const double l2 = nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2];
            const double inv = (l2 == 0.0) ? 0.0 : 1.0 / sqrt(l2);
            nv[0] *= inv;
            nv[1] *= inv;
            nv[2] *= inv;
        }
        for (int c = 0; c < CH; c++) {
            w64[c * n + i] = nv[c];
            w[c * n + i] = (float)nv[c];
        }
        return;
    }
    const float fdt = (float)dt;
    float nv[CH];
    for (int c = 0; c < CH; c++) {
        nv[c] = 0.f;
        if (c < c0 || c >= c1) continue;
        nv[c] = y0[c * n + i] + fdt * k0[c * n + i];
        bad |= !isfinite(nv[c]);
    }
    if (mode == IMP_BDF_SWEEP) {
        for (int c = c0; c < c1; c++) {
            const float pv = prev[c * n + i];
            dmax[c] = fmaxf(dmax[c], fabsf(pv - nv[c]));
            smax[c] = fmaxf(smax[c], fabsf(pv + nv[c]));
        }
    }
    if (normalize && c0 == 0) {
        const float l2 = nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2];
#ifdef __CUDA_ARCH__
        const float inv = (l2 == 0.f) ? 0.f : rsqrtf(l2);
#else
        const float inv = (l2 == 0.f) ? 0.f : 1.0f / sqrtf(l2);
#endif
        nv[0] *= inv;
        nv[1] *= inv;
        nv[2] *= inv;
    }
    for (int c = c0; c < c1; c++) w[c * n + i] = nv[c];
}
