// Host build of the device step-control rules (test support, compiled by the CPU tests with
// nvcc as host code): the same inline functions the controller kernels run, driven from
// Python through ctypes so the rules can be checked against the oracle without a GPU.
#include "hsb_desc.h"
#include "hsb_fft4.cuh"
#include "hsb_llg.cuh"
#include "hsb_rhs.cuh"

// One rk12 attempt on a fresh solver word.  out: dt_new, accepted (0/1), status, tries,
// active, err.
extern "C" void rk12_rule_host(double dt, double mindt, double maxdt, int tries, const float* err,
                               const double* maxerr, int neq, int nonfinite, double* out) {
    HsbSolverDev sd = {};
    sd.dt = dt;
    sd.mindt = mindt;
    sd.maxdt = maxdt;
    sd.tries = tries;
    sd.active = 1;
    sd.step_stop = -1;
    hsb_rk12_rule(sd, err, maxerr, neq, nonfinite != 0);
    out[0] = sd.dt;
    out[1] = (double)sd.step;
    out[2] = (double)sd.status;
    out[3] = (double)sd.tries;
    out[4] = (double)sd.active;
    out[5] = sd.err;
}

// ---- a solver word on the host, for step-by-step emulation of the implicit solvers' kernel
// sequences (tests/test_control_rules.py)
#include <string>

extern "C" HsbSolverDev* hsd_new(void) {
    HsbSolverDev* p = new HsbSolverDev();
    memset(p, 0, sizeof(*p));
    p->active = 1;
    p->step_stop = -1;
    return p;
}
extern "C" void hsd_free(HsbSolverDev* p) { delete p; }

#define HSD_FIELDS(X)                                                                           \
    X(t) X(dt) X(step) X(attempts) X(rejects) X(cur) X(active) X(status) X(err) X(mindt) X(maxdt) \
    X(t_stop) X(step_stop) X(tries) X(it_active) X(it_count) X(it_flags) X(aborts) X(dysel)        \
    X(prevsel) X(eq) X(rhs_due) X(alpha_max) X(nonfinite) X(kslot)

// hsb_dp45_rule (the DP45 controller kernel's rule) on a host solver word.
extern "C" void dp45_rule_host(HsbSolverDev* p, float err, int nonfinite) { hsb_dp45_rule(*p, err, nonfinite != 0); }

extern "C" double hsd_get(const HsbSolverDev* p, const char* name) {
    const std::string n(name);
#define X(f) if (n == #f) return (double)p->f;
    HSD_FIELDS(X)
#undef X
    if (n.size() == 3 && n[0] == 'e' && n[1] == 'r') return p->er[n[2] - '0'];
    if (n.size() == 6 && n.compare(0, 5, "alpha") == 0) return p->alpha[n[5] - '0'];
    return NAN;
}
extern "C" void hsd_set(HsbSolverDev* p, const char* name, double v) {
    const std::string n(name);
#define X(f) if (n == #f) { p->f = (decltype(p->f))v; return; }
    HSD_FIELDS(X)
#undef X
}
// red[c] = max(red[c], v) as the sweep kernels' atomics do (v >= 0 as float bits)
extern "C" void hsd_fold(HsbSolverDev* p, int c, float v) {
    unsigned int b;
    memcpy(&b, &v, 4);
    if (v > 0.f && b > p->red[c]) p->red[c] = b;
}
extern "C" void imp_rule_host(HsbSolverDev* p, int which, const double* abs_err, const double* rel_err,
                              double max_iter_err, int max_iter, int neq, int eq) {
    ImpLimits L;
    memset(&L, 0, sizeof(L));
    for (int q = 0; q < 3; q++) {
        L.abs_err[q] = abs_err[q];
        L.rel_err[q] = rel_err[q];
    }
    L.max_iter_err = max_iter_err;
    L.max_iter = max_iter;
    L.neq = neq;
    L.eq = eq;
    hsb_imp_rule(*p, L, which);
}

// ---- the Newell tensor's shared arithmetic (hsb_newell.cuh), for the oracle comparison
#include "hsb_newell.cuh"

extern "C" void newell_host(int i, int j, const double* R, const double* cs, double* out3) {
    out3[0] = newell_exact(i, j, R, cs);
    out3[1] = newell_asymptotic(i, j, R, cs);
    out3[2] = newell_N(i, j, R, cs);
}

// The folded K = -N of a logic grid (program order) as k_newell_kernel computes it:
// Kc[6][h0+1][h1+1][h2+1].
extern "C" void newell_kernel_host(const int* L, const int* pbc, const double* cs, double* Kc) {
    ArneGeom g;
    for (int a = 0; a < 3; a++) {
        g.size[a] = L[a];
        g.cs[a] = cs[a];
        g.h[a] = L[a] / 2;
        if (pbc[a] == 0) {
            g.r1[a] = -(long)((L[a] - 1) / 2);
            g.r2[a] = (long)((L[a] - 1) / 2);
        } else {
            g.r1[a] = -((long)L[a] * pbc[a] - 1);
            g.r2[a] = (long)L[a] * pbc[a] - 1;
        }
    }
    if (L[2] == 1 && pbc[2] == 0) g.r2[2] = 0;
    const long n1 = g.h[1] + 1, n2 = g.h[2] + 1, ncell = (g.h[0] + 1) * n1 * n2;
    const int full[3][3] = {{KXX, KXY, KXZ}, {KXY, KYY, KYZ}, {KXZ, KYZ, KZZ}};
    for (long q = 0; q < 3 * ncell; q++) {
        const int s = (int)(q / ncell);
        const long c = q - s * ncell;
        double acc[3];
        newell_target(g, s, (int)(c / (n1 * n2)), (int)((c / n2) % n1), (int)(c % n2), acc);
        for (int d = s; d < 3; d++) Kc[(long)full[s][d] * ncell + c] = acc[d];
    }
}

// ---- Kernel_Arne's quadrature split over the lanes of a warp (hsb_arne.cuh)
#include "hsb_arne.cuh"

// The folded Kernel_Arne tensor Kc[6][h0+1][h1+1][h2+1] of a logic grid with every target's
// quadrature split into `nparts` shares that are summed afterwards, as k_arne_kernel's lanes do.
extern "C" void arne_kernel_host(const int* L, const int* pbc, const double* cs, int accuracy, int nparts,
                                 double* Kc) {
    ArneGeom g;
    for (int a = 0; a < 3; a++) {
        g.size[a] = L[a];
        g.cs[a] = cs[a];
        g.h[a] = L[a] / 2;
        if (pbc[a] == 0) {
            g.r1[a] = -(long)((L[a] - 1) / 2);
            g.r2[a] = (long)((L[a] - 1) / 2);
        } else {
            g.r1[a] = -((long)L[a] * pbc[a] - 1);
            g.r2[a] = (long)L[a] * pbc[a] - 1;
        }
    }
    if (L[2] == 1 && pbc[2] == 0) g.r2[2] = 0;
    g.Lmin = fmin(cs[0], fmin(cs[1], cs[2]));
    g.accuracy = (double)accuracy;
    const long n1 = g.h[1] + 1, n2 = g.h[2] + 1, ncell = (g.h[0] + 1) * n1 * n2;
    const int full[3][3] = {{KXX, KXY, KXZ}, {KXY, KYY, KYZ}, {KXZ, KYZ, KZZ}};
    for (long q = 0; q < 3 * ncell; q++) {
        const int s = (int)(q / ncell);
        const long c = q - s * ncell;
        double acc[3] = {0, 0, 0};
        for (int part = 0; part < nparts; part++) {
            double p[3];
            arne_target_part(g, s, (int)(c / (n1 * n2)), (int)((c / n2) % n1), (int)(c % n2), part, nparts, p);
            for (int d = s; d < 3; d++) acc[d] += p[d];
        }
        for (int d = s; d < 3; d++) Kc[(long)full[s][d] * ncell + c] = acc[d];
    }
}

// ---- the LLBar second-order local relaxation terms of one cell (hsb_llbar02 in hsb_llg.cuh)
extern "C" void llbar02_host(const float* m, const float* H, float g, const float* mu_par, const float* mu_perp,
                             float* k) {
    k[0] = k[1] = k[2] = 0.f;
    hsb_llbar02(m, H, g, mu_par, mu_perp, k);
}

// ---- one fixed-point sweep over all cells with the kernel's own cell code (hsb_imp_sweep_cell)
extern "C" void imp_sweep_host(int ch, int mode, long n, double dt, int c0, int c1, int normalize, const float* y0,
                               float* w, const float* prev, const float* dy, const float* k0, double* w64,
                               const double* prev64, double* u64, const double* up64, const double* uc64, float* dmax,
                               float* smax, int* bad) {
    bool b = false;
    for (int c = 0; c < 5; c++) dmax[c] = smax[c] = 0.f;
    for (long i = 0; i < n; i++) {
        if (ch == 5)
            hsb_imp_sweep_cell<5>(mode, i, n, dt, c0, c1, normalize, y0, w, prev, dy, k0, w64, prev64, u64, up64, uc64,
                                  dmax, smax, b);
        else
            hsb_imp_sweep_cell<3>(mode, i, n, dt, c0, c1, normalize, y0, w, prev, dy, k0, w64, prev64, u64, up64, uc64,
                                  dmax, smax, b);
    }
    *bad = b ? 1 : 0;
}

// The generic stage kernel's per-cell right-hand side (rhs_cell) over every cell of a grid,
// with the physics the library derives from the descriptor (phys_from_desc).  Buffers are
// FP32 [channel][cell] as on the device: ys the state, hd the demag field (A/m, or null), yth
// the state whose Te sets the thermal amplitude; masks and tables optional (host copies).
// With the non-local relaxation term a first pass stores every cell's effective field in
// hbuf ([3][cell]), as the kernel's first launch does.  k: [channel][cell].
extern "C" void rhs_host(const hsb_sim_desc* d, const float* ys, const float* hd, const float* yth, double t,
                         double dt, long long step, const float* msat_mask, const float* lex_mask, float* hbuf,
                         float* k) {
    const int nch = d->ttm ? 5 : 3;
    const long n = (long)d->size[0] * d->size[1] * d->size[2];
    HsbPhys P;
    phys_from_desc(*d, nch, n, P);
    P.msat_mask = msat_mask;
    P.lex_mask = lex_mask;
    P.laser_tab = (const double2*)d->laser_table;
    P.laser_npts = d->laser_table ? d->laser_npts : 0;
    P.bext_tab = d->bext_table;
    P.bext_npts = d->bext_table ? d->bext_npts : 0;
    P.hbuf = hbuf;
    for (int pass = P.nonlocal ? 0 : 1; pass < 2; pass++) {
        for (long i = 0; i < n; i++) {
            const int a2 = (int)(i % P.N2);
            const long r = i / P.N2;
            const int a1 = (int)(r % P.N1);
            const int a0 = (int)(r / P.N1);
            float y[5], kk[5];
            float* hout = pass == 0 ? hbuf : nullptr;
            if (nch == 5) rhs_cell<5>(P, ys, hd, yth, t, dt, step, a0, a1, a2, i, y, kk, false, hout);
            else rhs_cell<3>(P, ys, hd, yth, t, dt, step, a0, a1, a2, i, y, kk, false, hout);
            if (pass == 1)
                for (int c = 0; c < nch; c++) k[c * n + i] = kk[c];
        }
    }
}

// The four-step register FFT of one sequence (fft4 in hsb_fft4.cuh) with its lanes run one
// after the other: every lane's first half (A-point FFT, twiddles, write to the shared slot),
// then every lane's second half (read back, B-point FFTs), as the warp does between its
// __syncwarp calls.  x and X interleaved (re, im), L points; tw4 the A x B twiddle matrix.
template <int L, int DIR, bool ZIN, bool HOUT>
static void fft4_run(const float* x, const float* tw, float* X) {
    constexpr int A = Split<L>::A, B = Split<L>::B;
    static float2 v[B][A];
    static float2 slot[Slot<L>::S];
    const float2* tw4 = (const float2*)tw;
    for (int t = 0; t < B; t++)
        for (int n1 = 0; n1 < A; n1++) v[t][n1] = make_float2(x[2 * (B * n1 + t)], x[2 * (B * n1 + t) + 1]);
    for (int t = 0; t < B; t++) fft4_first<L, DIR, ZIN>(v[t], slot, t, tw4);
    for (int t = 0; t < B; t++) fft4_second<L, DIR, HOUT>(v[t], slot, t);
    for (int t = 0; t < B; t++)
        for (int j = 0; j < A; j++) {
            const int k = fft4_out_index<L>(t, j);
            X[2 * k] = v[t][j].x;
            X[2 * k + 1] = v[t][j].y;
        }
}

template <int L>
static void fft4_dispatch(int dir, int zin, int hout, const float* x, const float* tw, float* X) {
    const int c = (dir > 0 ? 4 : 0) + (zin ? 2 : 0) + (hout ? 1 : 0);
    switch (c) {
        case 0: fft4_run<L, -1, false, false>(x, tw, X); break;
        case 1: fft4_run<L, -1, false, true>(x, tw, X); break;
        case 2: fft4_run<L, -1, true, false>(x, tw, X); break;
        case 3: fft4_run<L, -1, true, true>(x, tw, X); break;
        case 4: fft4_run<L, 1, false, false>(x, tw, X); break;
        case 5: fft4_run<L, 1, false, true>(x, tw, X); break;
        case 6: fft4_run<L, 1, true, false>(x, tw, X); break;
        default: fft4_run<L, 1, true, true>(x, tw, X); break;
    }
}

// Split<L>::B of a length (0 when fft4 has no such length).
extern "C" int fft4_lanes(int L) {
    switch (L) {
#define FB(N) case N: return Split<N>::B;
        FB(2) FB(4) FB(8) FB(16) FB(32) FB(64) FB(128) FB(256) FB(512) FB(1024) FB(2048)
#undef FB
        default: return 0;
    }
}

extern "C" int fft4_host(int L, int dir, int zin, int hout, const float* x, const float* tw, float* X) {
    switch (L) {
#define FD(N) case N: fft4_dispatch<N>(dir, zin, hout, x, tw, X); return 0;
        FD(2) FD(4) FD(8) FD(16) FD(32) FD(64) FD(128) FD(256) FD(512) FD(1024) FD(2048)
#undef FD
        default: return 1;
    }
}
