// The simulation descriptor as the library compiles it (the layout of hsb_sim_desc in
// include/hotspin_b200.h, field for field) and the FP32 / FP64 physics parameters of the
// stage kernels derived from it.  Host code: the handle (hsb_sim.cu) and host builds of the
// per-cell right-hand side (tests/native/rule_check.cu) share it.
#pragma once
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "hsb_llg.cuh"

static const double MU0 = 4.0e-7 * M_PI;
static const double KB = 1.38064881313131313e-23;

struct hsb_sim_desc {
    int32_t size[3];
    int32_t pbc[3];
    double cellsize[3];
    double msat0T0, lex, gamma_ll;
    double alpha[3];
    double ku;
    double anis_u[3];
    double b_ext[3];
    int32_t demag, normalize, llb;
    double tc, spin_j, n_spins, temperature;
    int32_t thermal;
    uint64_t seed;
    double cutoff_dt;
    int32_t ttm;
    double gamma_e, c_l, g_ep, k_e, k_l;
    double laser_p0, laser_t0, laser_fwhm, laser_sigma;
    int32_t solver;
    double dt, rtol, mindt, maxdt;
    const double* laser_table;   // 2 x laser_npts (t, factor); copied at creation
    int32_t laser_npts;
    const double* bext_table;    // 4 x bext_npts (t, Bx, By, Bz); copied at creation
    int32_t bext_npts;
    double maxerr[3];            // rk12: maxError; am12: maxAbsError; bdf-euler: maxIterError (m, Te, Tl)
    double maxrelerr[3];         // am12: maxRelError (m, Te, Tl)
    int32_t max_iter;            // bdf-euler: sweeps per equation
    int32_t demag_tensor;        // 0 Kernel_Arne, 1 Newell
    double mu_par[3];            // llbar/damping/nonconservative/02/local (0: not loaded)
    double mu_perp[3];           // llbar/damping/conservative/02/local (0: not loaded)
    double alpha_e[3];           // llbar/damping/nonconservative/00/nonlocal (0: not loaded)
};

inline bool has_llbar02(const hsb_sim_desc& d) {
    for (int a = 0; a < 3; a++)
        if (d.mu_par[a] != 0.0 || d.mu_perp[a] != 0.0) return true;
    return false;
}
inline bool has_nonlocal(const hsb_sim_desc& d) {
    return d.alpha_e[0] != 0.0 || d.alpha_e[1] != 0.0 || d.alpha_e[2] != 0.0;
}

// FP32 physics of one simulation (device table pointers, masks and hbuf left null).
inline void phys_from_desc(const hsb_sim_desc& d, int nch, long ncell, HsbPhys& P) {
    memset(&P, 0, sizeof(P));
    P.N0 = d.size[0];
    P.N1 = d.size[1];
    P.N2 = d.size[2];
    P.pbc0 = d.pbc[0];
    P.pbc1 = d.pbc[1];
    P.pbc2 = d.pbc[2];
    P.nch = nch;
    P.ncell = ncell;
    for (int a = 0; a < 3; a++) {
        P.ex_c[a] = (float)(d.msat0T0 * d.lex * d.lex / (d.cellsize[a] * d.cellsize[a]));
        P.lam[a] = (float)d.alpha[a];
        P.bext[a] = (float)(d.b_ext[a] / MU0);
        P.u[a] = (float)d.anis_u[a];
        P.ke_c[a] = (float)(d.k_e / (d.cellsize[a] * d.cellsize[a]));
        P.kl_c[a] = (float)(d.k_l / (d.cellsize[a] * d.cellsize[a]));
    }
    const double ul = sqrt(d.anis_u[0] * d.anis_u[0] + d.anis_u[1] * d.anis_u[1] + d.anis_u[2] * d.anis_u[2]);
    for (int a = 0; a < 3; a++) P.uhat[a] = ul > 0 ? (float)(d.anis_u[a] / ul) : 0.f;
    P.gamma = (float)d.gamma_ll;
    P.ku_pre = (float)(2.0 * d.ku / (MU0 * d.msat0T0));
    P.demag = d.demag;
    P.llb = d.llb;
    const double S_ = d.spin_j;
    const bool lang = S_ > 1.0e5;
    P.lf_langevin = lang;
    P.lf_pre = (float)(d.n_spins * KB / (MU0 * d.msat0T0));
    P.lf_b = (float)(3.0 * (lang ? 1.0 : S_ / (S_ + 1.0)) * d.tc);
    if (!lang && S_ > 0) {
        const double lpre = 1.0 / (2.0 * S_), gpre = (2.0 * S_ + 1.0) * lpre;
        P.lf_gpre = (float)gpre;
        P.lf_lpre = (float)lpre;
        P.lf_lim = (float)fmin(0.2 / gpre, 0.2 / lpre);
    }
    P.T_uniform = (float)d.temperature;
    P.thermal = d.thermal;
    P.seed_lo = (uint32_t)(d.seed & 0xFFFFFFFFu);
    P.seed_hi = (uint32_t)(d.seed >> 32);
    const double V = d.cellsize[0] * d.cellsize[1] * d.cellsize[2];
    P.th_pre = 2.0 * KB / (MU0 * V * d.gamma_ll * d.msat0T0);
    P.cutoff_dt = d.cutoff_dt;
    P.ttm = d.ttm;
    P.g_ep = (float)d.g_ep;
    P.gamma_e = (float)d.gamma_e;
    P.c_l = (float)d.c_l;
    P.laser_p0 = (float)d.laser_p0;
    P.laser_t0 = (float)d.laser_t0;
    P.laser_c = d.laser_fwhm > 0 ? (float)(4.0 * log(2.0) / (d.laser_fwhm * d.laser_fwhm)) : 0.f;
    P.laser_inv2s2 = d.laser_sigma > 0 ? (float)(1.0 / (2.0 * d.laser_sigma * d.laser_sigma)) : 0.f;
    P.cs1 = (float)d.cellsize[1];
    P.cs2 = (float)d.cellsize[2];
    P.normalize = d.normalize;
    P.ms0 = (float)d.msat0T0;
    P.llbar02 = has_llbar02(d) ? 1 : 0;
    P.nonlocal = has_nonlocal(d) ? 1 : 0;
    for (int a = 0; a < 3; a++) {
        P.mu_par[a] = (float)d.mu_par[a];
        P.mu_perp[a] = (float)d.mu_perp[a];
        P.lam_e[a] = (float)d.alpha_e[a];
        P.inv_cs2[a] = (float)(1.0 / (d.cellsize[a] * d.cellsize[a]));
    }
    hsb_fastdiv_init((unsigned)P.N2, &P.div2_mul, &P.div2_shr);
    hsb_fastdiv_init((unsigned)P.N1, &P.div1_mul, &P.div1_shr);
}
