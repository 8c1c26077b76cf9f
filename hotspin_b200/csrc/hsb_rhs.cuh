// Per-cell right-hand side of the fused LLBar / LLB / two-temperature equations, shared by the
// generic stage kernel (hsb_llg.cu) and host builds that check it against the oracle
// (tests/native/rule_check.cu).  Device builds use the read-only load and fast-division
// intrinsics (HSB_LDG, HSB_FDIV); host builds their plain forms.
#pragma once
#include <math.h>

#include "hsb_common.cuh"
#include "hsb_llg.cuh"
#include "hsb_philox.cuh"

// B_J(x) and B_J'(x) (common_func.h:72-138): the reference's 4-term series below the linear
// range; above it the same functions in forms that stay accurate in FP32:
// B_1/2 = tanh x, B_1/2' = 1/cosh^2 x; B_J' = l^2/sinh^2(l x) - g^2/sinh^2(g x), which equals
// the reference's (g^2 - l^2) + l^2 coth^2(l x) - g^2 coth^2(g x) without its cancellation;
// Langevin L = coth x - 1/x, L' = 1/x^2 - 1/sinh^2 x.
__host__ __device__ __forceinline__ void mfa_w(const HsbPhys& P, float x, float& W, float& dW) {
    if (P.lf_langevin) {
        if (fabsf(x) < 0.2f) {
            const float x2 = x * x;
            W = x / 3.0f - x * x2 / 45.0f + x * x2 * x2 * 2.0f / 945.0f - x * x2 * x2 * x2 / 4725.0f;
            dW = 1.0f / 3.0f - x2 / 15.0f + x2 * x2 * 2.0f / 189.0f - x2 * x2 * x2 / 675.0f;
        } else {
            const float sh = sinhf(x);
            W = 1.0f / tanhf(x) - 1.0f / x;
            dW = 1.0f / (x * x) - 1.0f / (sh * sh);
        }
        return;
    }
    const float g = P.lf_gpre, l = P.lf_lpre;
    if (fabsf(x) < P.lf_lim) {
        const float g2 = g * g, l2 = l * l, g4 = g2 * g2, l4 = l2 * l2, g6 = g4 * g2, l6 = l4 * l2,
                    g8 = g4 * g4, l8 = l4 * l4, x2 = x * x;
        W = (g2 - l2) * x / 3.0f - (g4 - l4) * x * x2 / 45.0f + (g6 - l6) * x * x2 * x2 * 2.0f / 945.0f -
            (g8 - l8) * x * x2 * x2 * x2 / 4725.0f;
        dW = (g2 - l2) / 3.0f - (g4 - l4) * x2 / 15.0f + (g6 - l6) * x2 * x2 * 2.0f / 189.0f -
             (g8 - l8) * x2 * x2 * x2 / 675.0f;
    } else if (l == 1.0f && g == 2.0f) {
        const float c = coshf(x);
        W = tanhf(x);
        dW = 1.0f / (c * c);
    } else {
        const float sg = sinhf(g * x), sl = sinhf(l * x);
        W = g / tanhf(g * x) - l / tanhf(l * x);
        dW = (l * l) / (sl * sl) - (g * g) / (sg * sg);
    }
}

// The longitudinal-field multiplier n kB T (W(am b) - am) / (mu0 Ms0 W'(am b) am), b = lf_b / T.
// For J = 1/2 above the series range it uses e = expm1(-2x): tanh x = -e / (2 + e) and
// 1 / cosh^2 x = 4 (1 + e) / (2 + e)^2, the same values as mfa_w's forms with one
// transcendental instead of two; with d = 2 + e, (W - am) d^2 = -d (e + am d), so the
// multiplier is -pre T d (e + am d) / (4 (1 + e) am).  Both divisions use the fast reciprocal
// form: T > 0 is kelvin-sized, and the denominator leaves the normal range only where
// exp(-2x) underflows (x > 43), where the field is unbounded in any arithmetic.
__host__ __device__ __forceinline__ float mfa_mult(const HsbPhys& P, float am, float Ts) {
    const float x = am * HSB_FDIV(P.lf_b, Ts);
    if (!P.lf_langevin && P.lf_lpre == 1.0f && P.lf_gpre == 2.0f && fabsf(x) >= P.lf_lim) {
        const float e = expm1f(-2.0f * x);
        const float d = 2.0f + e;
        return HSB_FDIV(-P.lf_pre * Ts * d * (e + am * d), 4.0f * (1.0f + e) * am);
    }
    float W, dW;
    mfa_w(P, x, W, dW);
    return P.lf_pre * Ts * (W - am) / dW / am;
}

template <int CH>
__host__ __device__ __forceinline__ void load_ch(const float* __restrict__ y, long n, long i, float* v) {
#pragma unroll
    for (int c = 0; c < CH; c++) v[c] = HSB_LDG(y + c * n + i);
}

// Right-hand side at cell (a0, a1, a2) = index i.  k[0..2] = dm/dt, k[3], k[4] = dTe/dt, dTl/dt.
template <int CH>
__host__ __device__ __forceinline__ void rhs_cell(const HsbPhys& P, const float* __restrict__ ys,
                                         const float* __restrict__ hd, const float* __restrict__ yth,
                                         double t, double dt, long long step, int a0, int a1, int a2,
                                         long i, float* y, float* k, bool torque_only = false,
                                         float* hout = nullptr) {
    const long n = P.ncell;
    const long s1 = P.N2, s0 = (long)P.N1 * P.N2;
    load_ch<CH>(ys, n, i, y);
    const float ms = P.msat_mask ? HSB_LDG(P.msat_mask + i) : 1.0f;
    float H[3] = {0.f, 0.f, 0.f};
    // ---- exchange (6 neighbours, clamp / wrap)
    {
        const float l0 = P.lex_mask ? HSB_LDG(P.lex_mask + i) : 1.0f;
        const float l02 = l0 * l0;
        const int lo[3] = {nb_lo(a0, P.N0, P.pbc0), nb_lo(a1, P.N1, P.pbc1), nb_lo(a2, P.N2, P.pbc2)};
        const int hi[3] = {nb_hi(a0, P.N0, P.pbc0), nb_hi(a1, P.N1, P.pbc1), nb_hi(a2, P.N2, P.pbc2)};
        const int me[3] = {a0, a1, a2};
        const long st[3] = {s0, s1, 1};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if (P.ex_c[d] == 0.f) continue;
            const long im = i + (long)(lo[d] - me[d]) * st[d];
            const long ip = i + (long)(hi[d] - me[d]) * st[d];
            float w1 = 1.f, w2 = 1.f;
            if (P.lex_mask) {
                const float lm = HSB_LDG(P.lex_mask + im), lp = HSB_LDG(P.lex_mask + ip);
                w1 = harm0(l02, lm * lm);
                w2 = harm0(l02, lp * lp);
            }
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float fm = HSB_LDG(ys + c * n + im), fp = HSB_LDG(ys + c * n + ip);
                H[c] += P.ex_c[d] * ((w1 * fm + w2 * fp) - (w1 * y[c] + w2 * y[c]));
            }
        }
    }
    // ---- uniaxial anisotropy
    if (P.ku_pre != 0.f && ms != 0.f) {
        const float pre = P.ku_pre / ms;
        const float mu = y[0] * P.uhat[0] + y[1] * P.uhat[1] + y[2] * P.uhat[2];
#pragma unroll
        for (int c = 0; c < 3; c++) H[c] += pre * mu * P.u[c];
    }
    // ---- demag + Zeeman
    if (hd) {
#pragma unroll
        for (int c = 0; c < 3; c++) H[c] += HSB_LDG(hd + c * n + i);
    }
    {
        float hb[3];
        hsb_bext(P, t, hb);
#pragma unroll
        for (int c = 0; c < 3; c++) H[c] += hb[c];
    }
    // ---- spin temperature
    float Ts = P.T_uniform;
    if (CH >= 5) Ts = y[3];
    // ---- MFA longitudinal field
    if (P.llb && ms != 0.f) {
        const float am = sqrtf(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]);
        if (am > 1e-30f && Ts > 0.f) {
            const float b = P.lf_b / Ts;
            float W, dW;
            mfa_w(P, am * b, W, dW);
            const float mult = P.lf_pre * Ts * (W - am) / (ms * dW);
            const float inv = 1.0f / am;
#pragma unroll
            for (int c = 0; c < 3; c++) H[c] += mult * y[c] * inv;
        }
    }
    // ---- thermal field: Philox normals of this cell and step, amplitude from the step start
    if (P.thermal && ms != 0.f) {
        float Tth = P.T_uniform;
        if (CH >= 5) Tth = HSB_LDG(yth + 3 * n + i);
        if (Tth > 0.f) {
            const double dte = dt > P.cutoff_dt ? dt : P.cutoff_dt;
            const float amp = sqrtf((float)(P.th_pre / dte) * Tth / ms);
            float g[3];
            philox_normals3((uint32_t)i, (uint64_t)step, P.seed_lo, P.seed_hi, g);
#pragma unroll
            for (int c = 0; c < 3; c++) H[c] += amp * sqrtf(P.lam[c]) * g[c];
        }
    }
    if (hout) {       // first pass of the non-local relaxation: the effective field only
#pragma unroll
        for (int c = 0; c < 3; c++) hout[c * n + i] = H[c];
        return;
    }
    // ---- LLBar torque cross(H, m) = m x H + zero-order local relaxation (zero in vacuum)
    if (ms == 0.f) {
        k[0] = k[1] = k[2] = 0.f;
    } else {
        const float g = P.gamma;
        const float r = torque_only ? 0.f : 1.f;
        k[0] = g * (-H[1] * y[2] + H[2] * y[1]) + r * g * P.lam[0] * H[0];
        k[1] = g * (-H[2] * y[0] + H[0] * y[2]) + r * g * P.lam[1] * H[1];
        k[2] = g * (-H[0] * y[1] + H[1] * y[0]) + r * g * P.lam[2] * H[2];
        if (P.llbar02 && !torque_only) hsb_llbar02(y, H, g, P.mu_par, P.mu_perp, k);
        // zero-order non-local relaxation -gamma alpha_e lap(H) with the stored fields of the
        // neighbours (llbar-nonlocal00nc.cu:11-205 with a uniform alpha_e: the harmonic means of
        // the cell's and each neighbour's alpha_e are alpha_e itself; clamp / wrap boundaries)
        if (P.nonlocal && !torque_only) {
            const int lo[3] = {nb_lo(a0, P.N0, P.pbc0), nb_lo(a1, P.N1, P.pbc1), nb_lo(a2, P.N2, P.pbc2)};
            const int hi[3] = {nb_hi(a0, P.N0, P.pbc0), nb_hi(a1, P.N1, P.pbc1), nb_hi(a2, P.N2, P.pbc2)};
            const int me[3] = {a0, a1, a2};
            const long st[3] = {s0, s1, 1};
            float lap[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const long im = i + (long)(lo[d] - me[d]) * st[d];
                const long ip = i + (long)(hi[d] - me[d]) * st[d];
#pragma unroll
                for (int c = 0; c < 3; c++)
                    lap[c] += P.inv_cs2[d] * ((P.hbuf[c * n + im] + P.hbuf[c * n + ip]) - (H[c] + H[c]));
            }
#pragma unroll
            for (int c = 0; c < 3; c++) k[c] -= g * P.lam_e[c] * lap[c];
        }
    }
    // ---- two-temperature model
    if (CH >= 5) {
        const float Te = y[3], Tl = y[4];
        float lapE = 0.f, lapL = 0.f;
        const int lo[3] = {nb_lo(a0, P.N0, P.pbc0), nb_lo(a1, P.N1, P.pbc1), nb_lo(a2, P.N2, P.pbc2)};
        const int hi[3] = {nb_hi(a0, P.N0, P.pbc0), nb_hi(a1, P.N1, P.pbc1), nb_hi(a2, P.N2, P.pbc2)};
        const int me[3] = {a0, a1, a2};
        const long st[3] = {s0, s1, 1};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const long im = i + (long)(lo[d] - me[d]) * st[d];
            const long ip = i + (long)(hi[d] - me[d]) * st[d];
            if (P.ke_c[d] != 0.f) lapE += P.ke_c[d] * ((HSB_LDG(ys + 3 * n + im) + HSB_LDG(ys + 3 * n + ip)) - (Te + Te));
            if (P.kl_c[d] != 0.f) lapL += P.kl_c[d] * ((HSB_LDG(ys + 4 * n + im) + HSB_LDG(ys + 4 * n + ip)) - (Tl + Tl));
        }
        float Qe = lapE + P.g_ep * (Tl - Te);
        if (P.laser_p0 != 0.f) {
            float q = hsb_laser_power(P, t);
            if (P.laser_inv2s2 != 0.f) {
                const float yy = ((float)a1 + 0.5f - 0.5f * (float)P.N1) * P.cs1;
                const float xx = ((float)a2 + 0.5f - 0.5f * (float)P.N2) * P.cs2;
                q *= expf(-(xx * xx + yy * yy) * P.laser_inv2s2);
            }
            Qe += q;
        }
        const float Ce = P.gamma_e * Te;
        k[3] = (Ce == 0.f) ? 0.f : Qe / Ce;
        const float Ql = lapL + P.g_ep * (Te - Tl);
        k[4] = (P.c_l == 0.f) ? 0.f : Ql / P.c_l;
    }
}
