// Fused LLBar / LLB / two-temperature right-hand side and Runge-Kutta stage update.
//
// One thread per cell evaluates, in registers, everything hotspin computes with a chain of
// separate kernels and host syncs per right-hand side (engine/quant.go:417-445 walking the
// updaters of the modules below):
//   H_eff = H_ex (exchange6.cu:11-127) + H_anis (uniaxialanisotropy.cu:12-52)
//         + B_ext/mu0 (mod_zeeman.go) + H_demag (input) + H_lf (long_field.cu:13-72)
//         + H_therm (temperature.cu:14-70 on Philox normals)
//   dm/dt = gamma (m x H) + gamma diag(lambda) H   (llbar-torque.cu computes cross(H, M)
//           with the reference's cross helper, which evaluates m x H; llbar-local00nc.cu)
//   dTe/dt = (ke lap Te + G (Tl - Te) + Q_laser) / (gamma_e Te),
//   dTl/dt = (kl lap Tl + G (Te - Tl)) / Cl       (Qspat.cu, Qinter.cu, div.cu, mod_ce.go)
// and then performs the stage arithmetic of the integrator (store k_s, form the next stage
// point / the new state, renormalise m, accumulate the error norm).  Storage is FP32 SoA
// [channel][a0][a1][a2]; the error norm is a max-norm (exact in any precision).
#include <math.h>
#include <string.h>

#include "hsb_common.cuh"
#include "hsb_llg.cuh"
#include "hsb_philox.cuh"
#include "hsb_rhs.cuh"

__device__ __forceinline__ float* resolve(const PtrSel& s, const HsbSolverDev* sd) {
    switch (s.sel) {
        case SEL_CUR: return s.p[sd->cur];
        case SEL_NEXT: return s.p[1 - sd->cur];
        case SEL_K1: return s.p[sd->kslot];
        case SEL_K7: return s.p[1 - sd->kslot];
        default: return s.p[0];
    }
}

__device__ __forceinline__ void atomic_max_nonneg(unsigned int* a, float v) {
    atomicMax(a, __float_as_uint(v));
}

// Per-equation absolute error of one cell (err_abs mode, hotspin's rk12 estimate
// dt max |k1 - k0|): eeq[0] over the three m components, eeq[1], eeq[2] for Te, Tl.
template <int CH, int W = 1>
__device__ __forceinline__ void err_abs_cell(const float (&e)[CH], float fdt, float (&eeq)[3], bool& bad) {
    float em = fmaxf(fabsf(e[0]), fmaxf(fabsf(e[1]), fabsf(e[2]))) * fdt;
    if (!(e[0] == e[0]) || !(e[1] == e[1]) || !(e[2] == e[2])) bad = true;
    eeq[0] = fmaxf(eeq[0], em);
#pragma unroll
    for (int c = 3; c < CH; c++) {
        const float ec = fabsf(e[c]) * fdt;
        if (!(ec == ec)) bad = true;
        eeq[c - 2] = fmaxf(eeq[c - 2], ec);
    }
}

// Warp maxima of the per-equation errors into the solver word.
template <int CH>
__device__ __forceinline__ void err_abs_store(float (&eeq)[3], HsbSolverDev* sd) {
#pragma unroll
    for (int q = 0; q < 3; q++) {
        const float v = warp_max_f(eeq[q]);
        if ((threadIdx.x & 31) == 0 && (q == 0 || q + 2 < CH)) atomic_max_nonneg(&sd->err_eq[q], v);
    }
}

template <int CH>
__global__ void __launch_bounds__(256) k_stage(const HsbPhys P, const StageArgs A, HsbSolverDev* sd) {
    if (!A.ungated && !hsb_gate(sd, A.gate_word)) return;
    const double t = sd->t;
    const double dt = sd->dt;
    const long long step = sd->step;
    const float* ys = resolve(A.ys, sd);
    const float* hd = resolve(A.hd, sd);
    const float* yth = resolve(A.ytherm, sd);
    float* kout = resolve(A.kout, sd);
    const float* kacc = resolve(A.kacc, sd);
    float* ynext = resolve(A.ynext, sd);
    const float* ybase = resolve(A.ybase, sd);
    const float* yerr0 = resolve(A.yerr0, sd);
    const float* kin[HSB_MAXK];
#pragma unroll
    for (int j = 0; j < HSB_MAXK; j++) kin[j] = (j < A.nk || A.err) ? resolve(A.kin[j], sd) : nullptr;
    const double ts = t + (double)A.tfrac * dt;
    const float fdt = (float)dt;
    const long n = P.ncell;
    float emax = 0.f;
    float eeq[3] = {0.f, 0.f, 0.f};
    bool bad = false;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int a2 = (int)(i % P.N2);
        const long r = i / P.N2;
        const int a1 = (int)(r % P.N1);
        const int a0 = (int)(r / P.N1);
        float y[CH], k[CH];
        rhs_cell<CH>(P, ys, hd, yth, ts, dt, step, a0, a1, a2, i, y, k, A.torque_only != 0, A.heff_out);
        if (A.heff_out) continue;
        if (kout) {
#pragma unroll
            for (int c = 0; c < CH; c++) {
                float v = A.kself_w * k[c];
                if (kacc) v += A.kacc_w * __ldg(kacc + c * n + i);
                kout[c * n + i] = v;
            }
        }
        if (ynext) {
            float acc[CH];
#pragma unroll
            for (int c = 0; c < CH; c++) acc[c] = A.cself * k[c];
#pragma unroll
            for (int j = 0; j < HSB_MAXK; j++) {
                if (j < A.nk && A.ck[j] != 0.f) {
#pragma unroll
                    for (int c = 0; c < CH; c++) acc[c] += A.ck[j] * __ldg(kin[j] + c * n + i);
                }
            }
            float out[CH];
#pragma unroll
            for (int c = 0; c < CH; c++) out[c] = __ldg(ybase + c * n + i) + fdt * acc[c];
            if (A.normalize) {
                const float l2 = out[0] * out[0] + out[1] * out[1] + out[2] * out[2];
                const float inv = (l2 == 0.f) ? 0.f : rsqrtf(l2);
                out[0] *= inv;
                out[1] *= inv;
                out[2] *= inv;
            }
#pragma unroll
            for (int c = 0; c < CH; c++) {
                ynext[c * n + i] = out[c];
                bad |= !isfinite(out[c]);
            }
        }
        if (A.err) {
            float e[CH];
#pragma unroll
            for (int c = 0; c < CH; c++) e[c] = A.ceself * k[c];
#pragma unroll
            for (int j = 0; j < HSB_MAXK; j++) {
                if (A.ce[j] != 0.f) {
#pragma unroll
                    for (int c = 0; c < CH; c++) e[c] += A.ce[j] * __ldg(kin[j] + c * n + i);
                }
            }
            if (A.err_abs) {
                err_abs_cell<CH>(e, fdt, eeq, bad);
            } else {
                float em = fmaxf(fabsf(e[0]), fmaxf(fabsf(e[1]), fabsf(e[2]))) * fdt / A.rtol;
#pragma unroll
                for (int c = 3; c < CH; c++) {
                    const float sc = A.rtol * fmaxf(fabsf(__ldg(yerr0 + c * n + i)), fabsf(y[c]));
                    const float ec = fabsf(e[c]) * fdt;
                    em = fmaxf(em, sc > 0.f ? ec / sc : (ec > 0.f ? INFINITY : 0.f));
                }
                if (!(em == em)) bad = true;   // NaN
                emax = fmaxf(emax, em);
            }
        }
    }
    if (A.err) {
        if (A.err_abs) {
            err_abs_store<CH>(eeq, sd);
        } else {
            emax = warp_max_f(emax);
            if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&sd->err_acc, emax);
        }
    }
    if (bad) atomicOr(&sd->nonfinite, 1u);
}

// ------------------------------------------------------------------ 4-cell vector variant
// Same arithmetic as k_stage, four consecutive cells along a2 per thread with 16-byte loads
// and stores (N2 % 4 == 0, no per-cell masks).  Neighbours along a0/a1 are float4 loads of
// the adjacent rows; along a2 the two outer neighbours are scalar loads (L1 hits).
__device__ __forceinline__ float4 ld4(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ void st4(float* p, const float v[4]) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void un4(float4 a, float v[4]) {
    v[0] = a.x;
    v[1] = a.y;
    v[2] = a.z;
    v[3] = a.w;
}

__device__ __forceinline__ float* resolve_off(const PtrSel& s, const HsbSolverDev* sd, long off) {
    float* p = resolve(s, sd);
    return p ? p + off : nullptr;
}

template <int CH, bool BATCH>
__global__ void __launch_bounds__(256, 2) k_stage4(const __grid_constant__ HsbPhys P0, const StageArgs A,
                                                   HsbSolverDev* sd0, const BatchArgs Bt) {
    const int slot = BATCH ? (int)blockIdx.z : 0;
    HsbSolverDev* sd = sd0 + slot;
    if (!A.ungated && !(A.prep_gated ? sd->prep : hsb_gate(sd, A.gate_word))) return;
    const HsbPhys& P = BATCH ? Bt.phys[slot] : P0;
    const long off = BATCH ? (long)slot * Bt.stride : 0;
    const int normalize = BATCH ? (A.normalize && P.normalize) : A.normalize;
    const double t = sd->t;
    const double dt = sd->dt;
    const long long step = sd->step;
    const float* ys = resolve_off(A.ys, sd, off);
    const float* hd = resolve_off(A.hd, sd, off);
    const float* yth = resolve_off(A.ytherm, sd, off);
    float* kout = resolve_off(A.kout, sd, off);
    const float* kacc = resolve_off(A.kacc, sd, off);
    float* ynext = resolve_off(A.ynext, sd, off);
    const float* ybase = resolve_off(A.ybase, sd, off);
    const float* yerr0 = resolve_off(A.yerr0, sd, off);
    const double ts = t + (double)A.tfrac * dt;
    const float fdt = (float)dt;
    const long n = P.ncell;
    const long s1 = P.N2, s0 = (long)P.N1 * P.N2;
    const long ngroups = n >> 2;
    // per-launch constants
    const double dte = dt > P.cutoff_dt ? dt : P.cutoff_dt;
    const float th_amp = (float)(P.th_pre / dte);
    const float laser_t = (CH >= 5) ? hsb_laser_power(P, ts) : 0.f;
    float hb[3];
    hsb_bext(P, ts, hb);
    float emax = 0.f;
    float eeq[3] = {0.f, 0.f, 0.f};
    bool bad = false;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < ngroups; g += (long)gridDim.x * blockDim.x) {
        const long i = g << 2;
        const int a2 = (int)(i % P.N2);
        const long r = i / P.N2;
        const int a1 = (int)(r % P.N1);
        const int a0 = (int)(r / P.N1);
        float y[CH][4];
#pragma unroll
        for (int c = 0; c < CH; c++) un4(ld4(ys + c * n + i), y[c]);
        float H[3][4];
        if (hd) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float h[4];
                un4(ld4(hd + c * n + i), h);
#pragma unroll
                for (int q = 0; q < 4; q++) H[c][q] = h[q] + hb[c];
            }
        } else {
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int q = 0; q < 4; q++) H[c][q] = hb[c];
        }
        float lapE[4] = {0.f, 0.f, 0.f, 0.f}, lapL[4] = {0.f, 0.f, 0.f, 0.f};
        // ---- a0 / a1 neighbours: whole float4 rows
#pragma unroll
        for (int d = 0; d < 2; d++) {
            const int me = d == 0 ? a0 : a1;
            const int nn = d == 0 ? P.N0 : P.N1;
            const int wr = d == 0 ? P.pbc0 : P.pbc1;
            const long st = d == 0 ? s0 : s1;
            const long im = i + (long)(nb_lo(me, nn, wr) - me) * st;
            const long ip = i + (long)(nb_hi(me, nn, wr) - me) * st;
            const float cx = P.ex_c[d];
            if (cx != 0.f) {
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    float lo[4], hi[4];
                    un4(ld4(ys + c * n + im), lo);
                    un4(ld4(ys + c * n + ip), hi);
#pragma unroll
                    for (int q = 0; q < 4; q++) H[c][q] += cx * ((lo[q] + hi[q]) - (y[c][q] + y[c][q]));
                }
            }
            if (CH >= 5) {
                if (P.ke_c[d] != 0.f) {
                    float lo[4], hi[4];
                    un4(ld4(ys + 3 * n + im), lo);
                    un4(ld4(ys + 3 * n + ip), hi);
#pragma unroll
                    for (int q = 0; q < 4; q++) lapE[q] += P.ke_c[d] * ((lo[q] + hi[q]) - (y[3][q] + y[3][q]));
                }
                if (P.kl_c[d] != 0.f) {
                    float lo[4], hi[4];
                    un4(ld4(ys + 4 * n + im), lo);
                    un4(ld4(ys + 4 * n + ip), hi);
#pragma unroll
                    for (int q = 0; q < 4; q++) lapL[q] += P.kl_c[d] * ((lo[q] + hi[q]) - (y[4][q] + y[4][q]));
                }
            }
        }
        // ---- a2 neighbours: inside the vector plus one scalar on each side
        {
            const long il = i + (long)(nb_lo(a2, P.N2, P.pbc2) - a2);
            const long ir = (i + 3) + (long)(nb_hi(a2 + 3, P.N2, P.pbc2) - (a2 + 3));
            const int nst = CH >= 5 ? 5 : 3;
#pragma unroll
            for (int c = 0; c < nst; c++) {
                const float cx = c < 3 ? P.ex_c[2] : (c == 3 ? P.ke_c[2] : P.kl_c[2]);
                if (cx == 0.f) continue;
                const float l = __ldg(ys + c * n + il), rr = __ldg(ys + c * n + ir);
                float v[4];
                v[0] = cx * ((l + y[c][1]) - (y[c][0] + y[c][0]));
                v[1] = cx * ((y[c][0] + y[c][2]) - (y[c][1] + y[c][1]));
                v[2] = cx * ((y[c][1] + y[c][3]) - (y[c][2] + y[c][2]));
                v[3] = cx * ((y[c][2] + rr) - (y[c][3] + y[c][3]));
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    if (c < 3) H[c][q] += v[q];
                    else if (c == 3) lapE[q] += v[q];
                    else lapL[q] += v[q];
                }
            }
        }
        float thT[4] = {P.T_uniform, P.T_uniform, P.T_uniform, P.T_uniform};
        if (CH >= 5 && P.thermal) un4(ld4(yth + 3 * n + i), thT);
        float k[CH][4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const float mx = y[0][q], my = y[1][q], mz = y[2][q];
            float hx = H[0][q], hy = H[1][q], hz = H[2][q];
            if (P.ku_pre != 0.f) {
                const float mu = mx * P.uhat[0] + my * P.uhat[1] + mz * P.uhat[2];
                hx += P.ku_pre * mu * P.u[0];
                hy += P.ku_pre * mu * P.u[1];
                hz += P.ku_pre * mu * P.u[2];
            }
            const float Ts = (CH >= 5) ? y[3][q] : P.T_uniform;
            if (P.llb) {
                const float am = sqrtf(mx * mx + my * my + mz * mz);
                if (am > 1e-30f && Ts > 0.f) {
                    const float b = P.lf_b / Ts;
                    float W, dW;
                    mfa_w(P, am * b, W, dW);
                    const float mult = P.lf_pre * Ts * (W - am) / dW / am;
                    hx += mult * mx;
                    hy += mult * my;
                    hz += mult * mz;
                }
            }
            if (P.thermal && thT[q] > 0.f) {
                const float amp = sqrtf(th_amp * thT[q]);
                float gg[3];
                philox_normals3((uint32_t)(i + q), (uint64_t)step, P.seed_lo, P.seed_hi, gg);
                hx += amp * sqrtf(P.lam[0]) * gg[0];
                hy += amp * sqrtf(P.lam[1]) * gg[1];
                hz += amp * sqrtf(P.lam[2]) * gg[2];
            }
            const float gm = P.gamma;
            k[0][q] = gm * (-hy * mz + hz * my) + gm * P.lam[0] * hx;
            k[1][q] = gm * (-hz * mx + hx * mz) + gm * P.lam[1] * hy;
            k[2][q] = gm * (-hx * my + hy * mx) + gm * P.lam[2] * hz;
            if (CH >= 5) {
                const float Te = y[3][q], Tl = y[4][q];
                float Qe = lapE[q] + P.g_ep * (Tl - Te);
                if (laser_t != 0.f) {
                    float q2 = laser_t;
                    if (P.laser_inv2s2 != 0.f) {
                        const float yy = ((float)a1 + 0.5f - 0.5f * (float)P.N1) * P.cs1;
                        const float xx = ((float)(a2 + q) + 0.5f - 0.5f * (float)P.N2) * P.cs2;
                        q2 *= expf(-(xx * xx + yy * yy) * P.laser_inv2s2);
                    }
                    Qe += q2;
                }
                const float Ce = P.gamma_e * Te;
                k[3][q] = (Ce == 0.f) ? 0.f : Qe / Ce;
                const float Ql = lapL[q] + P.g_ep * (Te - Tl);
                k[4][q] = (P.c_l == 0.f) ? 0.f : Ql / P.c_l;
            }
        }
        if (kout) {
#pragma unroll
            for (int c = 0; c < CH; c++) {
                float v[4];
#pragma unroll
                for (int q = 0; q < 4; q++) v[q] = A.kself_w * k[c][q];
                if (kacc) {
                    float a[4];
                    un4(ld4(kacc + c * n + i), a);
#pragma unroll
                    for (int q = 0; q < 4; q++) v[q] += A.kacc_w * a[q];
                }
                st4(kout + c * n + i, v);
            }
        }
        if (ynext) {
            float out[CH][4];
#pragma unroll
            for (int c = 0; c < CH; c++)
#pragma unroll
                for (int q = 0; q < 4; q++) out[c][q] = A.cself * k[c][q];
#pragma unroll
            for (int j = 0; j < HSB_MAXK; j++) {
                if (j < A.nk && A.ck[j] != 0.f) {
                    const float* kj = resolve_off(A.kin[j], sd, off);
#pragma unroll
                    for (int c = 0; c < CH; c++) {
                        float a[4];
                        un4(ld4(kj + c * n + i), a);
#pragma unroll
                        for (int q = 0; q < 4; q++) out[c][q] += A.ck[j] * a[q];
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < CH; c++) {
                float b[4];
                un4(ld4(ybase + c * n + i), b);
#pragma unroll
                for (int q = 0; q < 4; q++) out[c][q] = b[q] + fdt * out[c][q];
            }
            if (normalize) {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const float l2 = out[0][q] * out[0][q] + out[1][q] * out[1][q] + out[2][q] * out[2][q];
                    const float inv = (l2 == 0.f) ? 0.f : rsqrtf(l2);
                    out[0][q] *= inv;
                    out[1][q] *= inv;
                    out[2][q] *= inv;
                }
            }
#pragma unroll
            for (int c = 0; c < CH; c++) {
#pragma unroll
                for (int q = 0; q < 4; q++) bad |= !isfinite(out[c][q]);
                st4(ynext + c * n + i, out[c]);
            }
        }
        if (A.err) {
            float e[CH][4];
#pragma unroll
            for (int c = 0; c < CH; c++)
#pragma unroll
                for (int q = 0; q < 4; q++) e[c][q] = A.ceself * k[c][q];
#pragma unroll
            for (int j = 0; j < HSB_MAXK; j++) {
                if (A.ce[j] != 0.f) {
                    const float* kj = resolve_off(A.kin[j], sd, off);
#pragma unroll
                    for (int c = 0; c < CH; c++) {
                        float a[4];
                        un4(ld4(kj + c * n + i), a);
#pragma unroll
                        for (int q = 0; q < 4; q++) e[c][q] += A.ce[j] * a[q];
                    }
                }
            }
            if (A.err_abs) {
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    float ec[CH];
#pragma unroll
                    for (int c = 0; c < CH; c++) ec[c] = e[c][q];
                    err_abs_cell<CH>(ec, fdt, eeq, bad);
                }
            } else {
#pragma unroll
            for (int q = 0; q < 4; q++) {
                float em = fmaxf(fabsf(e[0][q]), fmaxf(fabsf(e[1][q]), fabsf(e[2][q]))) * fdt / A.rtol;
                if (!(em == em)) bad = true;
                emax = fmaxf(emax, em);
            }
            if (CH >= 5) {
#pragma unroll
                for (int c = 3; c < CH; c++) {
                    float y0v[4];
                    un4(ld4(yerr0 + c * n + i), y0v);
#pragma unroll
                    for (int q = 0; q < 4; q++) {
                        const float sc = A.rtol * fmaxf(fabsf(y0v[q]), fabsf(y[c][q]));
                        const float ec = fabsf(e[c][q]) * fdt;
                        const float em = sc > 0.f ? ec / sc : (ec > 0.f ? INFINITY : 0.f);
                        if (!(em == em)) bad = true;
                        emax = fmaxf(emax, em);
                    }
                }
            }
            }
        }
    }
    if (A.err) {
        if (A.err_abs) {
            err_abs_store<CH>(eeq, sd);
        } else {
            emax = warp_max_f(emax);
            if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&sd->err_acc, emax);
        }
    }
    if (bad) atomicOr(&sd->nonfinite, 1u);
}

// ------------------------------------------------------------------ load-first variant
// Same right-hand side as k_stage4 with W consecutive cells along a2 per thread, arranged so
// that a thread's global loads are issued back to back and consumed afterwards: (A) the
// stage derivatives the stage sums over (a compacted list of the nonzero coefficients, NK
// known at compile time) and the base state, (B) the state, its six neighbours and the demag
// field, all without data-dependent branches (an unused neighbour or field reads the cell
// itself and is discarded by a select).  Stores come last.  Two load round trips per cell
// instead of one per stage derivative and per stencil direction.  The stage combination is
// formed as (ybase + dt sum_j c_j k_j) + (dt c_s) k_s; the error estimate as
// (sum_j e_j k_j) + e_s k_s.
struct KList {
    PtrSel p[HSB_MAXK];
    float c[HSB_MAXK];
};

template <int W>
__device__ __forceinline__ void ldw(const float* p, float* v) {
    if (W == 4) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    } else if (W == 2) {
        const float2 a = __ldg(reinterpret_cast<const float2*>(p));
        v[0] = a.x; v[1] = a.y;
    } else {
        v[0] = __ldg(p);
    }
}
template <int W>
__device__ __forceinline__ void stw(float* p, const float* v) {
    if (W == 4) *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    else if (W == 2) *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    else *p = v[0];
}

template <int CH, bool BATCH, int W, int NK>
__global__ void __launch_bounds__(256, W == 1 ? 3 : (W == 2 ? 2 : 1))
    k_stagec(const __grid_constant__ HsbPhys P0, const StageArgs A, const KList KL, HsbSolverDev* sd0,
             const BatchArgs Bt) {
    const int slot = BATCH ? (int)blockIdx.z : 0;
    HsbSolverDev* sd = sd0 + slot;
    if (!A.ungated && !(A.prep_gated ? sd->prep : hsb_gate(sd, A.gate_word))) return;
    const HsbPhys& P = BATCH ? Bt.phys[slot] : P0;
    const long off = BATCH ? (long)slot * Bt.stride : 0;
    const int normalize = BATCH ? (A.normalize && P.normalize) : A.normalize;
    const double t = sd->t;
    const double dt = sd->dt;
    const long long step = sd->step;
    const float* ys = resolve_off(A.ys, sd, off);
    const float* hdp = resolve_off(A.hd, sd, off);
    const float* ythp = resolve_off(A.ytherm, sd, off);
    float* kout = resolve_off(A.kout, sd, off);
    const float* kaccp = resolve_off(A.kacc, sd, off);
    float* ynext = resolve_off(A.ynext, sd, off);
    const float* ybasep = resolve_off(A.ybase, sd, off);
    const float* yerr0p = resolve_off(A.yerr0, sd, off);
    const float* kl[NK > 0 ? NK : 1];
#pragma unroll
    for (int j = 0; j < NK; j++) kl[j] = resolve_off(KL.p[j], sd, off);
    // absent inputs read valid memory (the state) and are discarded
    const bool has_hd = hdp != nullptr, has_kacc = kaccp != nullptr;
    const bool form_y = ynext != nullptr;
    const bool form_e = !form_y && A.err;
    const float* hd = has_hd ? hdp : ys;
    const float* kacc = has_kacc ? kaccp : ys;
    const float* ybase = (form_y && ybasep) ? ybasep : ys;
    const float* yerr0 = yerr0p ? yerr0p : ys;
    const bool th_field = (CH >= 5) && P.thermal && ythp != nullptr;
    const float* yth = th_field ? ythp : ys;
    float* hth = resolve_off(A.hth, sd, off);
    const int hmode = hth ? A.hth_mode : 0;      // 0 generate, 1 generate + store, 2 load
    const double ts = t + (double)A.tfrac * dt;
    const float fdt = (float)dt;
    const long n = P.ncell;
    const long s1 = P.N2, s0 = (long)P.N1 * P.N2;
    const long ngroups = n / W;
    const double dte = dt > P.cutoff_dt ? dt : P.cutoff_dt;
    const float th_amp = (float)(P.th_pre / dte);
    const float laser_t = (CH >= 5) ? hsb_laser_power(P, ts) : 0.f;
    float hb[3];
    hsb_bext(P, ts, hb);
    float emax = 0.f;
    bool bad = false;
    const float dt_rtol = A.err ? fdt / A.rtol : 0.f;
    for (long g = blockIdx.x * (long)blockDim.x + threadIdx.x; g < ngroups; g += (long)gridDim.x * blockDim.x) {
        const long i = g * W;
        const unsigned iu = (unsigned)i;
        const unsigned ru = hsb_fastdiv(iu, P.div2_mul, P.div2_shr);
        const int a2 = (int)(iu - ru * (unsigned)P.N2);
        const unsigned a0u = hsb_fastdiv(ru, P.div1_mul, P.div1_shr);
        const int a1 = (int)(ru - a0u * (unsigned)P.N1);
        const int a0 = (int)a0u;
        // ---- (A) stage derivatives and base state
        float acc[CH][W];
        {
            float kv[NK > 0 ? NK : 1][CH][W];
#pragma unroll
            for (int j = 0; j < NK; j++)
#pragma unroll
                for (int c = 0; c < CH; c++) ldw<W>(kl[j] + c * n + i, kv[j][c]);
            float bv[CH][W];
#pragma unroll
            for (int c = 0; c < CH; c++) ldw<W>(ybase + c * n + i, bv[c]);
#pragma unroll
            for (int c = 0; c < CH; c++)
#pragma unroll
                for (int q = 0; q < W; q++) {
                    float sum = 0.f;
#pragma unroll
                    for (int j = 0; j < NK; j++) sum += KL.c[j] * kv[j][c][q];
                    acc[c][q] = form_y ? bv[c][q] + fdt * sum : sum;
                }
        }
        // ---- (B) state, neighbours, demag field
        float y[CH][W], H[3][W], lapE[W], lapL[W];
        float thT[W], hthv[3][W];
        {
            {
                // loaded unconditionally (the state's channels when there is no kept field,
                // then discarded) so the phase's loads carry no branch
                const float* hsrc = (hmode == 2) ? hth : ys;
#pragma unroll
                for (int c = 0; c < 3; c++) ldw<W>(hsrc + c * n + i, hthv[c]);
            }
            float hv[3][W], nb[4][CH][W], sl[CH], sr[CH];
#pragma unroll
            for (int c = 0; c < CH; c++) ldw<W>(ys + c * n + i, y[c]);
#pragma unroll
            for (int c = 0; c < 3; c++) ldw<W>(hd + c * n + i, hv[c]);
            long nidx[4];
            {
                const long im0 = i + (long)(nb_lo(a0, P.N0, P.pbc0) - a0) * s0;
                const long ip0 = i + (long)(nb_hi(a0, P.N0, P.pbc0) - a0) * s0;
                const long im1 = i + (long)(nb_lo(a1, P.N1, P.pbc1) - a1) * s1;
                const long ip1 = i + (long)(nb_hi(a1, P.N1, P.pbc1) - a1) * s1;
                nidx[0] = im0;
                nidx[1] = ip0;
                nidx[2] = im1;
                nidx[3] = ip1;
            }
#pragma unroll
            for (int d = 0; d < 4; d++)
#pragma unroll
                for (int c = 0; c < CH; c++) {
                    // temperature neighbours only where that diffusion term is on
                    const float kc = c < 3 ? 1.f : (c == 3 ? P.ke_c[d >> 1] : P.kl_c[d >> 1]);
                    const long ix = (c < 3 || kc != 0.f) ? nidx[d] : i;
                    ldw<W>(ys + c * n + ix, nb[d][c]);
                }
            const long il = i + (long)(nb_lo(a2, P.N2, P.pbc2) - a2);
            const long ir = (i + W - 1) + (long)(nb_hi(a2 + W - 1, P.N2, P.pbc2) - (a2 + W - 1));
#pragma unroll
            for (int c = 0; c < CH; c++) {
                sl[c] = __ldg(ys + c * n + il);
                sr[c] = __ldg(ys + c * n + ir);
            }
            if (CH >= 5) ldw<W>(yth + 3 * n + i, thT);   // yth is the state itself without a field
            // consume
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int q = 0; q < W; q++) H[c][q] = (has_hd ? hv[c][q] : 0.f) + hb[c];
#pragma unroll
            for (int q = 0; q < W; q++) lapE[q] = lapL[q] = 0.f;
#pragma unroll
            for (int dd = 0; dd < 2; dd++) {
                const float cx = P.ex_c[dd];
#pragma unroll
                for (int c = 0; c < 3; c++)
#pragma unroll
                    for (int q = 0; q < W; q++)
                        H[c][q] += cx * ((nb[2 * dd][c][q] + nb[2 * dd + 1][c][q]) - (y[c][q] + y[c][q]));
                if (CH >= 5) {
#pragma unroll
                    for (int q = 0; q < W; q++) {
                        lapE[q] += P.ke_c[dd] * ((nb[2 * dd][3][q] + nb[2 * dd + 1][3][q]) - (y[3][q] + y[3][q]));
                        lapL[q] += P.kl_c[dd] * ((nb[2 * dd][4 % CH][q] + nb[2 * dd + 1][4 % CH][q]) -
                                                 (y[4 % CH][q] + y[4 % CH][q]));
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < CH; c++) {
                const float cx = c < 3 ? P.ex_c[2] : (c == 3 ? P.ke_c[2] : P.kl_c[2]);
#pragma unroll
                for (int q = 0; q < W; q++) {
                    const float left = q == 0 ? sl[c] : y[c][q - 1];
                    const float right = q == W - 1 ? sr[c] : y[c][q + 1];
                    const float v = cx * ((left + right) - (y[c][q] + y[c][q]));
                    if (c < 3) H[c][q] += v;
                    else if (c == 3) lapE[q] += v;
                    else lapL[q] += v;
                }
            }
            if (!th_field) {
#pragma unroll
                for (int q = 0; q < W; q++) thT[q] = P.T_uniform;
            }
        }
        float k[CH][W];
#pragma unroll
        for (int q = 0; q < W; q++) {
            const float mx = y[0][q], my = y[1][q], mz = y[2][q];
            float hx = H[0][q], hy = H[1][q], hz = H[2][q];
            if (P.ku_pre != 0.f) {
                const float mu = mx * P.uhat[0] + my * P.uhat[1] + mz * P.uhat[2];
                hx += P.ku_pre * mu * P.u[0];
                hy += P.ku_pre * mu * P.u[1];
                hz += P.ku_pre * mu * P.u[2];
            }
            const float Ts = (CH >= 5) ? y[3 % CH][q] : P.T_uniform;
            if (P.llb) {
                const float am = sqrtf(mx * mx + my * my + mz * mz);
                if (am > 1e-30f && Ts > 0.f) {
                    const float mult = mfa_mult(P, am, Ts);
                    hx += mult * mx;
                    hy += mult * my;
                    hz += mult * mz;
                }
            }
            if (hmode == 2) {
                hx += hthv[0][q];
                hy += hthv[1][q];
                hz += hthv[2][q];
            } else {
                float t0 = 0.f, t1 = 0.f, t2 = 0.f;
                if (P.thermal && thT[q] > 0.f) {
                    const float amp = sqrtf(th_amp * thT[q]);
                    float gg[3];
                    philox_normals3((uint32_t)(i + q), (uint64_t)step, P.seed_lo, P.seed_hi, gg);
                    t0 = amp * sqrtf(P.lam[0]) * gg[0];
                    t1 = amp * sqrtf(P.lam[1]) * gg[1];
                    t2 = amp * sqrtf(P.lam[2]) * gg[2];
                }
                hx += t0;
                hy += t1;
                hz += t2;
                if (hmode == 1) {
                    hthv[0][q] = t0;
                    hthv[1][q] = t1;
                    hthv[2][q] = t2;
                }
            }
            const float gm = P.gamma;
            k[0][q] = gm * (-hy * mz + hz * my) + gm * P.lam[0] * hx;
            k[1][q] = gm * (-hz * mx + hx * mz) + gm * P.lam[1] * hy;
            k[2][q] = gm * (-hx * my + hy * mx) + gm * P.lam[2] * hz;
            if (CH >= 5) {
                const float Te = y[3 % CH][q], Tl = y[4 % CH][q];
                float Qe = lapE[q] + P.g_ep * (Tl - Te);
                if (laser_t != 0.f) {
                    float q2 = laser_t;
                    if (P.laser_inv2s2 != 0.f) {
                        const float yy = ((float)a1 + 0.5f - 0.5f * (float)P.N1) * P.cs1;
                        const float xx = ((float)(a2 + q) + 0.5f - 0.5f * (float)P.N2) * P.cs2;
                        q2 *= expf(-(xx * xx + yy * yy) * P.laser_inv2s2);
                    }
                    Qe += q2;
                }
                // heat capacities are ~1e4..1e7 J/(m^3 K): the fast reciprocal division applies
                const float Ce = P.gamma_e * Te;
                k[3 % CH][q] = (Ce == 0.f) ? 0.f : __fdividef(Qe, Ce);
                const float Ql = lapL[q] + P.g_ep * (Te - Tl);
                k[4 % CH][q] = (P.c_l == 0.f) ? 0.f : __fdividef(Ql, P.c_l);
            }
        }
        // ---- stores and the error norm
        if (hmode == 1) {
#pragma unroll
            for (int c = 0; c < 3; c++) stw<W>(hth + c * n + i, hthv[c]);
        }
        if (kout) {
#pragma unroll
            for (int c = 0; c < CH; c++) {
                float v[W];
#pragma unroll
                for (int q = 0; q < W; q++) v[q] = A.kself_w * k[c][q];
                if (has_kacc) {   // RK4's accumulated stage sum, read only where it exists
                    float ka[W];
                    ldw<W>(kacc + c * n + i, ka);
#pragma unroll
                    for (int q = 0; q < W; q++) v[q] += A.kacc_w * ka[q];
                }
                stw<W>(kout + c * n + i, v);
            }
        }
        if (form_y) {
            const float cs = fdt * A.cself;
#pragma unroll
            for (int c = 0; c < CH; c++)
#pragma unroll
                for (int q = 0; q < W; q++) acc[c][q] += cs * k[c][q];
            if (normalize) {
#pragma unroll
                for (int q = 0; q < W; q++) {
                    const float l2 = acc[0][q] * acc[0][q] + acc[1][q] * acc[1][q] + acc[2][q] * acc[2][q];
                    const float inv = (l2 == 0.f) ? 0.f : rsqrtf(l2);
                    acc[0][q] *= inv;
                    acc[1][q] *= inv;
                    acc[2][q] *= inv;
                }
            }
#pragma unroll
            for (int c = 0; c < CH; c++) {
#pragma unroll
                for (int q = 0; q < W; q++) bad |= !isfinite(acc[c][q]);
                stw<W>(ynext + c * n + i, acc[c]);
            }
        } else if (form_e) {
#pragma unroll
            for (int c = 0; c < CH; c++)
#pragma unroll
                for (int q = 0; q < W; q++) acc[c][q] += A.ceself * k[c][q];
#pragma unroll
            for (int q = 0; q < W; q++) {
                float em = fmaxf(fabsf(acc[0][q]), fmaxf(fabsf(acc[1][q]), fabsf(acc[2][q]))) * dt_rtol;
                if (!(em == em)) bad = true;
                emax = fmaxf(emax, em);
            }
            if (CH >= 5) {
#pragma unroll
                for (int c = 3; c < CH; c++) {
                    float ye[W];
                    ldw<W>(yerr0 + c * n + i, ye);
#pragma unroll
                    for (int q = 0; q < W; q++) {
                        const float sc = A.rtol * fmaxf(fabsf(ye[q]), fabsf(y[c][q]));
                        const float ec = fabsf(acc[c][q]) * fdt;
                        const float em = sc > 0.f ? __fdividef(ec, sc) : (ec > 0.f ? INFINITY : 0.f);
                        if (!(em == em)) bad = true;
                        emax = fmaxf(emax, em);
                    }
                }
            }
        }
    }
    if (A.err) {
        emax = warp_max_f(emax);
        if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&sd->err_acc, emax);
    }
    if (bad) atomicOr(&sd->nonfinite, 1u);
}

// Next stage point / new state without a right-hand-side evaluation:
// ynext = ybase + dt * sum_j ck[j] kin[j] (renormalised in LLG mode).
template <int CH, bool BATCH>
__global__ void __launch_bounds__(256) k_combine(const __grid_constant__ HsbPhys P0, const StageArgs A,
                                                 HsbSolverDev* sd0, const BatchArgs Bt) {
    const int slot = BATCH ? (int)blockIdx.z : 0;
    HsbSolverDev* sd = sd0 + slot;
    if (!sd->active) return;
    const HsbPhys& P = BATCH ? Bt.phys[slot] : P0;
    const long off = BATCH ? (long)slot * Bt.stride : 0;
    const float fdt = (float)sd->dt;
    const long n = P.ncell;
    float* ynext = resolve_off(A.ynext, sd, off);
    const float* ybase = resolve_off(A.ybase, sd, off);
    const float* kin[HSB_MAXK];
#pragma unroll
    for (int j = 0; j < HSB_MAXK; j++) kin[j] = (j < A.nk) ? resolve_off(A.kin[j], sd, off) : nullptr;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        float out[CH];
#pragma unroll
        for (int c = 0; c < CH; c++) {
            float acc = 0.f;
#pragma unroll
            for (int j = 0; j < HSB_MAXK; j++)
                if (j < A.nk && A.ck[j] != 0.f) acc += A.ck[j] * __ldg(kin[j] + c * n + i);
            out[c] = __ldg(ybase + c * n + i) + fdt * acc;
        }
        if (BATCH ? (A.normalize && P.normalize) : A.normalize) {
            const float l2 = out[0] * out[0] + out[1] * out[1] + out[2] * out[2];
            const float inv = (l2 == 0.f) ? 0.f : rsqrtf(l2);
            out[0] *= inv;
            out[1] *= inv;
            out[2] *= inv;
        }
#pragma unroll
        for (int c = 0; c < CH; c++) ynext[c * n + i] = out[c];
    }
}

// Dormand-Prince step-size control, one thread per slot (hsb_dp45_rule in hsb_llg.cuh).
// Consumes the attempt's error maximum.
__global__ void k_dp45_control(HsbSolverDev* sd0, int nslot) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nslot) return;
    HsbSolverDev* sd = sd0 + slot;
    if (!sd->active) return;
    const float ef = __uint_as_float(sd->err_acc);
    const unsigned int nf = sd->nonfinite;
    sd->err_acc = 0u;
    sd->nonfinite = 0u;
    hsb_dp45_rule(*sd, ef, nf != 0u);
}

// hotspin's adaptive Heun (rk12) step control, one thread per slot: consumes the attempt's
// per-equation errors (hsb_rk12_rule in hsb_llg.cuh).
struct Rk12Limits {
    double maxerr[3];
    int neq;
};

__global__ void k_rk12_control(HsbSolverDev* sd0, int nslot, const Rk12Limits lim) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nslot) return;
    HsbSolverDev* sd = sd0 + slot;
    if (!sd->active) return;
    float err[3];
    for (int q = 0; q < 3; q++) {
        err[q] = __uint_as_float(sd->err_eq[q]);
        sd->err_eq[q] = 0u;
    }
    const bool nf = sd->nonfinite != 0u;
    sd->nonfinite = 0u;
    hsb_rk12_rule(*sd, err, lim.maxerr, lim.neq, nf);
}

int hsb_launch_rk12_control(HsbSolverDev* sd, int nslot, const double* maxerr, int neq, cudaStream_t st) {
    Rk12Limits lim;
    for (int q = 0; q < 3; q++) lim.maxerr[q] = maxerr[q];
    lim.neq = neq;
    k_rk12_control<<<(nslot + 31) / 32, 32, 0, st>>>(sd, nslot, lim);
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}

// Fixed-step bookkeeping: t += dt, step++, swap state buffers, stop at the target.
__global__ void k_fixed_advance(HsbSolverDev* sd0, int nslot) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nslot) return;
    HsbSolverDev* sd = sd0 + slot;
    if (!sd->active) return;
    sd->t += sd->dt;
    sd->step += 1;
    sd->cur = 1 - sd->cur;
    sd->attempts += 1;
    if (sd->nonfinite) {     // consumed, as the adaptive controllers consume it
        sd->status |= 1;
        sd->active = 0;
        sd->nonfinite = 0u;
    }
    if (sd->step_stop >= 0 && sd->step >= sd->step_stop) sd->active = 0;
    if (sd->t_stop > 0.0 && sd->t_stop - sd->t <= 1e-6 * sd->dt) sd->active = 0;
}

// ------------------------------------------------------------------------------ launchers
// Stage-kernel variant for grids without masks: 0 = k_stage4, 1 / 2 / 4 = k_stagec with 1 / 2 /
// 4 cells per thread (the load-first form).  Each simulation passes the variant its tuning
// picked (hsb_sim.cu); hsb_set_stage_variant forces one for every launch (tuning sweeps), -1
// returns to the per-simulation choice.
static int g_stage_force = -1;
static const int STAGE_DEFAULT = 2;

static int stage_variant(int requested) {
    if (g_stage_force >= 0) return g_stage_force;
    return requested >= 0 ? requested : STAGE_DEFAULT;
}

HSB_EXPORT int hsb_set_stage_variant(int v) {
    const int old = g_stage_force;
    if (v == -1 || v == 0 || v == 1 || v == 2 || v == 4) g_stage_force = v;
    return old;
}

template <int CH, bool BATCH, int W>
static void launch_c(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, const BatchArgs& Bt, int nslot,
                     cudaStream_t st) {
    // compacted list of the stage derivatives the launch sums over, nonzero coefficients only
    KList KL;
    memset(&KL, 0, sizeof(KL));
    const bool form_y = A.ynext.p[0] || A.ynext.p[1];
    int nk = 0;
    for (int j = 0; j < HSB_MAXK; j++) {
        const float c = form_y ? (j < A.nk ? A.ck[j] : 0.f) : (A.err ? A.ce[j] : 0.f);
        if (c != 0.f) {
            KL.p[nk] = A.kin[j];
            KL.c[nk] = c;
            nk++;
        }
    }
    const int threads = 256;
    const int per_sm = W == 1 ? 3 : (W == 2 ? 2 : 1);
    long g = (P.ncell / W + threads - 1) / threads;
    const long cap = (long)hsb_sm_count() * per_sm;
    dim3 grid((unsigned)(g < cap ? g : cap), 1, (unsigned)nslot);
    switch (nk) {
#define KC(m) case m: k_stagec<CH, BATCH, W, m><<<grid, threads, 0, st>>>(P, A, KL, sd, Bt); break;
        KC(0) KC(1) KC(2) KC(3) KC(4) KC(5) KC(6) KC(7)
#undef KC
    }
}

template <int CH, bool BATCH>
static void launch_vec(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, const BatchArgs& Bt, int nslot,
                       cudaStream_t st, int variant) {
    // the load-first kernel forms either the next state or the DP45 error norm: launches that
    // need both, or the per-equation absolute errors, take the four-cell kernel
    const int v = (A.err && (A.ynext.p[0] || A.ynext.p[1] || A.err_abs)) ? 0 : stage_variant(variant);
    if (v == 0) {
        const int threads = 256;
        long g = (P.ncell / 4 + threads - 1) / threads;
        const long cap = (long)hsb_sm_count() * 2;
        dim3 grid((unsigned)(g < cap ? g : cap), 1, (unsigned)nslot);
        k_stage4<CH, BATCH><<<grid, threads, 0, st>>>(P, A, sd, Bt);
    } else if (v == 1) {
        launch_c<CH, BATCH, 1>(P, A, sd, Bt, nslot, st);
    } else if (v == 2) {
        launch_c<CH, BATCH, 2>(P, A, sd, Bt, nslot, st);
    } else {
        launch_c<CH, BATCH, 4>(P, A, sd, Bt, nslot, st);
    }
}

bool hsb_stage_tunable(const HsbPhys& P);

// True when stage launches of this simulation run the load-first kernel, which is the one
// that can keep the step's thermal field (StageArgs.hth_mode).
bool hsb_stage_keeps_thermal(const HsbPhys& P, int variant) {
    return hsb_stage_tunable(P) && stage_variant(variant) != 0;
}

// True when the stage launches of this geometry can take a variant (no masks, no second-order
// relaxation terms, a2 % 4 == 0); otherwise every stage runs the generic per-cell kernel.
bool hsb_stage_tunable(const HsbPhys& P) {
    return P.N2 % 4 == 0 && !P.msat_mask && !P.lex_mask && !P.llbar02 && !P.nonlocal;
}

int hsb_launch_stage_generic(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, cudaStream_t st);

int hsb_launch_stage(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, cudaStream_t st, int variant) {
    if (hsb_stage_tunable(P)) {
        BatchArgs nb = {0, nullptr, 1};
        if (P.nch == 5) launch_vec<5, false>(P, A, sd, nb, 1, st, variant);
        else launch_vec<3, false>(P, A, sd, nb, 1, st, variant);
        return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
    }
    return hsb_launch_stage_generic(P, A, sd, st);
}

// The generic per-cell kernel whatever the geometry (state queries such as the torque).  With
// the non-local relaxation term a first launch of the same kernel stores every cell's effective
// field, which the second reads at the neighbours.
int hsb_launch_stage_generic(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, cudaStream_t st) {
    const int threads = 256;
    const int grid = hsb_grid_1d(P.ncell, threads, 8);
    if (P.nonlocal && !A.torque_only) {
        if (!P.hbuf) return HSB_ERR_INVALID;
        StageArgs Hp = A;
        Hp.heff_out = P.hbuf;
        if (P.nch == 5) k_stage<5><<<grid, threads, 0, st>>>(P, Hp, sd);
        else k_stage<3><<<grid, threads, 0, st>>>(P, Hp, sd);
    }
    if (P.nch == 5) k_stage<5><<<grid, threads, 0, st>>>(P, A, sd);
    else k_stage<3><<<grid, threads, 0, st>>>(P, A, sd);
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}

int hsb_launch_combine(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, cudaStream_t st) {
    const int threads = 256;
    const int grid = hsb_grid_1d(P.ncell, threads, 8);
    BatchArgs nb = {0, nullptr, 1};
    if (P.nch == 5) k_combine<5, false><<<grid, threads, 0, st>>>(P, A, sd, nb);
    else k_combine<3, false><<<grid, threads, 0, st>>>(P, A, sd, nb);
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}

int hsb_launch_dp45_control(HsbSolverDev* sd, cudaStream_t st) {
    k_dp45_control<<<1, 1, 0, st>>>(sd, 1);
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}

// Batched variants: one grid plane per slot (blockIdx.z); Bt.phys / sd are slot arrays.
// P carries the class-wide geometry (size, channels; masks are not supported in batches).
int hsb_launch_stage_batched(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, const BatchArgs& Bt,
                             cudaStream_t st, int variant) {
    if (P.N2 % 4 != 0 || P.msat_mask || P.lex_mask || P.llbar02 || P.nonlocal) return HSB_ERR_UNSUPPORTED;
    if (P.nch == 5) launch_vec<5, true>(P, A, sd, Bt, Bt.nslot, st, variant);
    else launch_vec<3, true>(P, A, sd, Bt, Bt.nslot, st, variant);
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}

int hsb_launch_combine_batched(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, const BatchArgs& Bt,
                               cudaStream_t st) {
    const int threads = 256;
    long g = (P.ncell + threads - 1) / threads;
    const long cap = (long)hsb_sm_count() * 4;
    dim3 grid((unsigned)(g < cap ? g : cap), 1, (unsigned)Bt.nslot);
    if (P.nch == 5) k_combine<5, true><<<grid, threads, 0, st>>>(P, A, sd, Bt);
    else k_combine<3, true><<<grid, threads, 0, st>>>(P, A, sd, Bt);
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}

int hsb_launch_dp45_control_batched(HsbSolverDev* sd, int nslot, cudaStream_t st) {
    k_dp45_control<<<(nslot + 31) / 32, 32, 0, st>>>(sd, nslot);
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}

// Slots whose preparation just ran start stepping.
__global__ void k_activate_prepped(HsbSolverDev* sd0, int nslot) {
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nslot) return;
    HsbSolverDev* sd = sd0 + slot;
    if (sd->prep) {
        sd->prep = 0;
        sd->active = 1;
    }
}

int hsb_launch_fixed_advance_batched(HsbSolverDev* sd, int nslot, cudaStream_t st) {
    k_fixed_advance<<<(nslot + 31) / 32, 32, 0, st>>>(sd, nslot);
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}

int hsb_launch_activate_prepped(HsbSolverDev* sd, int nslot, cudaStream_t st) {
    k_activate_prepped<<<(nslot + 31) / 32, 32, 0, st>>>(sd, nslot);
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}

int hsb_launch_fixed_advance(HsbSolverDev* sd, cudaStream_t st) {
    k_fixed_advance<<<1, 1, 0, st>>>(sd, 1);
    return cudaGetLastError() == cudaSuccess ? HSB_OK : HSB_ERR_CUDA;
}
