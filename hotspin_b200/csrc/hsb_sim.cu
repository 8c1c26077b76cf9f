// Simulation handle: device-resident FP32 state, integrator sequencing, CUDA graphs.
//
// Replaces the per-step host sequencing of hotspin's engine (engine/engine.go:473-508,
// solve_euler.go, solve_heun.go, solve_rk12.go; the Quant.Update graph walk of
// engine/quant.go:417-445) for a fixed module set.  Each integrator step is a fixed
// sequence of kernels whose buffer choices and step-size decisions are resolved on the
// device (HsbSolverDev), so a run of steps is captured once into a CUDA graph and replayed
// with no host round trip; the host only checks completion between graph launches.
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "hsb_common.cuh"
#include "hsb_demag.h"
#include "hsb_llg.cuh"

int hsb_launch_stage(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, cudaStream_t st);
int hsb_launch_combine(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, cudaStream_t st);
int hsb_launch_dp45_control(HsbSolverDev* sd, cudaStream_t st);
int hsb_launch_fixed_advance(HsbSolverDev* sd, cudaStream_t st);

// Mirror of the public descriptor (include/hotspin_b200.h).
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
};

enum { SOLVER_EULER = 0, SOLVER_HEUN = 1, SOLVER_RK4 = 2, SOLVER_DP45 = 3 };

static const double MU0 = 4.0e-7 * M_PI;
static const double KB = 1.38064881313131313e-23;

// Dormand-Prince 5(4) tableau.
static const double DPA[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {1.0 / 5, 0, 0, 0, 0, 0},
    {3.0 / 40, 9.0 / 40, 0, 0, 0, 0},
    {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0, 0},
    {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0, 0},
    {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656, 0},
    {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}};
static const double DPC[7] = {0, 1.0 / 5, 3.0 / 10, 4.0 / 5, 8.0 / 9, 1, 1};
static const double DPE[7] = {71.0 / 57600, 0, -71.0 / 16695, 71.0 / 1920, -17253.0 / 339200, 22.0 / 525, -1.0 / 40};

struct hsb_sim_s {
    hsb_sim_desc d;
    HsbPhys P;
    int nch;
    long n;
    cudaStream_t st;
    hsb_demag_plan demag;
    float* y[2];        // state double buffer
    float* ystage[2];   // stage points (ping-pong: a kernel never reads and writes one)
    float* k[8];        // stage derivatives
    float* hd;          // demag field of the stage point
    float* hd01[2];     // demag field of y[0], y[1] (DP45 with a thermal field)
    float* msat_mask;
    float* lex_mask;
    HsbSolverDev* sd;   // device
    HsbSolverDev* sd_host;  // pinned mirror
    double* red;        // reduction scratch (device)
    double* red_host;   // pinned
    float* stage_f;     // device staging for FP64 <-> FP32 conversion
    double* stage_d;
    cudaGraphExec_t graph;
    int graph_steps;    // attempts captured in one graph launch
    bool initialized;   // k1 / hd01 of the current state computed (DP45)
    // eager profiling: events around every launch group of one attempt
    bool profiling;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof;  // category, start, stop
    int launches;       // kernel launches of one attempt (counted while enqueuing)
};

enum { PROF_STAGE = 0, PROF_XFWD = 1, PROF_YZ = 2, PROF_XINV = 3, PROF_OTHER = 4, PROF_NCAT = 5 };

static cudaEvent_t prof_event(hsb_sim_s* S) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    S->ev_pool.push_back(e);
    return e;
}

static PtrSel fixed(float* p) {
    PtrSel s;
    s.p[0] = p;
    s.p[1] = p;
    s.sel = SEL_FIXED;
    return s;
}
static PtrSel pair(float* a, float* b, int sel) {
    PtrSel s;
    s.p[0] = a;
    s.p[1] = b;
    s.sel = sel;
    return s;
}
static PtrSel none() { return fixed(nullptr); }

static StageArgs empty_args() {
    StageArgs A;
    memset(&A, 0, sizeof(A));
    A.ys = A.hd = A.ytherm = A.kout = A.kacc = A.ynext = A.ybase = A.yerr0 = none();
    for (int j = 0; j < HSB_MAXK; j++) A.kin[j] = none();
    A.rtol = 1.0f;
    return A;
}

// ------------------------------------------------------------------ conversion kernels
__global__ void k_d2f(const double* __restrict__ in, float* __restrict__ out, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] = (float)in[i];
}
__global__ void k_f2d(const float* __restrict__ in, double* __restrict__ out, long n) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        out[i] = (double)in[i];
}

#include "hsb_reduce.cuh"

// Energy-density terms (mod_energy.go:20-66): per cell, with ms = msat mask,
//   zeeman  -(m . Bext/mu0) ms          (times V mu0 Ms0)
//   exch    -0.5 (m . H_ex) ms          (times V mu0 Ms0)
//   demag   -0.5 (m . H_d) ms           (times V mu0 Ms0)
//   anis    -0.5 (m . H_anis) ms        (times V mu0 Ms0)
//   lf      -(m . H_lf) ms              (times V mu0 Ms0)
// plus sum of m (3) for the average.
__global__ void k_energy(const HsbPhys P, const float* __restrict__ y, const float* __restrict__ hd, int normalize,
                         double* partial, unsigned int* counter, double* out) {
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    double comp[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const long n = P.ncell;
    const long s1 = P.N2, s0 = (long)P.N1 * P.N2;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int a2 = (int)(i % P.N2);
        const long r = i / P.N2;
        const int a1 = (int)(r % P.N1);
        const int a0 = (int)(r / P.N1);
        float m[3] = {y[i], y[n + i], y[2 * n + i]};
        auto nrm = [&](float* a) {
            if (!normalize) return;
            float l2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
            float inv = l2 == 0.f ? 0.f : rsqrtf(l2);
            a[0] *= inv; a[1] *= inv; a[2] *= inv;
        };
        nrm(m);
        const float ms = P.msat_mask ? P.msat_mask[i] : 1.0f;
        double term[8];
        // exchange
        double hex[3] = {0, 0, 0};
        {
            const float l0 = P.lex_mask ? P.lex_mask[i] : 1.0f;
            const int lo[3] = {nb_lo(a0, P.N0, P.pbc0), nb_lo(a1, P.N1, P.pbc1), nb_lo(a2, P.N2, P.pbc2)};
            const int hi[3] = {nb_hi(a0, P.N0, P.pbc0), nb_hi(a1, P.N1, P.pbc1), nb_hi(a2, P.N2, P.pbc2)};
            const int me[3] = {a0, a1, a2};
            const long st[3] = {s0, s1, 1};
            for (int d = 0; d < 3; d++) {
                if (P.ex_c[d] == 0.f) continue;
                const long im = i + (long)(lo[d] - me[d]) * st[d];
                const long ip = i + (long)(hi[d] - me[d]) * st[d];
                float w1 = 1.f, w2 = 1.f;
                if (P.lex_mask) {
                    const float lm = P.lex_mask[im], lp = P.lex_mask[ip];
                    w1 = harm0(l0 * l0, lm * lm);
                    w2 = harm0(l0 * l0, lp * lp);
                }
                float mm[3] = {y[im], y[n + im], y[2 * n + im]};
                float mp[3] = {y[ip], y[n + ip], y[2 * n + ip]};
                nrm(mm);
                nrm(mp);
                for (int c = 0; c < 3; c++)
                    hex[c] += (double)P.ex_c[d] * ((w1 * mm[c] + w2 * mp[c]) - (w1 * m[c] + w2 * m[c]));
            }
        }
        term[0] = -(m[0] * (double)P.bext[0] + m[1] * (double)P.bext[1] + m[2] * (double)P.bext[2]) * ms;
        term[1] = -0.5 * (m[0] * hex[0] + m[1] * hex[1] + m[2] * hex[2]) * ms;
        term[2] = 0;
        if (hd) term[2] = -0.5 * (m[0] * (double)hd[i] + m[1] * (double)hd[n + i] + m[2] * (double)hd[2 * n + i]) * ms;
        term[3] = 0;
        if (P.ku_pre != 0.f && ms != 0.f) {
            const double mu = m[0] * (double)P.uhat[0] + m[1] * (double)P.uhat[1] + m[2] * (double)P.uhat[2];
            const double pre = (double)P.ku_pre / ms;
            term[3] = -0.5 * pre * mu * (m[0] * (double)P.u[0] + m[1] * (double)P.u[1] + m[2] * (double)P.u[2]) * ms;
        }
        term[4] = 0;
        if (P.llb && ms != 0.f) {
            const float Ts = (P.nch >= 5) ? y[3 * n + i] : P.T_uniform;
            const float am = sqrtf(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
            if (am > 1e-30f && Ts > 0.f) {
                const double b = (double)P.lf_b / Ts, x = am * b;
                double W, dW;
                if (P.lf_langevin) {
                    const double c = 1.0 / tanh(x);
                    W = c - 1.0 / x;
                    dW = 1.0 - c * c + 1.0 / (x * x);
                } else {
                    const double g = P.lf_gpre, l = P.lf_lpre;
                    const double cg = 1.0 / tanh(g * x), cl = 1.0 / tanh(l * x);
                    W = g * cg - l * cl;
                    dW = (g * g - l * l) + l * l * cl * cl - g * g * cg * cg;
                }
                const double mult = (double)P.lf_pre * Ts * (W - am) / (ms * dW);
                term[4] = -(mult * am) * ms;  // m . (mult m_hat) = mult |m|
            }
        }
        term[5] = m[0];
        term[6] = m[1];
        term[7] = m[2];
        for (int q = 0; q < 8; q++) {  // Kahan per thread
            double yv = term[q] - comp[q];
            double tv = v[q] + yv;
            comp[q] = (tv - v[q]) - yv;
            v[q] = tv;
        }
    }
    block_reduce_store<8>(v, partial, counter, out, gridDim.x);
}

// ------------------------------------------------------------------ helpers
static int set_sd_fields(hsb_sim_s* S) {
    HSB_CUDA_TRY(cudaMemcpyAsync(S->sd, S->sd_host, sizeof(HsbSolverDev), cudaMemcpyHostToDevice, S->st));
    return HSB_OK;
}
static int get_sd(hsb_sim_s* S) {
    HSB_CUDA_TRY(cudaMemcpyAsync(S->sd_host, S->sd, sizeof(HsbSolverDev), cudaMemcpyDeviceToHost, S->st));
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    return HSB_OK;
}

// Demag of one of the two state buffers (sel: -1 fixed pointer `m`, 0 = y[cur], 1 = y[next])
// into `h` (or into hd01[cur / next] when hsel >= 0).
static int run_demag(hsb_sim_s* S, const float* m, int msel, float* h, int hsel, bool gated = true) {
    if (!S->demag) return HSB_OK;
    HsbDemagIO io;
    if (msel < 0) {
        io.m[0] = io.m[1] = m;
        io.msel = nullptr;
        io.minv = 0;
    } else {
        io.m[0] = S->y[0];
        io.m[1] = S->y[1];
        io.msel = &S->sd->cur;
        io.minv = msel;
    }
    if (hsel < 0) {
        io.h[0] = io.h[1] = h;
        io.hsel = nullptr;
        io.hinv = 0;
    } else {
        io.h[0] = S->hd01[0];
        io.h[1] = S->hd01[1];
        io.hsel = &S->sd->cur;
        io.hinv = hsel;
    }
    io.ev = nullptr;
    cudaEvent_t ev[4];
    if (S->profiling) {
        for (int i = 0; i < 4; i++) ev[i] = prof_event(S);
        io.ev = ev;
    }
    S->launches += hsb_demag_nlaunch(S->demag);
    int rc = hsb_demag_launch(S->demag, io, S->msat_mask, (float)S->d.msat0T0, S->st,
                              gated ? &S->sd->active : nullptr);
    if (S->profiling) {
        S->prof.push_back({PROF_XFWD, {ev[0], ev[1]}});
        S->prof.push_back({PROF_YZ, {ev[1], ev[2]}});
        S->prof.push_back({PROF_XINV, {ev[2], ev[3]}});
    }
    return rc;
}

// Wrap one non-FFT launch for counting and (eager) profiling.
template <typename F>
static int timed(hsb_sim_s* S, int cat, F&& f) {
    S->launches += 1;
    if (!S->profiling) return f();
    cudaEvent_t a = prof_event(S), b = prof_event(S);
    cudaEventRecord(a, S->st);
    int rc = f();
    cudaEventRecord(b, S->st);
    S->prof.push_back({cat, {a, b}});
    return rc;
}

#define RC(x)                          \
    do {                               \
        int rc_ = (x);                 \
        if (rc_ != HSB_OK) return rc_; \
    } while (0)

// Enqueue one attempt (one step for the fixed-step methods) of the configured integrator.
// All buffer choices that depend on accept/reject are made on the device.
static int enqueue_attempt(hsb_sim_s* S) {
    HsbSolverDev* sd = S->sd;
    const int norm = S->d.normalize;
    float* hd = S->demag ? S->hd : nullptr;
    float* ya = S->ystage[0];
    float* yb = S->ystage[1];
    float* y0 = S->y[0];
    float* y1 = S->y[1];
    const PtrSel YC = pair(y0, y1, SEL_CUR);
    const PtrSel YN = pair(y0, y1, SEL_NEXT);
    switch (S->d.solver) {
        case SOLVER_EULER: {
            RC(run_demag(S, nullptr, 0, hd, -1));
            StageArgs A = empty_args();
            A.ys = YC;
            A.hd = fixed(hd);
            A.ytherm = YC;
            A.ynext = YN;
            A.ybase = YC;
            A.cself = 1.0f;
            A.normalize = norm;
            RC(timed(S, PROF_STAGE, [&] { return hsb_launch_stage(S->P, A, sd, S->st); }));
            RC(timed(S, PROF_OTHER, [&] { return hsb_launch_fixed_advance(sd, S->st); }));
            break;
        }
        case SOLVER_HEUN: {  // solve_heun.go:27-79
            RC(run_demag(S, nullptr, 0, hd, -1));
            StageArgs A = empty_args();
            A.ys = YC;
            A.hd = fixed(hd);
            A.ytherm = YC;
            A.kout = fixed(S->k[0]);
            A.kself_w = 1.0f;
            A.ynext = fixed(ya);
            A.ybase = YC;
            A.cself = 1.0f;
            A.normalize = norm;
            RC(timed(S, PROF_STAGE, [&] { return hsb_launch_stage(S->P, A, sd, S->st); }));
            RC(run_demag(S, ya, -1, hd, -1));
            StageArgs B = empty_args();
            B.ys = fixed(ya);
            B.hd = fixed(hd);
            B.ytherm = YC;
            B.tfrac = 1.0f;
            B.ynext = YN;
            B.ybase = fixed(ya);
            B.nk = 1;
            B.kin[0] = fixed(S->k[0]);
            B.ck[0] = -0.5f;
            B.cself = 0.5f;
            B.normalize = norm;
            RC(timed(S, PROF_STAGE, [&] { return hsb_launch_stage(S->P, B, sd, S->st); }));
            RC(timed(S, PROF_OTHER, [&] { return hsb_launch_fixed_advance(sd, S->st); }));
            break;
        }
        case SOLVER_RK4: {
            float* kacc = S->k[0];
            const float tf[4] = {0.f, 0.5f, 0.5f, 1.0f};
            const float cn[3] = {0.5f, 0.5f, 1.0f};
            float* in[4] = {nullptr, ya, yb, ya};
            for (int s = 0; s < 4; s++) {
                if (s == 0) RC(run_demag(S, nullptr, 0, hd, -1));
                else RC(run_demag(S, in[s], -1, hd, -1));
                StageArgs A = empty_args();
                A.ys = (s == 0) ? YC : fixed(in[s]);
                A.hd = fixed(hd);
                A.ytherm = YC;
                A.tfrac = tf[s];
                A.ybase = YC;
                A.normalize = norm;
                if (s < 3) {
                    A.kout = fixed(kacc);
                    A.kacc = (s == 0) ? none() : fixed(kacc);
                    A.kacc_w = 1.0f;
                    A.kself_w = (s == 0) ? 1.0f : 2.0f;
                    A.ynext = fixed(in[s + 1]);
                    A.cself = cn[s];
                } else {
                    A.ynext = YN;
                    A.nk = 1;
                    A.kin[0] = fixed(kacc);
                    A.ck[0] = 1.0f / 6.0f;
                    A.cself = 1.0f / 6.0f;
                }
                RC(timed(S, PROF_STAGE, [&] { return hsb_launch_stage(S->P, A, sd, S->st); }));
            }
            RC(timed(S, PROF_OTHER, [&] { return hsb_launch_fixed_advance(sd, S->st); }));
            break;
        }
        case SOLVER_DP45: {
            const PtrSel K1 = pair(S->k[0], S->k[6], SEL_K1);
            const PtrSel K7 = pair(S->k[0], S->k[6], SEL_K7);
            PtrSel kk[7];
            kk[0] = K1;
            for (int j = 1; j < 6; j++) kk[j] = fixed(S->k[j]);
            kk[6] = K7;
            const bool th = S->d.thermal != 0;
            if (th) {
                // the thermal field is redrawn for every step (and rescaled with dt), so
                // k1 is evaluated afresh; the demag field of y0 is kept from stage 7
                StageArgs A = empty_args();
                A.ys = YC;
                A.hd = S->demag ? pair(S->hd01[0], S->hd01[1], SEL_CUR) : none();
                A.ytherm = YC;
                A.kout = K1;
                A.kself_w = 1.0f;
                A.ynext = fixed(ya);
                A.ybase = YC;
                A.cself = (float)DPA[1][0];
                A.normalize = norm;
                RC(timed(S, PROF_STAGE, [&] { return hsb_launch_stage(S->P, A, sd, S->st); }));
            } else {
                StageArgs A = empty_args();
                A.ynext = fixed(ya);
                A.ybase = YC;
                A.nk = 1;
                A.kin[0] = K1;
                A.ck[0] = (float)DPA[1][0];
                A.normalize = norm;
                RC(timed(S, PROF_OTHER, [&] { return hsb_launch_combine(S->P, A, sd, S->st); }));
            }
            float* cur = ya;
            float* other = yb;
            for (int s = 1; s < 6; s++) {  // stages 2..6 -> k[s]
                RC(run_demag(S, cur, -1, hd, -1));
                StageArgs A = empty_args();
                A.ys = fixed(cur);
                A.hd = fixed(hd);
                A.ytherm = YC;
                A.tfrac = (float)DPC[s];
                A.kout = fixed(S->k[s]);
                A.kself_w = 1.0f;
                A.ybase = YC;
                A.ynext = (s < 5) ? fixed(other) : YN;
                A.nk = s;
                for (int j = 0; j < s; j++) {
                    A.kin[j] = kk[j];
                    A.ck[j] = (float)DPA[s + 1][j];
                }
                A.cself = (float)DPA[s + 1][s];
                A.normalize = norm;
                RC(timed(S, PROF_STAGE, [&] { return hsb_launch_stage(S->P, A, sd, S->st); }));
                float* t = cur;
                cur = other;
                other = t;
            }
            // stage 7 at the 5th-order solution y[next]: FSAL derivative + error norm
            PtrSel HD7;
            if (th && S->demag) {
                RC(run_demag(S, nullptr, 1, nullptr, 1));
                HD7 = pair(S->hd01[0], S->hd01[1], SEL_NEXT);
            } else {
                RC(run_demag(S, nullptr, 1, hd, -1));
                HD7 = fixed(hd);
            }
            StageArgs A = empty_args();
            A.ys = YN;
            A.hd = HD7;
            A.ytherm = YC;
            A.tfrac = 1.0f;
            A.kout = K7;
            A.kself_w = 1.0f;
            A.err = 1;
            A.nk = 0;
            for (int j = 0; j < 6; j++) {
                A.kin[j] = kk[j];
                A.ce[j] = (float)DPE[j];
            }
            A.ceself = (float)DPE[6];
            A.yerr0 = YC;
            A.rtol = (float)S->d.rtol;
            RC(timed(S, PROF_STAGE, [&] { return hsb_launch_stage(S->P, A, sd, S->st); }));
            RC(timed(S, PROF_OTHER, [&] { return hsb_launch_dp45_control(sd, S->st); }));
            break;
        }
        default:
            hsb_set_error("unknown solver %d", S->d.solver);
            return HSB_ERR_INVALID;
    }
    return HSB_OK;
}

// DP45 needs k1 = f(y0) (without a thermal field) and, with a thermal field, the demag
// field of y0 before the first attempt; recomputed whenever the state is replaced.
static int prepare(hsb_sim_s* S) {
    if (S->initialized || S->d.solver != SOLVER_DP45) {
        S->initialized = true;
        return HSB_OK;
    }
    float* y0 = S->y[0];
    float* y1 = S->y[1];
    const PtrSel YC = pair(y0, y1, SEL_CUR);
    if (S->d.thermal) {
        if (S->demag) RC(run_demag(S, nullptr, 0, nullptr, 0));
    } else {
        float* hd = S->demag ? S->hd : nullptr;
        RC(run_demag(S, nullptr, 0, hd, -1));
        StageArgs A = empty_args();
        A.ys = YC;
        A.hd = fixed(hd);
        A.ytherm = YC;
        A.kout = pair(S->k[0], S->k[6], SEL_K1);
        A.kself_w = 1.0f;
        RC(hsb_launch_stage(S->P, A, S->sd, S->st));
    }
    S->initialized = true;
    return HSB_OK;
}

static int build_graph(hsb_sim_s* S) {
    if (S->graph) return HSB_OK;
    cudaGraph_t g;
    HSB_CUDA_TRY(cudaStreamBeginCapture(S->st, cudaStreamCaptureModeThreadLocal));
    int rc = HSB_OK;
    S->launches = 0;
    for (int a = 0; a < S->graph_steps && rc == HSB_OK; a++) rc = enqueue_attempt(S);
    cudaError_t e = cudaStreamEndCapture(S->st, &g);
    if (rc != HSB_OK) return rc;
    if (e != cudaSuccess) {
        hsb_set_error("graph capture: %s", cudaGetErrorString(e));
        return HSB_ERR_CUDA;
    }
    e = cudaGraphInstantiate(&S->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        hsb_set_error("graph instantiate: %s", cudaGetErrorString(e));
        S->graph = nullptr;
        return HSB_ERR_CUDA;
    }
    return HSB_OK;
}

// Advance until the device clears `active` (step or time target reached).
static int advance(hsb_sim_s* S, int64_t nsteps, double t_stop) {
    RC(get_sd(S));
    HsbSolverDev* h = S->sd_host;
    if (h->status & 1) {
        hsb_set_error("state is not finite (status %d)", h->status);
        return HSB_ERR_NONFINITE;
    }
    h->active = 1;
    h->step_stop = nsteps >= 0 ? h->step + nsteps : -1;
    h->t_stop = t_stop;
    if (t_stop > 0.0) {
        if (t_stop - h->t <= 1e-6 * h->dt) return HSB_OK;
        if (h->dt > t_stop - h->t) h->dt = t_stop - h->t;
    }
    if (nsteps == 0) return HSB_OK;
    RC(set_sd_fields(S));
    RC(prepare(S));
    RC(build_graph(S));
    const bool fixed_step = S->d.solver != SOLVER_DP45;
    int64_t launched = 0;
    const int64_t max_attempts = fixed_step ? (nsteps >= 0 ? nsteps : INT64_MAX) : INT64_MAX;
    while (true) {
        HSB_CUDA_TRY(cudaGraphLaunch(S->graph, S->st));
        launched += S->graph_steps;
        if (fixed_step && nsteps >= 0) {
            if (launched >= max_attempts) break;
            continue;
        }
        HSB_CUDA_TRY(cudaMemcpyAsync(&S->sd_host->active, &S->sd->active, sizeof(int), cudaMemcpyDeviceToHost, S->st));
        HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
        if (!S->sd_host->active) break;
        if (launched > 100000000LL) {
            hsb_set_error("solver did not reach its target");
            return HSB_ERR_SOLVER;
        }
    }
    RC(get_sd(S));
    if (S->sd_host->status & 1) {
        hsb_set_error("state became non-finite at t = %g", S->sd_host->t);
        return HSB_ERR_NONFINITE;
    }
    return HSB_OK;
}

// ------------------------------------------------------------------ public API
static void fill_phys(hsb_sim_s* S) {
    const hsb_sim_desc& d = S->d;
    HsbPhys& P = S->P;
    memset(&P, 0, sizeof(P));
    P.N0 = d.size[0];
    P.N1 = d.size[1];
    P.N2 = d.size[2];
    P.pbc0 = d.pbc[0];
    P.pbc1 = d.pbc[1];
    P.pbc2 = d.pbc[2];
    P.nch = S->nch;
    P.ncell = S->n;
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
    P.msat_mask = S->msat_mask;
    P.lex_mask = S->lex_mask;
}

static void free_sim(hsb_sim_s* S) {
    if (!S) return;
    if (S->graph) cudaGraphExecDestroy(S->graph);
    for (auto e : S->ev_pool) cudaEventDestroy(e);
    if (S->demag) hsb_demag_plan_destroy(S->demag);
    cudaFree(S->y[0]);
    cudaFree(S->ystage[0]);
    cudaFree(S->k[0]);
    cudaFree(S->hd);
    cudaFree(S->hd01[0]);
    cudaFree(S->msat_mask);
    cudaFree(S->lex_mask);
    cudaFree(S->sd);
    cudaFree(S->red);
    cudaFree(S->stage_f);
    cudaFree(S->stage_d);
    if (S->sd_host) cudaFreeHost(S->sd_host);
    if (S->red_host) cudaFreeHost(S->red_host);
    if (S->st) cudaStreamDestroy(S->st);
    delete S;
}

#define STRY(x)                                                                       \
    do {                                                                              \
        cudaError_t e_ = (x);                                                         \
        if (e_ != cudaSuccess) {                                                      \
            hsb_set_error("hsb_sim_create: %s: %s", #x, cudaGetErrorString(e_));      \
            free_sim(S);                                                              \
            return e_ == cudaErrorMemoryAllocation ? HSB_ERR_NOMEM : HSB_ERR_CUDA;    \
        }                                                                             \
    } while (0)

static const int RED_BLOCKS = 296;

__global__ void k_fill(float* p, long n, float v) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) p[i] = v;
}

HSB_EXPORT int hsb_sim_create(const hsb_sim_desc* desc, hsb_sim_s** out) {
    if (!desc || !out) {
        hsb_set_error("hsb_sim_create: null argument");
        return HSB_ERR_INVALID;
    }
    *out = nullptr;
    const hsb_sim_desc& d = *desc;
    for (int a = 0; a < 3; a++) {
        if (d.size[a] < 1 || d.cellsize[a] <= 0 || d.pbc[a] < 0) {
            hsb_set_error("hsb_sim_create: bad size/cellsize/pbc on axis %d", a);
            return HSB_ERR_INVALID;
        }
    }
    if (d.solver < SOLVER_EULER || d.solver > SOLVER_DP45) {
        hsb_set_error("hsb_sim_create: unknown solver %d", d.solver);
        return HSB_ERR_INVALID;
    }
    if (!(d.dt > 0) || !(d.msat0T0 > 0) || (d.solver == SOLVER_DP45 && !(d.rtol > 0))) {
        hsb_set_error("hsb_sim_create: dt, msat0T0 (and rtol for DP45) must be positive");
        return HSB_ERR_INVALID;
    }
    if (d.llb && !(d.tc > 0 && d.spin_j > 0 && d.n_spins > 0)) {
        hsb_set_error("hsb_sim_create: llb needs tc, spin_j and n_spins > 0");
        return HSB_ERR_INVALID;
    }
    if (d.ttm && !(d.gamma_e > 0 && d.c_l > 0)) {
        hsb_set_error("hsb_sim_create: ttm needs gamma_e > 0 and c_l > 0");
        return HSB_ERR_INVALID;
    }
    const long n = (long)d.size[0] * d.size[1] * d.size[2];
    if (n > (1L << 31) / 8) {
        hsb_set_error("hsb_sim_create: %ld cells exceed the 2^28 limit", n);
        return HSB_ERR_UNSUPPORTED;
    }
    hsb_sim_s* S = new hsb_sim_s();
    S->d = d;
    S->n = n;
    S->nch = d.ttm ? 5 : 3;
    const long ny = (long)S->nch * n;
    STRY(cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking));
    STRY(cudaMalloc(&S->y[0], sizeof(float) * 2 * ny));
    S->y[1] = S->y[0] + ny;
    STRY(cudaMalloc(&S->ystage[0], sizeof(float) * 2 * ny));
    S->ystage[1] = S->ystage[0] + ny;
    const int nk = (d.solver == SOLVER_DP45) ? 7 : 1;
    STRY(cudaMalloc(&S->k[0], sizeof(float) * nk * ny));
    for (int j = 1; j < nk; j++) S->k[j] = S->k[0] + j * ny;
    STRY(cudaMalloc(&S->sd, sizeof(HsbSolverDev)));
    STRY(cudaMallocHost(&S->sd_host, sizeof(HsbSolverDev)));
    STRY(cudaMalloc(&S->red, sizeof(double) * (RED_BLOCKS * 8 + 16) + 64));
    STRY(cudaMallocHost(&S->red_host, sizeof(double) * 16));
    STRY(cudaMemsetAsync(S->red, 0, sizeof(double) * (RED_BLOCKS * 8 + 16) + 64, S->st));
    if (d.demag) {
        STRY(cudaMalloc(&S->hd, sizeof(float) * 3 * n));
        if (d.thermal && d.solver == SOLVER_DP45) {
            STRY(cudaMalloc(&S->hd01[0], sizeof(float) * 6 * n));
            S->hd01[1] = S->hd01[0] + 3 * n;
        }
        int rc = hsb_demag_plan_create(d.size, d.cellsize, d.pbc, 6, S->st, &S->demag);
        if (rc != HSB_OK) {
            free_sim(S);
            return rc;
        }
    }
    fill_phys(S);
    // initial state: m = (0, 0, 1) in program order (+x user would be component 2), T = bath
    k_fill<<<hsb_grid_1d(n, 256), 256, 0, S->st>>>(S->y[0], 2 * n, 0.f);
    k_fill<<<hsb_grid_1d(n, 256), 256, 0, S->st>>>(S->y[0] + 2 * n, n, 1.f);
    if (S->nch == 5) k_fill<<<hsb_grid_1d(n, 256), 256, 0, S->st>>>(S->y[0] + 3 * n, 2 * n, (float)d.temperature);
    memset(S->sd_host, 0, sizeof(HsbSolverDev));
    S->sd_host->dt = d.dt;
    S->sd_host->mindt = d.mindt > 0 ? d.mindt : 1e-22;
    S->sd_host->maxdt = d.maxdt > 0 ? d.maxdt : 1e-9;
    S->sd_host->step_stop = -1;
    S->sd_host->active = 1;
    STRY(cudaMemcpyAsync(S->sd, S->sd_host, sizeof(HsbSolverDev), cudaMemcpyHostToDevice, S->st));
    STRY(cudaStreamSynchronize(S->st));
    // launch-bound grids batch more steps per graph launch
    S->graph_steps = n < 65536 ? 16 : (n < 1048576 ? 8 : 4);
    if (d.solver == SOLVER_DP45) S->graph_steps = n < 65536 ? 8 : 4;
    *out = S;
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_destroy(hsb_sim_s* S) {
    if (S) cudaStreamSynchronize(S->st);
    free_sim(S);
    return HSB_OK;
}

HSB_EXPORT void* hsb_sim_stream(hsb_sim_s* S) { return S ? (void*)S->st : nullptr; }

static int channel_of(hsb_sim_s* S, const char* name, int* first, int* count) {
    std::string s(name ? name : "");
    if (s == "m") { *first = 0; *count = 3; return HSB_OK; }
    if (S->nch == 5 && s == "Te") { *first = 3; *count = 1; return HSB_OK; }
    if (S->nch == 5 && s == "Tl") { *first = 4; *count = 1; return HSB_OK; }
    hsb_set_error("unknown state quantity '%s'", name ? name : "(null)");
    return HSB_ERR_INVALID;
}

static int stage_buffers(hsb_sim_s* S, long count) {
    if (S->stage_f) return HSB_OK;
    long need = 5 * S->n;
    if (count > need) need = count;
    HSB_CUDA_TRY(cudaMalloc(&S->stage_f, sizeof(float) * need));
    HSB_CUDA_TRY(cudaMalloc(&S->stage_d, sizeof(double) * need));
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_set(hsb_sim_s* S, const char* name, const double* host, int64_t count) {
    if (!S || !name) {
        hsb_set_error("hsb_sim_set: null argument");
        return HSB_ERR_INVALID;
    }
    RC(stage_buffers(S, count));
    std::string s(name);
    if (s == "msat_mask" || s == "lex_mask") {
        float** dst = (s == "msat_mask") ? &S->msat_mask : &S->lex_mask;
        if (!host) {
            HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
            cudaFree(*dst);
            *dst = nullptr;
        } else {
            if (count != S->n) {
                hsb_set_error("hsb_sim_set(%s): expected %ld values, got %ld", name, S->n, (long)count);
                return HSB_ERR_INVALID;
            }
            if (!*dst) HSB_CUDA_TRY(cudaMalloc(dst, sizeof(float) * S->n));
            HSB_CUDA_TRY(cudaMemcpyAsync(S->stage_d, host, sizeof(double) * S->n, cudaMemcpyHostToDevice, S->st));
            k_d2f<<<hsb_grid_1d(S->n, 256), 256, 0, S->st>>>(S->stage_d, *dst, S->n);
        }
        fill_phys(S);
        if (S->graph) {
            cudaGraphExecDestroy(S->graph);
            S->graph = nullptr;
        }
        S->initialized = false;
        HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
        return HSB_OK;
    }
    int first, nc;
    RC(channel_of(S, name, &first, &nc));
    if (!host || count != (int64_t)nc * S->n) {
        hsb_set_error("hsb_sim_set(%s): expected %ld values, got %ld", name, (long)nc * S->n, (long)count);
        return HSB_ERR_INVALID;
    }
    RC(get_sd(S));
    float* y = S->y[S->sd_host->cur];
    HSB_CUDA_TRY(cudaMemcpyAsync(S->stage_d, host, sizeof(double) * count, cudaMemcpyHostToDevice, S->st));
    k_d2f<<<hsb_grid_1d(count, 256), 256, 0, S->st>>>(S->stage_d, y + (long)first * S->n, count);
    HSB_CUDA_TRY(cudaGetLastError());
    S->initialized = false;
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_get(hsb_sim_s* S, const char* name, double* host, int64_t count) {
    if (!S || !name || !host) {
        hsb_set_error("hsb_sim_get: null argument");
        return HSB_ERR_INVALID;
    }
    RC(stage_buffers(S, count));
    RC(get_sd(S));
    float* y = S->y[S->sd_host->cur];
    std::string s(name);
    const float* src = nullptr;
    long nv = 0;
    if (s == "H_demag") {
        if (!S->demag) {
            hsb_set_error("hsb_sim_get(H_demag): demag is not enabled");
            return HSB_ERR_INVALID;
        }
        RC(run_demag(S, y, -1, S->hd, -1, false));
        src = S->hd;
        nv = 3 * S->n;
    } else if (s == "k") {
        float* hd = S->demag ? S->hd : nullptr;
        if (S->demag) RC(run_demag(S, y, -1, hd, -1, false));
        StageArgs A = empty_args();
        A.ungated = 1;
        A.ys = fixed(y);
        A.hd = fixed(hd);
        A.ytherm = fixed(y);
        A.kout = fixed(S->ystage[1]);
        A.kself_w = 1.0f;
        RC(hsb_launch_stage(S->P, A, S->sd, S->st));
        src = S->ystage[1];
        nv = (long)S->nch * S->n;
        S->initialized = false;
    } else {
        int first, nc;
        RC(channel_of(S, name, &first, &nc));
        src = y + (long)first * S->n;
        nv = (long)nc * S->n;
    }
    if (count != nv) {
        hsb_set_error("hsb_sim_get(%s): expected %ld values, got %ld", name, nv, (long)count);
        return HSB_ERR_INVALID;
    }
    k_f2d<<<hsb_grid_1d(nv, 256), 256, 0, S->st>>>(src, S->stage_d, nv);
    HSB_CUDA_TRY(cudaMemcpyAsync(host, S->stage_d, sizeof(double) * nv, cudaMemcpyDeviceToHost, S->st));
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_step(hsb_sim_s* S, int64_t nsteps) {
    if (!S || nsteps < 0) {
        hsb_set_error("hsb_sim_step: bad argument");
        return HSB_ERR_INVALID;
    }
    return advance(S, nsteps, 0.0);
}

HSB_EXPORT int hsb_sim_run_until(hsb_sim_s* S, double t) {
    if (!S) {
        hsb_set_error("hsb_sim_run_until: null handle");
        return HSB_ERR_INVALID;
    }
    if (S->d.solver != SOLVER_DP45) {
        RC(get_sd(S));
        const double rem = t - S->sd_host->t;
        if (rem <= 0) return HSB_OK;
        const int64_t n = (int64_t)ceil(rem / S->sd_host->dt - 1e-9);
        return advance(S, n, 0.0);
    }
    return advance(S, -1, t);
}

HSB_EXPORT int hsb_sim_sync(hsb_sim_s* S) {
    if (!S) return HSB_ERR_INVALID;
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_status(hsb_sim_s* S, double* t, double* dt, int64_t* steps, int64_t* attempts,
                              int64_t* rejects, double* err, int32_t* status) {
    if (!S) return HSB_ERR_INVALID;
    RC(get_sd(S));
    const HsbSolverDev* h = S->sd_host;
    if (t) *t = h->t;
    if (dt) *dt = h->dt;
    if (steps) *steps = h->step;
    if (attempts) *attempts = h->attempts;
    if (rejects) *rejects = h->rejects;
    if (err) *err = h->err;
    if (status) *status = h->status;
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_set_time(hsb_sim_s* S, double t, double dt) {
    if (!S) return HSB_ERR_INVALID;
    RC(get_sd(S));
    S->sd_host->t = t;
    if (dt > 0) S->sd_host->dt = dt;
    RC(set_sd_fields(S));
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    return HSB_OK;
}

static int reduce_terms(hsb_sim_s* S, double* out8) {
    RC(get_sd(S));
    float* y = S->y[S->sd_host->cur];
    float* hd = nullptr;
    if (S->demag) {
        RC(run_demag(S, y, -1, S->hd, -1, false));
        hd = S->hd;
    }
    double* partial = S->red;
    double* res = S->red + RED_BLOCKS * 8;
    unsigned int* counter = (unsigned int*)(S->red + RED_BLOCKS * 8 + 8);
    k_energy<<<RED_BLOCKS, 256, 0, S->st>>>(S->P, y, hd, S->d.normalize, partial, counter, res);
    HSB_CUDA_TRY(cudaGetLastError());
    HSB_CUDA_TRY(cudaMemcpyAsync(S->red_host, res, sizeof(double) * 8, cudaMemcpyDeviceToHost, S->st));
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    for (int q = 0; q < 8; q++) out8[q] = S->red_host[q];
    return HSB_OK;
}

// Device time of one attempt split by kernel family, eager launches bracketed by CUDA
// events on the handle's stream: out[0] fused stage kernels, out[1] demag x-pass,
// out[2] demag y/z pass(es), out[3] demag inverse x-pass, out[4] combine/controller,
// out[5] kernel launches per attempt.  Averaged over `reps` attempts (each a real step of
// the simulation; the state advances).  out[6] accepted steps during the profile.
HSB_EXPORT int hsb_sim_profile(hsb_sim_s* S, int reps, double* out) {
    if (!S || !out || reps < 1) return HSB_ERR_INVALID;
    RC(get_sd(S));
    const long long step0 = S->sd_host->step;
    S->sd_host->active = 1;
    S->sd_host->step_stop = -1;
    S->sd_host->t_stop = 0.0;
    RC(set_sd_fields(S));
    RC(prepare(S));
    double acc[PROF_NCAT] = {0, 0, 0, 0, 0};
    int launches = 0;
    for (int r = 0; r < reps; r++) {
        S->profiling = true;
        S->prof.clear();
        S->launches = 0;
        int rc = enqueue_attempt(S);
        S->profiling = false;
        launches = S->launches;
        if (rc != HSB_OK) return rc;
        HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
        for (auto& p : S->prof) {
            float ms = 0;
            cudaEventElapsedTime(&ms, p.second.first, p.second.second);
            acc[p.first] += ms;
        }
        for (auto e : S->ev_pool) cudaEventDestroy(e);
        S->ev_pool.clear();
    }
    for (int c = 0; c < PROF_NCAT; c++) out[c] = acc[c] / reps;
    out[5] = launches;
    RC(get_sd(S));
    out[6] = (double)(S->sd_host->step - step0);
    return HSB_OK;
}

// Kernel launches enqueued per attempt (per step for the fixed-step methods).
HSB_EXPORT int hsb_sim_launches_per_attempt(hsb_sim_s* S, int* n) {
    if (!S || !n) return HSB_ERR_INVALID;
    if (!S->graph) {
        S->launches = 0;
        // count by capturing into a throw-away graph
        cudaGraph_t g;
        HSB_CUDA_TRY(cudaStreamBeginCapture(S->st, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_attempt(S);
        cudaStreamEndCapture(S->st, &g);
        if (g) cudaGraphDestroy(g);
        if (rc != HSB_OK) return rc;
        *n = S->launches;
        return HSB_OK;
    }
    *n = S->launches / (S->graph_steps > 0 ? S->graph_steps : 1);
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_energy(hsb_sim_s* S, double* energy) {
    if (!S || !energy) return HSB_ERR_INVALID;
    double r[8];
    RC(reduce_terms(S, r));
    const double V = S->d.cellsize[0] * S->d.cellsize[1] * S->d.cellsize[2];
    const double pre = V * MU0 * S->d.msat0T0;
    *energy = pre * (r[0] + r[1] + r[2] + r[3] + r[4]);
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_average_m(hsb_sim_s* S, double* avg3) {
    if (!S || !avg3) return HSB_ERR_INVALID;
    double r[8];
    RC(reduce_terms(S, r));
    for (int c = 0; c < 3; c++) avg3[c] = r[5 + c] / (double)S->n;
    return HSB_OK;
}
