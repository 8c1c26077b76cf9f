// Simulation handle: device-resident FP32 state, integrator sequencing, CUDA graphs.
//
// Replaces the per-step host sequencing of hotspin's engine (engine/engine.go:473-508,
// solve_euler.go, solve_heun.go, solve_rk12.go; the Quant.Update graph walk of
// engine/quant.go:417-445) for a fixed module set.  Each integrator step is a fixed
// sequence of kernels whose buffer choices and step-size decisions are resolved on the
// device (HsbSolverDev), so a run of steps is captured once into a CUDA graph and replayed
// with no host round trip; the host only checks completion between graph launches.
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "hsb_common.cuh"
#include "hsb_demag.h"
#include "hsb_desc.h"
#include "hsb_llg.cuh"

int hsb_launch_stage(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, cudaStream_t st, int variant = -1);
bool hsb_stage_keeps_thermal(const HsbPhys& P, int variant);
bool hsb_stage_tunable(const HsbPhys& P);
extern "C" int hsb_set_stage_variant(int v);
int hsb_launch_combine(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, cudaStream_t st);
int hsb_launch_stage_generic(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, cudaStream_t st);
int hsb_launch_dp45_control(HsbSolverDev* sd, cudaStream_t st);
int hsb_launch_fixed_advance(HsbSolverDev* sd, cudaStream_t st);
int hsb_launch_stage_batched(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, const BatchArgs& Bt,
                             cudaStream_t st, int variant = -1);
int hsb_launch_combine_batched(const HsbPhys& P, const StageArgs& A, HsbSolverDev* sd, const BatchArgs& Bt,
                               cudaStream_t st);
int hsb_launch_dp45_control_batched(HsbSolverDev* sd, int nslot, cudaStream_t st);
int hsb_launch_fixed_advance_batched(HsbSolverDev* sd, int nslot, cudaStream_t st);
int hsb_launch_activate_prepped(HsbSolverDev* sd, int nslot, cudaStream_t st);
int hsb_launch_rk12_control(HsbSolverDev* sd, int nslot, const double* maxerr, int neq, cudaStream_t st);

enum { SOLVER_EULER = 0, SOLVER_HEUN = 1, SOLVER_RK4 = 2, SOLVER_DP45 = 3, SOLVER_RK12 = 4, SOLVER_AM12 = 5,
       SOLVER_BDF_EULER = 6 };

// Solvers whose step size is chosen on the device (accept / reject per attempt).
static inline bool adaptive_solver(int s) { return s == SOLVER_DP45 || s == SOLVER_RK12 || s == SOLVER_AM12; }

// Fixed-point sweeps of the implicit solvers (hsb_implicit.cu).
int hsb_launch_imp_sweep(const HsbPhys& P, const ImpArgs& A, HsbSolverDev* sd, const BatchArgs& Bt, int nslot,
                         bool batched, cudaStream_t st);
int hsb_launch_imp_rule(HsbSolverDev* sd, int nslot, const ImpLimits& L, int which, cudaStream_t st);


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
    // Buffers of one simulation ("slot") lie in one arena; a batch holds nslot arenas at a
    // uniform stride, and every pointer below addresses slot 0's.
    float* arena;
    long slot_stride;   // floats between slots' arenas
    int nslot;
    bool batched;       // launches use the slot-batched kernels (per-slot physics and solver state)
    HsbPhys* phys_dev;  // batched: per-slot physics [nslot]
    std::vector<HsbPhys> phys_h;
    void* X1b;          // batched: per-slot demag spectra
    long x1_stride;     // complex elements
    float* kernb;       // batched: per-slot demag kernel spectra (each slot's own cell size)
    long kern_floats;
    hsb_demag_spec_s* spec;  // batched: FP64 scratch of the kernel-spectrum evaluation
    BatchArgs bt;
    bool prep_mode;     // enqueueing the preparation of newly admitted slots
    int stage_variant;  // stage-kernel variant picked by tune_stage (-1: the library default)
    int nprep;          // slots admitted since the last launch
    cudaEvent_t done_ev;
    bool launched;
    float* y[2];        // state double buffer
    float* ystage[2];   // stage points (ping-pong: a kernel never reads and writes one)
    double* y64[3];     // am12: FP64 iterates (renormalised, raw predictor, raw corrector)
    float* k[8];        // stage derivatives
    float* hd;          // demag field of the stage point
    float* hd01[2];     // demag field of y[0], y[1] (DP45 with a thermal field)
    float* hth;         // thermal field of the current step (kept across its stages)
    float* msat_mask;
    float* lex_mask;
    HsbSolverDev* sd;   // device [nslot]
    HsbSolverDev* sd_host;  // pinned mirror [nslot]
    double* red;        // reduction scratch (device)
    double* red_host;   // pinned
    float* stage_f;     // device staging for FP64 <-> FP32 conversion
    double* stage_d;
    void* stage_pin;    // batched: pinned per-slot staging of admissions
    cudaGraphExec_t graph;
    cudaGraphExec_t graph1;  // one attempt: short runs (a few steps) launch no gated attempts
    bool sd_fresh;      // sd_host equals the device words: read back, nothing enqueued since
    double2* laser_tab; // device copy of the pointwise laser profile (or null)
    double* bext_tab;   // device copy of the pointwise applied field (or null)
    int graph_steps;    // attempts captured in one graph launch
    bool initialized;   // k1 / hd01 of the current state computed (DP45)
    // eager profiling: events around every launch group of one attempt
    bool profiling;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof;  // category, start, stop
    int launches;       // kernel launches of one attempt (counted while enqueuing)
    int launches_g, launches_g1;  // kernels in the full graph and in the one-attempt graph
    long long launch_total;       // kernels enqueued for stepping since creation
    double rk12_maxerr[3];        // rk12: per-step error limits (m, Te, Tl; +inf = uncontrolled)
    ImpLimits imp;                // am12 / bdf-euler limits
    float* hbuf;                  // non-local relaxation: effective field of every cell [3][n]
    float* ckpt;                  // checkpoint: the state channels [nch][n] (device)
    HsbSolverDev* ckpt_sd;        // checkpoint: the solver word (device)
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
    A.ys = A.hd = A.ytherm = A.kout = A.kacc = A.ynext = A.ybase = A.yerr0 = A.hth = none();
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
                         double* partial, unsigned int* counter, double* out, double t) {
    float hb[3];
    hsb_bext(P, t, hb);       // the applied field at the state's time
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
        term[0] = -(m[0] * (double)hb[0] + m[1] * (double)hb[1] + m[2] * (double)hb[2]) * ms;
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
            // |m| in FP64: near equilibrium W(|m| b) - |m| is ~1e-9, so an FP32 |m| (biased by
            // the rounding of its sum of squares) would dominate this term
            const double am = sqrt((double)m[0] * m[0] + (double)m[1] * m[1] + (double)m[2] * m[2]);
            if (am > 1e-30 && Ts > 0.f) {
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
    S->sd_fresh = false;
    HSB_CUDA_TRY(cudaMemcpyAsync(S->sd, S->sd_host, sizeof(HsbSolverDev), cudaMemcpyHostToDevice, S->st));
    return HSB_OK;
}
static int get_sd(hsb_sim_s* S) {
    HSB_CUDA_TRY(cudaMemcpyAsync(S->sd_host, S->sd, sizeof(HsbSolverDev), cudaMemcpyDeviceToHost, S->st));
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    S->sd_fresh = true;
    return HSB_OK;
}

// Demag of one of the two state buffers (sel: -1 fixed pointer `m`, 0 = y[cur], 1 = y[next])
// into `h` (or into hd01[cur / next] when hsel >= 0).
static int run_demag(hsb_sim_s* S, const float* m, int msel, float* h, int hsel, bool gated = true,
                     const int* gate_word = nullptr) {
    S->sd_fresh = false;
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
    const int* gate = gated ? (gate_word ? gate_word : (S->prep_mode ? &S->sd->prep : &S->sd->active)) : nullptr;
    int rc;
    if (S->batched) {
        HsbDemagBatch b;
        b.nslot = S->nslot;
        b.m_stride = S->slot_stride;
        b.h_stride = S->slot_stride;
        b.sel_stride = (int)(sizeof(HsbSolverDev) / sizeof(int));
        b.X1 = S->X1b;
        b.x1_stride = S->x1_stride;
        b.scale = &S->phys_dev[0].ms0;
        b.scale_stride = (int)(sizeof(HsbPhys) / sizeof(float));
        b.kern = S->kernb;
        b.kern_stride = S->kern_floats;
        rc = hsb_demag_launch(S->demag, io, nullptr, 1.0f, S->st, gate, &b);
    } else {
        rc = hsb_demag_launch(S->demag, io, S->msat_mask, (float)S->d.msat0T0, S->st, gate);
    }
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

// Launches of one simulation or of a batch of slots.
static int L_stage(hsb_sim_s* S, StageArgs A) {
    S->sd_fresh = false;
    if (S->prep_mode) A.prep_gated = 1;
    if (S->batched) return hsb_launch_stage_batched(S->P, A, S->sd, S->bt, S->st, S->stage_variant);
    return hsb_launch_stage(S->P, A, S->sd, S->st, S->stage_variant);
}
static int L_combine(hsb_sim_s* S, const StageArgs& A) {
    S->sd_fresh = false;
    if (S->batched) return hsb_launch_combine_batched(S->P, A, S->sd, S->bt, S->st);
    return hsb_launch_combine(S->P, A, S->sd, S->st);
}
static int L_control(hsb_sim_s* S) {
    S->sd_fresh = false;
    if (S->batched) return hsb_launch_dp45_control_batched(S->sd, S->nslot, S->st);
    return hsb_launch_dp45_control(S->sd, S->st);
}
// Thermal field of the step: generated and kept by the attempt's first stage, read by the
// others (only the load-first stage kernel keeps it).
static void thermal_keep(hsb_sim_s* S, StageArgs& A, bool first) {
    if (!S->hth || !hsb_stage_keeps_thermal(S->P, S->stage_variant)) return;
    A.hth = fixed(S->hth);
    A.hth_mode = first ? 1 : 2;
}

static int L_sweep(hsb_sim_s* S, int mode, int eq = 0) {
    S->sd_fresh = false;
    ImpArgs A;
    memset(&A, 0, sizeof(A));
    A.y0 = pair(S->y[0], S->y[1], SEL_CUR);
    A.w = pair(S->y[0], S->y[1], SEL_NEXT);
    A.w64 = S->y64[0];
    A.up64 = S->y64[1];
    A.uc64 = S->y64[2];
    A.k0 = S->k[0];
    A.k1 = S->k[1];
    A.k2 = S->k[2];
    A.mode = mode;
    A.normalize = S->batched ? 1 : S->d.normalize;
    A.eq = eq;
    BatchArgs nb = {0, nullptr, 1};
    return hsb_launch_imp_sweep(S->P, A, S->sd, S->batched ? S->bt : nb, S->batched ? S->nslot : 1, S->batched,
                                S->st);
}
static int L_rule(hsb_sim_s* S, int which, int eq = 0) {
    S->sd_fresh = false;
    ImpLimits L = S->imp;
    L.eq = eq;
    return hsb_launch_imp_rule(S->sd, S->batched ? S->nslot : 1, L, which, S->st);
}

static int L_advance(hsb_sim_s* S) {
    S->sd_fresh = false;
    if (S->batched) return hsb_launch_fixed_advance_batched(S->sd, S->nslot, S->st);
    return hsb_launch_fixed_advance(S->sd, S->st);
}

// Enqueue one attempt (one step for the fixed-step methods) of the configured integrator.
// All buffer choices that depend on accept/reject are made on the device.
static int enqueue_attempt(hsb_sim_s* S) {
    // batched: every slot's own HsbPhys.normalize decides
    const int norm = S->batched ? 1 : S->d.normalize;
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
            RC(timed(S, PROF_STAGE, [&] { return L_stage(S, A); }));
            RC(timed(S, PROF_OTHER, [&] { return L_advance(S); }));
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
            thermal_keep(S, A, true);
            RC(timed(S, PROF_STAGE, [&] { return L_stage(S, A); }));
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
            thermal_keep(S, B, false);
            RC(timed(S, PROF_STAGE, [&] { return L_stage(S, B); }));
            RC(timed(S, PROF_OTHER, [&] { return L_advance(S); }));
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
                thermal_keep(S, A, s == 0);
                RC(timed(S, PROF_STAGE, [&] { return L_stage(S, A); }));
            }
            RC(timed(S, PROF_OTHER, [&] { return L_advance(S); }));
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
                thermal_keep(S, A, true);
                RC(timed(S, PROF_STAGE, [&] { return L_stage(S, A); }));
            } else {
                StageArgs A = empty_args();
                A.ynext = fixed(ya);
                A.ybase = YC;
                A.nk = 1;
                A.kin[0] = K1;
                A.ck[0] = (float)DPA[1][0];
                A.normalize = norm;
                RC(timed(S, PROF_OTHER, [&] { return L_combine(S, A); }));
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
                if (th) thermal_keep(S, A, false);
                RC(timed(S, PROF_STAGE, [&] { return L_stage(S, A); }));
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
            if (th) thermal_keep(S, A, false);
            RC(timed(S, PROF_STAGE, [&] { return L_stage(S, A); }));
            RC(timed(S, PROF_OTHER, [&] { return L_control(S); }));
            break;
        }
        case SOLVER_RK12: {  // solve_rk12.go:91-214: Euler predictor, Heun corrector, error |k1 - k0| dt
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
            thermal_keep(S, A, true);
            RC(timed(S, PROF_STAGE, [&] { return L_stage(S, A); }));
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
            B.err = 1;
            B.err_abs = 1;
            B.ce[0] = -1.0f;
            B.ceself = 1.0f;
            thermal_keep(S, B, false);
            RC(timed(S, PROF_STAGE, [&] { return L_stage(S, B); }));
            RC(timed(S, PROF_OTHER, [&] {
                S->sd_fresh = false;
                return hsb_launch_rk12_control(S->sd, S->batched ? S->nslot : 1, S->rk12_maxerr, S->nch == 5 ? 3 : 1,
                                               S->st);
            }));
            break;
        }
        case SOLVER_AM12: {  // solve_am01.go:45-318 (one try of the reference's loop per attempt)
            const int itw = (int)offsetof(HsbSolverDev, it_active);
            const int* itg = &S->sd->it_active;
            RC(timed(S, PROF_OTHER, [&] { return L_rule(S, IMP_RULE_AM_BEGIN); }));
            RC(run_demag(S, nullptr, 0, hd, -1));
            StageArgs A = empty_args();          // dy0 = f(t0, y0)
            A.ys = YC;
            A.hd = fixed(hd);
            A.ytherm = YC;
            A.kout = fixed(S->k[0]);
            A.kself_w = 1.0f;
            thermal_keep(S, A, true);
            RC(timed(S, PROF_STAGE, [&] { return L_stage(S, A); }));
            RC(timed(S, PROF_OTHER, [&] { return L_sweep(S, IMP_AM_EULER); }));  // the explicit Euler point
            StageArgs R = empty_args();          // f(t0 + dt, iterate)
            R.ys = YN;
            R.hd = fixed(hd);
            R.ytherm = YC;
            R.tfrac = 1.0f;
            R.kself_w = 1.0f;
            thermal_keep(S, R, false);
            RC(run_demag(S, nullptr, 1, hd, -1));
            R.kout = fixed(S->k[1]);
            RC(timed(S, PROF_STAGE, [&] { return L_stage(S, R); }));
            R.kout = fixed(S->k[2]);
            R.gate_word = itw;
            for (int phase = 0; phase < 2; phase++) {
                for (int j = 0; j < 6; j++) {
                    RC(timed(S, PROF_OTHER, [&] { return L_sweep(S, phase == 0 ? IMP_AM_PRED : IMP_AM_CORR); }));
                    RC(timed(S, PROF_OTHER, [&] {
                        return L_rule(S, phase == 0 ? IMP_RULE_AM_ITER_PRED : IMP_RULE_AM_ITER_CORR);
                    }));
                    if (j < 5) {
                        RC(run_demag(S, nullptr, 1, hd, -1, true, itg));
                        RC(timed(S, PROF_STAGE, [&] { return L_stage(S, R); }));
                    }
                }
                RC(timed(S, PROF_OTHER, [&] {
                    return L_rule(S, phase == 0 ? IMP_RULE_AM_PRED_END : IMP_RULE_AM_CORR_END);
                }));
            }
            RC(timed(S, PROF_OTHER, [&] { return L_sweep(S, IMP_AM_ERR); }));
            RC(timed(S, PROF_OTHER, [&] { return L_rule(S, IMP_RULE_AM_FINAL); }));
            break;
        }
        case SOLVER_BDF_EULER: {  // solve_euler_backward.go:29-91 (fixed step)
            const int rdw = (int)offsetof(HsbSolverDev, rhs_due);
            const int* rdg = &S->sd->rhs_due;
            RC(run_demag(S, nullptr, 0, hd, -1));
            StageArgs A = empty_args();          // inputs at t; the working state starts as y0
            A.ys = YC;
            A.hd = fixed(hd);
            A.ytherm = YC;
            A.kout = fixed(S->k[0]);
            A.kself_w = 1.0f;
            A.ynext = YN;
            A.ybase = YC;
            A.cself = 0.0f;
            thermal_keep(S, A, true);
            RC(timed(S, PROF_STAGE, [&] { return L_stage(S, A); }));
            StageArgs R = empty_args();          // f(t + dt, working state)
            R.ys = YN;
            R.hd = fixed(hd);
            R.ytherm = YC;
            R.tfrac = 1.0f;
            R.kout = fixed(S->k[0]);
            R.kself_w = 1.0f;
            thermal_keep(S, R, false);
            const int neq = S->nch == 5 ? 3 : 1;
            for (int q = 0; q < neq; q++) {
                RC(timed(S, PROF_OTHER, [&] { return L_rule(S, IMP_RULE_BDF_BEGIN, q); }));
                RC(timed(S, PROF_OTHER, [&] { return L_sweep(S, IMP_BDF_EULER, q); }));
                RC(run_demag(S, nullptr, 1, hd, -1));
                R.gate_word = 0;
                RC(timed(S, PROF_STAGE, [&] { return L_stage(S, R); }));
                R.gate_word = rdw;
                for (int j = 0; j <= S->imp.max_iter; j++) {
                    RC(timed(S, PROF_OTHER, [&] { return L_sweep(S, IMP_BDF_SWEEP, q); }));
                    RC(timed(S, PROF_OTHER, [&] { return L_rule(S, IMP_RULE_BDF_ITER, q); }));
                    RC(run_demag(S, nullptr, 1, hd, -1, true, rdg));
                    RC(timed(S, PROF_STAGE, [&] { return L_stage(S, R); }));
                    RC(timed(S, PROF_OTHER, [&] { return L_rule(S, IMP_RULE_BDF_CLEAR, q); }));
                }
            }
            RC(timed(S, PROF_OTHER, [&] { return L_advance(S); }));
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
    // ungated: the state's first-stage data are computed even when the run about to start is
    // already inactive (target reached), so `initialized` always describes the buffers
    if (S->d.thermal) {
        if (S->demag) {
            RC(run_demag(S, nullptr, 0, nullptr, 0, false));
            S->launch_total += hsb_demag_nlaunch(S->demag);
        }
    } else {
        float* hd = S->demag ? S->hd : nullptr;
        RC(run_demag(S, nullptr, 0, hd, -1, false));
        if (S->demag) S->launch_total += hsb_demag_nlaunch(S->demag);
        S->launch_total += 1;
        StageArgs A = empty_args();
        A.ungated = 1;
        A.ys = YC;
        A.hd = fixed(hd);
        A.ytherm = YC;
        A.kout = pair(S->k[0], S->k[6], SEL_K1);
        A.kself_w = 1.0f;
        RC(L_stage(S, A));
    }
    S->initialized = true;
    return HSB_OK;
}

// Capture `attempts` attempts into *out.  S->launches counts the kernels of the capture.
static int capture_attempts(hsb_sim_s* S, int attempts, cudaGraphExec_t* out) {
    cudaGraph_t g;
    HSB_CUDA_TRY(cudaStreamBeginCapture(S->st, cudaStreamCaptureModeThreadLocal));
    int rc = HSB_OK;
    S->launches = 0;
    for (int a = 0; a < attempts && rc == HSB_OK; a++) rc = enqueue_attempt(S);
    cudaError_t e = cudaStreamEndCapture(S->st, &g);
    if (rc != HSB_OK) return rc;
    if (e != cudaSuccess) {
        hsb_set_error("graph capture: %s", cudaGetErrorString(e));
        return HSB_ERR_CUDA;
    }
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        hsb_set_error("graph instantiate: %s", cudaGetErrorString(e));
        *out = nullptr;
        return HSB_ERR_CUDA;
    }
    return HSB_OK;
}

static int build_graph(hsb_sim_s* S) {
    if (S->graph) return HSB_OK;
    const int rc = capture_attempts(S, S->graph_steps, &S->graph);
    S->launches_g = S->launches;
    return rc;
}

// The one-attempt graph (S->launches keeps the count of the full graph).
static int build_graph1(hsb_sim_s* S) {
    if (S->graph1) return HSB_OK;
    const long keep = S->launches;
    const int rc = capture_attempts(S, 1, &S->graph1);
    S->launches_g1 = S->launches;
    S->launches = keep;
    return rc;
}

static void drop_graphs(hsb_sim_s* S) {
    if (S->graph) cudaGraphExecDestroy(S->graph);
    if (S->graph1) cudaGraphExecDestroy(S->graph1);
    S->graph = nullptr;
    S->graph1 = nullptr;
}

static int plain_only(hsb_sim_s* S, const char* who) {
    if (S && S->batched) {
        hsb_set_error("%s: a batch handle takes the hsb_batch_* functions", who);
        return HSB_ERR_INVALID;
    }
    return HSB_OK;
}

// Arms the solver words for a run on the device, so the host needs no read of them first:
// a non-finite state stays inactive (reported after the run); a time target already
// reached leaves it inactive; dt is clipped to land on the target.
__global__ void k_arm(HsbSolverDev* sd, long long nsteps, double t_stop) {
    sd->tries = 0;
    sd->aborts = 0;
    sd->it_flags = 0;
    if (sd->status & 1) {
        sd->active = 0;
        return;
    }
    sd->active = 1;
    sd->step_stop = nsteps >= 0 ? sd->step + nsteps : -1;
    sd->t_stop = t_stop;
    if (t_stop > 0.0) {
        if (t_stop - sd->t <= 1e-6 * sd->dt) sd->active = 0;
        else if (sd->dt > t_stop - sd->t) sd->dt = t_stop - sd->t;
    }
}

// Advance until the device clears `active` (step or time target reached).
static int advance(hsb_sim_s* S, int64_t nsteps, double t_stop) {
    RC(plain_only(S, "hsb_sim_step/run_until"));
    if (nsteps == 0) {
        RC(get_sd(S));
        if (S->sd_host->status & 1) {
            hsb_set_error("state is not finite (status %d)", S->sd_host->status);
            return HSB_ERR_NONFINITE;
        }
        return HSB_OK;
    }
    S->sd_fresh = false;
    k_arm<<<1, 1, 0, S->st>>>(S->sd, (long long)nsteps, t_stop);
    HSB_CUDA_TRY(cudaGetLastError());
    S->launch_total += 1;
    RC(prepare(S));
    RC(build_graph(S));
    const bool fixed_step = !adaptive_solver(S->d.solver);
    const int G = S->graph_steps;
    // fewer steps than a graph holds (e.g. one step per call): one-attempt graphs, so no
    // launch carries attempts that the device would gate off
    const bool short_run = nsteps >= 0 && nsteps < G;
    if (short_run || (fixed_step && nsteps >= 0 && nsteps % G != 0)) RC(build_graph1(S));
    int64_t launched = 0;
    while (true) {
        if (fixed_step && nsteps >= 0) {
            // whole graphs, then single attempts for the remainder
            if (nsteps - launched >= G) {
                HSB_CUDA_TRY(cudaGraphLaunch(S->graph, S->st));
                launched += G;
                S->launch_total += S->launches_g;
            } else {
                HSB_CUDA_TRY(cudaGraphLaunch(S->graph1, S->st));
                launched += 1;
                S->launch_total += S->launches_g1;
            }
            if (launched >= nsteps) break;
            continue;
        }
        HSB_CUDA_TRY(cudaGraphLaunch(short_run ? S->graph1 : S->graph, S->st));
        launched += short_run ? 1 : G;
        S->launch_total += short_run ? S->launches_g1 : S->launches_g;
        // the whole solver word block (one round trip either way): current when the loop ends
        RC(get_sd(S));
        if (!S->sd_host->active) break;
        if (launched > 100000000LL) {
            hsb_set_error("solver did not reach its target");
            return HSB_ERR_SOLVER;
        }
    }
    if (fixed_step && nsteps >= 0) RC(get_sd(S));
    if (S->sd_host->status & 1) {
        hsb_set_error("state became non-finite at t = %g", S->sd_host->t);
        return HSB_ERR_NONFINITE;
    }
    if (S->sd_host->status & 4) {
        hsb_set_error("rk12: the step at t = %g still exceeded maxerr after 10 retries", S->sd_host->t);
        return HSB_ERR_SOLVER;
    }
    return HSB_OK;
}

// ------------------------------------------------------------------ public API
static void fill_phys(hsb_sim_s* S) {
    phys_from_desc(S->d, S->nch, S->n, S->P);
    S->P.laser_tab = S->laser_tab;
    S->P.laser_npts = S->laser_tab ? S->d.laser_npts : 0;
    S->P.bext_tab = S->bext_tab;
    S->P.bext_npts = S->bext_tab ? S->d.bext_npts : 0;
    S->P.msat_mask = S->msat_mask;
    S->P.lex_mask = S->lex_mask;
    S->P.hbuf = S->hbuf;
}

// Offsets (floats) of one slot's buffers in its arena.
struct SlotLayout {
    long y, ystage, k, hd, hd01, hth, d64, total;
    int nk;
};
static SlotLayout slot_layout(const hsb_sim_desc& d, long n) {
    auto al = [](long x) { return (x + 63) & ~63L; };  // 256-byte boundaries
    SlotLayout L;
    const long ny = (long)(d.ttm ? 5 : 3) * n;
    L.nk = (d.solver == SOLVER_DP45) ? 7 : (d.solver == SOLVER_AM12 ? 3 : 1);
    long o = 0;
    L.y = o;
    o += al(2 * ny);
    L.ystage = o;
    o += al(2 * ny);
    L.k = o;
    o += al(L.nk * ny);
    L.hd = -1;
    L.hd01 = -1;
    if (d.demag) {
        L.hd = o;
        o += al(3 * n);
        if (d.thermal && d.solver == SOLVER_DP45) {
            L.hd01 = o;
            o += al(6 * n);
        }
    }
    L.hth = -1;
    if (d.thermal && d.solver != SOLVER_EULER) {
        L.hth = o;
        o += al(3 * n);
    }
    L.d64 = -1;
    if (d.solver == SOLVER_AM12) {  // FP64 iterates w64, up64, uc64 (2 floats per double)
        L.d64 = o;
        o += al(3 * 2 * ny);
    }
    L.total = o;
    return L;
}

static void point_slot0(hsb_sim_s* S, const SlotLayout& L) {
    const long ny = (long)S->nch * S->n;
    float* a = S->arena;
    S->y[0] = a + L.y;
    S->y[1] = S->y[0] + ny;
    S->ystage[0] = a + L.ystage;
    S->ystage[1] = S->ystage[0] + ny;
    for (int j = 0; j < 8; j++) S->k[j] = (j < L.nk) ? a + L.k + j * ny : nullptr;
    S->hd = L.hd >= 0 ? a + L.hd : nullptr;
    S->hd01[0] = L.hd01 >= 0 ? a + L.hd01 : nullptr;
    S->hd01[1] = L.hd01 >= 0 ? S->hd01[0] + 3 * S->n : nullptr;
    S->hth = L.hth >= 0 ? a + L.hth : nullptr;
    for (int j = 0; j < 3; j++) S->y64[j] = L.d64 >= 0 ? (double*)(a + L.d64) + j * ny : nullptr;
    S->slot_stride = L.total;
}

static void free_sim(hsb_sim_s* S) {
    if (!S) return;
    drop_graphs(S);
    for (auto e : S->ev_pool) cudaEventDestroy(e);
    if (S->demag) hsb_demag_plan_destroy(S->demag);
    cudaFree(S->arena);
    cudaFree(S->phys_dev);
    cudaFree(S->X1b);
    cudaFree(S->kernb);
    if (S->spec) hsb_demag_spectrum_scratch_destroy(S->spec);
    if (S->done_ev) cudaEventDestroy(S->done_ev);
    cudaFree(S->msat_mask);
    cudaFree(S->lex_mask);
    cudaFree(S->sd);
    cudaFree(S->red);
    cudaFree(S->laser_tab);
    cudaFree(S->bext_tab);
    cudaFree(S->stage_f);
    cudaFree(S->stage_d);
    cudaFree(S->ckpt);
    cudaFree(S->ckpt_sd);
    cudaFree(S->hbuf);
    if (S->sd_host) cudaFreeHost(S->sd_host);
    if (S->stage_pin) cudaFreeHost(S->stage_pin);
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

// Launch-shape tuning of the stage kernel: the load-first kernel with 1, 2 and 4 cells per
// thread is timed on a representative stage of this simulation (a DP45 mid-attempt stage with
// four stage derivatives, or an RK stage with one), ungated, on the simulation's own (zeroed)
// buffers with its outputs in the stage-point scratch; the fastest is kept.  Every variant
// computes each cell with the same arithmetic.  Results are cached per geometry, channel
// count, physics flags, solver and slot count for the process.  The solver words must hold a
// valid dt; the caller re-uploads them afterwards (a timing launch may flag them).
static std::mutex g_stune_mu;
static std::map<std::vector<long>, int> g_stune;

static int tune_stage(hsb_sim_s* S) {
    S->stage_variant = -1;
    if (!hsb_stage_tunable(S->P)) return HSB_OK;
    const hsb_sim_desc& d = S->d;
    const std::vector<long> key = {S->P.N0, S->P.N1, S->P.N2, S->nch, d.llb, d.thermal, d.solver, d.demag, S->nslot};
    {
        std::lock_guard<std::mutex> lk(g_stune_mu);
        auto it = g_stune.find(key);
        if (it != g_stune.end()) {
            S->stage_variant = it->second;
            return HSB_OK;
        }
    }
    StageArgs A = empty_args();
    A.ungated = 1;
    A.ys = fixed(S->y[0]);
    A.hd = S->demag ? fixed(S->hd) : none();
    A.ytherm = fixed(S->y[0]);
    A.tfrac = 0.5f;
    A.kout = fixed(S->ystage[1]);
    A.kself_w = 1.0f;
    A.ynext = fixed(S->ystage[0]);
    A.ybase = fixed(S->y[0]);
    A.nk = (d.solver == SOLVER_DP45) ? 4 : 1;
    for (int j = 0; j < A.nk; j++) {
        A.kin[j] = fixed(S->k[j]);
        A.ck[j] = (d.solver == SOLVER_DP45) ? (float)DPA[5][j] : 0.5f;
    }
    A.cself = 0.1f;
    A.normalize = S->batched ? 1 : d.normalize;
    cudaEvent_t e0, e1;
    HSB_CUDA_TRY(cudaEventCreate(&e0));
    HSB_CUDA_TRY(cudaEventCreate(&e1));
    const int cand[3] = {1, 2, 4};
    int best = -1;
    float best_ms = 1e30f;
    int rc = HSB_OK;
    for (int c = 0; c < 3 && rc == HSB_OK; c++) {
        float acc = 0.f;
        for (int rep = 0; rep < 4 && rc == HSB_OK; rep++) {
            cudaEventRecord(e0, S->st);
            rc = S->batched ? hsb_launch_stage_batched(S->P, A, S->sd, S->bt, S->st, cand[c])
                            : hsb_launch_stage(S->P, A, S->sd, S->st, cand[c]);
            cudaEventRecord(e1, S->st);
            if (cudaEventSynchronize(e1) != cudaSuccess) rc = HSB_ERR_CUDA;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0) acc += ms;   // the first launch is a warm-up
        }
        if (rc == HSB_OK && acc < best_ms) {
            best_ms = acc;
            best = cand[c];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != HSB_OK) {
        hsb_set_error("stage-kernel tuning failed: %s", cudaGetErrorString(cudaGetLastError()));
        return rc;
    }
    S->stage_variant = best;
    std::lock_guard<std::mutex> lk(g_stune_mu);
    g_stune[key] = best;
    return HSB_OK;
}

// rk12 per-step error limits of the handle's equations (m, Te, Tl): maxerr[0] or rtol for
// m; a temperature limit <= 0 leaves that equation uncontrolled (+inf).
static void set_rk12_limits(hsb_sim_s* S) {
    const hsb_sim_desc& d = S->d;
    S->rk12_maxerr[0] = d.maxerr[0] > 0 ? d.maxerr[0] : d.rtol;
    for (int q = 1; q < 3; q++) S->rk12_maxerr[q] = d.maxerr[q] > 0 ? d.maxerr[q] : INFINITY;
    // am12: maxAbsError / maxRelError per equation, the reference's defaults 1e-4 / 1e-3
    // (solve_am01.go:395-398); bdf-euler: maxIterError 1e-5 and 3 sweeps
    // (solve_euler_backward.go:129-130)
    ImpLimits& L = S->imp;
    memset(&L, 0, sizeof(L));
    for (int q = 0; q < 3; q++) {
        L.abs_err[q] = d.maxerr[q] > 0 ? d.maxerr[q] : 1e-4;
        L.rel_err[q] = d.maxrelerr[q] > 0 ? d.maxrelerr[q] : 1e-3;
    }
    L.max_iter_err = d.maxerr[0] > 0 ? d.maxerr[0] : 1e-5;
    L.max_iter = d.max_iter > 0 ? d.max_iter : 3;
    L.neq = S->nch == 5 ? 3 : 1;
}

static int check_desc(const hsb_sim_desc& d, const char* who) {
    for (int a = 0; a < 3; a++) {
        if (d.size[a] < 1 || d.cellsize[a] <= 0 || d.pbc[a] < 0) {
            hsb_set_error("%s: bad size/cellsize/pbc on axis %d", who, a);
            return HSB_ERR_INVALID;
        }
    }
    if (d.solver < SOLVER_EULER || d.solver > SOLVER_BDF_EULER) {
        hsb_set_error("%s: unknown solver %d", who, d.solver);
        return HSB_ERR_INVALID;
    }
    if (!(d.dt > 0) || !(d.msat0T0 > 0) || (d.solver == SOLVER_DP45 && !(d.rtol > 0))) {
        hsb_set_error("%s: dt, msat0T0 (and rtol for DP45) must be positive", who);
        return HSB_ERR_INVALID;
    }
    if (d.solver == SOLVER_RK12 && !(d.maxerr[0] > 0) && !(d.rtol > 0)) {
        hsb_set_error("%s: rk12 needs maxerr[0] (or rtol) > 0", who);
        return HSB_ERR_INVALID;
    }
    for (int q = 0; q < 3; q++) {
        if (isnan(d.maxerr[q]) || isnan(d.maxrelerr[q])) {
            hsb_set_error("%s: maxerr[%d] / maxrelerr[%d] is not a number", who, q, q);
            return HSB_ERR_INVALID;
        }
    }
    if (d.demag_tensor != 0 && d.demag_tensor != 1) {
        hsb_set_error("%s: demag_tensor %d is neither Kernel_Arne (0) nor Newell (1)", who, d.demag_tensor);
        return HSB_ERR_INVALID;
    }
    if (d.solver == SOLVER_BDF_EULER && d.max_iter > 64) {
        hsb_set_error("%s: bdf-euler max_iter %d above 64", who, d.max_iter);
        return HSB_ERR_INVALID;
    }
    if (d.llb && !(d.tc > 0 && d.spin_j > 0 && d.n_spins > 0)) {
        hsb_set_error("%s: llb needs tc, spin_j and n_spins > 0", who);
        return HSB_ERR_INVALID;
    }
    if (d.ttm && !(d.gamma_e > 0 && d.c_l > 0)) {
        hsb_set_error("%s: ttm needs gamma_e > 0 and c_l > 0", who);
        return HSB_ERR_INVALID;
    }
    const long n = (long)d.size[0] * d.size[1] * d.size[2];
    if (n > (1L << 31) / 8) {
        hsb_set_error("%s: %ld cells exceed the 2^28 limit", who, n);
        return HSB_ERR_UNSUPPORTED;
    }
    if (d.laser_npts != 0) {
        if (d.laser_npts < 2 || d.laser_npts > 4096 || !d.laser_table) {
            hsb_set_error("%s: laser_npts must be 0 or 2..4096 with a table, got %d", who, d.laser_npts);
            return HSB_ERR_INVALID;
        }
        for (int i = 0; i < d.laser_npts; i++) {
            const double t = d.laser_table[2 * i], v = d.laser_table[2 * i + 1];
            if (!isfinite(t) || !isfinite(v) || (i > 0 && !(t > d.laser_table[2 * i - 2]))) {
                hsb_set_error("%s: laser table point %d is not finite or its time is not increasing", who, i);
                return HSB_ERR_INVALID;
            }
        }
    }
    if (d.bext_npts != 0) {
        if (d.bext_npts < 2 || d.bext_npts > 4096 || !d.bext_table) {
            hsb_set_error("%s: bext_npts must be 0 or 2..4096 with a table, got %d", who, d.bext_npts);
            return HSB_ERR_INVALID;
        }
        for (int i = 0; i < d.bext_npts; i++) {
            const double* r = d.bext_table + 4 * i;
            if (!isfinite(r[0]) || !isfinite(r[1]) || !isfinite(r[2]) || !isfinite(r[3]) ||
                (i > 0 && !(r[0] > r[-4]))) {
                hsb_set_error("%s: field table point %d is not finite or its time is not increasing", who, i);
                return HSB_ERR_INVALID;
            }
        }
    }
    return HSB_OK;
}

// Size of the descriptor as compiled into the library, for bindings to check their layout.
HSB_EXPORT int hsb_sim_desc_bytes(void) { return (int)sizeof(hsb_sim_desc); }

// Bytes of the device solver word a step call reads back (the per-step device-to-host read).
HSB_EXPORT int hsb_solver_word_bytes(void) { return (int)sizeof(HsbSolverDev); }

HSB_EXPORT int hsb_sim_create(const hsb_sim_desc* desc, hsb_sim_s** out) {
    if (!desc || !out) {
        hsb_set_error("hsb_sim_create: null argument");
        return HSB_ERR_INVALID;
    }
    *out = nullptr;
    const hsb_sim_desc& d = *desc;
    RC(check_desc(d, "hsb_sim_create"));
    const long n = (long)d.size[0] * d.size[1] * d.size[2];
    hsb_sim_s* S = new hsb_sim_s();
    S->d = d;
    S->d.laser_table = nullptr;    // the caller's arrays are copied to the device below
    S->d.bext_table = nullptr;
    S->n = n;
    S->nch = d.ttm ? 5 : 3;
    S->nslot = 1;
    STRY(cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking));
    if (d.laser_npts >= 2) {
        STRY(cudaMalloc(&S->laser_tab, sizeof(double2) * d.laser_npts));
        STRY(cudaMemcpy(S->laser_tab, d.laser_table, sizeof(double2) * d.laser_npts, cudaMemcpyHostToDevice));
    }
    if (d.bext_npts >= 2) {
        STRY(cudaMalloc(&S->bext_tab, sizeof(double) * 4 * d.bext_npts));
        STRY(cudaMemcpy(S->bext_tab, d.bext_table, sizeof(double) * 4 * d.bext_npts, cudaMemcpyHostToDevice));
    }
    const SlotLayout L = slot_layout(d, n);
    STRY(cudaMalloc(&S->arena, sizeof(float) * L.total));
    if (has_nonlocal(d)) STRY(cudaMalloc(&S->hbuf, sizeof(float) * 3 * n));
    STRY(cudaMemsetAsync(S->arena, 0, sizeof(float) * L.total, S->st));
    point_slot0(S, L);
    STRY(cudaMalloc(&S->sd, sizeof(HsbSolverDev)));
    STRY(cudaMallocHost(&S->sd_host, sizeof(HsbSolverDev)));
    STRY(cudaMalloc(&S->red, sizeof(double) * (RED_BLOCKS * 8 + 16) + 64));
    STRY(cudaMallocHost(&S->red_host, sizeof(double) * 16));
    STRY(cudaMemsetAsync(S->red, 0, sizeof(double) * (RED_BLOCKS * 8 + 16) + 64, S->st));
    if (d.demag) {
        int rc = hsb_demag_plan_create_tensor(d.size, d.cellsize, d.pbc, 6, d.demag_tensor, S->st, &S->demag);
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
    {
        const int rc = tune_stage(S);
        if (rc != HSB_OK) {
            free_sim(S);
            return rc;
        }
    }
    STRY(cudaMemcpyAsync(S->sd, S->sd_host, sizeof(HsbSolverDev), cudaMemcpyHostToDevice, S->st));
    STRY(cudaStreamSynchronize(S->st));
    // launch-bound grids batch more steps per graph launch
    S->graph_steps = n < 65536 ? 16 : (n < 1048576 ? 8 : 4);
    if (adaptive_solver(d.solver)) S->graph_steps = n < 65536 ? 8 : 4;
    set_rk12_limits(S);
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
    RC(plain_only(S, "hsb_sim_set"));
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
        drop_graphs(S);
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
    if (!S->sd_fresh) RC(get_sd(S));   // the current buffer index
    float* y = S->y[S->sd_host->cur];
    // one copy (a DMA straight from the caller's array when it is page-locked) and one
    // conversion, then a single synchronisation so the caller may reuse its array on return
    HSB_CUDA_TRY(cudaMemcpyAsync(S->stage_d, host, sizeof(double) * count, cudaMemcpyHostToDevice, S->st));
    k_d2f<<<hsb_grid_1d(count, 256), 256, 0, S->st>>>(S->stage_d, y + (long)first * S->n, count);
    HSB_CUDA_TRY(cudaGetLastError());
    S->initialized = false;
    if (S->sd_host->status || S->sd_host->nonfinite) {   // the flags described the state just replaced
        S->sd_host->status = 0;
        S->sd_host->nonfinite = 0u;
        RC(set_sd_fields(S));
    }
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    S->sd_fresh = true;    // the device words equal the host mirror
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_get(hsb_sim_s* S, const char* name, double* host, int64_t count) {
    RC(plain_only(S, "hsb_sim_get"));
    if (!S || !name || !host) {
        hsb_set_error("hsb_sim_get: null argument");
        return HSB_ERR_INVALID;
    }
    RC(stage_buffers(S, count));
    if (!S->sd_fresh) RC(get_sd(S));
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
        RC(hsb_launch_stage(S->P, A, S->sd, S->st, S->stage_variant));
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

// State transfer between the handle and caller-owned FP64 device arrays (SoA, program order;
// hotspin's gpu.Array layout, gpu/array.go:26-37), enqueued on the handle's stream and
// completed before return: the conversion kernels read or write the caller's array directly,
// with no host copy and no allocation.  name: "m", "Te", "Tl".
HSB_EXPORT int hsb_sim_set_device(hsb_sim_s* S, const char* name, const double* dev, int64_t count) {
    RC(plain_only(S, "hsb_sim_set_device"));
    if (!S || !name || !dev) {
        hsb_set_error("hsb_sim_set_device: null argument");
        return HSB_ERR_INVALID;
    }
    int first, nc;
    RC(channel_of(S, name, &first, &nc));
    if (count != (int64_t)nc * S->n) {
        hsb_set_error("hsb_sim_set_device(%s): expected %ld values, got %ld", name, (long)nc * S->n, (long)count);
        return HSB_ERR_INVALID;
    }
    if (!S->sd_fresh) RC(get_sd(S));
    float* y = S->y[S->sd_host->cur];
    k_d2f<<<hsb_grid_1d(count, 256), 256, 0, S->st>>>(dev, y + (long)first * S->n, count);
    HSB_CUDA_TRY(cudaGetLastError());
    S->initialized = false;
    if (S->sd_host->status || S->sd_host->nonfinite) {
        S->sd_host->status = 0;
        S->sd_host->nonfinite = 0u;
        RC(set_sd_fields(S));
    }
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    S->sd_fresh = true;
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_get_device(hsb_sim_s* S, const char* name, double* dev, int64_t count) {
    RC(plain_only(S, "hsb_sim_get_device"));
    if (!S || !name || !dev) {
        hsb_set_error("hsb_sim_get_device: null argument");
        return HSB_ERR_INVALID;
    }
    int first, nc;
    RC(channel_of(S, name, &first, &nc));
    if (count != (int64_t)nc * S->n) {
        hsb_set_error("hsb_sim_get_device(%s): expected %ld values, got %ld", name, (long)nc * S->n, (long)count);
        return HSB_ERR_INVALID;
    }
    if (!S->sd_fresh) RC(get_sd(S));
    const float* y = S->y[S->sd_host->cur];
    k_f2d<<<hsb_grid_1d(count, 256), 256, 0, S->st>>>(y + (long)first * S->n, dev, count);
    HSB_CUDA_TRY(cudaGetLastError());
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
    if (!adaptive_solver(S->d.solver)) {
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
    RC(plain_only(S, "hsb_sim_status"));
    if (!S) return HSB_ERR_INVALID;
    if (!S->sd_fresh) RC(get_sd(S));   // after a step call the words were just read back
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
    RC(plain_only(S, "hsb_sim_set_time"));
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
    k_energy<<<RED_BLOCKS, 256, 0, S->st>>>(S->P, y, hd, S->d.normalize, partial, counter, res, S->sd_host->t);
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
    RC(plain_only(S, "hsb_sim_profile"));
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

// Device-side checkpoint of the whole solver position: the current state (every channel, FP32
// as held) and the solver word (time, dt, counters, buffer selectors).  hsb_sim_restore puts
// both back and recomputes the first-stage data of the restored state, so a run from a
// restored checkpoint repeats the original continuation bit for bit (the thermal field's
// Philox counter is the step count, restored with it).  The checkpoint buffer is allocated
// by the first checkpoint.
HSB_EXPORT int hsb_sim_checkpoint(hsb_sim_s* S) {
    RC(plain_only(S, "hsb_sim_checkpoint"));
    if (!S) return HSB_ERR_INVALID;
    if (!S->ckpt) {
        HSB_CUDA_TRY(cudaMalloc(&S->ckpt, sizeof(float) * S->nch * S->n));
        HSB_CUDA_TRY(cudaMalloc(&S->ckpt_sd, sizeof(HsbSolverDev)));
    }
    if (!S->sd_fresh) RC(get_sd(S));
    HSB_CUDA_TRY(cudaMemcpyAsync(S->ckpt, S->y[S->sd_host->cur], sizeof(float) * S->nch * S->n,
                                 cudaMemcpyDeviceToDevice, S->st));
    HSB_CUDA_TRY(cudaMemcpyAsync(S->ckpt_sd, S->sd, sizeof(HsbSolverDev), cudaMemcpyDeviceToDevice, S->st));
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_restore(hsb_sim_s* S) {
    RC(plain_only(S, "hsb_sim_restore"));
    if (!S) return HSB_ERR_INVALID;
    if (!S->ckpt) {
        hsb_set_error("hsb_sim_restore: no checkpoint taken");
        return HSB_ERR_INVALID;
    }
    HSB_CUDA_TRY(cudaMemcpyAsync(S->sd, S->ckpt_sd, sizeof(HsbSolverDev), cudaMemcpyDeviceToDevice, S->st));
    RC(get_sd(S));
    HSB_CUDA_TRY(cudaMemcpyAsync(S->y[S->sd_host->cur], S->ckpt, sizeof(float) * S->nch * S->n,
                                 cudaMemcpyDeviceToDevice, S->st));
    S->initialized = false;
    RC(prepare(S));
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    S->sd_fresh = false;
    return HSB_OK;
}

// Kernels this handle has enqueued for stepping since its creation: the arming kernel of
// each step or run call, the first-stage preparation and every kernel node of each graph
// launch (gated attempts included).
HSB_EXPORT int hsb_sim_launch_count(hsb_sim_s* S, int64_t* n) {
    RC(plain_only(S, "hsb_sim_launch_count"));
    if (!S || !n) return HSB_ERR_INVALID;
    *n = S->launch_total;
    return HSB_OK;
}

// Kernel launches enqueued per attempt (per step for the fixed-step methods).
HSB_EXPORT int hsb_sim_launches_per_attempt(hsb_sim_s* S, int* n) {
    RC(plain_only(S, "hsb_sim_launches_per_attempt"));
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
    RC(plain_only(S, "hsb_sim_energy"));
    if (!S || !energy) return HSB_ERR_INVALID;
    double r[8];
    RC(reduce_terms(S, r));
    const double V = S->d.cellsize[0] * S->d.cellsize[1] * S->d.cellsize[2];
    const double pre = V * MU0 * S->d.msat0T0;
    *energy = pre * (r[0] + r[1] + r[2] + r[3] + r[4]);
    return HSB_OK;
}

// The energy's terms (J): out5 = Zeeman, exchange, demag, uniaxial anisotropy, MFA
// longitudinal field (their sum is hsb_sim_energy).
HSB_EXPORT int hsb_sim_energy_terms(hsb_sim_s* S, double* out5) {
    RC(plain_only(S, "hsb_sim_energy_terms"));
    if (!S || !out5) return HSB_ERR_INVALID;
    double r[8];
    RC(reduce_terms(S, r));
    const double V = S->d.cellsize[0] * S->d.cellsize[1] * S->d.cellsize[2];
    const double pre = V * MU0 * S->d.msat0T0;
    for (int q = 0; q < 5; q++) out5[q] = pre * r[q];
    return HSB_OK;
}

// max over cells of |v| for a [3][n] FP32 field, into the FP64 word at `out` (non-negative
// doubles order like their bit patterns)
__global__ void k_maxnorm3(const float* __restrict__ v, long n, unsigned long long* out) {
    double m = 0.0;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double x = v[i], y = v[n + i], z = v[2 * n + i];
        m = fmax(m, sqrt(x * x + y * y + z * z));
    }
    m = warp_max_d(m);
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// Maximum over cells of |gamma (m x H_eff)| (1/s) of the current state, H_eff with every field
// term of the right-hand side (thermal field of the current step included).  hotspin's
// maxtorque module: max |torque| (mod_maxtorque.go, MaxNormUpdater update_reduce.go:132-142).
HSB_EXPORT int hsb_sim_max_torque(hsb_sim_s* S, double* out) {
    RC(plain_only(S, "hsb_sim_max_torque"));
    if (!S || !out) return HSB_ERR_INVALID;
    RC(get_sd(S));
    float* y = S->y[S->sd_host->cur];
    float* hd = nullptr;
    if (S->demag) {
        RC(run_demag(S, y, -1, S->hd, -1, false));
        hd = S->hd;
    }
    StageArgs A = empty_args();
    A.ungated = 1;
    A.torque_only = 1;
    A.ys = fixed(y);
    A.hd = fixed(hd);
    A.ytherm = fixed(y);
    A.kout = fixed(S->ystage[1]);
    A.kself_w = 1.0f;
    S->sd_fresh = false;
    RC(hsb_launch_stage_generic(S->P, A, S->sd, S->st));
    double* word = S->red + RED_BLOCKS * 8 + 10;
    HSB_CUDA_TRY(cudaMemsetAsync(word, 0, sizeof(double), S->st));
    k_maxnorm3<<<hsb_grid_1d(S->n, 256), 256, 0, S->st>>>(S->ystage[1], S->n, (unsigned long long*)word);
    HSB_CUDA_TRY(cudaGetLastError());
    HSB_CUDA_TRY(cudaMemcpyAsync(S->red_host, word, sizeof(double), cudaMemcpyDeviceToHost, S->st));
    HSB_CUDA_TRY(cudaStreamSynchronize(S->st));
    *out = S->red_host[0];
    S->initialized = false;    // the stage buffer used here may hold first-stage data
    return HSB_OK;
}

HSB_EXPORT int hsb_sim_average_m(hsb_sim_s* S, double* avg3) {
    RC(plain_only(S, "hsb_sim_average_m"));
    if (!S || !avg3) return HSB_ERR_INVALID;
    double r[8];
    RC(reduce_terms(S, r));
    for (int c = 0; c < 3; c++) avg3[c] = r[5 + c] / (double)S->n;
    return HSB_OK;
}

// ------------------------------------------------------------------ batches of simulations
// A batch ("size class") advances up to nslot independent simulations of one grid size with
// the same kernels: each slot has its own arena (state, stages, demag field), physics
// (HsbPhys) and solver word (HsbSolverDev), and every launch covers all slots (blockIdx.z).
// Slots are admitted and read back while the others keep running; a slot that reached its
// end time, or is empty, costs one early-returning block per launch.  The class fixes the
// grid size, boundary conditions, solver and its tolerance, channel count (two-temperature
// model or not) and demag on/off; everything else (Ms0, lex, cell size and with it the demag
// kernel spectrum, damping, field, anisotropy, temperature, LLB or LLG, seed) is per slot.
static int batch_check_class(const hsb_sim_desc& d, int32_t nslot, const char* who) {
    RC(check_desc(d, who));
    if (d.laser_npts != 0 || d.bext_npts != 0) {
        hsb_set_error("%s: pointwise laser profiles and field tables are not supported in batches", who);
        return HSB_ERR_UNSUPPORTED;
    }
    if (nslot < 1 || nslot > 65535) {
        hsb_set_error("%s: nslot = %d outside [1, 65535]", who, nslot);
        return HSB_ERR_INVALID;
    }
    if (d.size[2] % 4 != 0) {
        hsb_set_error("%s: batched kernels need the a2 (user x) size to be a multiple of 4, got %d", who,
                      d.size[2]);
        return HSB_ERR_UNSUPPORTED;
    }
    if (has_llbar02(d) || has_nonlocal(d)) {
        hsb_set_error("%s: the second-order and non-local relaxation terms run on the single-simulation handle only",
                      who);
        return HSB_ERR_UNSUPPORTED;
    }
    for (int a = 0; a < 3; a++) {
        const int n = d.size[a];
        if (d.demag && (n & (n - 1)) != 0) {
            hsb_set_error("%s: batches with demag need sizes that are powers of two, got %d on axis %d", who, n, a);
            return HSB_ERR_UNSUPPORTED;
        }
    }
    return HSB_OK;
}

// Device bytes a batch of `nslot` slots of this class holds (arenas, demag spectra and plan,
// solver words, physics, reduction scratch); host-pinned staging is not counted.
HSB_EXPORT int hsb_batch_footprint(const hsb_sim_desc* cls, int32_t nslot, int64_t* bytes) {
    if (!cls || !bytes) return HSB_ERR_INVALID;
    RC(batch_check_class(*cls, nslot, "hsb_batch_footprint"));
    const hsb_sim_desc& d = *cls;
    const long n = (long)d.size[0] * d.size[1] * d.size[2];
    const SlotLayout L = slot_layout(d, n);
    int64_t b = (int64_t)nslot * L.total * (int64_t)sizeof(float);
    b += (int64_t)nslot * (sizeof(HsbSolverDev) + sizeof(HsbPhys));
    b += sizeof(double) * (RED_BLOCKS * 8 + 16) + 64;
    if (d.demag) {
        int Lg[3];
        for (int a = 0; a < 3; a++) Lg[a] = (d.size[a] > 1 && d.pbc[a] == 0) ? 2 * d.size[a] : d.size[a];
        const long C2 = Lg[2] / 2 + 1;
        const long x1 = 3L * d.size[0] * C2 * d.size[1] * 8;
        b += (int64_t)(nslot + 1) * x1;                                   // batch spectra + the plan's own
        b += (int64_t)(nslot + 1) * C2 * (Lg[1] / 2 + 1) * (Lg[0] / 2 + 1) * 6 * 4;  // kernel spectra
        int twL = Lg[0] > Lg[1] ? Lg[0] : Lg[1];
        if (Lg[2] > twL) twL = Lg[2];
        b += (int64_t)twL * 8;
        // FP64 scratch of the per-slot kernel evaluation
        const int64_t nfold = (int64_t)(Lg[0] / 2 + 1) * (Lg[1] / 2 + 1) * (Lg[2] / 2 + 1);
        b += 8 * 6 * nfold + 8 * (int64_t)Lg[0] * Lg[1] * Lg[2] + 16 * (int64_t)Lg[0] * C2 * Lg[1] + 16 * twL + 256;
    }
    *bytes = b;
    return HSB_OK;
}

HSB_EXPORT int hsb_batch_create(const hsb_sim_desc* cls, int32_t nslot, hsb_sim_s** out) {
    if (!cls || !out) {
        hsb_set_error("hsb_batch_create: null argument");
        return HSB_ERR_INVALID;
    }
    *out = nullptr;
    const hsb_sim_desc& d = *cls;
    RC(batch_check_class(d, nslot, "hsb_batch_create"));
    const long n = (long)d.size[0] * d.size[1] * d.size[2];
    hsb_sim_s* S = new hsb_sim_s();
    S->d = d;
    S->n = n;
    S->nch = d.ttm ? 5 : 3;
    S->nslot = nslot;
    S->batched = true;
    STRY(cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking));
    const SlotLayout L = slot_layout(d, n);
    STRY(cudaMalloc(&S->arena, sizeof(float) * L.total * nslot));
    STRY(cudaMemsetAsync(S->arena, 0, sizeof(float) * L.total * nslot, S->st));
    point_slot0(S, L);
    STRY(cudaMalloc(&S->sd, sizeof(HsbSolverDev) * nslot));
    STRY(cudaMallocHost(&S->sd_host, sizeof(HsbSolverDev) * nslot));
    memset(S->sd_host, 0, sizeof(HsbSolverDev) * nslot);
    STRY(cudaMemsetAsync(S->sd, 0, sizeof(HsbSolverDev) * nslot, S->st));
    STRY(cudaMalloc(&S->phys_dev, sizeof(HsbPhys) * nslot));
    fill_phys(S);
    S->phys_h.assign(nslot, S->P);
    STRY(cudaMemcpyAsync(S->phys_dev, S->phys_h.data(), sizeof(HsbPhys) * nslot, cudaMemcpyHostToDevice, S->st));
    STRY(cudaMalloc(&S->red, sizeof(double) * (RED_BLOCKS * 8 + 16) + 64));
    STRY(cudaMallocHost(&S->red_host, sizeof(double) * 16));
    STRY(cudaEventCreateWithFlags(&S->done_ev, cudaEventDisableTiming));
    if (d.demag) {
        int rc = hsb_demag_plan_create_tensor(d.size, d.cellsize, d.pbc, 6, d.demag_tensor, S->st, &S->demag);
        if (rc != HSB_OK) {
            free_sim(S);
            return rc;
        }
        const long xb = hsb_demag_x1_bytes(S->demag);
        if (xb == 0) {
            hsb_set_error("hsb_batch_create: no batched FFT kernels for padded size (%d, %d, %d)",
                          d.size[0], d.size[1], d.size[2]);
            free_sim(S);
            return HSB_ERR_UNSUPPORTED;
        }
        STRY(cudaMalloc(&S->X1b, xb * nslot));
        S->x1_stride = xb / (long)sizeof(float2);
        S->kern_floats = hsb_demag_kern_floats(S->demag);
        STRY(cudaMalloc(&S->kernb, sizeof(float) * S->kern_floats * nslot));
        rc = hsb_demag_spectrum_scratch_create(S->demag, &S->spec);
        if (rc != HSB_OK) {
            free_sim(S);
            return rc;
        }
    }
    S->bt.stride = S->slot_stride;
    S->bt.phys = S->phys_dev;
    S->bt.nslot = nslot;
    const long tot = n * nslot;
    S->graph_steps = tot < 65536 ? 16 : (tot < 1048576 ? 8 : 4);
    if (adaptive_solver(d.solver)) S->graph_steps = tot < 65536 ? 8 : 4;
    set_rk12_limits(S);
    S->initialized = true;
    {
        // tune with a valid dt in every solver word, then clear them again (all slots empty)
        for (int k = 0; k < nslot; k++) S->sd_host[k].dt = d.dt;
        STRY(cudaMemcpyAsync(S->sd, S->sd_host, sizeof(HsbSolverDev) * nslot, cudaMemcpyHostToDevice, S->st));
        const int rc = tune_stage(S);
        if (rc != HSB_OK) {
            free_sim(S);
            return rc;
        }
        memset(S->sd_host, 0, sizeof(HsbSolverDev) * nslot);
        STRY(cudaMemsetAsync(S->sd, 0, sizeof(HsbSolverDev) * nslot, S->st));
    }
    STRY(cudaStreamSynchronize(S->st));
    *out = S;
    return HSB_OK;
}

static int batch_slot_ok(hsb_sim_s* B, int32_t slot, const char* who) {
    if (!B || !B->batched) {
        hsb_set_error("%s: not a batch handle", who);
        return HSB_ERR_INVALID;
    }
    if (slot < 0 || slot >= B->nslot) {
        hsb_set_error("%s: slot %d outside [0, %d)", who, slot, B->nslot);
        return HSB_ERR_INVALID;
    }
    return HSB_OK;
}

// Load one simulation into a free slot: its descriptor (same class), initial magnetization
// (3 x ncell FP64, program order; the temperatures of a two-temperature class start at the
// descriptor's bath temperature) and end time.  Enqueued on the batch's stream; the slot
// starts stepping with the next hsb_batch_launch.  Host arrays may be reused on return.
HSB_EXPORT int hsb_batch_admit(hsb_sim_s* B, int32_t slot, const hsb_sim_desc* desc, const double* m,
                               double t_stop) {
    RC(batch_slot_ok(B, slot, "hsb_batch_admit"));
    if (!desc || !m || !(t_stop > 0)) {
        hsb_set_error("hsb_batch_admit: need a descriptor, m and t_stop > 0");
        return HSB_ERR_INVALID;
    }
    const hsb_sim_desc& d = *desc;
    const hsb_sim_desc& c = B->d;
    RC(check_desc(d, "hsb_batch_admit"));
    if (d.laser_npts != 0 || d.bext_npts != 0) {
        hsb_set_error("hsb_batch_admit: pointwise laser profiles and field tables are not supported in batches");
        return HSB_ERR_UNSUPPORTED;
    }
    for (int a = 0; a < 3; a++) {
        if (d.size[a] != c.size[a] || d.pbc[a] != c.pbc[a]) {
            hsb_set_error("hsb_batch_admit: grid size / boundaries differ from the class");
            return HSB_ERR_INVALID;
        }
    }
    if (has_llbar02(d) || has_nonlocal(d)) {
        hsb_set_error("hsb_batch_admit: the second-order and non-local relaxation terms run on the single-simulation "
                      "handle only");
        return HSB_ERR_UNSUPPORTED;
    }
    if (d.solver != c.solver || d.ttm != c.ttm || d.demag != c.demag || (d.thermal && !c.thermal) ||
        d.demag_tensor != c.demag_tensor ||
        (adaptive_solver(c.solver) && d.rtol != c.rtol) ||
        (c.solver >= SOLVER_RK12 &&
         (d.maxerr[0] != c.maxerr[0] || d.maxerr[1] != c.maxerr[1] || d.maxerr[2] != c.maxerr[2] ||
          d.maxrelerr[0] != c.maxrelerr[0] || d.maxrelerr[1] != c.maxrelerr[1] || d.maxrelerr[2] != c.maxrelerr[2] ||
          d.max_iter != c.max_iter))) {
        hsb_set_error("hsb_batch_admit: solver, tolerance, two-temperature model, demag or thermal field differ "
                      "from the class");
        return HSB_ERR_INVALID;
    }
    const long n = B->n;
    const long ny = (long)B->nch * n;
    // pinned staging per slot: a copy from pageable memory may wait for the running graphs
    static_assert(sizeof(HsbPhys) % 8 == 0 && sizeof(HsbSolverDev) % 8 == 0, "staging layout");
    const size_t per = sizeof(float) * ny + sizeof(HsbPhys) + sizeof(HsbSolverDev);
    if (!B->stage_pin) HSB_CUDA_TRY(cudaMallocHost(&B->stage_pin, per * B->nslot));
    unsigned char* base = (unsigned char*)B->stage_pin + per * slot;
    float* hy = (float*)base;
    HsbPhys* hp = (HsbPhys*)(base + sizeof(float) * ny);
    HsbSolverDev* hs = (HsbSolverDev*)(base + sizeof(float) * ny + sizeof(HsbPhys));
    // the previous use of this staging (an earlier admission into this slot) completed
    // before that slot could finish, so it is free to overwrite
    for (long i = 0; i < 3 * n; i++) hy[i] = (float)m[i];
    for (long i = 3 * n; i < ny; i++) hy[i] = (float)d.temperature;
    phys_from_desc(d, B->nch, n, *hp);
    B->phys_h[slot] = *hp;
    memset(hs, 0, sizeof(HsbSolverDev));
    hs->dt = d.dt < t_stop ? d.dt : t_stop;
    hs->mindt = d.mindt > 0 ? d.mindt : 1e-22;
    hs->maxdt = d.maxdt > 0 ? d.maxdt : 1e-9;
    hs->step_stop = -1;
    hs->t_stop = t_stop;
    hs->prep = 1;
    float* y0 = B->y[0] + (long)slot * B->slot_stride;
    HSB_CUDA_TRY(cudaMemcpyAsync(y0, hy, sizeof(float) * ny, cudaMemcpyHostToDevice, B->st));
    HSB_CUDA_TRY(cudaMemcpyAsync(B->phys_dev + slot, hp, sizeof(HsbPhys), cudaMemcpyHostToDevice, B->st));
    HSB_CUDA_TRY(cudaMemcpyAsync(B->sd + slot, hs, sizeof(HsbSolverDev), cudaMemcpyHostToDevice, B->st));
    if (B->demag) {
        // this slot's own demag tensor (the reference evaluates Kernel_Arne in physical units,
        // so cells of equal shape but different size can round to different quadratures)
        RC(hsb_demag_spectrum_enqueue(B->demag, d.cellsize, 6, B->spec, nullptr,
                                      B->kernb + (long)slot * B->kern_floats, B->st));
    }
    B->nprep++;
    return HSB_OK;
}

// First-stage data of the newly admitted slots (DP45: demag of y0 with a thermal field,
// else k1 = f(y0)), gated on their `prep` word, then switch them to active.
static int prepare_slots(hsb_sim_s* B) {
    if (!B->nprep) return HSB_OK;
    B->prep_mode = true;
    int rc = HSB_OK;
    if (B->d.solver == SOLVER_DP45) {
        if (B->d.thermal) {
            if (B->demag) rc = run_demag(B, nullptr, 0, nullptr, 0);
        } else {
            float* hd = B->demag ? B->hd : nullptr;
            rc = run_demag(B, nullptr, 0, hd, -1);
            if (rc == HSB_OK) {
                StageArgs A = empty_args();
                A.ys = pair(B->y[0], B->y[1], SEL_CUR);
                A.hd = fixed(hd);
                A.ytherm = A.ys;
                A.kout = pair(B->k[0], B->k[6], SEL_K1);
                A.kself_w = 1.0f;
                rc = L_stage(B, A);
            }
        }
    }
    B->prep_mode = false;
    RC(rc);
    RC(hsb_launch_activate_prepped(B->sd, B->nslot, B->st));
    B->nprep = 0;
    return HSB_OK;
}

// Enqueue `graphs` launches of the class graph (each a fixed number of attempts for every
// slot), then a copy of all solver words to the host; hsb_batch_poll reports completion.
HSB_EXPORT int hsb_batch_launch(hsb_sim_s* B, int32_t graphs) {
    if (!B || !B->batched || graphs < 0) {
        hsb_set_error("hsb_batch_launch: bad argument");
        return HSB_ERR_INVALID;
    }
    RC(prepare_slots(B));
    RC(build_graph(B));
    B->sd_fresh = false;
    for (int g = 0; g < graphs; g++) HSB_CUDA_TRY(cudaGraphLaunch(B->graph, B->st));
    HSB_CUDA_TRY(cudaMemcpyAsync(B->sd_host, B->sd, sizeof(HsbSolverDev) * B->nslot, cudaMemcpyDeviceToHost,
                                 B->st));
    HSB_CUDA_TRY(cudaEventRecord(B->done_ev, B->st));
    B->launched = true;
    return HSB_OK;
}

// *done = 1 once everything enqueued by the last hsb_batch_launch has finished.
HSB_EXPORT int hsb_batch_poll(hsb_sim_s* B, int32_t* done) {
    if (!B || !B->batched || !done) return HSB_ERR_INVALID;
    if (!B->launched) {
        *done = 1;
        return HSB_OK;
    }
    cudaError_t e = cudaEventQuery(B->done_ev);
    if (e == cudaErrorNotReady) {
        *done = 0;
        return HSB_OK;
    }
    HSB_CUDA_TRY(e);
    *done = 1;
    return HSB_OK;
}

// Solver state of a slot as of the end of the last launch (waits for it).
HSB_EXPORT int hsb_batch_slot_status(hsb_sim_s* B, int32_t slot, double* t, double* dt, int64_t* steps,
                                     int64_t* attempts, int64_t* rejects, int32_t* status, int32_t* active) {
    RC(batch_slot_ok(B, slot, "hsb_batch_slot_status"));
    if (B->launched) HSB_CUDA_TRY(cudaEventSynchronize(B->done_ev));
    const HsbSolverDev* h = B->sd_host + slot;
    if (t) *t = h->t;
    if (dt) *dt = h->dt;
    if (steps) *steps = h->step;
    if (attempts) *attempts = h->attempts;
    if (rejects) *rejects = h->rejects;
    if (status) *status = h->status;
    if (active) *active = h->active | h->prep;
    return HSB_OK;
}

// Copy a slot's current m / Te / Tl to the host (FP64, program order); waits for the stream.
HSB_EXPORT int hsb_batch_slot_get(hsb_sim_s* B, int32_t slot, const char* name, double* host, int64_t count) {
    RC(batch_slot_ok(B, slot, "hsb_batch_slot_get"));
    if (!name || !host) {
        hsb_set_error("hsb_batch_slot_get: null argument");
        return HSB_ERR_INVALID;
    }
    int first, nc;
    RC(channel_of(B, name, &first, &nc));
    if (count != (int64_t)nc * B->n) {
        hsb_set_error("hsb_batch_slot_get(%s): expected %ld values, got %ld", name, (long)nc * B->n, (long)count);
        return HSB_ERR_INVALID;
    }
    RC(stage_buffers(B, count));
    HsbSolverDev h;
    HSB_CUDA_TRY(cudaMemcpyAsync(&h, B->sd + slot, sizeof(HsbSolverDev), cudaMemcpyDeviceToHost, B->st));
    HSB_CUDA_TRY(cudaStreamSynchronize(B->st));
    const float* src = B->y[h.cur] + (long)slot * B->slot_stride + (long)first * B->n;
    k_f2d<<<hsb_grid_1d(count, 256), 256, 0, B->st>>>(src, B->stage_d, count);
    HSB_CUDA_TRY(cudaGetLastError());
    HSB_CUDA_TRY(cudaMemcpyAsync(host, B->stage_d, sizeof(double) * count, cudaMemcpyDeviceToHost, B->st));
    HSB_CUDA_TRY(cudaStreamSynchronize(B->st));
    return HSB_OK;
}

// Stop a slot (it stays inactive until the next admission into it).
HSB_EXPORT int hsb_batch_release(hsb_sim_s* B, int32_t slot) {
    RC(batch_slot_ok(B, slot, "hsb_batch_release"));
    HSB_CUDA_TRY(cudaMemsetAsync(&B->sd[slot].active, 0, sizeof(int), B->st));
    HSB_CUDA_TRY(cudaMemsetAsync(&B->sd[slot].prep, 0, sizeof(int), B->st));
    HSB_CUDA_TRY(cudaStreamSynchronize(B->st));
    return HSB_OK;
}

HSB_EXPORT int hsb_batch_destroy(hsb_sim_s* B) { return hsb_sim_destroy(B); }

// Slots, attempts of every slot per class-graph launch, cells per slot.
// Stage-kernel variant a handle (simulation or batch) runs: picked by the tuning at creation,
// or forced by hsb_set_stage_variant.
HSB_EXPORT int hsb_stage_variant_of(hsb_sim_s* S) {
    if (!S) return -1;
    const int forced = hsb_set_stage_variant(-2);   // reads the forced value (-2 changes nothing)
    return forced >= 0 ? forced : (S->stage_variant >= 0 ? S->stage_variant : 2);
}

HSB_EXPORT int hsb_batch_info(hsb_sim_s* B, int32_t* nslot, int32_t* attempts_per_graph, int64_t* ncell) {
    if (!B || !B->batched) return HSB_ERR_INVALID;
    if (nslot) *nslot = B->nslot;
    if (attempts_per_graph) *attempts_per_graph = B->graph_steps;
    if (ncell) *ncell = B->n;
    return HSB_OK;
}
