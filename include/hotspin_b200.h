/*
 * hotspin_b200 -- B200 (sm_100a) implementation of the hotspin solver hot path.
 *
 * Two C-ABI surfaces, both exported by libhsb200.so:
 *
 *  1. Drop-in FP64 kernels with the names, argument order and meaning of hotspin's
 *     libhotspin.h (generated from src/libhotspin/*.h by src/libhotspin/Makefile:35-38).
 *     The Go layer (src/hotspin-core/gpu/libhotspin.go, wrap_*.go) binds them unchanged
 *     through cgo; they are declared in include/libhotspin_dropin.h.
 *
 *  2. The simulation handle API below: one call advances the whole per-step right-hand
 *     side and integrator (exchange, anisotropy, Zeeman, demag, MFA longitudinal field,
 *     Philox thermal field, two-temperature model; Euler / Heun / RK4 / Dormand-Prince 4(5))
 *     with FP32 state resident on the GPU.  It replaces the sequence that hotspin's
 *     engine drives per step (engine/engine.go:473-508 Engine.Step -> Solver.Step ->
 *     Quant.Update graph walk -> libhotspin kernels + cuFFT + host syncs).
 *
 * Conventions (reference engine/api.go:41-62, common/index.go:68-113): arrays are
 * structure-of-arrays in *program order* -- shape (N0, N1, N2), N2 fastest = the user's x --
 * and vector fields are component-major with component 0 = program X (user z).  All
 * host-facing values are double.  Every function returns an int status (HSB_OK = 0);
 * hsb_last_error() describes the last failure of the calling thread.  Nothing aborts.
 *
 * Dormand-Prince step control (device side, no host round trip):
 *   err = max( max_i |e_m,i| / rtol , max_i |e_T,i| / (rtol max(|T0_i|, |T1_i|)) )
 *   accept when err <= 1 (or dt == mindt); dt *= clamp(0.9 err^-1/5, 0.2, 5 | 1 on reject),
 *   clamped to [mindt, maxdt] and to the requested stop time.
 */
#ifndef HOTSPIN_B200_H
#define HOTSPIN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    HSB_OK = 0,
    HSB_ERR_INVALID = 1,
    HSB_ERR_CUDA = 2,
    HSB_ERR_NOMEM = 3,
    HSB_ERR_UNSUPPORTED = 4,
    HSB_ERR_NONFINITE = 5,
    HSB_ERR_SOLVER = 6
};

enum {
    HSB_SOLVER_EULER = 0,     /* solver/euler  (solve_euler.go:22-50)                  */
    HSB_SOLVER_HEUN = 1,      /* solver/heun   (solve_heun.go:27-79)                   */
    HSB_SOLVER_RK4 = 2,       /* classic RK4 (no reference counterpart)               */
    HSB_SOLVER_DP45 = 3,      /* Dormand-Prince 4(5) (no reference counterpart)       */
    HSB_SOLVER_RK12 = 4,      /* solver/rk12   (solve_rk12.go:91-214)                  */
    HSB_SOLVER_AM12 = 5,      /* solver/am12   (solve_am01.go:45-318)                  */
    HSB_SOLVER_BDF_EULER = 6  /* solver/bdf-euler (solve_euler_backward.go:29-91)      */
};

/* Simulation description.  Replaces the module graph a hotspin script builds with
 * load(...)/setv(...): exchange6, anisotropy/uniaxial, zeeman, demag, llbar +
 * llbar/torque + llbar/damping/nonconservative/00/local, normalizer, mfa/longfield,
 * temperature/brown, temperature/ETM + PTM + E-P + Drude + ETM/diffusion, solver/<x>. */
typedef struct hsb_sim_desc {
    int32_t size[3];        /* N0, N1, N2 (program order)                          */
    int32_t pbc[3];         /* periodic images per axis, 0 = open                  */
    double cellsize[3];     /* m, program order                                    */
    double msat0T0;         /* Ms(T=0), A/m   (msat0T0 multiplier)                 */
    double lex;             /* exchange length multiplier, m (lex)                 */
    double gamma_ll;        /* m/As  (gamma_LL)                                    */
    double alpha[3];        /* lambda diagonal, program components (alpha)         */
    double ku;              /* J/m^3 (Ku)                                          */
    double anis_u[3];       /* program components (anisU)                          */
    double b_ext[3];        /* tesla, program components (B_ext)                   */
    int32_t demag;          /* 1: demag module loaded                               */
    int32_t normalize;      /* 1: normalizer module on m (LLG mode)                 */
    int32_t llb;            /* 1: mfa/longfield added to H_eff                      */
    double tc;              /* K                                                   */
    double spin_j;          /* J                                                   */
    double n_spins;         /* 1/m^3                                               */
    double temperature;     /* K, bath temperature when ttm == 0                   */
    int32_t thermal;        /* 1: temperature/brown thermal field (mu = alpha)      */
    uint64_t seed;          /* Philox key                                          */
    double cutoff_dt;       /* s                                                   */
    int32_t ttm;            /* 1: two-temperature model (Te, Tl state channels)     */
    double gamma_e;         /* J/(m^3 K^2): Ce = gamma_e Te                        */
    double c_l;             /* J/(m^3 K)                                           */
    double g_ep;            /* W/(m^3 K)                                           */
    double k_e, k_l;        /* W/(m K)                                             */
    double laser_p0;        /* W/m^3 peak absorbed power                           */
    double laser_t0;        /* s, pulse centre                                     */
    double laser_fwhm;      /* s                                                   */
    double laser_sigma;     /* m, lateral Gaussian spot; 0 = uniform               */
    int32_t solver;         /* HSB_SOLVER_*                                        */
    double dt;              /* initial / fixed time step, s                        */
    double rtol;            /* DP45 tolerance                                      */
    double mindt, maxdt;    /* DP45 / RK12 step bounds                             */
    /* Pointwise laser time profile (hotspin's PointwiseOf quantities,
     * engine/update_pointwiseof.go:31-98): laser_npts >= 2 pairs (t_i in s, strictly
     * increasing; factor_i) as 2 * laser_npts doubles; the absorbed power is laser_p0 times
     * their piecewise-linear interpolation, zero outside [t_0, t_last] (the reference stops
     * with an error past the last point).  laser_npts = 0: the Gaussian pulse above.  Copied
     * at creation; not available in batches.                                            */
    const double* laser_table;
    int32_t laser_npts;     /* 0 or 2..4096                                          */
    /* Pointwise applied field: bext_npts >= 2 rows (t_i in s, strictly increasing; Bx, By,
     * Bz in tesla, program components) as 4 * bext_npts doubles, interpolated linearly at
     * each stage's time and zero outside [t_0, t_last]; replaces b_ext.  bext_npts = 0: the
     * constant b_ext.  Copied at creation; not available in batches.                     */
    const double* bext_table;
    int32_t bext_npts;      /* 0 or 2..4096                                          */
    /* Per-equation tolerances (m, Te, Tl) of hotspin's own solvers:
     *  HSB_SOLVER_RK12: maxerr = <q>_maxError, the largest dt max |k1 - k0| per step;
     *    maxerr[0] <= 0 takes rtol, a temperature entry <= 0 leaves that equation
     *    uncontrolled.
     *  HSB_SOLVER_AM12: maxerr = <q>_maxAbsError, maxrelerr = <q>_maxRelError
     *    (defaults when <= 0: 1e-4 and 1e-3, solve_am01.go:395-398).
     *  HSB_SOLVER_BDF_EULER: maxerr[0] = the iterator error of every equation (default
     *    1e-5), max_iter = sweeps per equation (default 3, at most 64;
     *    solve_euler_backward.go:129-130).                                                */
    double maxerr[3];
    double maxrelerr[3];
    int32_t max_iter;
    int32_t demag_tensor;   /* HSB_DEMAG_ARNE (default, the reference's) or HSB_DEMAG_NEWELL */
    /* Second-order local relaxation terms of the LLBar equation, diagonal tensors in program
     * components (0 = module not loaded): mu_par = mu_par of
     * llbar/damping/nonconservative/02/local, gamma diag(mu_par) (m . H) m
     * (llbar-local02nc.cu:11-73); mu_perp = mu_perp of llbar/damping/conservative/02/local,
     * gamma m x (diag(mu_perp) (H x m)) (llbar-local02c.cu:11-69).  Uniform values only; the
     * single-simulation handle runs them (batches refuse them). */
    double mu_par[3];
    double mu_perp[3];
    /* alpha_e of llbar/damping/nonconservative/00/nonlocal (llbar-nonlocal00nc.cu:11-205):
     * -gamma diag(alpha_e) lap(H_eff), uniform, program components (0 = not loaded); the
     * single-simulation handle runs it with one extra pass per right-hand side. */
    double alpha_e[3];
} hsb_sim_desc;

typedef struct hsb_sim_s* hsb_sim;

const char* hsb_last_error(void);
void hsb_clear_error(void);
int hsb_version(void);
/* sizeof(hsb_sim_desc) as compiled into the library (no reference counterpart): a binding
 * compares it with its own mirror of the struct. */
int hsb_sim_desc_bytes(void);
/* Bytes of the device solver word that each step call reads back (no reference
 * counterpart): the per-step device-to-host read of a stepping loop. */
int hsb_solver_word_bytes(void);
/* CRC-64 (ISO polynomial, Go hash/crc64 convention) that seals a #dump002 frame
 * (dump/writer.go:46-76); host function, no GPU needed.  Used by hotspin_b200.dump. */
uint64_t hsb_crc64_iso(const void* data, int64_t n);

/* Allocate device state, build the demag kernel (FP64 Kernel_Arne on the GPU), set the
 * initial state m = (0,0,1), Te = Tl = temperature.  Runs on the current CUDA device. */
int hsb_sim_create(const hsb_sim_desc* desc, hsb_sim* out);
int hsb_sim_destroy(hsb_sim sim);

/* Host <-> device state transfer in double.  name: "m" (3 N values), "Te", "Tl" (N),
 * "msat_mask", "lex_mask" (N; set before stepping, NULL host pointer clears the mask),
 * read-only "H_demag" (3 N, A/m, of the current state), "k" (3 N or 5 N, the right-hand
 * side of the current state).  Setting a state quantity clears the status flags, which
 * describe the state it replaces.  A page-locked host array is copied by DMA directly. */
int hsb_sim_set(hsb_sim sim, const char* name, const double* host, int64_t count);
int hsb_sim_get(hsb_sim sim, const char* name, double* host, int64_t count);
/* The same for caller-owned FP64 device arrays (hotspin's gpu.Array layout, SoA program order;
 * no reference counterpart): "m", "Te", "Tl" converted on the device, no host copy, no
 * allocation; completed before return. */
int hsb_sim_set_device(hsb_sim sim, const char* name, const double* dev, int64_t count);
int hsb_sim_get_device(hsb_sim sim, const char* name, double* dev, int64_t count);

/* Advance `nsteps` accepted steps / up to time t.  Asynchronous on the handle's stream
 * except for the periodic completion checks of the adaptive solver. */
int hsb_sim_step(hsb_sim sim, int64_t nsteps);
int hsb_sim_run_until(hsb_sim sim, double t);
int hsb_sim_sync(hsb_sim sim);

/* Solver bookkeeping: time, current dt, accepted steps, attempts, rejected attempts,
 * last error norm, status bits (1: non-finite state, 2: a step was taken at mindt without
 * meeting the tolerance, 4: an RK12 / AM12 step still failed after 10 retries or an
 * implicit iteration did not converge, where hotspin panics; the run stops with
 * HSB_ERR_SOLVER). */
int hsb_sim_status(hsb_sim sim, double* t, double* dt, int64_t* steps, int64_t* attempts,
                   int64_t* rejects, double* err, int32_t* status);
int hsb_sim_set_time(hsb_sim sim, double t, double dt);

/* Total energy (J) as hotspin's micromag/energy module sums it (mod_energy.go:20-66),
 * FP64 compensated reduction on the device; and the average of m (3 values). */
int hsb_sim_energy(hsb_sim sim, double* energy);
int hsb_sim_average_m(hsb_sim sim, double* avg3);
/* The energy's terms (J): Zeeman, exchange, demag, uniaxial anisotropy, MFA longitudinal
 * field (mod_energy.go:20-66 per term; their sum is hsb_sim_energy). */
int hsb_sim_energy_terms(hsb_sim sim, double* out5);
/* Maximum over cells of |gamma_LL (m x H_eff)| (1/s) of the current state, reduced on the device:
 * hotspin's maxtorque module (modules/mod_maxtorque.go, MaxNormUpdater
 * engine/update_reduce.go:132-142) applied to the LLBar torque (llbar-torque.cu:11-45). */
int hsb_sim_max_torque(hsb_sim sim, double* out);

/* Device time of one attempt by kernel family (eager launches between CUDA events on the
 * handle's stream; each profiled attempt is a real step): out[0] fused RHS+stage kernels,
 * out[1] demag x-pass, out[2] demag y/z pass(es), out[3] demag inverse x-pass,
 * out[4] combine / step control, out[5] launches per attempt, out[6] accepted steps. */
int hsb_sim_profile(hsb_sim sim, int reps, double* out7);
int hsb_sim_launches_per_attempt(hsb_sim sim, int* n);
/* Checkpoint / resume on the device (hotspin saves and reloads state through dump files,
 * dump/writer.go:46-76; this keeps the FP32 state and the solver word in device memory):
 * hsb_sim_checkpoint copies the current state and solver position (t, dt, counters) aside;
 * hsb_sim_restore puts them back, after which stepping repeats the original continuation
 * bit for bit (the thermal field's counter is restored with the step count). */
int hsb_sim_checkpoint(hsb_sim sim);
int hsb_sim_restore(hsb_sim sim);
/* Kernels the handle has enqueued for stepping since creation (no reference counterpart):
 * the arming kernel of each step / run call, the first-stage preparation and every kernel
 * node of each graph launch, gated attempts included. */
int hsb_sim_launch_count(hsb_sim sim, int64_t* n);

/* Mean-field tables in FP64 on the GPU: T_i = Tc i/(npts-1), m_e(T_i) by the Ridders
 * iteration of brillouinKern (src/libhotspin/brillouin.cu:88-138) and the reduced
 * longitudinal susceptibility chi(T_i) of kappaKern (kappa.cu:15-61) with unit masks
 * (times Ms0^2 mu0 / (n kB) for the physical value, mod_kappa.go:76-89).
 * hsb_mfa_equilibrium interpolates a 1024-point table. */
int hsb_mfa_table(double Tc, double J, int npts, double* T, double* me, double* chi);
int hsb_mfa_equilibrium(double T, double Tc, double J, double* me);

/* Average of a caller-owned FP32 SoA magnetization (3 x ncell, device memory) into
 * caller-owned device memory avg3[3], enqueued on `stream`; the library allocates nothing.
 * No counterpart in the reference: it is the device-finished FP64 reduction of
 * hsb_sim_average_m for callers that own all device memory (as hotspin's Go layer does),
 * with its scratch in a fixed static device array (about 7 KB per GPU, held until exit).
 * ncell must be in [1, 2^28]; larger sizes are rejected.  Every call resolves the scratch
 * address in the current context; the first call on a device also loads the library's
 * device code there (make it before any stream capture).  All calls share the
 * scratch: calls that overlap on the GPU race and must be serialised. */
int hsb_average_m_noalloc(const float* m, int64_t ncell, double* avg3, void* stream);

/* Stage-kernel variants (no reference counterpart): 0 = four cells per thread, loads as
 * needed; 1 / 2 / 4 = load-first kernel with 1 / 2 / 4 cells per thread.  Every simulation and
 * batch times variants 1, 2 and 4 on its own buffers at creation and keeps the fastest
 * (cached per geometry and physics flags for the process).  hsb_set_stage_variant forces one
 * variant for launches built afterwards (tuning sweeps); -1 returns to the per-handle choice;
 * other values change nothing.  Returns the previous forced value (-1 = none).  All variants
 * compute each cell identically up to FP32 rounding order. */
int hsb_set_stage_variant(int v);
/* The variant a handle (simulation or batch) runs. */
int hsb_stage_variant_of(hsb_sim sim);

/* The handle's CUDA stream (cudaStream_t) for callers that interleave their own work. */
void* hsb_sim_stream(hsb_sim sim);

/* ---- Batches of simulations (no reference counterpart: hotspin runs one simulation per
 * process, engine/engine.go).  A batch is a size class: up to nslot independent simulations
 * of one grid size, boundary conditions, solver (and tolerance) and channel count, advanced
 * together by the same kernels (one grid plane per slot) and CUDA graph.  Per slot: Ms0, lex,
 * cell size (each slot gets the demag kernel of its own cells, evaluated at admission), damping,
 * field, anisotropy, temperature, LLB/LLG (llb, normalize), thermal field and seed.  Not supported in batches: masks, a2 sizes that
 * are not multiples of 4, padded sizes outside the fast FFT kernels.
 *
 * A slot's trajectory is independent of what the other slots hold: every kernel reads and
 * writes only its own slot's arena and solver word.  A serving loop admits requests into free
 * slots (hsb_batch_admit), launches (hsb_batch_launch, asynchronous), polls for completion
 * (hsb_batch_poll), reads each slot's progress (hsb_batch_slot_status; active = 0 once its
 * end time is reached) and collects results (hsb_batch_slot_get).  One host thread per batch
 * handle; different handles may be driven from one thread and overlap on the GPU. */
typedef struct hsb_batch_s* hsb_batch;
/* Device bytes of a batch with `nslot` slots of the class `cls` (admission by footprint). */
int hsb_batch_footprint(const hsb_sim_desc* cls, int32_t nslot, int64_t* bytes);
int hsb_batch_create(const hsb_sim_desc* cls, int32_t nslot, hsb_batch* out);
int hsb_batch_destroy(hsb_batch b);
/* nslot, attempts of every slot per graph launch, cells per slot */
int hsb_batch_info(hsb_batch b, int32_t* nslot, int32_t* attempts_per_graph, int64_t* ncell);
/* Load a simulation into a free slot: descriptor of the same class, initial m (3 x ncell
 * FP64, program order), end time t_stop (s).  Enqueued; host arrays may be reused at once. */
int hsb_batch_admit(hsb_batch b, int32_t slot, const hsb_sim_desc* desc, const double* m, double t_stop);
/* Prepare newly admitted slots, enqueue `graphs` launches of the class graph and a copy of
 * every slot's solver state to the host.  Returns without waiting. */
int hsb_batch_launch(hsb_batch b, int32_t graphs);
/* *done = 1 when everything the last hsb_batch_launch enqueued has finished. */
int hsb_batch_poll(hsb_batch b, int32_t* done);
/* A slot's solver state as of the end of the last launch (waits for it). */
int hsb_batch_slot_status(hsb_batch b, int32_t slot, double* t, double* dt, int64_t* steps,
                          int64_t* attempts, int64_t* rejects, int32_t* status, int32_t* active);
/* A slot's m / Te / Tl (FP64, program order). */
int hsb_batch_slot_get(hsb_batch b, int32_t slot, const char* name, double* host, int64_t count);
/* Stop a slot until its next admission. */
int hsb_batch_release(hsb_batch b, int32_t slot);

/* Demag convolution on caller-owned FP32 device arrays (SoA [3][N0][N1][N2]):
 * H (A/m) = Ms0 * K (*) (m * mask); mask may be NULL.  The plan builds the Kernel_Arne
 * tensor (kernel_magnetostatic.go:25-241) on the GPU in FP64 (accuracy as the reference,
 * normally 6).  A periodic axis must be a power of two; an open axis of any size is padded to
 * twice its size or, when that is not a power of two, embedded in a grid of next_pow2(N) cells
 * (vacuum beyond the N cells), which gives the same field. */
typedef struct hsb_demag_plan_s* hsb_demag_plan;
int hsb_demag_plan_create(const int* size, const double* cellsize, const int* pbc, int accuracy,
                          void* stream, hsb_demag_plan* out);
/* The same with a choice of tensor: HSB_DEMAG_ARNE (hotspin's Kernel_Arne, as above) or
 * HSB_DEMAG_NEWELL (no reference counterpart: the closed-form cell-averaged tensor of Newell,
 * Williams and Dunlop (1993) in FP64 on the GPU, near field by its second differences and far
 * field by the multipole expansion through sixth order; it differs from Kernel_Arne by that
 * quadrature's error, about 1e-3 of the largest entry at accuracy 6). */
enum { HSB_DEMAG_ARNE = 0, HSB_DEMAG_NEWELL = 1 };
int hsb_demag_plan_create_tensor(const int* size, const double* cellsize, const int* pbc, int accuracy,
                                 int tensor, void* stream, hsb_demag_plan* out);
int hsb_demag_plan_destroy(hsb_demag_plan plan);
int hsb_demag_plan_info(hsb_demag_plan plan, int* logic3, int* fused, double* kern_max_imag);
int hsb_demag_field(hsb_demag_plan plan, const float* m, const float* mask, double msat0T0,
                    float* H, void* stream);
/* Device time of the three phases of one convolution (ms[0] x-pass, ms[1] y/z, ms[2]
 * inverse x), CUDA events on `stream`, averaged over reps after a warm-up. */
int hsb_demag_profile(hsb_demag_plan plan, const float* m, const float* mask, double msat0T0, float* H,
                      void* stream, int reps, double* ms3);
/* Folded FP32 kernel spectrum, layout [kx][k1][k0][6] (XX YY ZZ YZ XZ XY). */
int hsb_demag_kernel_copy(hsb_demag_plan plan, float* host_out, long count);

/* FP64 3-D real FFT plan with the semantics of hotspin's FFTPlanX (gpu/fftplanX.go:76-104), the
 * implementation behind hotspin's FFTInterface registry (fftPlans, gpu/fftinterface.go:16-42):
 *   hsb_fft_forward: the data block (N0, N1, N2) zero-padded to the logic size (L0, L1, L2),
 *     then the unnormalised real-to-complex transform into (L0, L1, L2/2 + 1) complex values
 *     (L2 + 2 doubles per row: cuFFT's packed layout);
 *   hsb_fft_inverse: the unnormalised complex-to-real transform of such a spectrum, cropped to
 *     the data block (the spectrum itself is left unchanged).
 * Device pointers, program order.  Each call runs on the plan's stream and synchronises it, as
 * FFTPlanX does.  Logic sizes: powers of two, at least the data size, at most 4096, the last
 * at least 2. */
typedef struct hsb_fft_plan_s* hsb_fft_plan;
int hsb_fft_plan_create(const int* data_size, const int* logic_size, void* stream, hsb_fft_plan* out);
int hsb_fft_forward(hsb_fft_plan plan, const double* in, double* out);
int hsb_fft_inverse(hsb_fft_plan plan, const double* in, double* out);
int hsb_fft_plan_destroy(hsb_fft_plan plan);

#ifdef __cplusplus
}
#endif
#endif
