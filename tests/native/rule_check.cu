// Host build of the device step-control rules (test support, compiled by the CPU tests with
// nvcc as host code): the same inline functions the controller kernels run, driven from
// Python through ctypes so the rules can be checked against the oracle without a GPU.
#include "hsb_llg.cuh"

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
    X(prevsel) X(eq) X(rhs_due) X(alpha_max) X(nonfinite)

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
