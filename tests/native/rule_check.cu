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
