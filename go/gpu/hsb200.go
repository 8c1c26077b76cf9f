//  Bindings of the B200 simulation handle (libhsb200.so, include/hotspin_b200.h) for
//  hotspin's Go engine.  Drop into src/hotspin-core/gpu/ beside libhotspin.go; the library and
//  its header must be on the cgo search paths (CGO_CFLAGS=-I<repo>/include,
//  CGO_LDFLAGS=-L<repo>/hotspin_b200).  Not compiled in this repository: no Go toolchain here.

package gpu

/*
#cgo LDFLAGS: -lhsb200
#include <stdlib.h>
#include "hotspin_b200.h"
*/
import "C"

import (
	"fmt"
	"unsafe"

	cu "cuda/driver"
)

// Solver choices of the handle (HSB_SOLVER_* in hotspin_b200.h).
const (
	HsbEuler    = 0
	HsbHeun     = 1
	HsbRK4      = 2
	HsbDP45     = 3
	HsbRK12     = 4
	HsbAM12     = 5
	HsbBDFEuler = 6
)

// HsbDesc mirrors hsb_sim_desc: every length, vector and size in program order (the engine's
// internal order), physical values in SI units as the engine's multipliers hold them.
type HsbDesc struct {
	Size       [3]int
	PBC        [3]int
	CellSize   [3]float64
	Msat0T0    float64
	Lex        float64
	GammaLL    float64
	Alpha      [3]float64
	Ku         float64
	AnisU      [3]float64
	BExt       [3]float64 // tesla
	Demag      bool
	Normalize  bool
	LLB        bool
	Tc         float64
	SpinJ      float64
	NSpins     float64
	Temp       float64
	Thermal    bool
	Seed       uint64
	CutoffDt   float64
	TTM        bool
	GammaE     float64
	Cl         float64
	Gep        float64
	Ke, Kl     float64
	LaserP0    float64
	LaserT0    float64
	LaserFWHM  float64
	LaserSigma float64
	Solver     int
	Dt         float64
	Rtol       float64
	MinDt      float64
	MaxDt      float64
	MaxErr     [3]float64 // rk12 maxError / am12 maxAbsError / bdf-euler maxIterError (m, Te, Tl)
	MaxRelErr  [3]float64 // am12 maxRelError
	MaxIter    int
	Newell     bool       // the FP64 Newell tensor instead of Kernel_Arne
	MuPar      [3]float64 // llbar/damping/nonconservative/02/local (0: not loaded)
	MuPerp     [3]float64 // llbar/damping/conservative/02/local (0: not loaded)
	AlphaE     [3]float64 // llbar/damping/nonconservative/00/nonlocal (0: not loaded)
}

func b2i(b bool) C.int32_t {
	if b {
		return 1
	}
	return 0
}

func (d *HsbDesc) c() C.hsb_sim_desc {
	var c C.hsb_sim_desc
	for i := 0; i < 3; i++ {
		c.size[i] = C.int32_t(d.Size[i])
		c.pbc[i] = C.int32_t(d.PBC[i])
		c.cellsize[i] = C.double(d.CellSize[i])
		c.alpha[i] = C.double(d.Alpha[i])
		c.anis_u[i] = C.double(d.AnisU[i])
		c.b_ext[i] = C.double(d.BExt[i])
		c.maxerr[i] = C.double(d.MaxErr[i])
		c.maxrelerr[i] = C.double(d.MaxRelErr[i])
		c.mu_par[i] = C.double(d.MuPar[i])
		c.mu_perp[i] = C.double(d.MuPerp[i])
		c.alpha_e[i] = C.double(d.AlphaE[i])
	}
	c.msat0T0, c.lex, c.gamma_ll, c.ku = C.double(d.Msat0T0), C.double(d.Lex), C.double(d.GammaLL), C.double(d.Ku)
	c.demag, c.normalize, c.llb = b2i(d.Demag), b2i(d.Normalize), b2i(d.LLB)
	c.tc, c.spin_j, c.n_spins, c.temperature = C.double(d.Tc), C.double(d.SpinJ), C.double(d.NSpins), C.double(d.Temp)
	c.thermal, c.seed, c.cutoff_dt = b2i(d.Thermal), C.uint64_t(d.Seed), C.double(d.CutoffDt)
	c.ttm, c.gamma_e, c.c_l, c.g_ep = b2i(d.TTM), C.double(d.GammaE), C.double(d.Cl), C.double(d.Gep)
	c.k_e, c.k_l = C.double(d.Ke), C.double(d.Kl)
	c.laser_p0, c.laser_t0, c.laser_fwhm, c.laser_sigma = C.double(d.LaserP0), C.double(d.LaserT0),
		C.double(d.LaserFWHM), C.double(d.LaserSigma)
	c.solver, c.dt, c.rtol = C.int32_t(d.Solver), C.double(d.Dt), C.double(d.Rtol)
	c.mindt, c.maxdt = C.double(d.MinDt), C.double(d.MaxDt)
	c.max_iter = C.int32_t(d.MaxIter)
	if d.Newell {
		c.demag_tensor = 1
	}
	return c
}

// HsbSim is one device-resident simulation (FP32 state, fused stage kernels, device-side step
// control, CUDA graphs).
type HsbSim struct {
	h C.hsb_sim
}

func hsbErr(rc C.int, what string) error {
	if rc == 0 {
		return nil
	}
	return fmt.Errorf("%s: %s (status %d)", what, C.GoString(C.hsb_last_error()), int(rc))
}

// NewHsbSim builds the handle on the current CUDA device (the engine's context).
func NewHsbSim(d *HsbDesc) (*HsbSim, error) {
	if int(C.hsb_sim_desc_bytes()) != int(unsafe.Sizeof(C.hsb_sim_desc{})) {
		return nil, fmt.Errorf("hsb_sim_desc layout differs between the header and libhsb200.so")
	}
	cd := d.c()
	s := new(HsbSim)
	if err := hsbErr(C.hsb_sim_create(&cd, &s.h), "hsb_sim_create"); err != nil {
		return nil, err
	}
	return s, nil
}

func (s *HsbSim) Free() {
	if s.h != nil {
		C.hsb_sim_destroy(s.h)
		s.h = nil
	}
}

func cstr(name string) *C.char { return C.CString(name) }

// SetFromArray loads m, Te or Tl from an engine array (FP64 on the device), without a host copy.
func (s *HsbSim) SetFromArray(name string, a *Array) error {
	n := cstr(name)
	defer C.free(unsafe.Pointer(n))
	p := (*C.double)(unsafe.Pointer(uintptr(a.Pointer())))
	return hsbErr(C.hsb_sim_set_device(s.h, n, p, C.int64_t(a.Len())), "hsb_sim_set_device("+name+")")
}

// CopyToArray writes m, Te or Tl into an engine array (FP64 on the device).
func (s *HsbSim) CopyToArray(name string, a *Array) error {
	n := cstr(name)
	defer C.free(unsafe.Pointer(n))
	p := (*C.double)(unsafe.Pointer(uintptr(a.Pointer())))
	return hsbErr(C.hsb_sim_get_device(s.h, n, p, C.int64_t(a.Len())), "hsb_sim_get_device("+name+")")
}

// Step advances n accepted steps (adaptive solvers) or n fixed steps.
func (s *HsbSim) Step(n int) error { return hsbErr(C.hsb_sim_step(s.h, C.int64_t(n)), "hsb_sim_step") }

// RunUntil advances to time t.
func (s *HsbSim) RunUntil(t float64) error {
	return hsbErr(C.hsb_sim_run_until(s.h, C.double(t)), "hsb_sim_run_until")
}

// SetTime sets the solver's time and, when dt > 0, its step.
func (s *HsbSim) SetTime(t, dt float64) error {
	return hsbErr(C.hsb_sim_set_time(s.h, C.double(t), C.double(dt)), "hsb_sim_set_time")
}

// HsbStatus is the solver word the step call read back.
type HsbStatus struct {
	T, Dt, Err               float64
	Steps, Attempts, Rejects int64
	Flags                    int
}

func (s *HsbSim) Status() (HsbStatus, error) {
	var t, dt, e C.double
	var st, at, rj C.int64_t
	var fl C.int32_t
	err := hsbErr(C.hsb_sim_status(s.h, &t, &dt, &st, &at, &rj, &e, &fl), "hsb_sim_status")
	return HsbStatus{float64(t), float64(dt), float64(e), int64(st), int64(at), int64(rj), int(fl)}, err
}

// Energy is the total energy (J) with the device's compensated FP64 reduction.
func (s *HsbSim) Energy() (float64, error) {
	var e C.double
	err := hsbErr(C.hsb_sim_energy(s.h, &e), "hsb_sim_energy")
	return float64(e), err
}

// Stream is the handle's CUDA stream (work on the engine's arrays can be ordered after it).
func (s *HsbSim) Stream() cu.Stream { return cu.Stream(uintptr(C.hsb_sim_stream(s.h))) }
