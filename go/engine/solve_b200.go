//  Solver modules that hand hotspin's time step to the B200 simulation handle
//  (go/gpu/hsb200.go -> libhsb200.so).  Drop into src/hotspin-core/engine/; scripts select them
//  with load('solver/rk45') etc. like any other solver.  The module builds one handle from the
//  engine's quantities on the first step (the same quantities and module names the script
//  API mirror hotspin_b200/api.py reads), moves the state in and out of the engine's own device
//  arrays with no host copy, and keeps the engine's t, dt and step in step with the handle.
//  Not compiled in this repository: no Go toolchain here.

package engine

import (
	"fmt"

	. "hotspin-core/common"
	"hotspin-core/gpu"
)

// B200Solver advances the whole step (right-hand side, demag, integrator, step control) on
// the device; the engine's updaters for m (and Te, Tp) are bypassed while it runs.
type B200Solver struct {
	kind   int
	sim    *gpu.HsbSim
	minDt  *Quant
	maxDt  *Quant
	maxErr *Quant // m_maxerror: DP45 relative tolerance, rk12 maxError of m
}

func loadB200(kind int) func(e *Engine) {
	return func(e *Engine) {
		s := &B200Solver{kind: kind}
		s.minDt = e.AddNewQuant("mindt", SCALAR, VALUE, Unit("s"), "Minimum time step")
		s.minDt.SetScalar(1e-22)
		s.maxDt = e.AddNewQuant("maxdt", SCALAR, VALUE, Unit("s"), "Maximum time step")
		s.maxDt.SetScalar(1e-12)
		s.maxErr = e.AddNewQuant("m_maxerror", SCALAR, VALUE, Unit(""), "Error tolerance per step for m")
		s.maxErr.SetScalar(1e-5)
		e.SetSolver(s)
	}
}

func init() {
	RegisterModule("solver/rk45", "Dormand-Prince 4(5), fused FP32 kernels and device step control (B200)",
		loadB200(gpu.HsbDP45))
	RegisterModule("solver/rk4", "Classic Runge-Kutta 4, fused FP32 kernels (B200)", loadB200(gpu.HsbRK4))
	RegisterModule("solver/rk12-b200", "hotspin's adaptive Heun solver on the device (B200)", loadB200(gpu.HsbRK12))
	RegisterModule("solver/am12-b200", "hotspin's adaptive Adams-Moulton 1-2 solver on the device (B200)",
		loadB200(gpu.HsbAM12))
}

func scalarOr(e *Engine, name string, def float64) float64 {
	if e.HasQuant(name) {
		return e.Quant(name).Scalar()
	}
	return def
}

func vec3Or(e *Engine, name string, def [3]float64) [3]float64 {
	if !e.HasQuant(name) {
		return def
	}
	m := e.Quant(name).Multiplier()
	return [3]float64{m[0], m[1], m[2]}
}

// desc reads the module graph the script built into a handle descriptor.
func (s *B200Solver) desc(e *Engine) gpu.HsbDesc {
	var d gpu.HsbDesc
	size, cs, pbc := e.GridSize(), e.CellSize(), e.Periodic()
	for i := 0; i < 3; i++ {
		d.Size[i], d.CellSize[i], d.PBC[i] = size[i], cs[i], pbc[i]
	}
	d.Msat0T0 = scalarOr(e, "msat0T0", 0)
	if e.HasModule("exchange6") {
		d.Lex = scalarOr(e, "lex", 0)
	}
	d.GammaLL = scalarOr(e, "γ_LL", 2.211e5)
	if e.HasModule("llbar/damping/nonconservative/00/local") {
		d.Alpha = vec3Or(e, "α", [3]float64{})
	}
	if e.HasModule("llbar/damping/nonconservative/02/local") {
		d.MuPar = vec3Or(e, "μ∥", [3]float64{})
	}
	if e.HasModule("llbar/damping/conservative/02/local") {
		d.MuPerp = vec3Or(e, "μ⊥", [3]float64{})
	}
	if e.HasModule("llbar/damping/nonconservative/00/nonlocal") {
		d.AlphaE = vec3Or(e, "αₑ", [3]float64{})
	}
	if e.HasModule("anisotropy/uniaxial") {
		d.Ku = scalarOr(e, "Ku", 0)
		d.AnisU = vec3Or(e, "anisU", [3]float64{0, 0, 1})
	}
	if e.HasModule("zeeman") {
		d.BExt = vec3Or(e, "B_ext", [3]float64{})
	}
	d.Demag = e.HasModule("demag")
	d.Normalize = e.HasModule("normalizer")
	d.LLB = e.HasModule("mfa/longfield")
	d.Tc, d.SpinJ, d.NSpins = scalarOr(e, "Tc", 0), scalarOr(e, "J", 0.5), scalarOr(e, "n", 0)
	d.Temp = scalarOr(e, "Temp", 0)
	d.Thermal = e.HasModule("temperature/brown")
	d.Seed = uint64(scalarOr(e, "Therm_seed", 0))
	d.CutoffDt = scalarOr(e, "cutoff_dt", 0)
	d.TTM = e.HasModule("temperature/ETM")
	if d.TTM {
		d.GammaE = scalarOr(e, "γ", 0) * scalarOr(e, "n", 0) / Na
		d.Cl, d.Gep = scalarOr(e, "Cp", 0), scalarOr(e, "Ge-p", 0)
		if e.HasModule("temperature/ETM/diffusion") {
			d.Ke = scalarOr(e, "Ke", 0)
		}
	}
	d.Solver = s.kind
	d.Dt = scalarOr(e, "dt", 1e-15)
	d.Rtol = s.maxErr.Scalar()
	d.MinDt, d.MaxDt = s.minDt.Scalar(), s.maxDt.Scalar()
	d.MaxErr[0] = s.maxErr.Scalar()
	return d
}

func (s *B200Solver) check(err error) {
	if err != nil {
		panic(InputErr(fmt.Sprint("B200 solver: ", err)))
	}
}

// Step takes one accepted step (one fixed step for rk4) on the device.
func (s *B200Solver) Step() {
	e := GetEngine()
	if s.sim == nil {
		d := s.desc(e)
		sim, err := gpu.NewHsbSim(&d)
		s.check(err)
		s.sim = sim
		s.check(s.sim.SetFromArray("m", e.Quant("m").Array()))
		if e.HasQuant("Te") && d.TTM {
			s.check(s.sim.SetFromArray("Te", e.Quant("Te").Array()))
			s.check(s.sim.SetFromArray("Tl", e.Quant("Tp").Array()))
		}
		s.check(s.sim.SetTime(e.time.Scalar(), e.dt.Scalar()))
	}
	s.check(s.sim.Step(1))
	st, err := s.sim.Status()
	s.check(err)
	m := e.Quant("m")
	s.check(s.sim.CopyToArray("m", m.Array()))
	m.Invalidate()
	if e.HasQuant("Te") && e.HasModule("temperature/ETM") {
		s.check(s.sim.CopyToArray("Te", e.Quant("Te").Array()))
		s.check(s.sim.CopyToArray("Tl", e.Quant("Tp").Array()))
		e.Quant("Te").Invalidate()
		e.Quant("Tp").Invalidate()
	}
	e.time.SetScalar(st.T)
	e.dt.SetScalar(st.Dt)
	e.step.SetScalar(e.step.Scalar() + 1)
}

func (s *B200Solver) Dependencies() (children, parents []string) {
	children = []string{"dt", "step", "t"}
	parents = []string{"dt", "mindt", "maxdt", "m_maxerror"}
	return
}
