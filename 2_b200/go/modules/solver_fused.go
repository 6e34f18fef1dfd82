// Package modules (addition to mumax/2's src/mumax/modules): solver modules that step the
// engine's magnetisation with the fused B200 path of libmm_b200.so.  "solver/rk23" and
// "solver/rk45" are new adaptive solvers (the reference has RK12 as its adaptive one);
// "solver/rk12fused" is the reference's RK12 semantics on the fused kernels.  They
// register like the reference's solvers (engine.RegisterModule, solve_rk12.go:87) and
// implement engine.Solver (solver.go:14-17).
//
// Not built in this repository's image (there is no Go toolchain); written against the
// reference's engine API (module.go, engine.go, quant.go) and checked by reading only.
package modules

import (
	. "mumax/common"
	. "mumax/engine"
	"mumax/gpu"
)

func init() {
	RegisterModule("solver/rk23", "Adaptive Bogacki-Shampine 3(2) on the fused B200 path", func(e *Engine) { loadFused(e, gpu.RK23) })
	RegisterModule("solver/rk45", "Adaptive Dormand-Prince 5(4) on the fused B200 path", func(e *Engine) { loadFused(e, gpu.RK45) })
	RegisterModule("solver/rk12fused", "Adaptive Heun (RK12 semantics) on the fused B200 path", func(e *Engine) { loadFused(e, gpu.RK12) })
}

type fusedSolver struct {
	kind  int
	plan  *gpu.FusedPlan
	dirty bool // m was changed by the script since the last step
}

func loadFused(e *Engine, kind int) {
	s := &fusedSolver{kind: kind, dirty: true}
	e.AddNewQuant("mindt", SCALAR, VALUE, Unit("s"), "Minimum time step").SetScalar(1e-38)
	e.AddNewQuant("maxdt", SCALAR, VALUE, Unit("s"), "Maximum time step").SetScalar(1e38)
	e.AddNewQuant("badsteps", SCALAR, VALUE, Unit(""), "Number of time steps that had to be re-done")
	e.AddNewQuant("m_maxerror", SCALAR, VALUE, Unit(""), "Maximum error per step").SetScalar(1e-5)
	e.AddNewQuant("m_error", SCALAR, VALUE, Unit(""), "Error/step estimate")
	e.AddNewQuant("m_peakerror", SCALAR, VALUE, Unit(""), "All-time maximum error/step")
	e.SetSolver(s)
}

// problem collects the loaded modules' parameters from the engine's quantities (their
// multipliers; masks are passed through as device arrays).
func (s *fusedSolver) problem(e *Engine) *gpu.FusedProblem {
	f := new(gpu.FusedProblem)
	size, cell, per := e.GridSize(), e.CellSize(), e.Periodic()
	for i := 0; i < 3; i++ {
		f.Size[i], f.CellSize[i], f.Periodic[i] = size[i], cell[i], per[i]
	}
	has := func(name string) bool { return e.HasQuant(name) }
	f.Demag, f.Exchange = has("B"), has("H_ex")
	f.Anis, f.Zeeman, f.Thermal = has("H_anis"), has("B_ext"), has("H_therm")
	f.Msat = e.Quant("Msat").Multiplier()[0]
	f.Gamma = e.Quant("gamma").Scalar()
	f.Alpha = e.Quant("alpha").Multiplier()[0]
	if f.Exchange {
		f.Aex = e.Quant("Aex").Multiplier()[0]
	}
	if f.Anis {
		f.Ku = e.Quant("Ku").Multiplier()[0]
		u := e.Quant("anisU").Multiplier()
		f.AnisU = [3]float64{u[0], u[1], u[2]}
	}
	if f.Zeeman {
		b := e.Quant("B_ext").Multiplier()
		f.Bext = [3]float64{b[0], b[1], b[2]}
	}
	if !e.Quant("Msat").Array().IsNil() {
		f.MsatMask = e.Quant("Msat").Array()
	}
	return f
}

func (s *fusedSolver) Step() {
	e := GetEngine()
	m := e.Quant("m")
	if s.plan == nil {
		p, err := gpu.NewFusedPlan(s.problem(e))
		if err != nil {
			panic(InputErr(err.Error()))
		}
		s.plan = p
		dt := e.Quant("dt").Scalar()
		if err := p.Solver(s.kind, dt, e.Quant("mindt").Scalar(), e.Quant("maxdt").Scalar(),
			e.Quant("m_maxerror").Scalar()); err != nil {
			panic(InputErr(err.Error()))
		}
	}
	if s.dirty {
		if err := s.plan.SetState(m.Array()); err != nil {
			panic(Bug(err.Error()))
		}
		s.dirty = false
	}
	if err := s.plan.Step(); err != nil {
		panic(Bug(err.Error()))
	}
	if err := s.plan.GetState(m.Array()); err != nil {
		panic(Bug(err.Error()))
	}
	m.Invalidate()
	st, err := s.plan.Stats()
	if err != nil {
		panic(Bug(err.Error()))
	}
	e.Quant("t").SetScalar(st.T)
	e.Quant("dt").SetScalar(st.Dt)
	e.Quant("m_error").SetScalar(st.Err)
	e.Quant("m_peakerror").SetScalar(st.PeakErr)
	e.Quant("badsteps").SetScalar(float64(st.BadSteps))
}

func (s *fusedSolver) Dependencies() (children, parents []string) {
	children = []string{"dt", "m_error", "m_peakerror", "badsteps"}
	parents = []string{"dt", "mindt", "maxdt", "m_maxerror"}
	return
}
