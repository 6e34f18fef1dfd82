// Package gpu (addition to mumax/2's src/mumax/gpu): cgo binding of the fused tier of
// libmm_b200.so (include/mm_b200.h).  The compatibility tier needs no Go changes: the
// reference's own wrappers (libmumax2.go) link against libmm_b200.so unchanged.
//
// Not built in this repository's image (there is no Go toolchain); written against the
// reference's gpu.Array (array.go: one contiguous SoA allocation per array, part 0 on
// the single device) and checked by reading only.
package gpu

/*
#cgo CFLAGS: -I${SRCDIR}/../../../include
#cgo LDFLAGS: -L${SRCDIR}/../.. -lmm_b200 -lcudart
#include "mm_b200.h"
*/
import "C"

import (
	"fmt"
	"unsafe"
)

// FusedProblem mirrors mm_problem for the terms the engine's modules load.  Sizes and
// vectors are in the engine's internal axis order (Z, Y, X).
type FusedProblem struct {
	Size                                             [3]int
	CellSize                                         [3]float64
	Periodic                                         [3]int
	Demag, Exchange, Anis, Zeeman, Thermal, ZhangLi  bool
	Slonczewski, DemagExchange                       bool
	Newell                                           bool // Newell tensor instead of Kernel_Arne
	Msat, Aex, Alpha, Gamma, Ku, Temp                float64
	Bext, AnisU, J                                   [3]float64
	Seed                                             uint64
	MsatMask, AexMask, AlphaMask                     *Array // nil = uniform (the NULL-mask rule)
}

func b2i(b bool) C.int {
	if b {
		return 1
	}
	return 0
}

func maskPtr(a *Array) *C.float {
	if a == nil || a.IsNil() {
		return nil
	}
	return (*C.float)(unsafe.Pointer(uintptr(a.DevicePtr()[0])))
}

// FusedPlan owns the demag tensor, its transform and every workspace of one geometry
// (mm_plan_create; replaces MaxwellPlan.init/EnableDemag, maxwell_convolution.go:72-120).
type FusedPlan struct {
	p C.mm_plan
}

func lastError(what string) error {
	return fmt.Errorf("%s: %s", what, C.GoString(C.mm_last_error()))
}

func NewFusedPlan(f *FusedProblem) (*FusedPlan, error) {
	var pr C.mm_problem
	for i := 0; i < 3; i++ {
		pr.n[i] = C.int(f.Size[i])
		pr.cell[i] = C.double(f.CellSize[i])
		pr.pbc[i] = C.int(f.Periodic[i])
		pr.bext[i] = C.double(f.Bext[i])
		pr.anisu[i] = C.double(f.AnisU[i])
		pr.j[i] = C.double(f.J[i])
	}
	pr.demag, pr.exchange, pr.anis, pr.zeeman = b2i(f.Demag), b2i(f.Exchange), b2i(f.Anis), b2i(f.Zeeman)
	pr.thermal, pr.zhangli, pr.slonczewski = b2i(f.Thermal), b2i(f.ZhangLi), b2i(f.Slonczewski)
	pr.demag_exchange = b2i(f.DemagExchange)
	pr.demag_accuracy = 6
	if f.Newell {
		pr.demag_tensor = C.MM_TENSOR_NEWELL
	}
	pr.msat, pr.aex, pr.alpha, pr.gamma = C.double(f.Msat), C.double(f.Aex), C.double(f.Alpha), C.double(f.Gamma)
	pr.ku, pr.temp, pr.seed = C.double(f.Ku), C.double(f.Temp), C.ulonglong(f.Seed)
	pr.msat_mask, pr.aex_mask, pr.alpha_mask = maskPtr(f.MsatMask), maskPtr(f.AexMask), maskPtr(f.AlphaMask)
	var p C.mm_plan
	if C.mm_plan_create(&pr, &p) != C.MM_OK {
		return nil, lastError("mm_plan_create")
	}
	return &FusedPlan{p}, nil
}

func (f *FusedPlan) Destroy() {
	if f.p != nil {
		C.mm_plan_destroy(f.p)
		f.p = nil
	}
}

// Solver kinds of mm_solver_init.
const (
	Euler = C.MM_EULER
	Heun  = C.MM_HEUN
	RK12  = C.MM_RK12
	RK23  = C.MM_RK23
	RK45  = C.MM_RK45
	AM12  = C.MM_AM12
)

func (f *FusedPlan) Solver(kind int, dt, mindt, maxdt, maxerr float64) error {
	if C.mm_solver_init(f.p, C.int(kind), C.double(dt), C.double(mindt), C.double(maxdt), C.double(maxerr)) != C.MM_OK {
		return lastError("mm_solver_init")
	}
	return nil
}

// SetState copies m (the engine's 3-component device array) into the plan (normalised).
func (f *FusedPlan) SetState(m *Array) error {
	if C.mm_set_state(f.p, (*C.float)(unsafe.Pointer(uintptr(m.DevicePtr()[0]))), 0, nil) != C.MM_OK {
		return lastError("mm_set_state")
	}
	return nil
}

// GetState copies the plan's accepted state into m.
func (f *FusedPlan) GetState(m *Array) error {
	if C.mm_get_state(f.p, (*C.float)(unsafe.Pointer(uintptr(m.DevicePtr()[0]))), 0, nil) != C.MM_OK {
		return lastError("mm_get_state")
	}
	return nil
}

// Step replaces Solver.Step (solve_rk12.go:91): one accepted step, all step control
// on the device; the host waits for nothing but the returned status.
func (f *FusedPlan) Step() error {
	if C.mm_step(f.p, nil) != C.MM_OK {
		return lastError("mm_step")
	}
	return nil
}

// Run advances the simulated time by duration (api.go Run).
func (f *FusedPlan) Run(duration float64) error {
	if C.mm_run(f.p, C.double(duration), nil) != C.MM_OK {
		return lastError("mm_run")
	}
	return nil
}

// RunUntilMaxTorque is the relax idiom run_until_smaller("maxtorque", thr) (api.go:122-131).
func (f *FusedPlan) RunUntilMaxTorque(thr float64, maxSteps int64) error {
	if C.mm_run_until_maxtorque(f.p, C.double(thr), C.longlong(maxSteps), nil) != C.MM_OK {
		return lastError("mm_run_until_maxtorque")
	}
	return nil
}

// Stats of the solver: time, dt, error estimates, step counters (the engine's t, dt,
// m_error, m_peakerror, badsteps).
type FusedStats struct {
	T, Dt, Err, PeakErr, MaxTorque float64
	Step, BadSteps                 int64
}

func (f *FusedPlan) Stats() (FusedStats, error) {
	var s C.mm_stats
	if C.mm_get_stats(f.p, &s, nil) != C.MM_OK {
		return FusedStats{}, lastError("mm_get_stats")
	}
	return FusedStats{float64(s.t), float64(s.dt), float64(s.err), float64(s.peakerr), float64(s.maxtorque),
		int64(s.step), int64(s.badsteps)}, nil
}

// Average is <m> (update_reduce.go AverageUpdater), compensated on the device.
func (f *FusedPlan) Average() ([3]float64, error) {
	var out [3]C.double
	if C.mm_average(f.p, &out[0], nil) != C.MM_OK {
		return [3]float64{}, lastError("mm_average")
	}
	return [3]float64{float64(out[0]), float64(out[1]), float64(out[2])}, nil
}

// Energy returns E_zeeman, E_ex, E_demag, E_anis and E (mod_energy.go), in J.
func (f *FusedPlan) Energy() ([5]float64, error) {
	var out [5]C.double
	if C.mm_energy(f.p, &out[0], nil) != C.MM_OK {
		return [5]float64{}, lastError("mm_energy")
	}
	var e [5]float64
	for i := range e {
		e[i] = float64(out[i])
	}
	return e, nil
}
