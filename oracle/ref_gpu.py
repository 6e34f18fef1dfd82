"""Test and baseline infrastructure, not the product: the reference's own CUDA path of the
micromagnetic step on this GPU.

The kernels are the reference's libmumax2 (src/libmumax2/*.cu), built from its sources
for sm_100a by oracle/build_ref.sh into oracle/_ref/libmumax2_ref.so.  The host loop that
drives them restates the reference's Go code, one call for one call, with cuFFT (through
torch.fft, the library the reference's FFTPlanX calls) for the transforms:

  RK12Solver.Step                 src/mumax/engine/solve_rk12.go:91-214
  MaxwellPlan.UpdateB / update    src/mumax/modules/maxwell_convolution.go:222-309
      (fftOut zeroed, per input component: FFTPlanX.Forward, then one CMaddAsync per
       non-zero kernel component with a stream sync; per output component
       FFTPlanX.Inverse)
  FFTPlanX.Forward / Inverse      src/mumax/gpu/fftplanX.go:80-109
      (buffer zeroed, CopyPad3D, R2C; C2R, CopyUnPad3D)
  H_eff = B/mu0 + H_ex + H_anis   src/mumax/modules/hfield.go:18-30,
                                  src/mumax/engine/update_sum.go:29-75 (zero, VecMadd per parent)
  exchange6, uniaxial anisotropy, torque
                                  src/mumax/modules/mod_exchange6.go:40-51,
                                  mod_uniaxialanisotropy.go:44-57, mod_llg.go:59-70
  normalisation of m on update    src/mumax/modules/update_norm.go
  MaxDiff (partial + host finish) src/mumax/gpu/reductor.go:26-45,141-154
  Madd / MAdd2Async (+ sync)      src/mumax/gpu/libmumax2.go:131-176

Uniform material parameters only (the maps are NULL parts, the reference's convention
for a uniform mask), no external field, open boundaries.  The demag tensor is given as
the transformed octant (Plan.demag_kernel(): the FP64 Kernel_Arne of this repository,
checked against the oracle) and expanded to the reference's full real layout
[L0][L1][L2/2+1] per (i, j); building it is setup, outside any timed region.
"""
import ctypes as C
import os

import numpy as np

MU0 = 4e-7 * np.pi
REF_LIB = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "libmumax2_ref.so")
F = C.c_float
I = C.c_int


_LIB = None


def available():
    return os.path.exists(REF_LIB)


def ref_lib():
    """The reference library, loaded once per process.  Its setUsedGPUs (multigpu.cu)
    asserts that it runs only once, so every user of the library in a process goes
    through here."""
    global _LIB
    if _LIB is None:
        import torch
        lib = C.CDLL(REF_LIB)
        lib.setUsedGPUs((C.c_int * 1)(torch.cuda.current_device()), 1)
        _LIB = lib
    return _LIB


def padded(n):
    return tuple(2 * x if x > 1 else 1 for x in n)


def expand_octant(octant, L):
    """{(i, j): [L0][L1][L2/2+1] float32} from the octant [6][kd0][kd1][kd2] (components
    00 11 22 12 02 01): K_ij with i != j flips sign under k -> L-k along axes i and j
    (axis 2 never needs it in the half spectrum); zero components are left out."""
    L0, L1, L2 = L
    h = L2 // 2 + 1
    f0, f1 = np.arange(L0), np.arange(L1)
    o0, o1 = np.minimum(f0, L0 - f0) % max(L0, 1), np.minimum(f1, L1 - f1) % max(L1, 1)
    s0 = np.where(f0 > L0 // 2, -1.0, 1.0)[:, None, None]
    s1 = np.where(f1 > L1 // 2, -1.0, 1.0)[None, :, None]
    pairs = {0: (0, 0), 1: (1, 1), 2: (2, 2), 3: (1, 2), 4: (0, 2), 5: (0, 1)}
    out = {}
    for q, (i, j) in pairs.items():
        k = octant[q][o0][:, o1][:, :, :h].astype(np.float64)
        if i != j:
            if 0 in (i, j):
                k = k * s0
            if 1 in (i, j):
                k = k * s1
        if not np.any(k):
            continue
        k = np.ascontiguousarray(k, dtype=np.float32)
        out[(i, j)] = k
        out[(j, i)] = k
    return out


class RefPath:
    """The reference's RK12 step on the GPU.  n, cell, anisu in the internal axis order."""

    def __init__(self, n, cell, msat, aex, alpha, gamma, ku, anisu, octant, dt=1e-15, mindt=1e-38, maxdt=1e38,
                 maxerr=1.0 / 2000):
        import torch
        self.torch = torch
        self.lib = ref_lib()
        self.n = tuple(int(x) for x in n)
        self.L = padded(self.n)
        self.N = int(np.prod(self.n))
        self.cell = cell
        self.msat, self.aex, self.alpha, self.gamma, self.ku = msat, aex, alpha, gamma, ku
        self.anisu = anisu
        self.dt, self.mindt, self.maxdt, self.maxerr = dt, mindt, maxdt, maxerr
        self.step_count = 0
        self.bad_steps = 0
        self.evals = 0
        dev = torch.device("cuda")
        z = lambda *s: torch.zeros(*s, dtype=torch.float32, device=dev)
        N, L = self.N, self.L
        h = L[2] // 2 + 1
        self.m, self.tau, self.H = z(3, N), z(3, N), z(3, N)
        self.B, self.Hex, self.Hanis = z(3, N), z(3, N), z(3, N)
        self.dybuf, self.y0buf = z(3, N), z(3, N)
        self.pad = z(*L)
        self.spec = torch.zeros(L[0], L[1], h, dtype=torch.complex64, device=dev)
        self.fftout = torch.zeros(3, L[0], L[1], h, dtype=torch.complex64, device=dev)
        self.kern = {k: torch.tensor(v, device=dev) for k, v in expand_octant(octant, L).items()}
        self.nc = L[0] * L[1] * h
        # reductor of 3N floats (reductor.go:26-45)
        threads = 512
        while 3 * N <= threads:
            threads //= 2
        self.red_threads = threads
        self.red_blocks = (3 * N + threads * 2 - 1) // (threads * 2)
        self.red = z(self.red_blocks)
        self.stream = (C.c_void_p * 1)(None)

    # ---- helpers
    @staticmethod
    def _p(t):
        return (C.c_void_p * 1)(t.data_ptr() if t is not None else None)

    def _sync(self):
        self.torch.cuda.synchronize()

    def set_state(self, m):
        self.m.copy_(self.torch.as_tensor(np.asarray(m, dtype=np.float32).reshape(3, -1)))

    def state(self):
        return self.m.cpu().numpy().ravel()

    # ---- field and torque (one Update() of the torque quantity)
    def _normalize(self):
        p = self._p
        self.lib.normalizeAsync(p(self.m[0]), p(self.m[1]), p(self.m[2]), p(None), self.stream, I(self.N))
        self._sync()

    def _demag(self):
        torch, p = self.torch, self._p
        L, n = self.L, self.n
        self.fftout.zero_()
        for i in range(3):
            # FFTPlanX.Forward: zero the buffer, CopyPad3D, R2C
            self.pad.zero_()
            self.lib.copyPad3DAsync(p(self.pad), I(L[0]), I(L[1]), I(L[2]), p(self.m[i]), I(n[0]), I(n[1]), I(n[2]),
                                    I(1), self.stream)
            torch.fft.rfftn(self.pad, norm="backward", out=self.spec)
            self._sync()
            for j in range(3):
                k = self.kern.get((i, j))
                if k is None:
                    continue
                mul = self.msat * MU0  # BInMul = Msat mu0 (maxwell_convolution.go:239-241)
                self.lib.cmaddAsync(p(self.fftout[j]), F(mul), F(0.0), p(k), p(self.spec), self.stream, I(self.nc))
                self._sync()
        for j in range(3):
            # FFTPlanX.Inverse: C2R (unnormalised), CopyUnPad3D
            torch.fft.irfftn(self.fftout[j], s=L, norm="forward", out=self.pad)
            self._sync()
            self.lib.copyUnPad3DAsync(p(self.B[j]), I(n[0]), I(n[1]), I(n[2]), p(self.pad), I(L[0]), I(L[1]),
                                      I(L[2]), I(1), self.stream)
            self._sync()

    def evaluate(self):
        p = self._p
        self._normalize()
        self._demag()
        n, cell = self.n, self.cell
        self.lib.exchange6Async(p(self.Hex[0]), p(self.Hex[1]), p(self.Hex[2]), p(self.m[0]), p(self.m[1]),
                                p(self.m[2]), p(None), p(None), F(2 * self.aex / (MU0 * self.msat)), I(n[0]),
                                I(n[1]), I(n[2]), I(0), I(0), I(0), F(cell[0]), F(cell[1]), F(cell[2]), self.stream)
        self._sync()
        u = self.anisu
        self.lib.uniaxialAnisotropyAsync(p(self.Hanis[0]), p(self.Hanis[1]), p(self.Hanis[2]), p(self.m[0]),
                                         p(self.m[1]), p(self.m[2]), p(None), p(None),
                                         F(2 * self.ku / (MU0 * self.msat)), p(None), F(u[0]), p(None), F(u[1]),
                                         p(None), F(u[2]), self.stream, I(self.N))
        self._sync()
        # SumUpdater: zero, then one VecMadd per parent (B with weight 1/mu0, H_ex, H_anis)
        self.H.zero_()
        for par, w in ((self.B, 1.0 / MU0), (self.Hex, 1.0), (self.Hanis, 1.0)):
            self.lib.vecMaddAsync(p(self.H[0]), p(self.H[1]), p(self.H[2]), p(self.H[0]), p(self.H[1]), p(self.H[2]),
                                  p(par[0]), p(par[1]), p(par[2]), F(w), F(w), F(w), self.stream, I(self.N))
            self._sync()
        self.lib.torqueAsync(p(self.tau[0]), p(self.tau[1]), p(self.tau[2]), p(self.m[0]), p(self.m[1]),
                             p(self.m[2]), p(self.H[0]), p(self.H[1]), p(self.H[2]), p(None), F(self.alpha),
                             self.stream, I(self.N))
        self._sync()
        self.evals += 1

    def _max_diff(self):
        p = self._p
        self.lib.partialMaxDiffAsync(p(self.tau), p(self.dybuf), p(self.red), I(self.red_blocks),
                                     I(self.red_threads), I(3 * self.N), self.stream)
        return float(self.red.cpu().numpy().max())

    # ---- RK12Solver.Step
    def step(self):
        p = self._p
        self.evaluate()                        # inputs updated (the state was invalidated)
        self.dybuf.copy_(self.tau)
        self.y0buf.copy_(self.m)
        max_try, head_room = 10, 0.8
        tries = 0
        while True:
            dt = self.dt
            if tries > 0:
                self.m.copy_(self.y0buf)
                self.tau.copy_(self.dybuf)
            self.lib.maddAsync(p(self.m), p(self.m), p(self.tau), F(dt * self.gamma), self.stream, I(3 * self.N))
            self._sync()
            self.evaluate()
            hstep = float(np.float32(dt * self.gamma))
            self.lib.madd2Async(p(self.m), p(self.tau), F(0.5 * hstep), p(self.dybuf), F(-0.5 * hstep), self.stream,
                                I(3 * self.N))
            self._sync()
            err = float(np.float32(self._max_diff()) * np.float32(hstep))
            bad = err > self.maxerr
            if bad:
                self.bad_steps += 1
            factor = np.sqrt(self.maxerr / err) if not bad else (self.maxerr / err) ** (1.0 / 3.0)
            factor = min(1.5, max(0.1, factor * head_room))
            new_dt = min(self.maxdt, max(self.mindt, dt * factor))
            self.dt = new_dt
            if not bad or new_dt == self.mindt:
                break
            if tries > max_try:
                raise RuntimeError("the solver cannot converge after %d bad steps" % max_try)
            tries += 1
        self.step_count += 1
