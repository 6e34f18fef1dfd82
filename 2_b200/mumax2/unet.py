"""Learned warm start for relaxations: a 4-level convolutional U-Net (32/64/128/256
channels, 3x3 kernels, BF16 weights and activations, FP32 accumulation) trained on the
GPU by this library's own kernels (unet.cu) on relaxed states that the plain relaxer
produced.  torch supplies device memory only; every operation is a libmm_b200 kernel.

Tensors are NHWC bf16 [pixels][channels] with pixel = (b, y, x) in the engine's cell
order (internal n1 = y, n2 = x for single-layer films).  Input features (16 channels,
9 used): mask, Ms/1e6, Aex/1e-11, Ku1/1e5, the anisotropy axis (x, y), B_ext (x, y)/0.05 T,
and a constant 1, each except B and the constant multiplied by the mask.  Output: the
three user-order components of m (normalised and masked by `predict`).
"""
import ctypes as C

import numpy as np

from . import _native as nat

FEAT = 16   # input channels (9 used, zero padded for the tensor-core K slices)
OUTC = 16   # output rows of the last convolution (3 used)

# (name, input view, input channels, output view, output channels, relu)
# views: (buffer, channel offset); buffers are listed in BUFFERS as (level, channels)
BUFFERS = {
    "in": (0, FEAT), "x0a": (0, 32), "d0cat": (0, 96), "p0": (1, 32),
    "x1a": (1, 64), "d1cat": (1, 192), "p1": (2, 64),
    "x2a": (2, 128), "d2cat": (2, 384), "p2": (3, 128),
    "x3a": (3, 256), "x3b": (3, 256),
    "x2d": (2, 128), "x2e": (2, 128),
    "x1d": (1, 64), "x1e": (1, 64),
    "x0d": (0, 32), "x0e": (0, 32), "out": (0, OUTC),
}
CONVS = [
    ("e0a", ("in", 0), FEAT, ("x0a", 0), 32, True),
    ("e0b", ("x0a", 0), 32, ("d0cat", 64), 32, True),
    ("e1a", ("p0", 0), 32, ("x1a", 0), 64, True),
    ("e1b", ("x1a", 0), 64, ("d1cat", 128), 64, True),
    ("e2a", ("p1", 0), 64, ("x2a", 0), 128, True),
    ("e2b", ("x2a", 0), 128, ("d2cat", 256), 128, True),
    ("e3a", ("p2", 0), 128, ("x3a", 0), 256, True),
    ("e3b", ("x3a", 0), 256, ("x3b", 0), 256, True),
    ("d2a", ("d2cat", 0), 384, ("x2d", 0), 128, True),
    ("d2b", ("x2d", 0), 128, ("x2e", 0), 128, True),
    ("d1a", ("d1cat", 0), 192, ("x1d", 0), 64, True),
    ("d1b", ("x1d", 0), 64, ("x1e", 0), 64, True),
    ("d0a", ("d0cat", 0), 96, ("x0d", 0), 32, True),
    ("d0b", ("x0d", 0), 32, ("x0e", 0), 32, True),
    ("out", ("x0e", 0), 32, ("out", 0), OUTC, False),
]
# (source view, destination view, channels, source level) in forward order
POOLS = [(("d0cat", 64), ("p0", 0), 32, 0), (("d1cat", 128), ("p1", 0), 64, 1), (("d2cat", 256), ("p2", 0), 128, 2)]
UPS = [(("x3b", 0), ("d2cat", 0), 256, 3), (("x2e", 0), ("d1cat", 0), 128, 2), (("x1e", 0), ("d0cat", 0), 64, 1)]
# forward schedule: convs by name, "pool<i>" and "up<i>"
SCHEDULE = ["e0a", "e0b", "pool0", "e1a", "e1b", "pool1", "e2a", "e2b", "pool2", "e3a", "e3b",
            "up0", "d2a", "d2b", "up1", "d1a", "d1b", "up2", "d0a", "d0b", "out"]


def conv_flops(H, W):
    """Multiply-adds x 2 of one forward pass of one sample."""
    total = 0
    for _, (src, _), cin, _, cout, _ in CONVS:
        lvl = BUFFERS[src][0]
        total += 2 * 9 * cin * cout * (H >> lvl) * (W >> lvl)
    return total


def init_params(seed=0):
    """He-normal weights [cout][9][cin] (rows beyond the real outputs of the last layer
    are zero), zero biases; FP32 numpy."""
    rng = np.random.default_rng(seed)
    params = {}
    for name, _, cin, _, cout, _ in CONVS:
        fan_in = 9 * (9 if name == "e0a" else cin)
        w = rng.normal(0.0, np.sqrt(2.0 / fan_in), size=(cout, 9, cin)).astype(np.float32)
        if name == "e0a":
            w[:, :, 9:] = 0.0
        if name == "out":
            w[3:] = 0.0
            w *= 0.05   # start near zero output: the first steps fit the mean state
        params[name] = (w, np.zeros(cout, dtype=np.float32))
    return params


# feature channels that carry the y components of the anisotropy axis and the field,
# and their columns in param_table
FEAT_AXIS_Y = 5
FEAT_B_Y = 7
PRM_AXIS_Y = 4
PRM_B_Y = 6


def features(sims, masks, n):
    """Input features [nsim][H*W][FEAT] (float32) of relaxation problems (workloads.relax_set)."""
    ny, nx = n[1], n[2]
    P = ny * nx
    out = np.zeros((len(sims), P, FEAT), dtype=np.float32)
    for b, (s, mk) in enumerate(zip(sims, masks)):
        mk = np.asarray(mk, dtype=np.float32).reshape(-1)
        u = s["anisu"]   # internal (z, y, x)
        bext = s["bext"]
        out[b, :, 0] = mk
        out[b, :, 1] = mk * s["msat"] / 1e6
        out[b, :, 2] = mk * s["aex"] / 1e-11
        out[b, :, 3] = mk * s["ku"] / 1e5
        out[b, :, 4] = mk * u[2]
        out[b, :, 5] = mk * u[1]
        out[b, :, 6] = bext[2] / 0.05
        out[b, :, 7] = bext[1] / 0.05
        out[b, :, 8] = 1.0
    return out


def param_table(sims):
    """[nsim][8] float32: Ms, Aex, Ku1, axis x, axis y, B_x, B_y, 0 (user axes) for the
    features kernel."""
    t = np.zeros((len(sims), 8), dtype=np.float32)
    for q, s in enumerate(sims):
        u, b = s["anisu"], s["bext"]   # internal (z, y, x)
        t[q] = (s["msat"], s["aex"], s["ku"], u[2], u[1], b[2], b[1], 0.0)
    return t


def target_from_state(m_int, n):
    """Relaxed internal SoA state [3][N] -> [N][3] user order (mx, my, mz)."""
    m = np.asarray(m_int, dtype=np.float32).reshape(3, -1)
    return np.ascontiguousarray(np.stack([m[2], m[1], m[0]], axis=1))


def state_from_output(out3, masks):
    """Network output [nsim][N][3] (user order) -> normalised, masked internal SoA states."""
    o = np.asarray(out3, dtype=np.float32)
    nrm = np.linalg.norm(o, axis=2, keepdims=True)
    nrm[nrm == 0] = 1.0
    o = o / nrm * np.asarray(masks, dtype=np.float32).reshape(o.shape[0], -1, 1)
    return np.ascontiguousarray(np.stack([o[..., 2], o[..., 1], o[..., 0]], axis=1).reshape(o.shape[0], -1))


class UNet:
    """Buffers for one batch size; forward, backward and Adam on the GPU."""

    def __init__(self, batch, H=64, W=64, device=0, seed=0, params=None, tcgen05=True, tcgen05_wgrad=False):
        """tcgen05: forward and data-gradient convolutions on the tcgen05 kernel (else
        mma.sync); tcgen05_wgrad: weight gradients on the tcgen05 kernel (measured slower
        than the mma.sync one at these sizes, so off by default)."""
        import torch
        self.torch = torch
        self.tcgen05 = tcgen05
        self.tcgen05_wgrad = tcgen05_wgrad
        self.device = torch.device("cuda", device) if isinstance(device, int) else torch.device(device)
        self.B, self.H, self.W = batch, H, W
        bf = torch.bfloat16
        self.buf, self.grad = {}, {}
        for k, (lvl, ch) in BUFFERS.items():
            npx = batch * (H >> lvl) * (W >> lvl)
            self.buf[k] = torch.zeros(npx * ch, dtype=bf, device=self.device)
            self.grad[k] = torch.zeros(npx * ch, dtype=bf, device=self.device)
        self.p = {}
        params = params or init_params(seed)
        for name, _, cin, _, cout, _ in CONVS:
            w, b = params[name]
            d = {"w": torch.tensor(w, device=self.device).reshape(-1), "b": torch.tensor(b, device=self.device)}
            d["wb"] = d["w"].to(bf)
            cin_t = ((cout + 15) // 16) * 16
            d["wt"] = torch.zeros(cin * 9 * cin_t, dtype=bf, device=self.device)
            d["cin_t"] = cin_t
            for k in ("gw", "mw", "vw"):
                d[k] = torch.zeros_like(d["w"])
            for k in ("gb", "mb", "vb"):
                d[k] = torch.zeros_like(d["b"])
            self.p[name] = d
        self.t = 0
        self.target = None
        self.mask = None
        self.loss_buf = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._flip_all()

    # ---- helpers
    def _lvl(self, view):
        return BUFFERS[view[0]][0]

    def _ptr(self, t):
        return C.c_void_p(t.data_ptr())

    def _need(self, t, count, what):
        """t must be a contiguous device tensor of `count` elements: the kernels read and
        write exactly that many."""
        if t.numel() != count or not t.is_contiguous() or t.device.type != "cuda":
            raise ValueError("%s: contiguous device tensor of %d elements needed, got %d" % (what, count, t.numel()))
        return t

    def _cs(self, view):
        return BUFFERS[view[0]][1]

    def _conv(self, src, s_cs, s_co, cin, w, b, dst, d_cs, d_co, cout, H, W, relu):
        """One 3x3 convolution: tcgen05 (TMEM accumulators) or the mma.sync kernel."""
        L = nat.lib()
        fp = self._ptr
        bp = fp(b) if b is not None else None
        if self.tcgen05:
            nat.check(L.mm_nn_conv3x3_tc(fp(src), s_cs, s_co, cin, fp(w), bp, fp(dst), d_cs, d_co, cout, self.B, H, W,
                                         relu, fp(self.err), None))
        else:
            nat.check(L.mm_nn_conv3x3(fp(src), s_cs, s_co, cin, fp(w), bp, fp(dst), d_cs, d_co, cout, self.B, H, W,
                                      relu, None))

    def check(self):
        """Raises if a tcgen05 convolution reported a timed-out wait since the last check."""
        if int(self.err.item()):
            self.err.zero_()
            raise RuntimeError("tcgen05 convolution: an mbarrier wait ran out")

    def _flip_all(self):
        for name, _, cin, _, cout, _ in CONVS:
            d = self.p[name]
            nat.check(nat.lib().mm_nn_flip(self._ptr(d["wb"]), cout, cin, self._ptr(d["wt"]), d["cin_t"], cin, None))

    def params_numpy(self):
        out = {}
        for name, _, cin, _, cout, _ in CONVS:
            d = self.p[name]
            out[name] = (d["w"].reshape(cout, 9, cin).cpu().numpy(), d["b"].cpu().numpy())
        return out

    # ---- forward
    def set_features(self, masks_dev, prm_dev):
        """Builds the input features on the GPU from masks [B][H*W] and param_table rows
        (device float32 tensors)."""
        P = self.H * self.W
        self._need(masks_dev, self.B * P, "masks")
        self._need(prm_dev, self.B * 8, "parameter table")
        nat.check(nat.lib().mm_nn_features(self._ptr(masks_dev), self._ptr(prm_dev), self.B, P,
                                           self._ptr(self.buf["in"]), None))

    def set_input(self, feats):
        """feats: float32 [B][H*W][FEAT] (numpy or device tensor)."""
        torch = self.torch
        f = torch.as_tensor(feats, device=self.device, dtype=torch.float32).reshape(-1).contiguous()
        P = self.B * self.H * self.W
        self._need(f, P * FEAT, "features")
        nat.check(nat.lib().mm_nn_to_bf16(self._ptr(f), P, FEAT, self._ptr(self.buf["in"]), FEAT, 0, None))

    def forward(self):
        L = nat.lib()
        B, H, W = self.B, self.H, self.W
        convs = {c[0]: c for c in CONVS}
        for op in SCHEDULE:
            if op.startswith("pool"):
                (sv, so), (dv, do), ch, lvl = POOLS[int(op[4:])]
                nat.check(L.mm_nn_pool(self._ptr(self.buf[sv]), self._cs((sv,)), so, self._ptr(self.buf[dv]),
                                       self._cs((dv,)), do, ch, B, H >> (lvl + 1), W >> (lvl + 1), 0, None))
            elif op.startswith("up"):
                (sv, so), (dv, do), ch, lvl = UPS[int(op[2:])]
                nat.check(L.mm_nn_upsample(self._ptr(self.buf[sv]), self._cs((sv,)), so, self._ptr(self.buf[dv]),
                                           self._cs((dv,)), do, ch, B, H >> lvl, W >> lvl, 0, None))
            else:
                name, (iv, io), cin, (ov, oo), cout, relu = convs[op]
                lvl = BUFFERS[iv][0]
                d = self.p[name]
                self._conv(self.buf[iv], self._cs((iv,)), io, cin, d["wb"], d["b"], self.buf[ov], self._cs((ov,)), oo,
                           cout, H >> lvl, W >> lvl, 1 if relu else 0)
        return self.buf["out"]

    # ---- loss and backward
    def set_target(self, target, mask, mask_count=None):
        """target float32 [B][H*W][3] (user order), mask float32 [B][H*W]; mask_count (the
        sum of the mask, if the caller knows it) spares a device-to-host read."""
        torch = self.torch
        self.target = torch.as_tensor(target, device=self.device, dtype=torch.float32).reshape(-1).contiguous()
        self.mask = torch.as_tensor(mask, device=self.device, dtype=torch.float32).reshape(-1).contiguous()
        P = self.B * self.H * self.W
        self._need(self.target, P * 3, "target")
        self._need(self.mask, P, "mask")
        cnt = float(mask_count) if mask_count is not None else float(self.mask.sum().item())
        self.norm = max(1.0, cnt) * 3.0

    def loss_and_grad(self):
        L = nat.lib()
        self.loss_buf.zero_()
        P = self.B * self.H * self.W
        nat.check(L.mm_nn_mse(self._ptr(self.buf["out"]), OUTC, self._ptr(self.target), self._ptr(self.mask), P,
                              C.c_float(self.norm), self._ptr(self.grad["out"]), OUTC, self._ptr(self.loss_buf),
                              None))
        return self.loss_buf

    def backward(self):
        L = nat.lib()
        B, H, W = self.B, self.H, self.W
        convs = {c[0]: c for c in CONVS}
        fp = self._ptr
        for d in self.p.values():
            d["gw"].zero_()
            d["gb"].zero_()
        for op in reversed(SCHEDULE):
            if op.startswith("pool"):
                (sv, so), (dv, do), ch, lvl = POOLS[int(op[4:])]
                nat.check(L.mm_nn_pool(self._ptr(self.grad[dv]), self._cs((dv,)), do, self._ptr(self.grad[sv]),
                                       self._cs((sv,)), so, ch, B, H >> (lvl + 1), W >> (lvl + 1), 1, None))
            elif op.startswith("up"):
                (sv, so), (dv, do), ch, lvl = UPS[int(op[2:])]
                nat.check(L.mm_nn_upsample(self._ptr(self.grad[dv]), self._cs((dv,)), do, self._ptr(self.grad[sv]),
                                           self._cs((sv,)), so, ch, B, H >> lvl, W >> lvl, 1, None))
            else:
                name, (iv, io), cin, (ov, oo), cout, relu = convs[op]
                lvl = BUFFERS[iv][0]
                P = B * (H >> lvl) * (W >> lvl)
                d = self.p[name]
                # ReLU backward (in place) and the bias gradient in one pass
                nat.check(L.mm_nn_relu_bias_bwd(self._ptr(self.buf[ov]), self._cs((ov,)), oo, self._ptr(self.grad[ov]),
                                                self._cs((ov,)), oo, cout, P, 1 if relu else 0, fp(d["gb"]), None))
                if self.tcgen05_wgrad:
                    nat.check(L.mm_nn_conv3x3_wgrad_tc(self._ptr(self.grad[ov]), self._cs((ov,)), oo, cout,
                                                       self._ptr(self.buf[iv]), self._cs((iv,)), io, cin, fp(d["gw"]),
                                                       B, H >> lvl, W >> lvl, fp(self.err), None))
                else:
                    nat.check(L.mm_nn_conv3x3_wgrad(self._ptr(self.grad[ov]), self._cs((ov,)), oo, cout,
                                                    self._ptr(self.buf[iv]), self._cs((iv,)), io, cin, fp(d["gw"]),
                                                    B, H >> lvl, W >> lvl, None))
                if name != "e0a":
                    # dX over the whole input view (a concatenated input gets both parts)
                    self._conv(self.grad[ov], self._cs((ov,)), oo, d["cin_t"], d["wt"], None, self.grad[iv],
                               self._cs((iv,)), io, cin, H >> lvl, W >> lvl, 0)

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        L = nat.lib()
        self.t += 1
        fp = self._ptr
        for name, d in self.p.items():
            nat.check(L.mm_nn_adam(fp(d["w"]), fp(d["gw"]), fp(d["mw"]), fp(d["vw"]), d["w"].numel(), C.c_float(lr),
                                   C.c_float(b1), C.c_float(b2), C.c_float(eps), self.t, self._ptr(d["wb"]), None))
            nat.check(L.mm_nn_adam(fp(d["b"]), fp(d["gb"]), fp(d["mb"]), fp(d["vb"]), d["b"].numel(), C.c_float(lr),
                                   C.c_float(b1), C.c_float(b2), C.c_float(eps), self.t, None, None))
        # the last layer's unused output rows stay zero
        dl = self.p["out"]
        w = dl["w"].reshape(OUTC, -1)
        w[3:].zero_()
        dl["wb"].copy_(dl["w"].to(self.torch.bfloat16))
        self._flip_all()

    def states(self, masks_dev, dst):
        """Initial states of this batch from the output: dst (float32 device tensor
        [B][3][H*W], internal SoA) = masks_dev [B][H*W] * normalised output."""
        P = self.H * self.W
        self._need(masks_dev, self.B * P, "masks")
        self._need(dst, self.B * 3 * P, "states")
        nat.check(nat.lib().mm_nn_output_state(self._ptr(self.buf["out"]), OUTC, self._ptr(masks_dev), self.B, P,
                                               self._ptr(dst), None))

    def output3(self):
        """[B][H*W][3] float32 numpy of the first three output channels."""
        o = self.buf["out"].reshape(self.B * self.H * self.W, OUTC)[:, :3]
        return o.float().cpu().numpy().reshape(self.B, self.H * self.W, 3)
