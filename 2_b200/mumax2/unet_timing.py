"""Per-layer timing of the U-Net's 3x3 convolutions through the C-ABI, for profiling.

Every convolution of the network (`unet.CONVS`) at a batch size, with seeded random bf16
inputs and weights of the layer's shape, timed with CUDA events on the current stream:
the tcgen05 forward kernel (the one-tile halo-band kernel and the persistent
warp-specialised one), the mma.sync forward kernel, and the two weight-gradient kernels
(mma.sync, tcgen05).

    PYTHONPATH=2_b200 python -m mumax2.unet_timing [--batch 256] [--reps 20]
    PYTHONPATH=2_b200 python -m mumax2.unet_timing --layer d2a --launches 4 [--persistent]

The second form only launches that layer's tcgen05 forward convolution N times (a small
case for an ncu capture of one kernel).  One JSON line per layer, then the totals.
"""
import argparse
import ctypes as C
import json

from . import _native as nat
from .unet import BUFFERS, CONVS


def layer_shapes(H=64, W=64):
    """(name, Cin, Cout, H, W, relu) of every convolution of the network."""
    for name, (iv, _io), cin, (_ov, _oo), cout, relu in CONVS:
        lvl = BUFFERS[iv][0]
        yield name, cin, cout, H >> lvl, W >> lvl, relu


class _Layer:
    def __init__(self, batch, cin, cout, H, W, relu, device, seed):
        import torch
        dev = torch.device("cuda", device)
        g = torch.Generator(device=dev).manual_seed(seed)
        P = batch * H * W
        self.shape = (batch, cin, cout, H, W, int(relu))
        self.x = ((torch.rand(P * cin, generator=g, device=dev) - 0.5)).to(torch.bfloat16)
        self.dy = ((torch.rand(P * cout, generator=g, device=dev) - 0.5)).to(torch.bfloat16)
        self.w = ((torch.rand(cout * 9 * cin, generator=g, device=dev) - 0.5) * 0.1).to(torch.bfloat16)
        self.b = torch.zeros(cout, device=dev)
        self.y = torch.empty(P * cout, dtype=torch.bfloat16, device=dev)
        self.dw = torch.zeros(cout * 9 * cin, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)

    @staticmethod
    def _p(t):
        return C.c_void_p(t.data_ptr())

    def fwd_tc(self):
        B, cin, cout, H, W, relu = self.shape
        p = self._p
        nat.check(nat.lib().mm_nn_conv3x3_tc(p(self.x), cin, 0, cin, p(self.w), p(self.b), p(self.y), cout, 0, cout,
                                             B, H, W, relu, p(self.err), None))

    def fwd_mma(self):
        B, cin, cout, H, W, relu = self.shape
        p = self._p
        nat.check(nat.lib().mm_nn_conv3x3(p(self.x), cin, 0, cin, p(self.w), p(self.b), p(self.y), cout, 0, cout,
                                          B, H, W, relu, None))

    def wgrad_mma(self):
        B, cin, cout, H, W, _ = self.shape
        p = self._p
        nat.check(nat.lib().mm_nn_conv3x3_wgrad(p(self.dy), cout, 0, cout, p(self.x), cin, 0, cin, p(self.dw),
                                                B, H, W, None))

    def wgrad_tc(self):
        B, cin, cout, H, W, _ = self.shape
        p = self._p
        nat.check(nat.lib().mm_nn_conv3x3_wgrad_tc(p(self.dy), cout, 0, cout, p(self.x), cin, 0, cin, p(self.dw),
                                                   B, H, W, p(self.err), None))

    def check(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("a bounded wait inside a tcgen05 kernel ran out")


def _time(fn, reps, warmup):
    import torch
    for _ in range(warmup):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) * 1000.0 / reps


def time_layers(batch=256, reps=20, warmup=3, device=0, layers=None):
    """Microseconds per launch of each kernel on each layer: a list of dicts."""
    import torch
    torch.cuda.set_device(device)
    L = nat.lib()
    out = []
    try:
        for k, (name, cin, cout, H, W, relu) in enumerate(layer_shapes()):
            if layers and name not in layers:
                continue
            ly = _Layer(batch, cin, cout, H, W, relu, device, seed=k)
            flops = 2.0 * 9 * cin * cout * batch * H * W
            row = {"layer": name, "cin": cin, "cout": cout, "hw": H}
            nat.check(L.mm_nn_set_conv_kernel(0))
            row["tc_us"] = _time(ly.fwd_tc, reps, warmup)
            nat.check(L.mm_nn_set_conv_kernel(1))
            row["tc_persistent_us"] = _time(ly.fwd_tc, reps, warmup)
            nat.check(L.mm_nn_set_conv_kernel(0))
            row["mma_us"] = _time(ly.fwd_mma, reps, warmup)
            row["wgrad_mma_us"] = _time(ly.wgrad_mma, reps, warmup)
            row["wgrad_tc_us"] = _time(ly.wgrad_tc, reps, warmup)
            ly.check()
            row["tc_tflops"] = flops / (row["tc_us"] * 1e-6) / 1e12
            out.append(row)
    finally:
        nat.check(L.mm_nn_set_conv_kernel(0))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--layer", default=None, help="only this layer's tcgen05 forward convolution")
    ap.add_argument("--launches", type=int, default=4)
    ap.add_argument("--persistent", action="store_true", help="with --layer: the persistent kernel")
    a = ap.parse_args(argv)
    if a.layer:
        import torch
        torch.cuda.set_device(a.device)
        shape = {s[0]: s for s in layer_shapes()}[a.layer]
        ly = _Layer(a.batch, *shape[1:], a.device, seed=0)
        L = nat.lib()
        nat.check(L.mm_nn_set_conv_kernel(1 if a.persistent else 0))
        try:
            for _ in range(a.launches):
                ly.fwd_tc()
            torch.cuda.synchronize()
        finally:
            nat.check(L.mm_nn_set_conv_kernel(0))
        ly.check()
        print(json.dumps({"layer": a.layer, "launches": a.launches, "persistent": a.persistent}))
        return
    rows = time_layers(a.batch, a.reps, a.warmup, a.device)
    for r in rows:
        print(json.dumps(r))
    tot = {k: sum(r[k] for r in rows) for k in ("tc_us", "tc_persistent_us", "mma_us", "wgrad_mma_us", "wgrad_tc_us")}
    print(json.dumps({"total": tot, "batch": a.batch}))


if __name__ == "__main__":
    main()
