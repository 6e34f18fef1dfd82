"""BF16 tensor-core kernels of the warm-start U-Net against the numpy oracle
(oracle/unet_ref.py, float64 with bf16 rounding where the GPU stores bf16).

Tolerances: a convolution output may differ from the oracle by one bf16 rounding step
(2^-8 relative) because the FP32 sums run in another order; weight gradients (FP32
accumulation of bf16 products) agree to 1e-3 relative in norm; the gradients of the whole
network, where a flipped rounding of an activation propagates, to 3e-2.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    import torch
    return torch.tensor(np.asarray(a, dtype=np.float32), device="cuda").to(dtype).reshape(-1).contiguous()


def _p(t):
    return C.c_void_p(t.data_ptr())


def _relnorm(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("cin,cout,B,H,W,relu", [(16, 32, 2, 8, 8, 1), (64, 128, 1, 16, 16, 0), (96, 32, 2, 8, 16, 1),
                                                 (32, 16, 1, 4, 4, 0)])
def test_conv3x3_forward_and_data_gradient(cin, cout, B, H, W, relu):
    import torch
    import unet_ref as R
    from mumax2 import _native as nat
    rng = np.random.default_rng(cin + cout)
    x = R.bf16(rng.normal(size=(B, H, W, cin)))
    w = R.bf16(rng.normal(size=(cout, 9, cin)) / np.sqrt(9 * cin))
    b = rng.normal(size=cout).astype(np.float32)
    xd, wd = _dev(x, torch.bfloat16), _dev(w, torch.bfloat16)
    bd = torch.tensor(b, device="cuda")
    out = torch.zeros(B * H * W * cout, dtype=torch.bfloat16, device="cuda")
    nat.check(nat.lib().mm_nn_conv3x3(_p(xd), cin, 0, cin, _p(wd), _p(bd), _p(out), cout, 0, cout, B, H, W, relu,
                                      None))
    ref = R.conv3x3(x, w, b)
    if relu:
        ref = np.maximum(ref, 0)
    got = out.float().cpu().numpy().reshape(ref.shape)
    assert np.abs(got - ref).max() <= 2 ** -7 * np.abs(ref).max() + 1e-6
    # data gradient through the flipped weights
    dy = R.bf16(rng.normal(size=(B, H, W, cout)))
    dyd = _dev(dy, torch.bfloat16)
    cin_t = ((cout + 15) // 16) * 16
    wt = torch.zeros(cin * 9 * cin_t, dtype=torch.bfloat16, device="cuda")
    nat.check(nat.lib().mm_nn_flip(_p(wd), cout, cin, _p(wt), cin_t, cin, None))
    dx = torch.zeros(B * H * W * cin, dtype=torch.bfloat16, device="cuda")
    nat.check(nat.lib().mm_nn_conv3x3(_p(dyd), cout, 0, cin_t, _p(wt), None, _p(dx), cin, 0, cin, B, H, W, 0, None))
    rdx, rdw, rdb = R.conv3x3_backward(x, w, dy)
    gdx = dx.float().cpu().numpy().reshape(rdx.shape)
    assert np.abs(gdx - rdx).max() <= 2 ** -7 * np.abs(rdx).max() + 1e-6
    # weight and bias gradients
    dw = torch.zeros(cout * 9 * cin, dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    nat.check(nat.lib().mm_nn_conv3x3_wgrad(_p(dyd), cout, 0, cout, _p(xd), cin, 0, cin, _p(dw), B, H, W, None))
    nat.check(nat.lib().mm_nn_bias_grad(_p(dyd), cout, 0, cout, B * H * W, _p(db), None))
    assert _relnorm(dw.cpu().numpy().reshape(rdw.shape), rdw) < 1e-3
    assert _relnorm(db.cpu().numpy(), rdb) < 1e-3


@pytest.mark.parametrize("tcgen05,wgrad", [(True, False), (False, False), (True, True)])
def test_network_gradients_match_oracle(tcgen05, wgrad):
    import unet_ref as R
    from mumax2 import unet as U
    B, H, W = 2, 16, 16
    rng = np.random.default_rng(7)
    params = U.init_params(seed=3)
    for name in params:   # non-zero biases exercise the bias paths
        w, b = params[name]
        params[name] = (w, (0.05 * rng.normal(size=b.shape)).astype(np.float32))
    feats = np.zeros((B, H * W, U.FEAT), dtype=np.float32)
    feats[..., :9] = rng.normal(size=(B, H * W, 9))
    target = rng.normal(size=(B, H * W, 3)).astype(np.float32)
    mask = (rng.uniform(size=(B, H * W)) > 0.2).astype(np.float32)
    net = U.UNet(B, H, W, params=params, tcgen05=tcgen05, tcgen05_wgrad=wgrad)
    net.set_input(feats)
    net.forward()
    net.set_target(target, mask)
    loss = float(net.loss_and_grad().item())
    net.backward()
    net.check()
    arch = (U.BUFFERS, U.CONVS, U.POOLS, U.UPS, U.SCHEDULE)
    rloss, rgrads, rout = R.forward_backward(arch, params, feats, target, mask, H, W)
    assert loss == pytest.approx(rloss, rel=1e-2)
    errs, berrs = {}, {}
    for name, (dw, db) in rgrads.items():
        d = net.p[name]
        errs[name] = _relnorm(d["gw"].cpu().numpy().reshape(dw.shape), dw)
        berrs[name] = _relnorm(d["gb"].cpu().numpy(), db)
    print(errs, berrs)
    assert max(errs.values()) < 3e-2
    assert max(berrs.values()) < 3e-2


def test_training_lowers_the_loss():
    """A few Adam steps on a fixed batch fit a smooth target."""
    from mumax2 import unet as U
    B, H, W = 4, 16, 16
    rng = np.random.default_rng(1)
    feats = np.zeros((B, H * W, U.FEAT), dtype=np.float32)
    feats[..., 0] = 1.0
    feats[..., 6:8] = rng.normal(size=(B, 1, 2))
    feats[..., 8] = 1.0
    target = np.zeros((B, H * W, 3), dtype=np.float32)
    target[..., 0] = np.cos(feats[..., 6])
    target[..., 1] = np.sin(feats[..., 6])
    mask = np.ones((B, H * W), dtype=np.float32)
    net = U.UNet(B, H, W, seed=0)
    net.set_input(feats)
    net.set_target(target, mask)
    losses = []
    for _ in range(60):
        net.forward()
        losses.append(float(net.loss_and_grad().item()))
        net.backward()
        net.adam(lr=3e-3)
    print(losses[0], losses[-1])
    assert losses[-1] < 0.2 * losses[0]


@pytest.mark.parametrize("persistent", [0, 1])
@pytest.mark.parametrize("cin,cout,B,H,W,relu", [(16, 32, 2, 8, 8, 1), (64, 128, 1, 16, 16, 0), (96, 32, 2, 8, 16, 1),
                                                 (32, 16, 1, 4, 4, 0), (384, 128, 2, 16, 16, 1), (256, 256, 4, 8, 8, 1),
                                                 (32, 32, 2, 64, 64, 1), (16, 16, 3, 5, 7, 1), (48, 64, 2, 1, 9, 0)])
def test_conv3x3_tcgen05_matches(cin, cout, B, H, W, relu, persistent):
    """The tcgen05 convolution (TMEM accumulators, halo band over padded positions), the
    one-tile-per-block kernel and the persistent warp-specialised one, against the numpy
    oracle, including widths that are not multiples of 8, single-row images and tiles
    that span several images."""
    import torch
    import unet_ref as R
    from mumax2 import _native as nat
    nat.check(nat.lib().mm_nn_set_conv_kernel(persistent))
    rng = np.random.default_rng(cin * 7 + cout)
    x = R.bf16(rng.normal(size=(B, H, W, cin)))
    w = R.bf16(rng.normal(size=(cout, 9, cin)) / np.sqrt(9 * cin))
    b = rng.normal(size=cout).astype(np.float32)
    xd, wd = _dev(x, torch.bfloat16), _dev(w, torch.bfloat16)
    bd = torch.tensor(b, device="cuda")
    out = torch.zeros(B * H * W * cout, dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.check(nat.lib().mm_nn_conv3x3_tc(_p(xd), cin, 0, cin, _p(wd), _p(bd), _p(out), cout, 0, cout, B, H, W, relu,
                                         _p(err), None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = R.conv3x3(x, w, b)
    if relu:
        ref = np.maximum(ref, 0)
    got = out.float().cpu().numpy().reshape(ref.shape)
    nat.check(nat.lib().mm_nn_set_conv_kernel(0))
    assert np.abs(got - ref).max() <= 2 ** -7 * np.abs(ref).max() + 1e-6


def test_feature_kernel_matches_host_features():
    """mm_nn_features builds the same bf16 inputs as unet.features followed by the cast."""
    import torch
    import unet_ref as R
    from mumax2 import unet as U
    from mumax2 import workloads as W
    problem, sims, masks = W.relax_set(6, seed=11)
    n = problem["n"]
    net = U.UNet(6, n[1], n[2], seed=0)
    mk = torch.tensor(np.stack(masks).astype(np.float32), device="cuda")
    prm = torch.tensor(U.param_table(sims), device="cuda")
    net.set_features(mk, prm)
    got = net.buf["in"].float().cpu().numpy().reshape(6, -1, U.FEAT)
    ref = R.bf16(U.features(sims, masks, n))
    assert np.abs(got - ref).max() <= 2 ** -8 * np.abs(ref).max()


def test_output_state_kernel_matches_host_conversion():
    """mm_nn_output_state equals unet.state_from_output on the same network output."""
    import torch
    from mumax2 import unet as U
    B, H, W = 3, 8, 8
    rng = np.random.default_rng(5)
    net = U.UNet(B, H, W, seed=0)
    o = rng.normal(size=(B * H * W, U.OUTC)).astype(np.float32)
    o[5, :3] = 0.0
    net.buf["out"].copy_(torch.tensor(o.ravel(), device="cuda").to(torch.bfloat16))
    masks = (rng.uniform(size=(B, H * W)) > 0.3).astype(np.float32)
    md = torch.tensor(masks, device="cuda")
    dst = torch.zeros((B, 3 * H * W), device="cuda")
    net.states(md, dst)
    ref = U.state_from_output(net.output3(), masks)
    assert np.abs(dst.cpu().numpy() - ref).max() < 1e-6


@pytest.mark.parametrize("cin,cout,B,H,W", [(32, 32, 2, 8, 8), (16, 32, 2, 64, 64), (384, 128, 2, 16, 16),
                                            (128, 256, 3, 8, 8), (32, 16, 1, 5, 7), (48, 64, 2, 1, 9),
                                            (96, 32, 2, 8, 16)])
def test_wgrad_tcgen05_matches(cin, cout, B, H, W):
    """The tcgen05 weight gradient (nine TMEM accumulators over the halo band, MN-major
    operands) against the numpy oracle, 1e-3 relative in norm (FP32 sums of bf16
    products in another order)."""
    import torch
    import unet_ref as R
    from mumax2 import _native as nat
    rng = np.random.default_rng(cin + 3 * cout + W)
    x = R.bf16(rng.normal(size=(B, H, W, cin)))
    w = R.bf16(rng.normal(size=(cout, 9, cin)) / np.sqrt(9 * cin))
    dy = R.bf16(rng.normal(size=(B, H, W, cout)))
    xd, dyd = _dev(x, torch.bfloat16), _dev(dy, torch.bfloat16)
    dw = torch.zeros(cout * 9 * cin, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    nat.check(nat.lib().mm_nn_conv3x3_wgrad_tc(_p(dyd), cout, 0, cout, _p(xd), cin, 0, cin, _p(dw), B, H, W, _p(err),
                                               None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    _, rdw, _ = R.conv3x3_backward(x, w, dy)
    assert _relnorm(dw.cpu().numpy().reshape(rdw.shape), rdw) < 1e-3


def test_tcgen05_wait_timeout_is_reported():
    """Failure detection without a fault: with the wait limit at 0 every mbarrier wait of
    the tcgen05 kernels runs out, each kernel sets its error flag and returns after its
    MMAs in flight are done; with the default limit restored the next calls are correct."""
    import torch
    import unet_ref as R
    from mumax2 import _native as nat
    L = nat.lib()
    rng = np.random.default_rng(12)
    cin, cout, B, H, W = 64, 32, 2, 16, 16
    x = R.bf16(rng.normal(size=(B, H, W, cin)))
    w = R.bf16(rng.normal(size=(cout, 9, cin)) / np.sqrt(9 * cin))
    dy = R.bf16(rng.normal(size=(B, H, W, cout)))
    xd, wd, dyd = _dev(x, torch.bfloat16), _dev(w, torch.bfloat16), _dev(dy, torch.bfloat16)
    out = torch.zeros(B * H * W * cout, dtype=torch.bfloat16, device="cuda")
    dw = torch.zeros(cout * 9 * cin, dtype=torch.float32, device="cuda")
    err = torch.zeros(2, dtype=torch.int32, device="cuda")
    ep0 = C.c_void_p(err.data_ptr())
    ep1 = C.c_void_p(err.data_ptr() + 4)
    nat.check(L.mm_nn_set_wait_limit(0))
    try:
        nat.check(L.mm_nn_conv3x3_tc(_p(xd), cin, 0, cin, _p(wd), None, _p(out), cout, 0, cout, B, H, W, 0, ep0, None))
        nat.check(L.mm_nn_conv3x3_wgrad_tc(_p(dyd), cout, 0, cout, _p(xd), cin, 0, cin, _p(dw), B, H, W, ep1, None))
        torch.cuda.synchronize()
        assert err.cpu().tolist() == [1, 1]
    finally:
        nat.check(L.mm_nn_set_wait_limit(-1))
    err.zero_()
    dw.zero_()
    nat.check(L.mm_nn_conv3x3_tc(_p(xd), cin, 0, cin, _p(wd), None, _p(out), cout, 0, cout, B, H, W, 0, ep0, None))
    nat.check(L.mm_nn_conv3x3_wgrad_tc(_p(dyd), cout, 0, cout, _p(xd), cin, 0, cin, _p(dw), B, H, W, ep1, None))
    torch.cuda.synchronize()
    assert err.cpu().tolist() == [0, 0]
    ref = R.conv3x3(x, w)
    got = out.float().cpu().numpy().reshape(ref.shape)
    assert np.abs(got - ref).max() <= 2 ** -7 * np.abs(ref).max() + 1e-6
    _, rdw, _ = R.conv3x3_backward(x, w, dy)
    assert _relnorm(dw.cpu().numpy().reshape(rdw.shape), rdw) < 1e-3


@pytest.mark.parametrize("C,P,relu", [(16, 5000, 1), (32, 70000, 1), (384, 3000, 1), (64, 777, 0), (256, 12345, 1)])
def test_relu_bias_bwd_matches(C, P, relu):
    """The fused ReLU backward and bias gradient: the masked gradient exactly, the channel
    sums to 1e-5 relative (FP32 sums in another order)."""
    import torch
    import unet_ref as R
    from mumax2 import _native as nat
    rng = np.random.default_rng(C + P)
    out = R.bf16(rng.normal(size=(P, C)))
    d = R.bf16(rng.normal(size=(P, C)))
    od, dd = _dev(out, torch.bfloat16), _dev(d, torch.bfloat16)
    db = torch.zeros(C, dtype=torch.float32, device="cuda")
    nat.check(nat.lib().mm_nn_relu_bias_bwd(_p(od), C, 0, _p(dd), C, 0, C, P, relu, _p(db), None))
    ref = np.where(out > 0, d, 0.0) if relu else d
    assert np.array_equal(dd.float().cpu().numpy().reshape(P, C), ref)
    assert _relnorm(db.cpu().numpy(), ref.sum(axis=0)) < 1e-5


@pytest.mark.parametrize("co", [16, 2])
@pytest.mark.parametrize("kernel", ["tcgen05", "tcgen05-persistent", "mma.sync"])
@pytest.mark.parametrize("cin,cout,B,H,W", [(384, 128, 4, 16, 16), (32, 32, 3, 64, 64), (96, 32, 2, 8, 16),
                                            (16, 16, 3, 5, 7)])
def test_convolution_writes_only_its_output(kernel, cin, cout, B, H, W, co):
    """Output canary: the convolution writes a channel slice (offset co, Cout channels) of a
    wider pixel-major buffer that sits between two guard regions (offset 16: 16-byte
    vector stores; offset 2: the pair stores).  Every element outside
    the slice -- the other channels of each pixel and both guards -- must keep its canary
    value, and the slice must match the oracle."""
    import torch
    import unet_ref as R
    from mumax2 import _native as nat
    rng = np.random.default_rng(cin + 3 * cout + B)
    x = R.bf16(rng.normal(size=(B, H, W, cin)))
    w = R.bf16(rng.normal(size=(cout, 9, cin)) / np.sqrt(9 * cin))
    b = rng.normal(size=cout).astype(np.float32)
    xd, wd = _dev(x, torch.bfloat16), _dev(w, torch.bfloat16)
    bd = torch.tensor(b, device="cuda")
    P = B * H * W
    cs, guard = cout + 48, 1 << 16                    # row stride, guard elements
    canary = 0x7F7B                                   # a bf16 NaN payload no kernel computes
    buf = torch.full((2 * guard + P * cs,), canary, dtype=torch.int16, device="cuda")
    out = buf[guard:guard + P * cs]
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    L = nat.lib()
    if kernel.startswith("tcgen05"):
        nat.check(L.mm_nn_set_conv_kernel(1 if kernel.endswith("persistent") else 0))
        nat.check(L.mm_nn_conv3x3_tc(_p(xd), cin, 0, cin, _p(wd), _p(bd), _p(out), cs, co, cout, B, H, W, 1,
                                     _p(err), None))
        nat.check(L.mm_nn_set_conv_kernel(0))
    else:
        nat.check(L.mm_nn_conv3x3(_p(xd), cin, 0, cin, _p(wd), _p(bd), _p(out), cs, co, cout, B, H, W, 1, None))
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    h = buf.cpu().numpy()
    assert (h[:guard] == canary).all() and (h[guard + P * cs:] == canary).all(), "store outside the buffer"
    body = h[guard:guard + P * cs].reshape(P, cs)
    outside = np.ones(cs, dtype=bool)
    outside[co:co + cout] = False
    assert (body[:, outside] == canary).all(), "store into a channel outside the slice"
    got = torch.from_numpy(body[:, co:co + cout].copy()).view(torch.bfloat16).float().numpy()
    ref = np.maximum(R.conv3x3(x, w, b), 0).reshape(P, cout)
    assert np.abs(got - ref).max() <= 2 ** -7 * np.abs(ref).max() + 1e-6
