"""The numpy U-Net oracle pinned by finite differences (exact float64 arithmetic, bf16
rounding switched off): its analytic weight gradients are the derivative of its loss."""
import numpy as np
import pytest


def test_oracle_gradients_are_the_loss_derivative(monkeypatch):
    import unet_ref as R
    from mumax2 import unet as U
    monkeypatch.setattr(R, "bf16", lambda x: np.asarray(x, dtype=np.float64))
    B, H, W = 1, 8, 8
    rng = np.random.default_rng(0)
    params = U.init_params(1)
    for n in params:
        w, b = params[n]
        params[n] = (w.astype(np.float64), 0.05 * rng.normal(size=b.shape))
    feats = np.zeros((B, H * W, U.FEAT))
    feats[..., :9] = rng.normal(size=(B, H * W, 9))
    target = rng.normal(size=(B, H * W, 3))
    mask = np.ones((B, H * W))
    arch = (U.BUFFERS, U.CONVS, U.POOLS, U.UPS, U.SCHEDULE)
    L0, g, _ = R.forward_backward(arch, params, feats, target, mask, H, W)
    checked = 0
    for name in ["e0a", "e1a", "d1a", "d0b", "out"]:
        w, b = params[name]
        for _ in range(4):
            idx = tuple(int(rng.integers(0, s)) for s in w.shape)
            if name == "out":
                idx = (int(rng.integers(0, 3)),) + idx[1:]
            if name == "e0a":
                idx = idx[:2] + (int(rng.integers(0, 9)),)
            if g[name][0][idx] == 0.0:
                continue
            eps = 1e-6 * max(1.0, abs(w[idx]))
            w2 = w.copy()
            w2[idx] += eps
            p2 = dict(params)
            p2[name] = (w2, b)
            L1, _, _ = R.forward_backward(arch, p2, feats, target, mask, H, W)
            assert (L1 - L0) / eps == pytest.approx(g[name][0][idx], rel=1e-3, abs=1e-9)
            checked += 1
    assert checked >= 8
