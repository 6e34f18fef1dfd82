"""Test infrastructure: numpy restatement of the warm-start U-Net (2_b200/mumax2/unet.py
architecture) in float64, with bf16 rounding at the points where the GPU kernels store
bf16 values (activations, pooled and upsampled maps, activation gradients), used as the
checker of the GPU forward pass and gradients.  It is never part of the product path.
"""
import numpy as np


def bf16(x):
    """Round to bfloat16 (round to nearest even) and return float64."""
    f = np.asarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def conv3x3(x, w, b=None):
    """x [B,H,W,Ci], w [Co,9,Ci] -> [B,H,W,Co] (zero padding), float64."""
    B, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    out = np.zeros((B, H, W, w.shape[0]))
    for tap in range(9):
        dy, dx = tap // 3, tap % 3
        out += np.einsum("bhwc,oc->bhwo", xp[:, dy:dy + H, dx:dx + W, :], w[:, tap, :])
    if b is not None:
        out += b
    return out


def conv3x3_backward(x, w, dpre):
    """-> (dx [B,H,W,Ci], dw [Co,9,Ci], db [Co])"""
    B, H, W, _ = x.shape
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w, dtype=np.float64)
    for tap in range(9):
        dy, dx = tap // 3, tap % 3
        dw[:, tap, :] = np.einsum("bhwo,bhwc->oc", dpre, xp[:, dy:dy + H, dx:dx + W, :])
        dxp[:, dy:dy + H, dx:dx + W, :] += np.einsum("bhwo,oc->bhwc", dpre, w[:, tap, :])
    return dxp[:, 1:-1, 1:-1, :], dw, dpre.sum(axis=(0, 1, 2))


def pool(x):
    B, H, W, C = x.shape
    return x.reshape(B, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def upsample(x):
    return x.repeat(2, axis=1).repeat(2, axis=2)


def forward_backward(arch, params, feats, target, mask, H, W):
    """arch: the (BUFFERS, CONVS, POOLS, UPS, SCHEDULE) tuple of unet.py; params {name:
    (w [Co,9,Ci], b)}; feats [B,H*W,FEAT]; target [B,H*W,3]; mask [B,H*W].
    Returns (loss, grads {name: (dw, db)}, out [B,H*W,Co_out])."""
    BUFFERS, CONVS, POOLS, UPS, SCHEDULE = arch
    B = feats.shape[0]
    buf = {}
    for k, (lvl, ch) in BUFFERS.items():
        buf[k] = np.zeros((B, H >> lvl, W >> lvl, ch))
    buf["in"][...] = bf16(feats).reshape(B, H, W, -1)
    wq = {n: bf16(params[n][0]) for n in params}
    convs = {c[0]: c for c in CONVS}
    for op in SCHEDULE:
        if op.startswith("pool"):
            (sv, so), (dv, do), ch, _ = POOLS[int(op[4:])]
            buf[dv][..., do:do + ch] = bf16(pool(buf[sv][..., so:so + ch]))
        elif op.startswith("up"):
            (sv, so), (dv, do), ch, _ = UPS[int(op[2:])]
            buf[dv][..., do:do + ch] = upsample(buf[sv][..., so:so + ch])
        else:
            name, (iv, io), cin, (ov, oo), cout, relu = convs[op]
            y = conv3x3(buf[iv][..., io:io + cin], wq[name], params[name][1])
            if relu:
                y = np.maximum(y, 0.0)
            buf[ov][..., oo:oo + cout] = bf16(y)
    out = buf["out"]
    o3 = out[..., :3].reshape(B, H * W, 3)
    norm = max(1.0, mask.sum()) * 3.0
    diff = o3 - target
    loss = float((mask[..., None] * diff * diff).sum() / norm)
    grad = {k: np.zeros_like(v) for k, v in buf.items()}
    g = np.zeros_like(out)
    g[..., :3] = bf16(2.0 * mask[..., None] * diff / norm).reshape(B, H, W, 3)
    grad["out"] = g
    grads = {}
    for op in reversed(SCHEDULE):
        if op.startswith("pool"):
            (sv, so), (dv, do), ch, _ = POOLS[int(op[4:])]
            up = upsample(grad[dv][..., do:do + ch]) * 0.25
            grad[sv][..., so:so + ch] = bf16(grad[sv][..., so:so + ch] + up)
        elif op.startswith("up"):
            (sv, so), (dv, do), ch, _ = UPS[int(op[2:])]
            d = grad[dv][..., do:do + ch]
            Bq, Hh, Ww, _ = d.shape
            grad[sv][..., so:so + ch] = bf16(d.reshape(Bq, Hh // 2, 2, Ww // 2, 2, ch).sum(axis=(2, 4)))
        else:
            name, (iv, io), cin, (ov, oo), cout, relu = convs[op]
            dpre = grad[ov][..., oo:oo + cout].copy()
            if relu:
                dpre[buf[ov][..., oo:oo + cout] <= 0] = 0.0
                grad[ov][..., oo:oo + cout] = dpre
            dx, dw, db = conv3x3_backward(buf[iv][..., io:io + cin], wq[name], dpre)
            grads[name] = (dw, db)
            if name != "e0a":
                grad[iv][..., io:io + cin] = bf16(dx)
    return loss, grads, out.reshape(B, H * W, -1)
