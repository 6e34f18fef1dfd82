"""The per-layer convolution timing module (`mumax2.unet_timing`): its layer shapes follow
the network's definition (CPU), and both of its modes run through the C-ABI (GPU, a
batch of 2)."""
import pytest


def test_layer_shapes_follow_the_network():
    from mumax2 import unet as U
    from mumax2 import unet_timing as T
    shapes = list(T.layer_shapes())
    assert [s[0] for s in shapes] == [c[0] for c in U.CONVS]
    by = {s[0]: s for s in shapes}
    assert by["e0a"][1:5] == (U.FEAT, 32, 64, 64)
    assert by["d2a"][1:5] == (384, 128, 16, 16)
    assert by["e3b"][1:5] == (256, 256, 8, 8)
    assert by["out"][2] == U.OUTC and by["out"][5] is False


@pytest.mark.gpu
def test_timing_modes_run():
    from mumax2 import unet_timing as T
    rows = T.time_layers(batch=2, reps=1, warmup=1, layers={"e0b", "d2a"})
    assert [r["layer"] for r in rows] == ["e0b", "d2a"]
    for r in rows:
        for k in ("tc_us", "tc_persistent_us", "mma_us", "wgrad_mma_us", "wgrad_tc_us"):
            assert r[k] > 0
    T.main(["--batch", "2", "--layer", "e1a", "--launches", "1"])
