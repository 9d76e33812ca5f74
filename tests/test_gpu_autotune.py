"""The fused kernel's register-cap variants and the autotuner: every variant
gives the same positions bit for bit, and autotuning neither advances nor
perturbs the scene."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _spec():
    from ysim_b200 import generators as G
    return G.config_c2(P=40, level=3, height=0.33, gravity=-9.81)


def test_fused_variants_agree_and_autotune_keeps_state(cuda_lib):
    from ysim_b200.scene import Scene
    spec = _spec()
    outs = []
    for v in (8, 7, 4):
        s = Scene(spec)
        try:
            s.set_fused_variant(v)
            s.step(30)
            outs.append((s.get("x"), s.get("v"), s.totals()))
            assert s.stats()["flags"] == 0
        finally:
            s.close()
    for x, v, t in outs[1:]:
        assert np.array_equal(x.view(np.uint32), outs[0][0].view(np.uint32))
        assert np.array_equal(v.view(np.uint32), outs[0][1].view(np.uint32))
        assert t == outs[0][2]
    s = Scene(spec)
    try:
        s.step(20)
        x0, t0 = s.get("x"), s.totals()
        chosen, ms = s.autotune(reps=3)
        assert chosen in (8, 7, 4) and all(m > 0 for m in ms)
        assert np.array_equal(s.get("x").view(np.uint32), x0.view(np.uint32))
        assert s.totals() == t0
        s.step(10)
        assert np.array_equal(s.get("x").view(np.uint32), outs[0][0].view(np.uint32))
        assert s.totals() == outs[0][2]
    finally:
        s.close()
