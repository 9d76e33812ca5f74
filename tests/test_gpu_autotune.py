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


def test_per_class_autotune_keeps_results(cuda_lib):
    """A batch of instances spanning three size classes: every per-class
    choice (register-cap variant, Morton or vertex thread order) gives the
    same states bit for bit, and the per-class autotuner neither advances nor
    perturbs the scene."""
    from ysim_b200 import generators as G
    from ysim_b200.scene import Scene
    spec = G.config_c4(instances=12, lo=16, hi=140, level=2, drop=0.001)
    sizes = sorted({m.nV for m in spec.meshes if m.grid_n})
    assert sizes[0] <= 4096 < sizes[-1] and any(4096 < n <= 16384 for n in sizes)
    runs = []
    for variant, order in ((8, True), (7, False), (4, True)):
        s = Scene(spec)
        try:
            s.set_fused_variant(variant)
            s.set_thread_order(order)
            s.step(110)
            runs.append((s.get("x"), s.get("v"), s.totals()))
            assert s.stats()["flags"] == 0
        finally:
            s.close()
    for x, v, t in runs[1:]:
        assert np.array_equal(x.view(np.uint32), runs[0][0].view(np.uint32))
        assert np.array_equal(v.view(np.uint32), runs[0][1].view(np.uint32))
        assert t == runs[0][2]
    s = Scene(spec)
    try:
        s.step(90)
        x0, t0 = s.get("x"), s.totals()
        classes = s.autotune_classes(reps=2)
        assert len(classes) >= 2 and sum(c["vertices"] for c in classes) == sum(m.nV for m in spec.meshes
                                                                               if m.grid_n)
        assert all(c["ctas_per_sm"] in (8, 7, 4) and c["thread_order"] in ("morton", "vertex", "tile") for c in classes)
        assert np.array_equal(s.get("x").view(np.uint32), x0.view(np.uint32)) and s.totals() == t0
        s.step(20)
        assert np.array_equal(s.get("x").view(np.uint32), runs[0][0].view(np.uint32))
        assert s.totals() == runs[0][2] and s.totals()[1] > 0
    finally:
        s.close()
