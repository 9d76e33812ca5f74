"""Batched scenes: many independent cloth instances (each with its own
obstacle, group-separated) in one scene equal the same instances run one
scene each, bit for bit, through rebuilds and contacts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batched_equals_plain_per_instance(cuda_lib):
    from ysim_b200 import generators as G
    from ysim_b200.scene import Scene
    spec = G.config_c4(instances=6, lo=8, hi=24, level=2, drop=0.001)
    parts = G.split_instances(spec)
    assert len(parts) == 6
    batched = Scene(spec)
    plain = [Scene(p) for p in parts]
    try:
        n = 120  # crosses the rebuild at substep 100 (10 frames of 10)
        batched.step(n)
        for p in plain:
            p.step(n)
        xb = batched.get("x")
        off = 0
        contacts = 0
        for p, q in zip(parts, plain):
            xp = q.get("x")
            assert np.array_equal(xb[off:off + p.nV].view(np.uint32), xp.view(np.uint32))
            off += p.nV
            contacts += q.totals()[1]
            assert q.stats()["flags"] == 0
        assert off == spec.nV
        assert batched.stats()["flags"] == 0
        assert batched.totals()[1] == contacts > 0
    finally:
        batched.close()
        for q in plain:
            q.close()
