"""Tile thread order of the fused substep (YS_ORDER_TILE): each CTA is one
16 x 8 tile of a FastGridCloth whose positions and velocities (with a
2-vertex halo) come into shared memory by TMA, and every stencil spring with
an end in the tile is evaluated once for both ends.  The force on the second
end is the exact negation of the force on the first, and each vertex sums its
12 springs in compute_cloth_grid_forces_fast's order (physics.metal:197-218),
so the states must equal the per-vertex stencil's bit for bit: on ragged
sides (tiles cut by the mesh edge), on the smallest grids, through contacts
and rebuilds, with per-spring stiffness and rest length, and against the
oracle."""
import ctypes as C

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu


def _run(spec, order, steps, variant=None, springs=None):
    import torch
    from ysim_b200 import _lib
    from ysim_b200.scene import Scene
    s = Scene(spec)
    try:
        if variant:
            s.set_fused_variant(variant)
        s.set_thread_order(order)
        keep = None
        if springs is not None:
            keep = [torch.from_numpy(a).cuda() for a in springs]
            torch.cuda.synchronize()
            _lib.check(s.lib.ys_scene_set_grid_springs(s.h, 0, C.c_void_p(keep[0].data_ptr()),
                                                       C.c_void_p(keep[1].data_ptr())))
        s.step(steps)
        st = s.stats()
        return s.get("x"), s.get("v"), s.totals(), st["flags"]
    finally:
        s.close()


def _same(a, b):
    assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32))
    assert np.array_equal(a[1].view(np.uint32), b[1].view(np.uint32))
    assert a[2] == b[2]


def test_tile_order_ragged_batch_is_bit_identical(cuda_lib):
    """Instances of sides 3..70 (every remainder of 16 and 8, tiles that are
    mostly padding) through first contacts and the frame-10 rebuild: tile
    order equals vertex and Morton order bit for bit, at every register cap."""
    from ysim_b200 import generators as G
    spec = G.config_c4(instances=24, lo=3, hi=70, level=2, drop=0.001)
    sides = sorted({m.grid_n for m in spec.meshes if m.grid_n})
    assert sides[0] < 8 and any(n % 16 not in (0, 8) for n in sides)
    ref = _run(spec, "vertex", 110)
    assert ref[3] == 0 and ref[2][1] > 0  # contacts were made
    for order, variant in (("tile", 8), ("tile", 7), ("tile", 4), ("morton", 8)):
        out = _run(spec, order, 110, variant)
        assert out[3] == 0, (order, variant)
        _same(out, ref)


def test_tile_order_per_spring_parameters(cuda_lib):
    """Random per-spring stiffness and rest length (the adjoint's form, each
    spring's own id in the tile table) give the per-vertex result."""
    from ysim_b200 import generators as G
    spec = G.config_c5(N=37, level=2, height=0.2995)
    c = spec.meshes[0]
    k, L = G.grid_spring_params(c.grid_n, c.grid_rest, (c.kstretch, c.kshear, c.kbend))
    rng = np.random.default_rng(11)
    k = (k * np.exp(rng.normal(0, 0.3, k.shape))).astype(np.float32)
    L = (L * (1 + rng.uniform(-0.05, 0.05, L.shape))).astype(np.float32)
    ref = _run(spec, "vertex", 60, springs=(k, L))
    out = _run(spec, "tile", 60, springs=(k, L))
    assert out[3] == 0
    _same(out, ref)
    plain = _run(spec, "vertex", 60)
    assert not np.array_equal(plain[0].view(np.uint32), ref[0].view(np.uint32))  # the arrays did act


def test_tile_order_matches_oracle(cuda_lib, oracle):
    """C1's cloth (64 x 64 over the level-4 icosphere) in tile order against
    the oracle, substep by substep, in contact with the obstacle."""
    from ysim_b200 import generators as G
    from ysim_b200.scene import Scene
    spec = G.config_c1(height=0.2999)  # starts on the obstacle top
    s = Scene(spec)
    o = oracle.OracleScene(spec)
    try:
        s.set_thread_order("tile")
        for sub in range(60):
            s.step(1)
            o.step(1)
            assert rel_err(s.get("x"), o.get("x")) <= 1e-5, sub
            assert rel_err(s.get("v"), o.get("v")) <= 1e-5, sub
        assert s.totals()[1] > 0  # contacts were made
        assert np.array_equal(s.get("x").view(np.uint32), o.get("x").view(np.uint32))
        assert s.stats()["flags"] == 0
    finally:
        s.close()


def test_tile_order_with_triangle_cloth_in_class(cuda_lib):
    """A size class holding a TriangularCloth beside a grid cloth: in tile
    order the triangle cloth keeps vertex order from a CTA boundary with its
    CSR springs, and the scene equals vertex order bit for bit."""
    from ysim_b200 import generators as G
    spec = G.config_c1(P=40, level=2, height=0.2999)
    tri = G.config_c2(P=21, level=2, obstacle=False).meshes[0]
    tri.x = (tri.x + np.array([0.2, 0.1, 0.0], np.float32)).astype(np.float32)
    spec.meshes.append(tri)
    ref = _run(spec, "vertex", 80)
    assert ref[3] == 0 and ref[2][1] > 0
    for variant in (8, 4):
        out = _run(spec, "tile", 80, variant)
        assert out[3] == 0
        _same(out, ref)


def test_tile_order_signed_zeros(cuda_lib):
    """Gravity with -0 components on a cloth at rest: the first substep's
    spring forces are signed zeros (zero strain, zero velocity) and the force
    sums start at -0, so a spring shared by its two ends must give the second
    end the value it would compute itself (a component with dx exactly zero
    keeps its sign) for the states to stay bit-identical."""
    import dataclasses
    from ysim_b200 import generators as G
    spec = G.config_c1(P=37, level=2, height=0.2999)
    spec = dataclasses.replace(spec, params=dataclasses.replace(spec.params, gravity=(-0.0, -9.81, -0.0)))
    for steps in (1, 2, 30):
        ref = _run(spec, "vertex", steps)
        out = _run(spec, "tile", steps)
        _same(out, ref)


def test_thread_order_rejects_unknown_order(cuda_lib):
    """Only vertex (0), Morton (1) and tile (2) order exist."""
    from ysim_b200 import _lib
    from ysim_b200 import generators as G
    from ysim_b200.scene import Scene
    s = Scene(G.config_c1(P=16, level=1, height=0.2999))
    try:
        assert s.lib.ys_scene_set_thread_order(s.h, 3) == _lib.YS_ERR_BAD_ARG
        assert s.lib.ys_scene_set_thread_order(s.h, -1) == _lib.YS_ERR_BAD_ARG
        s.set_thread_order("tile")
        s.step(2)
        assert s.stats()["flags"] == 0
    finally:
        s.close()
