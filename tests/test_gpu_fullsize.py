"""Parity on the benchmark configurations at their full sizes.

C2: the 512x512 TriangularCloth (262,144 vertices, 522,242 triangles) with
hash-semantics self rows over the displaced level-7 icosphere (327,680
triangles), pre-rolled on the GPU into the contact phase of the drape (500
substeps: about 11k contacts and 1.4M candidate rows per substep).  The
state is copied into a fresh GPU scene and a fresh oracle scene, which then
step side by side: the substep body of Simulator::update
(simulator.hpp:3512-3815), a frame-0 tree rebuild from the draped state, and
a later frame boundary with a rebuild.  Candidate-row counts, per-vertex
contact offsets and (object, triangle) lists must be equal; positions and
velocities within 1e-5 relative max-abs per substep (they come out
bit-identical).

C4: all 256 batched instances (sides U{16..256}, 6.0M cloth vertices) in one
scene against the same instances as 256 scenes, bit for bit, through
contacts and a rebuild.
"""
import dataclasses

import numpy as np
import pytest

from helpers import canon_rows, rel_err

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

TOL = 1e-5       # relative max-abs per substep (positions, velocities, forces)
PREROLL = 500    # substeps into the drape: first contacts come near substep 370


@pytest.fixture(scope="module")
def c2_draped(cuda_lib):
    """The C2 scene pre-rolled on the GPU into the contact phase: (spec, x, v,
    xprev).  The pre-roll follows the oracle bit for bit (the small-scene
    tests check the trajectory), so this is the oracle's state too."""
    from ysim_b200 import generators as G
    from ysim_b200.scene import Scene
    spec = G.config_c2()
    s = Scene(spec)
    try:
        s.step(PREROLL)
        st = s.stats()
        assert st["flags"] == 0, st
        assert st["contacts"] > 5000, st
        return spec, s.get("x"), s.get("v"), s.get("xprev")
    finally:
        s.close()


def _every_frame_rebuilds(spec):
    """The same scene with a tree rebuild at every frame start.  Trees change
    no result (every leaf box is exact whenever it was built), so the
    trajectory is the benchmark's; the frame boundary at substep 20 then also
    rebuilds."""
    return dataclasses.replace(spec, params=dataclasses.replace(spec.params, rebuild_frames=1))


def _pair(spec, state, oracle, **kw):
    from ysim_b200.scene import Scene
    s = Scene(spec, **kw)
    o = oracle.OracleScene(spec)
    for k, a in zip(("x", "v", "xprev"), state):
        s.set(k, a)
        o.set(k, a)
    return s, o


def test_c2_full_size_fused_matches_oracle(c2_draped, oracle):
    """The fused substep (the benchmark's path) against the oracle for 22
    substeps from the draped state: the frame-0 rebuild, 19 refit-only
    substeps, then the frame-1 boundary with its rebuild."""
    spec, *state = c2_draped
    spec = _every_frame_rebuilds(spec)
    s, o = _pair(spec, state, oracle)
    try:
        s.set_record(True)
        seen = 0
        for sub in range(22):
            s.step(1)
            o.step(1)
            gs, os_ = s.stats(), o.stats()
            assert gs["broad_rows"] == os_["broad_rows"], (sub, gs, os_)
            goff, gc = s.contacts()
            ooff, oc = o.contacts()
            assert np.array_equal(goff, ooff), f"contact offsets differ at substep {sub}"
            assert np.array_equal(gc["tobj"], oc["tobj"]) and np.array_equal(gc["tri"], oc["tri"]), sub
            assert np.array_equal(np.stack([gc["nx"], gc["ny"], gc["nz"], gc["d"]], 1).view(np.uint32),
                                  np.concatenate([oc["n"], oc["d"][:, None]], 1).view(np.uint32)), sub
            assert rel_err(s.get("x"), o.get("x")) <= TOL, sub
            assert rel_err(s.get("v"), o.get("v")) <= TOL, sub
            seen += int(goff[-1])
            # the per-vertex contact list (32 entries) never overflowed
            assert gs["flags"] == 0, (sub, gs)
        assert seen > 22 * 5000
        assert np.array_equal(s.get("x").view(np.uint32), o.get("x").view(np.uint32))
    finally:
        s.close()


def test_c2_full_size_wide_refit_boxes_exact(c2_draped):
    """The cloth's 4-wide tree after a refit of the draped state: leaf slots
    are the swept leaf boxes, internal slots the unions of their children."""
    from test_gpu_parity import check_wide_boxes
    from ysim_b200.scene import Scene
    spec, *state = c2_draped
    s = Scene(spec)
    try:
        for k, a in zip(("x", "v", "xprev"), state):
            s.set(k, a)
        s.step(3)
        assert check_wide_boxes(s, spec) > 100_000
    finally:
        s.close()


def test_c2_full_size_staged_matches_oracle(c2_draped, oracle):
    """The staged path, stage by stage (broad rows, narrow contacts, forces,
    integration), for 3 substeps from the draped state."""
    spec, *state = c2_draped
    s, o = _pair(spec, state, oracle)
    try:
        for sub in range(3):
            o.stage(0); o.stage(1); o.stage(2)
            orows = o.rows()
            o.stage(3)
            ooff, oc = o.contacts()
            o.stage(4)
            o.stage(5)
            s.broad_phase.build(); s.broad_phase.refit_swept(); s.broad_phase.detect_collisions()
            grows = s.rows()
            assert len(grows) == len(orows) > 1_000_000, sub
            assert np.array_equal(canon_rows(grows), canon_rows(orows)), f"rows differ at substep {sub}"
            s.narrow_phase.narrow_and_sort_by_vertices()
            goff, gc = s.contacts()
            assert int(goff[-1]) > 5000
            assert np.array_equal(goff, ooff)
            assert np.array_equal(gc["tobj"], oc["tobj"]) and np.array_equal(gc["tri"], oc["tri"])
            s.system.snapshot_xprev()
            s.system.update()
            assert rel_err(s.get("f"), o.get("f")) <= TOL
            assert rel_err(s.get("x"), o.get("x")) <= TOL
            assert rel_err(s.get("v"), o.get("v")) <= TOL
            assert rel_err(s.get("xprev"), o.get("xprev")) <= TOL
        assert s.stats()["flags"] == 0
    finally:
        s.close()


@pytest.mark.parametrize("variant", ["bvh_self", "reference_tree"])
def test_c2_full_size_variants_match_oracle(c2_draped, oracle, variant):
    """The other two forms of C2 from the draped state, fused, 3 substeps:
    BVH self rows (checkSelfCollisions, the reference's YSIM_CPUSH_SELF=0
    path) and the reference's own tree layout (per-axis Morton box)."""
    from ysim_b200 import _lib
    spec, *state = c2_draped
    kw = {}
    if variant == "bvh_self":
        spec = dataclasses.replace(spec, params=dataclasses.replace(spec.params, self_mode=_lib.SELF_BVH))
    else:
        kw["tree_layout"] = _lib.TREE_REFERENCE
    s, o = _pair(spec, state, oracle, **kw)
    try:
        s.set_record(True)
        for sub in range(3):
            s.step(1)
            o.step(1)
            assert s.stats()["broad_rows"] == o.stats()["broad_rows"], sub
            goff, gc = s.contacts()
            ooff, oc = o.contacts()
            assert int(goff[-1]) > 5000
            assert np.array_equal(goff, ooff), sub
            assert np.array_equal(gc["tobj"], oc["tobj"]) and np.array_equal(gc["tri"], oc["tri"]), sub
            assert rel_err(s.get("x"), o.get("x")) <= TOL, sub
            assert rel_err(s.get("v"), o.get("v")) <= TOL, sub
        assert s.stats()["flags"] == 0
    finally:
        s.close()


def test_c4_full_256_batched_equals_plain(cuda_lib):
    """All 256 C4 instances as one scene against 256 scenes, bit for bit,
    for 120 substeps (contacts from about substep 85, the rebuild at 100)."""
    from ysim_b200 import generators as G
    from ysim_b200.scene import Scene
    spec = G.config_c4(drop=0.001)
    parts = G.split_instances(spec)
    assert len(parts) == 256
    n = 120
    batched = Scene(spec)
    try:
        batched.step(n)
        xb, vb = batched.get("x"), batched.get("v")
        assert batched.stats()["flags"] == 0
        bc = batched.totals()[1]
    finally:
        batched.close()
    off = contacts = 0
    for p in parts:
        q = Scene(p)
        try:
            q.step(n)
            assert np.array_equal(xb[off:off + p.nV].view(np.uint32), q.get("x").view(np.uint32))
            assert np.array_equal(vb[off:off + p.nV].view(np.uint32), q.get("v").view(np.uint32))
            assert q.stats()["flags"] == 0
            contacts += q.totals()[1]
            off += p.nV
        finally:
            q.close()
    assert off == spec.nV
    assert bc == contacts > 0
