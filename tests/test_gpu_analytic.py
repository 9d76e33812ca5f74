"""GPU analytic colliders (narrow_pt_analytic, src/metal/bruteforce.metal:236-499,
with the broad-phase markers of bvh.hpp:2886-2941) through the C ABI: the
standalone narrow phase against the reference kernel's golden contacts and the
oracle, and whole substeps of a scene with every collider kind -- static and
moving -- against the oracle on the staged and the fused path."""
import ctypes as C
import os

import numpy as np
import pytest

from analytic_cases import RADIUS, THICKNESS, canon_contacts, cases
from helpers import rel_err

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-5  # relative max-abs per substep (positions, velocities)


def _narrow(cuda_lib, shapes, x, xp, so, beh, pairs, radius, thickness, cap=None):
    import torch
    from oracle.oracle import CONTACT_DTYPE
    from ysim_b200 import _lib
    dx = torch.from_numpy(np.ascontiguousarray(x).reshape(-1)).cuda()
    dxp = torch.from_numpy(np.ascontiguousarray(xp).reshape(-1)).cuda()
    cap = len(x) * max(len(pairs), 1) if cap is None else cap
    out = torch.zeros(max(cap, 1) * 48, dtype=torch.uint8, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    sh = np.ascontiguousarray(shapes)
    so = np.ascontiguousarray(so, np.uint32)
    be = np.ascontiguousarray(beh, np.uint32)
    pr = np.ascontiguousarray(pairs, np.uint32)
    vp = C.c_void_p
    _lib.check(cuda_lib.ys_narrow_analytic(vp(dx.data_ptr()), vp(dxp.data_ptr()), so.ctypes.data_as(vp),
                                           be.ctypes.data_as(vp), len(be), sh.ctypes.data_as(vp), len(sh),
                                           pr.ctypes.data_as(vp), len(pr), float(radius), float(thickness),
                                           vp(out.data_ptr()), cap, vp(cnt.data_ptr()), None), "ys_narrow_analytic")
    torch.cuda.synchronize()
    n = int(cnt.item())
    return out.cpu().numpy().view(CONTACT_DTYPE)[: min(n, cap)], n


def test_gpu_analytic_matches_golden(cuda_lib, oracle):
    g = np.load(os.path.join(GOLD, "analytic.npz"))
    shapes = g["shapes"].view(oracle.SHAPE_DTYPE)
    ref = g["contacts"].view(oracle.CONTACT_DTYPE)
    gc, n = _narrow(cuda_lib, shapes, g["x"], g["xprev"], g["state_off"], g["beh"], g["pairs"], g["radius"],
                    g["thickness"])
    assert n == len(ref) > 1000
    assert np.array_equal(canon_contacts(gc).view(np.uint8), ref.view(np.uint8))


def test_gpu_analytic_matches_oracle_and_caps(cuda_lib, oracle):
    shapes, x, xp, so, beh, pairs = cases(seed=31, per_shape=20_000)
    oc, n = oracle.narrow_analytic(x, xp, so, beh, shapes, pairs, RADIUS, THICKNESS)
    gc, gn = _narrow(cuda_lib, shapes, x, xp, so, beh, pairs, RADIUS, THICKNESS)
    assert gn == n > 10_000
    assert np.array_equal(canon_contacts(gc).view(np.uint8), canon_contacts(oc).view(np.uint8))
    # more pairs than one launch carries, in a shuffled order, with unknown
    # colliders mixed in: the same contacts
    rep = np.concatenate([pairs] * 3)
    rep = rep[np.random.default_rng(0).permutation(len(rep))]
    rep = np.concatenate([rep, [[0, 9999]]]).astype(np.uint32)
    gc3, gn3 = _narrow(cuda_lib, shapes, x, xp, so, beh, rep, RADIUS, THICKNESS)
    assert gn3 == 3 * n
    # contacts beyond the capacity are counted, not written
    gcc, gnc = _narrow(cuda_lib, shapes, x, xp, so, beh, pairs, RADIUS, THICKNESS, cap=100)
    assert gnc == n and len(gcc) == 100


def _scene_spec():
    from ysim_b200 import generators as G
    base = G.config_c1(P=24, level=1, height=0.3)
    cloth = base.meshes[0]
    shapes = [
        G.analytic_collider(1, (0.0, 0.0, 0.0), (0.3, 0.3, 0.3)),
        G.analytic_collider(2, (0.3, 0.27, 0.3), (0.12, 0.04, 0.1), G.quat_axis_angle((0, 0, 1), 0.35)),
        G.analytic_collider(3, (-0.3, 0.22, -0.3), (0.08, 0.2, 0.08), G.quat_axis_angle((1, 0, 0), np.pi / 2)),
        G.analytic_collider(1, (-0.3, 0.26, 0.3), (0.12, 0.05, 0.08), G.quat_axis_angle((0, 1, 0), 0.5)),
        G.analytic_collider(4, (0.0, 0.285, 0.0)),
    ]
    return G.SceneSpec("analytic_kinds", base.params, [cloth] + shapes, 0)


def _move(frame):
    """Collider 1 (the sphere) drifts and spins from frame 1 on."""
    from ysim_b200 import generators as G
    return (1, 1, (0.0, -0.002 * frame, 0.001 * frame), (0.3, 0.3, 0.3),
            G.quat_axis_angle((0.3, 1.0, 0.2), 0.05 * frame))


def _check_shapes(s, o):
    a, b = s.colliders(), o.shapes()
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_scene_analytic_staged_and_fused_match_oracle(cuda_lib, oracle):
    from ysim_b200.scene import Scene
    spec = _scene_spec()
    sub = spec.params.substeps
    for fused in (False, True):
        s = Scene(spec)
        o = oracle.OracleScene(spec)
        try:
            if fused:
                s.set_record(True)
            total = 0
            for k in range(3 * sub + 2):
                if k % sub == 0 and k:
                    mv = _move(k // sub)
                    s.set_collider(*mv)
                    o.set_collider(*mv)
                if fused:
                    s.step(1)
                    o.step(1)
                else:
                    o.stage(0); o.stage(1); o.stage(2); o.stage(3)
                    s.broad_phase.build(); s.broad_phase.refit_swept(); s.broad_phase.detect_collisions()
                    s.narrow_phase.narrow_and_sort_by_vertices()
                if k % sub == 0:
                    _check_shapes(s, o)
                ooff, oc = o.contacts()
                goff, gc = s.contacts()
                assert np.array_equal(goff, ooff), f"contact offsets differ at substep {k}"
                assert np.array_equal(gc["tobj"], oc["tobj"]) and np.array_equal(gc["tri"], oc["tri"])
                assert np.array_equal(np.stack([gc["nx"], gc["ny"], gc["nz"], gc["d"]], 1).view(np.uint32),
                                      np.concatenate([oc["n"], oc["d"][:, None]], 1).view(np.uint32))
                total += len(oc)
                if not fused:
                    o.stage(4); o.stage(5)
                    s.system.snapshot_xprev(); s.system.update()
                assert rel_err(s.get("x"), o.get("x")) <= TOL
                assert rel_err(s.get("v"), o.get("v")) <= TOL
            kinds = set(np.unique(oc["tobj"]).tolist())
            assert {1, 2, 3, 4, 5} <= kinds, kinds  # every collider in contact
            assert total > 1000
            st = s.stats()
            assert st["flags"] == 0 and st["broad_rows"] == 0, st
        finally:
            s.close()


def test_scene_analytic_c1_drape_matches_oracle(cuda_lib, oracle):
    """C1's cloth draped over the analytic sphere, box, cylinder and floor
    (fused path, CUDA graphs on) for two frames from a mid-fall state."""
    from ysim_b200 import generators as G
    from ysim_b200.scene import Scene
    spec = G.config_c1_analytic(P=64, height=0.305)
    s = Scene(spec)
    o = oracle.OracleScene(spec)
    try:
        for f in range(2):
            o.step(spec.params.substeps)
            s.step(spec.params.substeps)
            assert rel_err(s.get("x"), o.get("x")) <= TOL
            assert rel_err(s.get("v"), o.get("v")) <= TOL
        assert s.stats()["contacts"] > 0 and s.stats()["flags"] == 0
    finally:
        s.close()
