"""Scene files on the GPU: a scene loaded from the reference's file format
(cloth over primitive colliders: the analytic sphere, box and cylinder the
primitives default to, a plane, and a sphere kept as triangles) steps like
the oracle on the fused and the staged path, and the headless runner writes
the FrameProfiler CSV and the sidecar run config."""
import os

import numpy as np
import pytest

from helpers import rel_err

pytestmark = pytest.mark.gpu

SCENES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scenes")
TOL = 1e-5


@pytest.mark.parametrize("fused", [True, False], ids=["fused", "staged"])
def test_loaded_scene_steps_like_the_oracle(cuda_lib, oracle, fused):
    from ysim_b200 import loader as L
    from ysim_b200.scene import Scene
    ls = L.load(os.path.join(SCENES, "drape.json"))
    assert ls.ext is None
    kinds = [m.collider[0] if m.collider else 0 for m in ls.spec.meshes]
    assert kinds == [0, 1, 2, 3, 4, 0]
    s = Scene(ls.spec)
    o = oracle.OracleScene(ls.spec)
    try:
        n = ls.spec.params.substeps
        for f in range(3):
            if fused:
                s.step(n)
            else:
                s.step_staged(n)
            o.step(n)
            assert rel_err(s.get("x"), o.get("x")) <= TOL, f
            assert rel_err(s.get("v"), o.get("v")) <= TOL, f
        st, ot = s.stats(), o.stats()
        assert st["flags"] == 0 and ot["contacts"] > 0
        if not fused:
            assert st["broad_rows"] == ot["broad_rows"] and st["contacts"] == ot["contacts_kept"]
    finally:
        s.close()


@pytest.mark.parametrize("level", ["in_frame", "per_frame", "none"])
def test_headless_run_writes_the_profile(cuda_lib, tmp_path, level):
    from ysim_b200 import run as RUN
    from ysim_b200 import scene_format as SF
    csv = str(tmp_path / "out" / "drape-3f.csv")
    summary = RUN.run(os.path.join(SCENES, "drape.json"), frames=3, csv_path=csv, level=level, quiet=True)
    assert summary["finite"] and summary["flags"] == 0 and summary["frames"] == 3
    if level == "none":
        assert not os.path.exists(csv)
        return
    rows = open(csv).read().splitlines()
    head = rows[0].split(",")
    assert head[:6] == ["frame_sequence", "wall_time_seconds", "frame_ms", "fps", "broad_collisions",
                        "narrow_collisions"]
    assert ("broad_refit" in head) == (level == "in_frame") and "physics_total" in head
    assert len(rows) == 4 and [r.split(",")[0] for r in rows[1:]] == ["0", "1", "2"]
    vals = np.array([[float(v) for v in r.split(",")] for r in rows[1:]])
    assert np.isfinite(vals).all() and (vals[:, 2] > 0).all() and (vals[:, 5] > 0).all()
    side = SF.read_run_config(SF.sidecar_scene_path(csv))
    assert len(side.scene.objects) == 6 and side.profile.frames == 4


def test_all_fields_scene_matches_the_oracle(cuda_lib, oracle, tmp_path):
    """Pins, a Rigid body, a plane collider, wind gates and the unsupported
    motion constraints (reported, not applied), staged: the same states and
    flags as the oracle.  The fixture's cloth (k / m = 1.5e6 at subh = 1/1200)
    is beyond the explicit integrator's stability limit, so both sides
    sanitise vertices and raise the non-finite flag alike."""
    from ysim_b200 import loader as L
    from ysim_b200 import run as RUN
    from ysim_b200.scene import Scene
    ls = L.load(os.path.join(SCENES, "all_fields.json"))
    s = Scene(ls.spec)
    o = oracle.OracleScene(ls.spec)
    try:
        for _ in range(2):
            s.step_staged(ls.spec.params.substeps)
            o.step(ls.spec.params.substeps)
            assert rel_err(s.get("x"), o.get("x")) <= TOL
            assert rel_err(s.get("v"), o.get("v")) <= TOL
        assert s.stats()["flags"] == o.stats()["flags"]
    finally:
        s.close()
    summary = RUN.run(os.path.join(SCENES, "all_fields.json"), frames=2, csv_path=str(tmp_path / "a.csv"),
                      quiet=True)
    assert summary["finite"] and any("spline" in w for w in summary["warnings"])


def test_external_force_buffer_equals_internal_gravity(cuda_lib):
    """applyEnvironmentForces' output given as a host buffer
    (ys_scene_set_external_forces) with g * m on the cloth and zero elsewhere
    steps the scene bit for bit like the kernels' own g * m, fused and
    staged, through contacts."""
    import ctypes as C
    from ysim_b200 import _lib, generators as G
    from ysim_b200.scene import Scene
    spec = G.config_c2(P=40, level=3, height=0.315, gravity=-9.81)
    g = np.asarray(spec.params.gravity, np.float32)
    ext = np.concatenate([(m.mass[:, None] * g[None, :]).astype(np.float32) if m.behavior in (0, 1)
                          else np.zeros((m.nV, 3), np.float32) for m in spec.meshes])
    for fused in (True, False):
        a, b = Scene(spec), Scene(spec)
        try:
            _lib.check(cuda_lib.ys_scene_set_external_forces(b.h, ext.ctypes.data_as(C.c_void_p)), "ext")
            for _ in range(3):
                for s in (a, b):
                    s.step(spec.params.substeps) if fused else s.step_staged(spec.params.substeps)
            assert np.array_equal(a.get("x").view(np.uint32), b.get("x").view(np.uint32))
            assert np.array_equal(a.get("v").view(np.uint32), b.get("v").view(np.uint32))
            assert a.totals() == b.totals()
            assert a.stats()["contacts"] == b.stats()["contacts"] > 0
        finally:
            a.close()
            b.close()


@pytest.mark.parametrize("gravity", [True, False], ids=["gravity_and_wind", "wind_only"])
def test_wind_scene_matches_the_oracle(cuda_lib, oracle, gravity):
    """The drape scene with wind (0.4, 0, -0.25) on the cloth, with and
    without its gravity gate: the loader's external-force buffer on the GPU
    against the oracle's own applyEnvironmentForces (simulator.hpp:3123-3166:
    g * m under the gravity gate, plus the wind vector per particle on
    wind-gated cloth, zero on Float meshes)."""
    import ctypes as C
    from ysim_b200 import _lib
    from ysim_b200 import loader as L
    from ysim_b200 import scene_format as SF
    from ysim_b200.scene import Scene
    cfg = SF.read_run_config(os.path.join(SCENES, "drape.json"))
    snap = cfg.scene
    snap.environment.wind = (0.4, 0.0, -0.25)
    snap.objects[0].apply_gravity = gravity
    ls = L.load(cfg, os.path.join(SCENES, "drape.json"))
    assert ls.ext is not None
    s = Scene(ls.spec)
    o = oracle.OracleScene(ls.spec)
    o.set_environment(snap.environment.wind, [(ob.apply_gravity, ob.apply_wind) for ob in snap.objects])
    try:
        ext = np.ascontiguousarray(ls.ext, np.float32)
        _lib.check(cuda_lib.ys_scene_set_external_forces(s.h, ext.ctypes.data_as(C.c_void_p)), "ext")
        n = ls.spec.params.substeps
        for f in range(3):
            s.step(n)
            o.step(n)
            assert np.array_equal(ext, o.get("ext")), f
            assert rel_err(s.get("x"), o.get("x")) <= TOL, f
            assert rel_err(s.get("v"), o.get("v")) <= TOL, f
        assert s.stats()["flags"] == 0
        x0 = ls.spec.meshes[0].x
        drift = (s.get("x")[: len(x0)] - x0).mean(0)
        assert drift[0] > 0 and drift[2] < 0  # blown along the wind
    finally:
        s.close()
