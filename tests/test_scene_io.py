"""Scene files, run configs, primitive meshes and profiles against the reference.

The loader (ysim_b200.scene_format, ysim_b200.primitives, ysim_b200.profiler)
is checked against the reference's own headers compiled for the host
(include/scene_format.hpp, sim_config.hpp, primitive_geometry.hpp,
FrameProfiler.hpp; oracle/ref_sceneio.cpp) when the reference checkout is
present, and always against the fixtures those produced
(tests/golden/make_golden.py).  ysim_b200.loader (snapshot -> scene) is
checked by the properties the reference's pack gives the packed state.
"""
import json
import os

import numpy as np
import pytest

import scene_cases as SCN

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gold():
    with open(os.path.join(GOLD, "scene_io.json")) as f:
        return json.load(f)


def _refk():
    try:
        from oracle import refkernels as R
    except Exception:
        return None
    return R if R.available() else None


def test_round_trips_match_the_reference_byte_for_byte(gold):
    from ysim_b200 import scene_format as SF
    R = _refk()
    for name in SCN.fixture_names():
        t = SCN.fixture_text(name)
        mine, mine_rc = SF.to_string(SF.parse_string(t)), SF.run_config_to_string(SF.parse_run_config(t))
        assert mine == gold["roundtrip"][name], name
        assert mine_rc == gold["runconfig"][name], name
        # a re-encoded file loads to the same text again
        assert SF.to_string(SF.parse_string(mine)) == mine
        if R:
            assert R.scene_roundtrip(t)[1] == mine and R.scene_roundtrip(t, runconfig=True)[1] == mine_rc


def test_load_errors_match_the_reference(gold):
    from ysim_b200 import scene_format as SF
    cases = dict(SCN.error_cases())
    assert len(gold["errors"]) == len(cases)
    for e in gold["errors"]:
        t = cases[e["name"]]
        for key, parse in (("scene", SF.parse_string), ("runconfig", SF.parse_run_config)):
            ok, msg = e[key]
            try:
                got = parse(t)
                mine_ok, mine = True, (SF.to_string(got) if key == "scene" else SF.run_config_to_string(got))
            except SF.SceneFormatError as err:
                mine_ok, mine = False, str(err)
            assert mine_ok == ok, (e["name"], key, mine)
            if msg.startswith("JSON parse error: "):  # the parser's own wording differs
                assert mine.startswith("JSON parse error: ")
            else:
                assert mine == msg, (e["name"], key)


def test_primitive_meshes_match_the_reference():
    from ysim_b200 import primitives as PR
    g = np.load(os.path.join(GOLD, "scene_io_geom.npz"))
    R = _refk()
    fn = {"sphere": PR.sphere, "cube": PR.cube, "cylinder": PR.cylinder}
    for k, s, t in SCN.PRIMITIVE_CASES:
        x, f = fn[k](s, t)
        assert np.array_equal(x.view(np.uint32), g[f"{k}_{s}_{t}_x"].view(np.uint32)), (k, s, t)
        assert np.array_equal(f, g[f"{k}_{s}_{t}_f"]), (k, s, t)
    if R:  # larger tessellations, live
        for k in fn:
            for t in (32, 64):
                rx, rf = R.primitive(k, 0.5, t)
                x, f = fn[k](0.5, t)
                assert np.array_equal(x.view(np.uint32), rx.view(np.uint32)) and np.array_equal(f, rf)
    # vertex / facet counts of the reference's formulas
    assert len(PR.sphere(1, 12)[0]) == 11 * 12 + 2 and len(PR.sphere(1, 12)[1]) == 2 * 12 * 11
    assert len(PR.cube(1, 5)[0]) == 6 * 25 + 2 and len(PR.cube(1, 5)[1]) == 12 * 25
    assert len(PR.cylinder(1, 9)[0]) == 10 * 9 + 2 and len(PR.cylinder(1, 9)[1]) == 2 * 81 + 18


def test_jiggle_draws_match_libstdcxx(gold):
    from ysim_b200 import primitives as PR
    for seed, want in gold["jiggle"].items():
        got = PR.uniform_float(int(seed), 0.0, 1.0 / 10000.0, len(want))
        assert np.array_equal(got.view(np.uint32), np.array(want, np.uint32)), seed


def test_profiler_csv_matches_the_reference(gold, tmp_path):
    from ysim_b200.profiler import FrameProfiler, FrameSnapshot
    pf = gold["profiler_frames"]
    p = FrameProfiler(pf["max_frames"])
    for nm in pf["names"]:
        p.ensure_section(nm)
    for i in range(len(pf["seq"])):
        fm = pf["frame_ms"][i]
        p.push(FrameSnapshot(pf["seq"][i], pf["wall"][i], fm, 1000.0 / fm if fm > 0 else 0.0, pf["sec_ms"][i],
                             pf["broad"][i], pf["narrow"][i]))
    assert p.csv() == gold["profiler_csv"]
    path = tmp_path / "sub" / "p.csv"
    assert p.export_csv(str(path)) and path.read_text() == gold["profiler_csv"]
    # begin / sample / end accumulate per frame
    q = FrameProfiler(2)
    for f in range(3):
        q.begin_frame(f, 0.5 * f)
        q.add_collision_counts(10, 2)
        q.add_collision_counts(5, 1)
        q.add_sample("a b", 1.0)
        q.add_sample("a b", 2.0)
        q.end_frame(4.0)
    rows = q.csv().splitlines()
    assert rows[0].endswith(",a_b") and len(rows) == 3 and rows[1].startswith("1,0.5,4,250,15,3,3")


def test_profile_paths_match_the_reference(gold):
    from ysim_b200 import scene_format as SF
    for csv, side, root, sp, frames in gold["paths"]:
        got = SF.default_profile_path(root, SF.path_stem(sp), frames)
        assert got == csv and SF.sidecar_scene_path(got) == side


def test_loader_builds_the_packed_scene():
    from ysim_b200 import _lib, loader as L, primitives as PR
    ls = L.load(os.path.join(GOLD, "scenes", "all_fields.json"))
    sheet, ball, crate, post, floor = ls.spec.meshes
    p = ls.spec.params
    assert p.substeps == 20 and np.float32(p.subh) == np.float32(np.float32(1 / 60) / np.float32(20))
    assert p.self_mode == _lib.SELF_HASH and p.margin == 0.015 and p.radius == 0.012
    # FastGridCloth: stiffness x cloth_stiffness_scale, rests from the packed grid, pins
    assert sheet.behavior == _lib.FAST_GRID_CLOTH and sheet.grid_n == 24 and sheet.nV == 576
    assert np.float32(sheet.kstretch) == np.float32(1000.0) * np.float32(1.5)
    assert sheet.mask[0] == 0 and sheet.mask[23] == 0 and sheet.mask.sum() == 574
    assert np.array_equal(sheet.x[23], np.float32([0.5, 0.45, -0.5]))
    assert np.allclose(sheet.x[1:23, 1], 0.45, atol=2.5e-4)  # two jiggles below 1e-4 each
    assert np.allclose(sheet.grid_rest[0], 1.0 / 23, rtol=1e-3)
    assert np.allclose(sheet.mass, 0.001)
    # sphere primitive: default Sphere collider, half extents = size / 2 x scale
    assert ball.collider[0] == _lib.COLLIDER_SPHERE and ball.flags & _lib.MESH_STATIC
    assert np.allclose(ball.collider[2], (0.25, 0.2, 0.25))
    assert np.allclose(ball.x[:, 1].max() - 0.1, 0.25 * 0.8, rtol=1e-6)  # scaled about the centre
    # cube: default Box collider, rotated about +y by 45 degrees
    assert crate.collider[0] == _lib.COLLIDER_BOX and np.allclose(crate.collider[2], (0.15, 0.15, 0.15))
    ref = L.rotate(crate.collider[3], (PR.cube(0.3, 3)[0]).astype(np.float32)) + np.float32([-0.3, 0.0, 0.2])
    assert np.allclose(crate.x, ref, atol=1e-6)
    # collider_kind "mesh" overrides the cylinder's default; not collidable; Rigid
    assert post.collider is None and not post.flags & _lib.MESH_COLLIDABLE and post.behavior == _lib.RIGID
    # plane collider on a grid (fitted extents unused)
    assert floor.collider[0] == _lib.COLLIDER_PLANE
    assert ls.ext is None  # gravity on everywhere, wind only on objects that do not take it
    assert any("spline" in w for w in ls.warnings) and any("reference-point" in w for w in ls.warnings)


def test_loader_forces_imports_and_errors(tmp_path):
    from ysim_b200 import loader as L, scene_format as SF
    j = json.loads(SCN.fixture_text("all_fields.json"))
    # wind on the cloth, gravity off on it: an external-force buffer
    j["objects"][0]["apply_wind"] = True
    j["objects"][0]["apply_gravity"] = False
    # an .obj import (quads, negative indices, v/t/n) relative to the scene file
    (tmp_path / "m").mkdir()
    (tmp_path / "m" / "quad.obj").write_text(
        "# quad\nv 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvn 0 0 1\ns off\nf 1/1/1 2/1/1 3/1/1 4/1/1\n"
        "f -3 -2 -1\n")
    j["objects"][1]["source"] = {"type": "import", "path": "m/quad.obj", "scale": 2.0, "mass": 0.5}
    path = tmp_path / "scene.json"
    path.write_text(json.dumps(j))
    ls = L.load(str(path))
    sheet, quad = ls.spec.meshes[:2]
    assert ls.ext is not None and ls.ext.shape == (ls.spec.nV, 3)
    assert np.allclose(ls.ext[: sheet.nV], [0.5, 0.0, -0.25]) and not ls.ext[sheet.nV:].any()
    # negative indices resolve as the reference's reader does (k - 1 + nV)
    assert quad.nV == 4 and quad.facets.tolist() == [[0, 1, 2], [0, 2, 3], [0, 1, 2]]
    # v * import scale + position, then the object's scale (1, 0.8, 1) about it
    assert np.allclose(quad.x[2], np.float32([2.1, 1.7, 0.0]))
    j["engine"]["system"] = "PBD"
    with pytest.raises(SF.SceneFormatError, match="Explicit only"):
        L.load(SF.run_config_from_json(j))
    j["engine"]["system"] = "Explicit"
    j["objects"][0]["behavior"]["params"]["particle_num_1d"] = 20
    with pytest.raises(SF.SceneFormatError, match="particle_num_1d"):
        L.load(SF.run_config_from_json(j))


@pytest.mark.parametrize("gravity,wind", [(True, True), (False, True), (True, False), (False, False)])
def test_loader_environment_forces_equal_the_oracle(oracle, gravity, wind):
    """The loader's external-force buffer (applyEnvironmentForces,
    simulator.hpp:3123-3166) equals the oracle's own restatement for every
    combination of the cloth's gravity and wind gates, with wind on the Float
    meshes' gates too (they get zero)."""
    import numpy as np
    from ysim_b200 import loader as L
    from ysim_b200 import scene_format as SF
    path = os.path.join(GOLD, "scenes", "drape.json")
    cfg = SF.read_run_config(path)
    snap = cfg.scene
    snap.environment.wind = (0.4, 0.0, -0.25)
    snap.objects[0].apply_gravity = gravity
    snap.objects[0].apply_wind = wind
    ls = L.load(cfg, path)
    o = oracle.OracleScene(ls.spec)
    o.set_environment(snap.environment.wind, [(ob.apply_gravity, ob.apply_wind) for ob in snap.objects])
    o.step(1)
    want = o.get("ext")
    got = np.ascontiguousarray(ls.ext, np.float32) if ls.ext is not None else None
    if gravity and not wind:
        assert got is None  # the kernels' own g * m
        g = np.asarray(ls.spec.params.gravity, np.float32)
        c = ls.spec.meshes[0]
        assert np.array_equal(want[: c.nV], (c.mass[:, None] * g[None, :]).astype(np.float32))
        assert not want[c.nV:].any()
    else:
        assert np.array_equal(got, want)
