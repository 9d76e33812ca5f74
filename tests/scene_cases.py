"""Scene-file cases shared by the golden generator and the tests: the fixture
files under tests/golden/scenes, and invalid variants of the all-fields
fixture (each one field broken) for the loader's error messages."""
from __future__ import annotations

import copy
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
SCENES = os.path.join(HERE, "golden", "scenes")


def fixture_names():
    return sorted(f for f in os.listdir(SCENES) if f.endswith(".json"))


def fixture_text(name: str) -> str:
    with open(os.path.join(SCENES, name)) as f:
        return f.read()


def _mutations():
    o0 = lambda j: j["objects"][0]  # noqa: E731
    src = lambda j: j["objects"][0]["source"]  # noqa: E731
    return [
        ("no format_version", lambda j: j.pop("format_version")),
        ("float format_version", lambda j: j.__setitem__("format_version", 1.0)),
        ("format_version 2", lambda j: j.__setitem__("format_version", 2)),
        ("string format_version", lambda j: j.__setitem__("format_version", "1")),
        ("objects not an array", lambda j: j.__setitem__("objects", {})),
        ("no id", lambda j: o0(j).pop("id")),
        ("string id", lambda j: o0(j).__setitem__("id", "x")),
        ("float id", lambda j: o0(j).__setitem__("id", 1.7)),
        ("boolean id", lambda j: o0(j).__setitem__("id", True)),
        ("numeric name", lambda j: o0(j).__setitem__("name", 3)),
        ("unknown shape", lambda j: src(j).__setitem__("shape", "torus")),
        ("unknown source type", lambda j: src(j).__setitem__("type", "procedural")),
        ("string size", lambda j: src(j).__setitem__("size", "big")),
        ("boolean size", lambda j: src(j).__setitem__("size", True)),
        ("float tessellation", lambda j: src(j).__setitem__("tessellation", 24.9)),
        ("no tessellation", lambda j: src(j).pop("tessellation")),
        ("fbx import", lambda j: j["objects"][1].__setitem__("source", {"type": "import", "path": "a/b.fbx"})),
        ("OBJ import", lambda j: j["objects"][1].__setitem__("source", {"type": "import", "path": "a/B.OBJ",
                                                                         "scale": 2})),
        ("short position", lambda j: o0(j)["transform"].__setitem__("position", [0, 1])),
        ("string in position", lambda j: o0(j)["transform"].__setitem__("position", [0, "a", 1])),
        ("zero rotation", lambda j: o0(j)["transform"].__setitem__("rotation", [0, 0, 0, 0])),
        ("no rotation", lambda j: o0(j)["transform"].pop("rotation")),
        ("no metallic", lambda j: o0(j)["material"].pop("metallic")),
        ("reserved behavior", lambda j: o0(j)["behavior"].__setitem__("type", "Elastic")),
        ("unknown behavior", lambda j: o0(j)["behavior"].__setitem__("type", "Jelly")),
        ("integer apply_gravity", lambda j: o0(j).__setitem__("apply_gravity", 1)),
        ("string stiffness scale", lambda j: o0(j).__setitem__("cloth_stiffness_scale", "2")),
        ("zero substeps", lambda j: j["simulation"].__setitem__("substeps", 0)),
        ("float substeps", lambda j: j["simulation"].__setitem__("substeps", 2.0)),
        ("negative time per frame", lambda j: j["simulation"].__setitem__("time_per_frame", -1)),
        ("simulation not an object", lambda j: j.__setitem__("simulation", [])),
        ("short gravity", lambda j: j["environment"].__setitem__("gravity", [0, 0])),
        ("unknown backend", lambda j: j["engine"].__setitem__("backend", "VULKAN")),
        ("unknown system", lambda j: j["engine"].__setitem__("system", "FEM")),
        ("zero profile frames", lambda j: j["profile"].__setitem__("frames", 0)),
        ("unknown profile level", lambda j: j["profile"].__setitem__("level", "max")),
        ("string profile enabled", lambda j: j["profile"].__setitem__("enabled", "yes")),
    ]


def error_cases():
    """(name, text) of each variant; the loader must answer as the reference does."""
    base = json.loads(fixture_text("all_fields.json"))
    out = [("truncated JSON", "{"), ("root array", "[]")]
    for name, mut in _mutations():
        j = copy.deepcopy(base)
        mut(j)
        out.append((name, json.dumps(j)))
    return out


PRIMITIVE_CASES = [(k, s, t) for k in ("sphere", "cube", "cylinder") for s in (1.0, 0.3, 2.7, 1e-3)
                   for t in (1, 3, 7, 12)]
JIGGLE_SEEDS = (0, 1, 7, 12345, 0xDEADBEEF)
