"""Scene files and run configs of the reference, read and written in Python.

The schema and its rules follow include/scene_format.hpp (SceneSnapshot:
objects with source / transform / material / behavior / collider fields,
environment, simulation timing, reference constraints; format_version 1) and
include/sim_config.hpp (RunConfig: the same root plus the optional "engine"
and "profile" blocks).  Loading validates as the reference does and fails with
the reference's messages; encoding produces the reference's JSON (keys sorted,
two-space indent, optional keys omitted when unset), so a file round-trips
byte for byte.  Turning a snapshot into a packed scene is ysim_b200.loader.
"""
from __future__ import annotations

import dataclasses
import json
import math
import os
from typing import Any, Dict, List, Optional, Tuple

FORMAT_VERSION = 1

Vec3 = Tuple[float, float, float]
Quat = Tuple[float, float, float, float]


class SceneFormatError(ValueError):
    """A scene file or run config that does not load (LoadError)."""


# ---------------------------------------------------------------- snapshot types
@dataclasses.dataclass
class PrimitiveSource:
    shape: str = "grid"
    size: float = 1.0
    tessellation: int = 32
    direction: str = "XZPlane"  # XYPlane | YZPlane | XZPlane
    mass: float = 0.1
    jiggle: bool = False


@dataclasses.dataclass
class ImportSource:
    path: str = ""
    scale: float = 1.0
    mass: float = 0.1


@dataclasses.dataclass
class Source:
    kind: str = "primitive"  # primitive | import
    primitive: PrimitiveSource = dataclasses.field(default_factory=PrimitiveSource)
    imported: ImportSource = dataclasses.field(default_factory=ImportSource)


@dataclasses.dataclass
class Transform:
    position: Vec3 = (0.0, 0.0, 0.0)
    rotation: Quat = (1.0, 0.0, 0.0, 0.0)  # w, x, y, z; unit length after a load
    scale: Vec3 = (1.0, 1.0, 1.0)


@dataclasses.dataclass
class Material:
    base_color: Vec3 = (1.0, 1.0, 1.0)
    metallic: float = 0.0
    roughness: float = 0.5
    specular_weight: float = 1.0
    emission_color: Vec3 = (0.0, 0.0, 0.0)


@dataclasses.dataclass
class Behavior:
    type: str = "Float"
    params: Dict[str, Any] = dataclasses.field(default_factory=dict)


@dataclasses.dataclass
class FixedParticle:
    vid: int = 0
    pos: Vec3 = (0.0, 0.0, 0.0)


@dataclasses.dataclass
class SplineConstraint:
    vid: int = 0
    closed: bool = False
    duration: float = 4.0
    points: List[Vec3] = dataclasses.field(default_factory=list)


@dataclasses.dataclass
class Object:
    id: int = 0
    name: str = ""
    source: Source = dataclasses.field(default_factory=Source)
    transform: Transform = dataclasses.field(default_factory=Transform)
    material: Material = dataclasses.field(default_factory=Material)
    behavior: Behavior = dataclasses.field(default_factory=Behavior)
    apply_gravity: bool = True
    apply_wind: bool = True
    is_static: bool = False
    cloth_stiffness_scale: float = 1.0
    collider_kind: str = ""  # "" = the kind the source implies
    collidable: bool = True
    self_collide: bool = False
    fixed_particles: List[FixedParticle] = dataclasses.field(default_factory=list)
    spline_constraints: List[SplineConstraint] = dataclasses.field(default_factory=list)


@dataclasses.dataclass
class Environment:
    gravity: Vec3 = (0.0, -9.81, 0.0)
    wind: Vec3 = (0.0, 0.0, 0.0)
    background_color: Vec3 = (0.68, 0.85, 0.95)


@dataclasses.dataclass
class Simulation:
    time_per_frame: float = 1.0 / 60.0
    substeps: int = 60


@dataclasses.dataclass
class ReferenceConstraint:
    query_object: int = 0
    query_vertex: int = 0
    target_object: int = 0
    target_vertex: int = 0


@dataclasses.dataclass
class SceneSnapshot:
    format_version: int = FORMAT_VERSION
    objects: List[Object] = dataclasses.field(default_factory=list)
    environment: Environment = dataclasses.field(default_factory=Environment)
    simulation: Simulation = dataclasses.field(default_factory=Simulation)
    reference_constraints: List[ReferenceConstraint] = dataclasses.field(default_factory=list)
    warnings: List[str] = dataclasses.field(default_factory=list)


KNOWN_BEHAVIORS = ("Float", "TriangularCloth", "FastGridCloth", "Rigid")
RESERVED_BEHAVIORS = ("Elastic", "Fluid", "Generator")
KNOWN_SHAPES = ("grid", "sphere", "cube", "cylinder")
COLLIDER_KINDS = ("mesh", "sphere", "box", "cylinder", "plane")


# ---------------------------------------------------------------- json value rules
# nlohmann's conversions (3.12): a number converts to a double or an integer,
# a boolean only to an integer; a string or a boolean must be exactly that
# type.  Type errors carry nlohmann's own message.
def _is_number(v) -> bool:
    return isinstance(v, (int, float))


def _is_integer(v) -> bool:
    return isinstance(v, int) and not isinstance(v, bool)


def _type_name(v) -> str:
    if v is None:
        return "null"
    if isinstance(v, bool):
        return "boolean"
    if isinstance(v, (int, float)):
        return "number"
    if isinstance(v, str):
        return "string"
    if isinstance(v, list):
        return "array"
    return "object"


def _type_error(expected: str, v) -> SceneFormatError:
    return SceneFormatError(f"[json.exception.type_error.302] type must be {expected}, but is {_type_name(v)}")


def _as_float(v, what: str = "") -> float:
    # a boolean is not a number for a double ...
    if not _is_number(v) or isinstance(v, bool):
        raise _type_error("number", v)
    return float(v)


def _as_int(v, what: str = "") -> int:
    # ... but converts for an integer (true -> 1); a float truncates
    if not _is_number(v):
        raise _type_error("number", v)
    return int(v)


def _as_str(v, what: str = "") -> str:
    if not isinstance(v, str):
        raise _type_error("string", v)
    return v


def _as_bool(v, what: str = "") -> bool:
    if not isinstance(v, bool):
        raise _type_error("boolean", v)
    return v


def _field(j: dict, key: str, path: str, conv):
    """detail::readField: missing key or wrong type fails the load."""
    if key not in j:
        raise SceneFormatError(f"missing '{key}' at {path}")
    try:
        return conv(j[key])
    except SceneFormatError as e:
        raise SceneFormatError(f"wrong type for '{key}' at {path}: {e}") from None


def _vec3(v, path: str) -> Vec3:
    if not isinstance(v, list) or len(v) != 3:
        raise SceneFormatError(f"expected 3-element array at {path}")
    for i, c in enumerate(v):
        if not _is_number(c) or isinstance(c, bool):
            raise SceneFormatError(f"expected number at {path}[{i}]")
    return (float(v[0]), float(v[1]), float(v[2]))


def _quat(v, path: str) -> Quat:
    if not isinstance(v, list) or len(v) != 4:
        raise SceneFormatError(f"expected 4-element [w,x,y,z] array at {path}")
    for i, c in enumerate(v):
        if not _is_number(c) or isinstance(c, bool):
            raise SceneFormatError(f"expected number at {path}[{i}]")
    return (float(v[0]), float(v[1]), float(v[2]), float(v[3]))


def normalize_quat(q: Quat) -> Quat:
    n = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    if n == 0.0:
        return (1.0, 0.0, 0.0, 0.0)
    return (q[0] / n, q[1] / n, q[2] / n, q[3] / n)


def _clamp01(x: float) -> float:
    return 0.0 if x < 0.0 else (1.0 if x > 1.0 else x)


# ---------------------------------------------------------------- decode
def _source(j, idx: int) -> Source:
    path = f"objects[{idx}].source"
    s = Source()
    typ = _field(j, "type", path, _as_str)
    if typ == "primitive":
        p = s.primitive
        p.shape = _field(j, "shape", path, _as_str)
        if p.shape not in KNOWN_SHAPES:
            raise SceneFormatError(f"unknown source.shape '{p.shape}' at objects[{idx}]")
        p.size = _field(j, "size", path, _as_float)
        p.tessellation = _field(j, "tessellation", path, _as_int)
        if "direction" in j:
            p.direction = _as_str(j["direction"], "direction")
        if "mass" in j:
            p.mass = _as_float(j["mass"], "mass")
        if "jiggle" in j:
            p.jiggle = _as_bool(j["jiggle"], "jiggle")
    elif typ == "import":
        s.kind = "import"
        m = s.imported
        m.path = _field(j, "path", path, _as_str)
        dot = m.path.rfind(".")
        ext = "" if dot < 0 else m.path[dot:].lower()
        if ext != ".obj":
            raise SceneFormatError(f"unsupported source.path extension '{m.path}' at objects[{idx}]")
        if "scale" in j:
            m.scale = _as_float(j["scale"], "scale")
        if "mass" in j:
            m.mass = _as_float(j["mass"], "mass")
    else:
        raise SceneFormatError(f"unknown source.type '{typ}' at objects[{idx}]")
    return s


def _transform(j, idx: int) -> Transform:
    path = f"objects[{idx}].transform"
    t = Transform()
    if "position" not in j:
        raise SceneFormatError(f"missing 'position' at {path}")
    t.position = _vec3(j["position"], path + ".position")
    if "rotation" not in j:
        raise SceneFormatError(f"missing 'rotation' at {path}")
    t.rotation = normalize_quat(_quat(j["rotation"], path + ".rotation"))
    if "scale" in j:
        t.scale = _vec3(j["scale"], path + ".scale")
    return t


def _material(j, idx: int, warnings: List[str]) -> Material:
    path = f"objects[{idx}].material"
    m = Material()
    if "base_color" not in j:
        raise SceneFormatError(f"missing 'base_color' at {path}")
    m.base_color = _vec3(j["base_color"], path + ".base_color")
    m.metallic = _field(j, "metallic", path, _as_float)
    m.roughness = _field(j, "roughness", path, _as_float)
    m.specular_weight = _field(j, "specular_weight", path, _as_float)
    if "emission_color" not in j:
        raise SceneFormatError(f"missing 'emission_color' at {path}")
    m.emission_color = _vec3(j["emission_color"], path + ".emission_color")
    clamped = (tuple(_clamp01(c) for c in m.base_color), _clamp01(m.metallic), _clamp01(m.roughness),
               _clamp01(m.specular_weight), tuple(max(c, 0.0) for c in m.emission_color))
    changed = clamped != (m.base_color, m.metallic, m.roughness, m.specular_weight, m.emission_color)
    m.base_color, m.metallic, m.roughness, m.specular_weight, m.emission_color = clamped
    if changed:
        warnings.append(f"clamped out-of-range material values at {path}")
    return m


def _behavior(j, idx: int) -> Behavior:
    path = f"objects[{idx}].behavior"
    b = Behavior()
    b.type = _field(j, "type", path, _as_str)
    if b.type in RESERVED_BEHAVIORS:
        raise SceneFormatError(f"behavior '{b.type}' not available in this build (objects[{idx}])")
    if b.type not in KNOWN_BEHAVIORS:
        raise SceneFormatError(f"unknown behavior.type '{b.type}' at {path}")
    if "params" in j:
        b.params = j["params"]
    return b


def _object(j, idx: int, warnings: List[str]) -> Object:
    path = f"objects[{idx}]"
    if not isinstance(j, dict):
        raise SceneFormatError(f"missing 'id' at {path}")
    o = Object()
    o.id = _field(j, "id", path, _as_int)
    o.name = _field(j, "name", path, _as_str)
    if "source" not in j:
        raise SceneFormatError(f"missing 'source' at {path}")
    o.source = _source(j["source"], idx)
    if "transform" not in j:
        raise SceneFormatError(f"missing 'transform' at {path}")
    o.transform = _transform(j["transform"], idx)
    if "material" not in j:
        raise SceneFormatError(f"missing 'material' at {path}")
    o.material = _material(j["material"], idx, warnings)
    if "behavior" not in j:
        raise SceneFormatError(f"missing 'behavior' at {path}")
    o.behavior = _behavior(j["behavior"], idx)
    # optional keys of the right type are taken, others ignored
    for key, attr in (("apply_gravity", "apply_gravity"), ("apply_wind", "apply_wind"),
                      ("is_static", "is_static"), ("collidable", "collidable"), ("self_collide", "self_collide")):
        if isinstance(j.get(key), bool):
            setattr(o, attr, j[key])
    v = j.get("cloth_stiffness_scale")
    if _is_number(v) and not isinstance(v, bool):
        o.cloth_stiffness_scale = float(v)
    if isinstance(j.get("collider_kind"), str):
        o.collider_kind = j["collider_kind"]
    for e in j.get("fixed_particles", []) if isinstance(j.get("fixed_particles"), list) else []:
        if not isinstance(e, dict) or not _is_integer(e.get("vid")) or "pos" not in e:
            continue
        try:
            o.fixed_particles.append(FixedParticle(e["vid"], _vec3(e["pos"], path)))
        except SceneFormatError:
            continue
    for e in j.get("spline_constraints", []) if isinstance(j.get("spline_constraints"), list) else []:
        if not isinstance(e, dict) or not _is_integer(e.get("vid")):
            continue
        s = SplineConstraint(vid=e["vid"])
        if isinstance(e.get("closed"), bool):
            s.closed = e["closed"]
        if _is_number(e.get("duration")) and not isinstance(e.get("duration"), bool):
            s.duration = float(e["duration"])
        pts = e.get("points")
        if not isinstance(pts, list):
            continue
        try:
            s.points = [_vec3(p, path) for p in pts]
        except SceneFormatError:
            continue
        if len(s.points) < 2:
            continue
        o.spline_constraints.append(s)
    return o


def _environment(j) -> Environment:
    e = Environment()
    if "gravity" in j:
        e.gravity = _vec3(j["gravity"], "environment.gravity")
    if "wind" in j:
        e.wind = _vec3(j["wind"], "environment.wind")
    if "background_color" in j:
        e.background_color = _vec3(j["background_color"], "environment.background_color")
    return e


def _simulation(j) -> Simulation:
    s = Simulation()
    if "time_per_frame" in j:
        v = j["time_per_frame"]
        if not _is_number(v) or isinstance(v, bool):
            raise SceneFormatError("simulation.time_per_frame must be a number")
        if not float(v) > 0.0:
            raise SceneFormatError("simulation.time_per_frame must be > 0")
        s.time_per_frame = float(v)
    if "substeps" in j:
        v = j["substeps"]
        if not _is_integer(v):
            raise SceneFormatError("simulation.substeps must be an integer")
        if v < 1:
            raise SceneFormatError("simulation.substeps must be >= 1")
        s.substeps = v
    return s


def from_json(j) -> SceneSnapshot:
    """scene_format::fromJson (scene_format.hpp:686-760)."""
    if not isinstance(j, dict):
        raise SceneFormatError("scene root must be a JSON object")
    if "format_version" not in j:
        raise SceneFormatError("missing format_version")
    fv = j["format_version"]
    if not _is_integer(fv):
        raise SceneFormatError(f"format_version must be an integer (got {_type_name(fv)})")
    if fv != FORMAT_VERSION:
        raise SceneFormatError(f"format_version mismatch: found {fv}, expected {FORMAT_VERSION}")
    s = SceneSnapshot(format_version=fv)
    objs = j.get("objects")
    if not isinstance(objs, list):
        raise SceneFormatError("missing or invalid 'objects' array")
    for i, o in enumerate(objs):
        s.objects.append(_object(o, i, s.warnings))
    if "environment" in j:
        s.environment = _environment(j["environment"])
    if "simulation" in j:
        if not isinstance(j["simulation"], dict):
            raise SceneFormatError("'simulation' must be a JSON object")
        s.simulation = _simulation(j["simulation"])
    for e in j.get("reference_constraints", []) if isinstance(j.get("reference_constraints"), list) else []:
        q, t = (e.get("query"), e.get("target")) if isinstance(e, dict) else (None, None)
        if not isinstance(q, dict) or not isinstance(t, dict):
            continue
        vals = (q.get("object"), q.get("vertex"), t.get("object"), t.get("vertex"))
        if not all(_is_integer(v) for v in vals):
            continue
        s.reference_constraints.append(ReferenceConstraint(*vals))
    return s


def parse_string(text: str) -> SceneSnapshot:
    try:
        j = json.loads(text)
    except json.JSONDecodeError as e:
        raise SceneFormatError(f"JSON parse error: {e}") from None
    return from_json(j)


def read_file(path: str) -> SceneSnapshot:
    try:
        with open(path) as f:
            text = f.read()
    except OSError:
        raise SceneFormatError(f"cannot open '{path}' for reading") from None
    return parse_string(text)


# ---------------------------------------------------------------- encode
def _source_json(s: Source) -> dict:
    if s.kind == "primitive":
        p = s.primitive
        return {"type": "primitive", "shape": p.shape, "size": p.size, "tessellation": p.tessellation,
                "direction": p.direction, "mass": p.mass, "jiggle": p.jiggle}
    m = s.imported
    return {"type": "import", "path": m.path, "scale": m.scale, "mass": m.mass}


def _object_json(o: Object) -> dict:
    t = o.transform
    tj = {"position": list(t.position), "rotation": list(normalize_quat(t.rotation))}
    if tuple(t.scale) != (1.0, 1.0, 1.0):
        tj["scale"] = list(t.scale)
    m = o.material
    j = {"id": o.id, "name": o.name, "source": _source_json(o.source), "transform": tj,
         "material": {"base_color": list(m.base_color), "metallic": m.metallic, "roughness": m.roughness,
                      "specular_weight": m.specular_weight, "emission_color": list(m.emission_color)},
         "behavior": {"type": o.behavior.type, "params": o.behavior.params},
         "apply_gravity": o.apply_gravity, "apply_wind": o.apply_wind, "is_static": o.is_static,
         "cloth_stiffness_scale": o.cloth_stiffness_scale, "collidable": o.collidable,
         "self_collide": o.self_collide}
    if o.collider_kind:
        j["collider_kind"] = o.collider_kind
    if o.fixed_particles:
        j["fixed_particles"] = [{"vid": f.vid, "pos": list(f.pos)} for f in o.fixed_particles]
    if o.spline_constraints:
        j["spline_constraints"] = [{"vid": s.vid, "closed": s.closed, "duration": s.duration,
                                    "points": [list(p) for p in s.points]} for s in o.spline_constraints]
    return j


def to_json(s: SceneSnapshot) -> dict:
    """scene_format::toJson (scene_format.hpp:377-416)."""
    e, sm = s.environment, s.simulation
    j = {"format_version": s.format_version, "objects": [_object_json(o) for o in s.objects],
         "environment": {"gravity": list(e.gravity), "wind": list(e.wind),
                         "background_color": list(e.background_color)},
         "simulation": {"time_per_frame": sm.time_per_frame, "substeps": sm.substeps}}
    if s.reference_constraints:
        j["reference_constraints"] = [{"query": {"object": c.query_object, "vertex": c.query_vertex},
                                       "target": {"object": c.target_object, "vertex": c.target_vertex}}
                                      for c in s.reference_constraints]
    return j


def dumps(j: dict) -> str:
    """nlohmann::json::dump(2): sorted keys, two-space indent, ": " separators."""
    return json.dumps(j, indent=2, sort_keys=True, ensure_ascii=False)


def to_string(s: SceneSnapshot) -> str:
    return dumps(to_json(s))


def write_file(s: SceneSnapshot, path: str) -> None:
    with open(path, "w") as f:
        f.write(to_string(s))


# ---------------------------------------------------------------- run config
BACKENDS = ("METAL", "CPU", "CUDA")
SYSTEMS = ("Explicit", "PBD", "PD", "LargeSteps")
PROFILE_LEVELS = ("none", "per_frame", "in_frame")


@dataclasses.dataclass
class EngineConfig:
    backend: str = "METAL"
    system: str = "Explicit"


@dataclasses.dataclass
class ProfileConfig:
    enabled: bool = False
    frames: int = 30
    realtime_sync: bool = False
    output_path: str = ""
    level: str = "in_frame"


@dataclasses.dataclass
class RunConfig:
    scene: SceneSnapshot = dataclasses.field(default_factory=SceneSnapshot)
    engine: EngineConfig = dataclasses.field(default_factory=EngineConfig)
    profile: ProfileConfig = dataclasses.field(default_factory=ProfileConfig)


def run_config_from_json(j) -> RunConfig:
    """sim_config::fromJson (sim_config.hpp:189-211): the scene blocks, then
    the optional engine and profile blocks."""
    c = RunConfig(scene=from_json(j))
    if "engine" in j:
        e = j["engine"]
        if not isinstance(e, dict):
            raise SceneFormatError("'engine' must be a JSON object")
        if "backend" in e:
            if not isinstance(e["backend"], str):
                raise SceneFormatError("engine.backend must be a string")
            if e["backend"] not in BACKENDS:
                raise SceneFormatError(f"unknown engine.backend '{e['backend']}' (expected METAL | CPU | CUDA)")
            c.engine.backend = e["backend"]
        if "system" in e:
            if not isinstance(e["system"], str):
                raise SceneFormatError("engine.system must be a string")
            if e["system"] not in SYSTEMS:
                raise SceneFormatError(f"unknown engine.system '{e['system']}' (expected Explicit)")
            c.engine.system = e["system"]
    if "profile" in j:
        p = j["profile"]
        if not isinstance(p, dict):
            raise SceneFormatError("'profile' must be a JSON object")
        if "enabled" in p:
            if not isinstance(p["enabled"], bool):
                raise SceneFormatError("profile.enabled must be a boolean")
            c.profile.enabled = p["enabled"]
        if "frames" in p:
            if not _is_integer(p["frames"]):
                raise SceneFormatError("profile.frames must be an integer")
            if p["frames"] < 1:
                raise SceneFormatError("profile.frames must be >= 1")
            c.profile.frames = p["frames"]
        if "realtime_sync" in p:
            if not isinstance(p["realtime_sync"], bool):
                raise SceneFormatError("profile.realtime_sync must be a boolean")
            c.profile.realtime_sync = p["realtime_sync"]
        if "output_path" in p:
            if not isinstance(p["output_path"], str):
                raise SceneFormatError("profile.output_path must be a string")
            c.profile.output_path = p["output_path"]
        if "level" in p:
            if not isinstance(p["level"], str):
                raise SceneFormatError("profile.level must be a string")
            if p["level"] not in PROFILE_LEVELS:
                raise SceneFormatError(f"unknown profile.level '{p['level']}' (expected none | per_frame | in_frame)")
            c.profile.level = p["level"]
    return c


def run_config_to_json(c: RunConfig) -> dict:
    j = to_json(c.scene)
    j["engine"] = {"backend": c.engine.backend, "system": c.engine.system}
    p = c.profile
    j["profile"] = {"enabled": p.enabled, "frames": p.frames, "realtime_sync": p.realtime_sync,
                    "output_path": p.output_path, "level": p.level}
    return j


def parse_run_config(text: str) -> RunConfig:
    try:
        j = json.loads(text)
    except json.JSONDecodeError as e:
        raise SceneFormatError(f"JSON parse error: {e}") from None
    return run_config_from_json(j)


def read_run_config(path: str) -> RunConfig:
    try:
        with open(path) as f:
            text = f.read()
    except OSError:
        raise SceneFormatError(f"cannot open '{path}' for reading") from None
    return parse_run_config(text)


def run_config_to_string(c: RunConfig) -> str:
    return dumps(run_config_to_json(c))


def path_stem(path: str) -> str:
    """sim_config::pathStem: the file name without its last extension."""
    base = path[path.rfind("/") + 1:]
    dot = base.rfind(".")
    return base if dot < 0 else base[:dot]


def default_profile_path(project_root: str, scene_stem: str, frames: int) -> str:
    """sim_config::defaultProfilePath: <root>/profiles/<stem>-<N>f.csv."""
    d = "profiles" if not project_root else project_root + "/profiles"
    return f"{d}/{scene_stem or 'scene'}-{frames}f.csv"


def sidecar_scene_path(csv_path: str) -> str:
    """sim_config::sidecarScenePath: <dir>/<stem>.scene.json beside a CSV."""
    dot, slash = csv_path.rfind("."), csv_path.rfind("/")
    base = csv_path[:dot] if dot >= 0 and (slash < 0 or dot > slash) else csv_path
    return base + ".scene.json"


def resolve_import_path(scene_dir: str, import_path: str) -> str:
    """scene_format::resolveImportPath: relative to the scene file's directory."""
    if import_path.startswith("/") or not scene_dir:
        return import_path
    return scene_dir + import_path if scene_dir.endswith("/") else scene_dir + "/" + import_path


def scene_dir(scene_path: str) -> str:
    pos = scene_path.rfind("/")
    return "" if pos < 0 else scene_path[:pos]
