"""A scene file (or run config) of the reference turned into a scene for this path.

Follows Simulator::applySnapshot (include/sim/simulator.hpp:4573-4858) and the
parts of Scene::pack that shape the packed state (scene.hpp:900-1080):

* behavior: TriangularCloth (stretch / shear / bend / thickness), FastGridCloth
  (particle_num_1d, k_stretch / k_shear / k_bend, thickness; the six rest
  lengths re-measured from the packed positions, recomputeFastGridRest), Float,
  Rigid (not integrated: the rigid-body backend is out of scope);
  cloth_stiffness_scale multiplies the stiffnesses (collision_pod.hpp:483-487);
* source: grid / sphere / cube / cylinder initializers, or a .obj import
  relative to the scene file; mass is per vertex (MeshState::memoryAllocation);
* transform: scale -> rotate -> translate about the initializer's centre, then
  the pack-time cloth jiggle of a cloth grid (seed object id ^ mesh id), rest
  lengths from the result, pinned vertices (fixed_particles: position held,
  integration mask 0);
* collider_kind (default: sphere / box / cylinder for those primitives, mesh
  otherwise) with the half extents of Scene::fitAnalyticLocalHalf
  (scene.hpp:600-641): size / 2 x scale for a matching primitive, else the
  smallest origin-centred box around the packed vertices in the collider frame;
* environment: gravity and wind per object (applyEnvironmentForces,
  simulator.hpp:3123-3166) as an external-force buffer when any object departs
  from "gravity on, no wind";
* simulation: subh = h / substeps; margin, radius, rebuild period and the
  CPU-hash self rows are the Simulator's defaults.

Spline and reference-point constraints (motion), materials (rendering) and
the PBD / PD / Large-Steps solvers are outside this path: they load, are
reported in `warnings`, and do not act.
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional

import numpy as np

from . import generators as G
from . import primitives as PR
from . import scene_format as SF

F32 = np.float32

_DEFAULT_COLLIDER = {"sphere": "sphere", "cube": "box", "cylinder": "cylinder"}
_COLLIDER_CODE = {"mesh": 0, "sphere": 1, "box": 2, "cylinder": 3, "plane": 4}


def _qmul(a, b):
    """Quat operator* (Hamilton product, material_quat.hpp:27-33), float32,
    each term in the reference's order (components may be arrays)."""
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return (aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
            aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw)


def rotate(q, v: np.ndarray) -> np.ndarray:
    """rotateVector (material_quat.hpp:59-63): q (0, v) q*, float32 per row."""
    q = tuple(F32(c) for c in q)
    qc = (q[0], -q[1], -q[2], -q[3])
    v = np.asarray(v, F32)
    zero = np.zeros(len(v), F32)
    r = _qmul(_qmul(q, (zero, v[:, 0], v[:, 1], v[:, 2])), qc)
    return np.stack([r[1], r[2], r[3]], 1).astype(F32)


@dataclasses.dataclass
class LoadedScene:
    spec: G.SceneSpec
    ext: Optional[np.ndarray]      # (V, 3) external forces, or None for g * m on cloth
    config: SF.RunConfig
    warnings: List[str]


def _behavior(o: SF.Object, warnings: List[str]):
    from ._lib import FAST_GRID_CLOTH, FLOAT, RIGID, TRIANGULAR_CLOTH
    p = o.behavior.params or {}
    s = F32(o.cloth_stiffness_scale)
    t = o.behavior.type
    if t == "TriangularCloth":
        return TRIANGULAR_CLOTH, dict(kstretch=F32(p.get("stretch", 0.0)) * s, kshear=F32(p.get("shear", 0.0)) * s,
                                      kbend=F32(p.get("bend", 0.0)) * s, thickness=F32(p.get("thickness", 0.0)))
    if t == "FastGridCloth":
        return FAST_GRID_CLOTH, dict(kstretch=F32(p.get("k_stretch", 0.0)) * s, kshear=F32(p.get("k_shear", 0.0)) * s,
                                     kbend=F32(p.get("k_bend", 0.0)) * s, thickness=F32(p.get("thickness", 0.0)),
                                     grid_n=int(p.get("particle_num_1d", 0)))
    if t == "Rigid":
        warnings.append(f"object {o.id} ({o.name}): Rigid bodies are not integrated (no rigid-body backend)")
        return RIGID, {}
    return FLOAT, {}


def _geometry(o: SF.Object, scene_dir: str, seed: int):
    """(positions, facets, pivot, primitive size or None) from the source."""
    pos = tuple(F32(c) for c in o.transform.position)
    src = o.source
    if src.kind == "import":
        path = SF.resolve_import_path(scene_dir, src.imported.path)
        x, f = PR.load_obj(path, src.imported.scale, pos)
        return x, f, pos, None, float(src.imported.mass)
    p = src.primitive
    if p.shape == "sphere":
        x, f = PR.sphere(p.size, p.tessellation, pos)
    elif p.shape == "cube":
        x, f = PR.cube(p.size, p.tessellation, pos)
    elif p.shape == "cylinder":
        x, f = PR.cylinder(p.size, p.tessellation, pos)
    else:
        x, f = PR.grid(p.direction, pos, p.tessellation, p.size, p.jiggle, seed)
    return x, f, pos, F32(p.size), float(p.mass)


def load(source, scene_path: str = "") -> LoadedScene:
    """A RunConfig, SceneSnapshot or the path of a scene / run-config file."""
    if isinstance(source, str):
        scene_path = source
        cfg = SF.read_run_config(source)
    elif isinstance(source, SF.SceneSnapshot):
        cfg = SF.RunConfig(scene=source)
    else:
        cfg = source
    if cfg.engine.system != "Explicit":
        raise SF.SceneFormatError(f"engine.system '{cfg.engine.system}' is not built here (Explicit only)")
    snap = cfg.scene
    warnings = list(snap.warnings)
    if cfg.engine.backend != "CUDA":
        warnings.append(f"engine.backend '{cfg.engine.backend}' requested; this path runs CUDA")
    if snap.reference_constraints:
        warnings.append(f"{len(snap.reference_constraints)} reference-point constraints are not applied")
    sdir = SF.scene_dir(scene_path)
    from ._lib import FAST_GRID_CLOTH, MESH_COLLIDABLE, MESH_SELF_COLLIDE, MESH_STATIC, SELF_HASH, TRIANGULAR_CLOTH
    meshes, ext_parts, custom_forces = [], [], False
    g = tuple(F32(c) for c in snap.environment.gravity)
    w = tuple(F32(c) for c in snap.environment.wind)
    for i, o in enumerate(snap.objects):
        beh, bp = _behavior(o, warnings)
        cloth = beh in (TRIANGULAR_CLOTH, FAST_GRID_CLOTH)
        x, fac, pivot, psize, mass = _geometry(o, sdir, o.id & 0xFFFFFFFF)
        # scale -> rotate -> translate about the pivot (Scene::pack)
        sc = tuple(F32(c) for c in o.transform.scale)
        q = tuple(F32(c) for c in o.transform.rotation)
        unit_s = all(abs(c - F32(1)) < F32(1e-7) for c in sc)
        id_q = abs(q[0] - F32(1)) < F32(1e-7) and all(abs(c) < F32(1e-7) for c in q[1:])
        if not unit_s or not id_q:
            pv = np.array(pivot, F32)
            d = (x - pv) * np.array(sc, F32)
            if not id_q:
                d = rotate(q, d)
            x = (pv + d).astype(F32)
        if cloth and o.source.kind == "primitive" and o.source.primitive.shape == "grid":
            x = PR.cloth_jiggle(x, o.source.primitive.direction, (o.id ^ i) & 0xFFFFFFFF)
        nV = len(x)
        mask = np.ones(nV, F32)
        for fp in o.fixed_particles:
            if 0 <= fp.vid < nV:
                x[fp.vid] = np.array(fp.pos, F32)
                mask[fp.vid] = F32(0)
        if o.spline_constraints:
            warnings.append(f"object {o.id} ({o.name}): {len(o.spline_constraints)} spline constraints are not applied")
        flags = (MESH_STATIC if o.is_static else 0) | (MESH_COLLIDABLE if o.collidable else 0) | \
                (MESH_SELF_COLLIDE if o.self_collide else 0)
        m = G.Mesh(behavior=beh, flags=flags, x=x, facets=fac, v=np.zeros_like(x), mass=np.full(nV, F32(mass), F32),
                   mask=mask, kstretch=float(bp.get("kstretch", 0.0)), kshear=float(bp.get("kshear", 0.0)),
                   kbend=float(bp.get("kbend", 0.0)), thickness=float(bp.get("thickness", 0.0)))
        if beh == FAST_GRID_CLOTH:
            n = bp["grid_n"]
            if n * n != nV:
                raise SF.SceneFormatError(f"object {o.id} ({o.name}): particle_num_1d {n} does not match "
                                          f"the {nV}-vertex source")
            m.grid_n = n
            m.grid_rest = G.fast_grid_rest(x, n)
        # collider
        kind = o.collider_kind if o.collider_kind in _COLLIDER_CODE else \
            (_DEFAULT_COLLIDER.get(o.source.primitive.shape, "mesh") if o.source.kind == "primitive" else "mesh")
        if kind != "mesh":
            match = o.source.kind == "primitive" and _DEFAULT_COLLIDER.get(o.source.primitive.shape) == kind
            if match:
                hh = psize * F32(0.5)
                half = tuple(float(hh * c) for c in sc)
            else:  # geometry fit in the collider frame
                loc = rotate((q[0], -q[1], -q[2], -q[3]), (x - np.array(pivot, F32)).astype(F32))
                half = tuple(float(max(F32(0), np.abs(loc[:, k]).max() if nV else F32(0))) for k in range(3))
            m.collider = (_COLLIDER_CODE[kind], tuple(float(c) for c in pivot), half, tuple(float(c) for c in q))
        meshes.append(m)
        # environment forces of this mesh
        e = np.zeros((nV, 3), F32)
        if cloth:
            if o.apply_gravity:
                e = (m.mass[:, None] * np.array(g, F32)[None, :]).astype(F32)
            if o.apply_wind:
                e = (e + np.array(w, F32)[None, :]).astype(F32)
            if not o.apply_gravity or (o.apply_wind and any(c != 0 for c in w)):
                custom_forces = True
        ext_parts.append(e)
    sim = snap.simulation
    subh = F32(F32(sim.time_per_frame) / F32(sim.substeps))
    prm = G.Params(subh=float(subh), substeps=int(sim.substeps), gravity=tuple(float(c) for c in g),
                   self_mode=SELF_HASH)
    name = SF.path_stem(scene_path) if scene_path else "scene"
    spec = G.SceneSpec(name, prm, meshes, 0)
    ext = np.concatenate(ext_parts) if (custom_forces and ext_parts) else None
    return LoadedScene(spec, ext, cfg, warnings)
