"""Host mirror of the reference's stage surfaces over the C ABI.

Names follow the reference so a caller of ysim finds the same stages:
  Scene.pack()                          Scene<BE,PR>::pack            (scene.hpp:783)
  Scene.broad_phase.build/refit_swept/detect_collisions
                                        BVH<SCENE,OBJECT>             (bvh.hpp:2537-2949)
  Scene.narrow_phase.narrow_and_sort_by_vertices
                                        BruteForce::narrowAndSortByVertices (bruteforce.hpp:311)
  Scene.system.snapshot_xprev / update  SymplecticSystem              (symplectic_system.hpp:230, 341)
  Simulator.update()                    one frame of substeps         (simulator.hpp:3169-3870)
Every call goes through the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from .generators import SceneSpec

ROW_DTYPE = np.dtype([("point", "<u4"), ("tri", "<u4"), ("qobj", "<u4"), ("tobj", "<u4"), ("qbeh", "<u4"),
                      ("tbeh", "<u4"), ("qshape", "<u4"), ("tshape", "<u4")])
VCONTACT_DTYPE = np.dtype([("tobj", "<u4"), ("tri", "<u4"), ("nx", "<f4"), ("ny", "<f4"), ("nz", "<f4"),
                           ("d", "<f4")])
NODE_DTYPE = np.dtype([("mn", "<f4", 3), ("a", "<i4"), ("mx", "<f4", 3), ("b", "<i4")])
WIDE_DTYPE = np.dtype([("lo", "<f4", (3, 4)), ("hi", "<f4", (3, 4)), ("child", "<i4", 4), ("nchild", "<u4"),
                       ("parent", "<i4"), ("slot", "<u4"), ("pad", "<u4")])
W4_EMPTY = 0x7FFFFFFF


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class _BroadPhase:
    def __init__(self, scene: "Scene"):
        self._s = scene

    def build(self):
        """Frame preamble: rebuild due trees (frame % rebuild_frames == 0)."""
        _lib.check(self._s.lib.ys_frame_preamble(self._s.h), "ys_frame_preamble")

    def refit_swept(self):
        _lib.check(self._s.lib.ys_broad_refit(self._s.h), "ys_broad_refit")

    def detect_collisions(self):
        _lib.check(self._s.lib.ys_broad_detect(self._s.h), "ys_broad_detect")


class _NarrowPhase:
    def __init__(self, scene: "Scene"):
        self._s = scene

    def narrow_and_sort_by_vertices(self):
        _lib.check(self._s.lib.ys_narrow_and_sort(self._s.h), "ys_narrow_and_sort")


class _System:
    def __init__(self, scene: "Scene"):
        self._s = scene

    def snapshot_xprev(self):
        _lib.check(self._s.lib.ys_snapshot_xprev(self._s.h), "ys_snapshot_xprev")

    def update(self):
        _lib.check(self._s.lib.ys_system_update(self._s.h), "ys_system_update")


class Scene:
    """A packed scene on one GPU (one CUDA stream)."""

    def __init__(self, spec: SceneSpec, device: int = 0, pack: bool = True, tree_layout: Optional[int] = None,
                 tree_builder: Optional[int] = None):
        self.lib = _lib.load()
        self.spec = spec
        p = spec.params
        sp = _lib.SimParams(p.subh, p.kair, p.kd, (C.c_float * 3)(*p.gravity), p.margin, p.radius, p.substeps,
                            p.rebuild_frames, p.self_mode, p.cols_per_point)
        h = C.c_void_p()
        _lib.check(self.lib.ys_scene_create(C.byref(h), C.byref(sp), device), "ys_scene_create")
        self.h = h
        self._keep = []
        for m in spec.meshes:
            x = np.ascontiguousarray(m.x, np.float32)
            v = np.ascontiguousarray(m.v if m.v is not None else np.zeros_like(x), np.float32)
            mass = np.ascontiguousarray(m.mass if m.mass is not None else np.ones(m.nV, np.float32), np.float32)
            mask = np.ascontiguousarray(m.mask if m.mask is not None else np.ones(m.nV, np.float32), np.float32)
            fac = np.ascontiguousarray(m.facets, np.uint32)
            d = _lib.MeshDesc(m.behavior, m.flags, m.nV, m.nF, _ptr(x), _ptr(v), _ptr(mass), _ptr(mask), _ptr(fac),
                              m.kstretch, m.kshear, m.kbend, m.thickness, m.grid_n,
                              (C.c_float * 6)(*m.grid_rest), m.group)
            idx = C.c_int()
            _lib.check(self.lib.ys_scene_add_mesh(self.h, C.byref(d), C.byref(idx)), "ys_scene_add_mesh")
            if m.collider is not None:
                self.set_collider(idx.value, *m.collider)
        if tree_layout is not None:
            _lib.check(self.lib.ys_scene_set_tree_layout(self.h, int(tree_layout)), "ys_scene_set_tree_layout")
        if tree_builder is not None:
            _lib.check(self.lib.ys_scene_set_tree_builder(self.h, int(tree_builder)), "ys_scene_set_tree_builder")
        self.nV = spec.nV
        self.broad_phase = _BroadPhase(self)
        self.narrow_phase = _NarrowPhase(self)
        self.system = _System(self)
        if pack:
            self.pack()

    def autotune(self, reps: int = 5):
        """Pick the fused kernel's register cap by timing each variant on the
        current state (the scene does not advance); returns (chosen, ms[3])."""
        chosen = C.c_int()
        ms = (C.c_float * 3)()
        _lib.check(self.lib.ys_scene_autotune(self.h, reps, C.byref(chosen), ms), "ys_scene_autotune")
        return chosen.value, list(ms)

    def autotune_classes(self, reps: int = 5):
        """Per size class of the working meshes, the fastest (register-cap
        variant, thread order) on the current state (the scene does not
        advance): a list of dicts for the non-empty classes."""
        out = (_lib.FusedClass * 4)()
        n = C.c_uint32()
        _lib.check(self.lib.ys_scene_autotune_classes(self.h, reps, out, 4, C.byref(n)), "ys_scene_autotune_classes")
        res = []
        for c in out[: n.value]:
            if c.vertices == 0:
                continue
            res.append({"max_mesh_vertices": int(c.max_mesh_vertices), "meshes": int(c.meshes),
                        "vertices": int(c.vertices), "ctas_per_sm": int(c.ctas_per_sm),
                        "thread_order": _lib.ORDER_NAMES[c.thread_order],
                        "ms": {name: [float(v) for v in c.ms[k]] for k, name in enumerate(_lib.ORDER_NAMES)}})
        return res

    def set_collider(self, mesh: int, kind: int, center, half=(0.0, 0.0, 0.0), q=(1.0, 0.0, 0.0, 0.0)):
        """Analytic collider kind and pose of a mesh (before pack: declares
        it; after: moves it from the next frame on)."""
        c = (C.c_float * 3)(*center)
        h = (C.c_float * 3)(*half)
        r = (C.c_float * 4)(*q)
        _lib.check(self.lib.ys_scene_set_collider(self.h, mesh, kind, c, h, r), "ys_scene_set_collider")

    def colliders(self) -> np.ndarray:
        """The analytic shape table as of the last frame start."""
        from .generators import SHAPE_DTYPE
        n = C.c_uint32()
        _lib.check(self.lib.ys_scene_colliders(self.h, None, 0, C.byref(n)), "ys_scene_colliders")
        out = np.zeros(n.value, SHAPE_DTYPE)
        _lib.check(self.lib.ys_scene_colliders(self.h, _ptr(out), n.value, C.byref(n)), "ys_scene_colliders")
        return out

    def set_fused_variant(self, min_blocks: int):
        _lib.check(self.lib.ys_scene_set_fused_variant(self.h, min_blocks), "ys_scene_set_fused_variant")

    def set_thread_order(self, order):
        """Fused-kernel threads over the working vertices in per-mesh Morton
        order ("morton" or True, default), vertex order ("vertex" or False),
        or 16 x 8 tiles of each grid cloth with TMA-staged spring tables
        ("tile"); the results are the same in every order."""
        if isinstance(order, str):
            code = _lib.ORDER_NAMES.index(order)
        else:
            code = _lib.ORDER_MORTON if order is True else _lib.ORDER_VERTEX if order is False else int(order)
        _lib.check(self.lib.ys_scene_set_thread_order(self.h, code), "ys_scene_set_thread_order")

    def pack(self):
        _lib.check(self.lib.ys_scene_pack(self.h), "ys_scene_pack")

    def close(self):
        if self.h:
            self.lib.ys_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- stepping
    def step(self, n: int = 1):
        """n substeps on the fused path."""
        _lib.check(self.lib.ys_scene_step(self.h, n), "ys_scene_step")

    def step_staged(self, n: int = 1):
        """n substeps, one kernel group per reference stage."""
        _lib.check(self.lib.ys_scene_step_staged(self.h, n), "ys_scene_step_staged")

    def set_record(self, on: bool):
        _lib.check(self.lib.ys_scene_set_record(self.h, 1 if on else 0), "ys_scene_set_record")

    def set_graphs(self, on: bool):
        _lib.check(self.lib.ys_scene_set_graphs(self.h, 1 if on else 0), "ys_scene_set_graphs")

    def sync(self):
        _lib.check(self.lib.ys_scene_sync(self.h), "ys_scene_sync")

    def stream(self) -> int:
        s = C.c_void_p()
        _lib.check(self.lib.ys_scene_stream(self.h, C.byref(s)), "ys_scene_stream")
        return s.value or 0

    # ---- state
    def get(self, which: str) -> np.ndarray:
        code = {"x": 0, "v": 1, "xprev": 2, "f": 3}[which]
        out = np.empty((self.nV, 3), np.float32)
        _lib.check(self.lib.ys_scene_get_state(self.h, code, _ptr(out)), "ys_scene_get_state")
        return out

    def set(self, which: str, arr: np.ndarray):
        code = {"x": 0, "v": 1, "xprev": 2}[which]
        a = np.ascontiguousarray(arr, np.float32)
        _lib.check(self.lib.ys_scene_set_state(self.h, code, _ptr(a)), "ys_scene_set_state")

    def stats(self) -> dict:
        out = (C.c_uint64 * 8)()
        _lib.check(self.lib.ys_scene_stats(self.h, out), "ys_scene_stats")
        keys = ("frame", "cursor", "broad_rows", "contacts", "anomaly", "flags", "num_vertices", "substeps")
        return dict(zip(keys, (int(v) for v in out)))

    def totals(self):
        out = (C.c_uint64 * 2)()
        _lib.check(self.lib.ys_scene_totals(self.h, out), "ys_scene_totals")
        return int(out[0]), int(out[1])

    def clear_flags(self):
        _lib.check(self.lib.ys_scene_clear_flags(self.h), "ys_scene_clear_flags")

    def rows(self) -> np.ndarray:
        n = C.c_uint64()
        _lib.check(self.lib.ys_scene_rows(self.h, None, 0, C.byref(n)), "ys_scene_rows")
        out = np.empty(n.value, ROW_DTYPE)
        _lib.check(self.lib.ys_scene_rows(self.h, _ptr(out), n.value, C.byref(n)), "ys_scene_rows")
        return out

    def contacts(self):
        n = C.c_uint64()
        off = np.empty(self.nV + 1, np.uint32)
        _lib.check(self.lib.ys_scene_contacts(self.h, _ptr(off), None, 0, C.byref(n)), "ys_scene_contacts")
        out = np.empty(n.value, VCONTACT_DTYPE)
        _lib.check(self.lib.ys_scene_contacts(self.h, _ptr(off), _ptr(out), n.value, C.byref(n)),
                   "ys_scene_contacts")
        return off, out

    def wide_tree(self, mesh: int) -> np.ndarray:
        """The 4-wide form of a mesh's tree as the last refit left it (cube
        layout; empty otherwise): WIDE_DTYPE records, lo/hi[axis][slot]."""
        n = C.c_uint32()
        _lib.check(self.lib.ys_scene_wide_tree(self.h, mesh, None, 0, C.byref(n)), "ys_scene_wide_tree")
        out = np.zeros(n.value, WIDE_DTYPE)
        if n.value:
            _lib.check(self.lib.ys_scene_wide_tree(self.h, mesh, _ptr(out), n.value, C.byref(n)),
                       "ys_scene_wide_tree")
        return out

    def tree(self, mesh: int):
        n = C.c_uint32()
        _lib.check(self.lib.ys_scene_tree(self.h, mesh, None, None, None, None, C.byref(n)), "ys_scene_tree")
        N = n.value
        nodes = np.empty(max(2 * N - 1, 0), NODE_DTYPE)
        parent = np.empty(max(2 * N - 1, 0), np.int32)
        codes = np.empty(N, np.uint32)
        idx = np.empty(N, np.uint32)
        _lib.check(self.lib.ys_scene_tree(self.h, mesh, _ptr(nodes), _ptr(parent), _ptr(codes), _ptr(idx),
                                          C.byref(n)), "ys_scene_tree")
        return nodes, parent, codes, idx


class Simulator:
    """Frame driver: Simulator::update (simulator.hpp:3169-3870) over a Scene."""

    def __init__(self, scene: Scene, fused: bool = True):
        self.scene = scene
        self.fused = fused

    def update(self):
        n = self.scene.spec.params.substeps
        if self.fused:
            self.scene.step(n)
        else:
            self.scene.step_staged(n)
