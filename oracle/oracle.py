"""ctypes wrapper of the CPU oracle (oracle/ys_oracle.cpp).

TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build_oracle import OUT, build

NODE_DTYPE = np.dtype([("mn", "<f4", 3), ("a", "<i4"), ("mx", "<f4", 3), ("b", "<i4")])
ROW_DTYPE = np.dtype([("point", "<u4"), ("tri", "<u4"), ("qobj", "<u4"), ("tobj", "<u4"), ("qbeh", "<u4"),
                      ("tbeh", "<u4"), ("qshape", "<u4"), ("tshape", "<u4")])
SHAPE_DTYPE = np.dtype([("cr", "<f4", 4), ("he", "<f4", 4), ("rq", "<f4", 4), ("pc", "<f4", 4), ("prq", "<f4", 4),
                        ("kind", "<u4"), ("obj", "<u4"), ("beh", "<u4"), ("flags", "<u4")])
CONTACT_DTYPE = np.dtype([("point", "<u4"), ("tri", "<u4"), ("qobj", "<u4"), ("tobj", "<u4"), ("n", "<f4", 3),
                          ("d", "<f4"), ("qbeh", "<u4"), ("tbeh", "<u4"), ("qshape", "<u4"), ("tshape", "<u4")])

_lib = None
vp = C.c_void_p


def lib():
    global _lib
    if _lib is None:
        path = OUT if os.path.exists(OUT) else build()
        L = C.CDLL(path)
        sig = {
            "yso_set_threads": (None, [C.c_int]),
            "yso_max_threads": (C.c_int, []),
            "yso_scene_box": (None, [vp, C.c_uint32, vp]),
            "yso_fill_mortons": (None, [vp, vp, C.c_uint32, vp, vp, vp]),
            "yso_radix_sort": (None, [vp, vp, C.c_uint32]),
            "yso_karras": (None, [vp, vp, C.c_uint32, vp, vp]),
            "yso_leaves": (None, [vp, vp, C.c_float, C.c_int, vp, C.c_uint32, vp]),
            "yso_bottom_up": (None, [vp, C.c_uint32]),
            "yso_build_tree": (None, [vp, C.c_uint32, vp, C.c_uint32, vp, vp, vp, vp]),
            "yso_build_tree_apetrei": (C.c_int, [vp, C.c_uint32, vp, C.c_uint32, vp, vp, vp, vp]),
            "yso_scene_set_builder": (None, [vp, C.c_int]),
            "yso_query_points": (C.c_uint64, [vp, C.c_uint32, vp, vp, C.c_uint32, C.c_float, C.c_int, vp,
                                              C.c_uint64]),
            "yso_self_hash": (C.c_uint64, [vp, vp, C.c_uint32, vp, C.c_uint32, C.c_float, vp, C.c_uint64]),
            "yso_brute_q1": (C.c_uint64, [vp, vp, C.c_uint32, vp, C.c_uint32, C.c_float, C.c_int, vp, C.c_uint64]),
            "yso_brute_h1": (C.c_uint64, [vp, vp, C.c_uint32, vp, C.c_uint32, C.c_float, vp, C.c_uint64]),
            "yso_point_tri_sq": (C.c_float, [vp, vp, vp, vp]),
            "yso_narrow_one": (C.c_int, [vp, vp, vp, vp, vp, C.c_float, vp, vp]),
            "yso_adj_new": (vp, [vp, C.c_uint32, vp, C.c_uint32]),
            "yso_adj_size": (C.c_uint64, [vp, C.c_int]),
            "yso_adj_get": (None, [vp, C.c_int, vp]),
            "yso_adj_free": (None, [vp]),
            "yso_scene_new": (vp, [vp, vp]),
            "yso_scene_free": (None, [vp]),
            "yso_scene_add_mesh": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint32, vp, vp, vp, vp, C.c_uint32, vp,
                                             vp, C.c_uint32, vp]),
            "yso_scene_pack": (None, [vp]),
            "yso_scene_step": (None, [vp, C.c_uint32]),
            "yso_scene_stage": (None, [vp, C.c_int]),
            "yso_scene_get": (None, [vp, C.c_int, vp]),
            "yso_scene_set": (None, [vp, C.c_int, vp]),
            "yso_scene_stats": (None, [vp, vp]),
            "yso_scene_nrows": (C.c_uint64, [vp]),
            "yso_scene_rows": (None, [vp, vp]),
            "yso_scene_ncontacts": (C.c_uint64, [vp]),
            "yso_scene_contacts": (None, [vp, vp, vp]),
            "yso_scene_tree_nodes": (C.c_uint64, [vp, C.c_int]),
            "yso_scene_tree": (None, [vp, C.c_int, vp, vp, vp, vp]),
            "yso_scene_set_collider": (C.c_int, [vp, C.c_int, C.c_uint32, vp, vp, vp]),
            "yso_scene_shapes": (C.c_uint64, [vp, vp]),
            "yso_scene_set_wind": (None, [vp, vp]),
            "yso_scene_set_mesh_env": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
            "yso_analytic_one": (C.c_int, [vp, vp, vp, C.c_float, C.c_float, C.c_float, vp, vp]),
            "yso_rot_margin": (C.c_float, [vp, C.c_float, C.c_float]),
            "yso_broad_box": (C.c_int, [vp, C.c_float, vp]),
            "yso_narrow_analytic": (C.c_uint64, [vp, vp, vp, vp, C.c_uint32, vp, C.c_uint32, vp, C.c_uint32,
                                                 C.c_float, C.c_float, vp, C.c_uint64]),
            "yso_sh_face_face": (C.c_uint64, [vp, vp, vp, vp, vp, vp, C.c_uint32, C.c_float, C.c_int, vp,
                                              C.c_uint64, vp]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def P(a):
    return None if a is None else a.ctypes.data_as(vp)


def set_threads(n: int):
    lib().yso_set_threads(n)


def max_threads() -> int:
    return lib().yso_max_threads()


def build_tree(x: np.ndarray, F: np.ndarray, builder: int = 0):
    """Box, Morton, sort and the Karras (builder 0) or Apetrei (1) build."""
    x = np.ascontiguousarray(x, np.float32)
    F = np.ascontiguousarray(F, np.uint32)
    n = len(F)
    nodes = np.zeros(2 * n - 1, NODE_DTYPE)
    parent = np.full(2 * n - 1, -1, np.int32)
    codes = np.zeros(n, np.uint32)
    idx = np.zeros(n, np.uint32)
    if builder == 1:
        lib().yso_build_tree_apetrei(P(x), len(x), P(F), n, P(nodes), P(parent), P(codes), P(idx))
    else:
        lib().yso_build_tree(P(x), len(x), P(F), n, P(nodes), P(parent), P(codes), P(idx))
    return nodes, parent, codes, idx


def morton(x, F):
    x = np.ascontiguousarray(x, np.float32)
    F = np.ascontiguousarray(F, np.uint32)
    box = np.zeros(6, np.float32)
    lib().yso_scene_box(P(x), len(x), P(box))
    codes = np.zeros(len(F), np.uint32)
    idx = np.zeros(len(F), np.uint32)
    lib().yso_fill_mortons(P(x), P(F), len(F), P(box), P(codes), P(idx))
    return codes, idx


def radix_sort(keys, vals):
    k = np.ascontiguousarray(keys, np.uint32).copy()
    v = np.ascontiguousarray(vals, np.uint32).copy()
    lib().yso_radix_sort(P(k), P(v), len(k))
    return k, v


def refit(nodes, x, v, F, dt, swept):
    nodes = nodes.copy()
    n = (len(nodes) + 1) // 2
    x = np.ascontiguousarray(x, np.float32)
    v = None if v is None else np.ascontiguousarray(v, np.float32)
    F = np.ascontiguousarray(F, np.uint32)
    lib().yso_leaves(P(x), P(v), dt, 1 if swept else 0, P(F), n, P(nodes))
    lib().yso_bottom_up(P(nodes), len(nodes))
    return nodes


def query_points(nodes, F, q, margin, self_query=False, cap=None):
    q = np.ascontiguousarray(q, np.float32)
    F = np.ascontiguousarray(F, np.uint32)
    n = lib().yso_query_points(P(nodes), len(nodes), P(F), P(q), len(q), margin, int(self_query), None, 0)
    out = np.zeros((n, 2), np.uint32)
    lib().yso_query_points(P(nodes), len(nodes), P(F), P(q), len(q), margin, int(self_query), P(out), n)
    return out


def pack_meshes(meshes):
    """Packed-scene arrays of a mesh list (Scene::pack, scene.hpp:783-1180):
    x (V, 3), per-mesh vertex and face offsets, facets with mesh-local vertex
    ids, behaviours, shapes (0 = triangle mesh)."""
    x = np.concatenate([np.asarray(m.x, np.float32) for m in meshes])
    so = np.concatenate([[0], np.cumsum([m.nV for m in meshes])]).astype(np.uint32)
    fo = np.concatenate([[0], np.cumsum([m.nF for m in meshes])]).astype(np.uint32)
    F = np.concatenate([np.asarray(m.facets, np.uint32) for m in meshes])
    beh = np.array([m.behavior for m in meshes], np.uint32)
    shape = np.zeros(len(meshes), np.uint32)
    return x, so, fo, F, beh, shape


def sh_face_face(x, so, fo, F, beh, shape, margin, self_rows=True):
    """H2 rows (ROW_DTYPE) of the face-face spatial hash, and stats (entries,
    cells, candidate pairs, grid resolution)."""
    a = [np.ascontiguousarray(t, d) for t, d in ((x, np.float32), (so, np.uint32), (F, np.uint32), (fo, np.uint32),
                                                  (beh, np.uint32), (shape, np.uint32))]
    st = np.zeros(6, np.uint32)
    n = lib().yso_sh_face_face(*[P(t) for t in a], len(beh), margin, int(self_rows), None, 0, P(st))
    out = np.zeros(n, ROW_DTYPE)
    lib().yso_sh_face_face(*[P(t) for t in a], len(beh), margin, int(self_rows), P(out), n, P(st))
    return out, st


def brute_q1(x, F, q, margin, self_query=False):
    x = np.ascontiguousarray(x, np.float32)
    F = np.ascontiguousarray(F, np.uint32)
    q = np.ascontiguousarray(q, np.float32)
    n = lib().yso_brute_q1(P(x), P(F), len(F), P(q), len(q), margin, int(self_query), None, 0)
    out = np.zeros((n, 2), np.uint32)
    lib().yso_brute_q1(P(x), P(F), len(F), P(q), len(q), margin, int(self_query), P(out), n)
    return out


def self_hash(x, xp, F, m):
    x = np.ascontiguousarray(x, np.float32)
    xp = np.ascontiguousarray(xp, np.float32)
    F = np.ascontiguousarray(F, np.uint32)
    n = lib().yso_self_hash(P(x), P(xp), len(x), P(F), len(F), m, None, 0)
    out = np.zeros((n, 2), np.uint32)
    lib().yso_self_hash(P(x), P(xp), len(x), P(F), len(F), m, P(out), n)
    return out


def brute_h1(x, xp, F, m):
    x = np.ascontiguousarray(x, np.float32)
    xp = np.ascontiguousarray(xp, np.float32)
    F = np.ascontiguousarray(F, np.uint32)
    n = lib().yso_brute_h1(P(x), P(xp), len(x), P(F), len(F), m, None, 0)
    out = np.zeros((n, 2), np.uint32)
    lib().yso_brute_h1(P(x), P(xp), len(x), P(F), len(F), m, P(out), n)
    return out


def adjacency(x, F):
    x = np.ascontiguousarray(x, np.float32)
    F = np.ascontiguousarray(F, np.uint32)
    h = lib().yso_adj_new(P(x), len(x), P(F), len(F))
    names = ["vaf_off", "vaf", "edges", "rest_edge", "vae_off", "vae", "opp_off", "opp", "rest_opp"]
    out = {}
    for i, nm in enumerate(names):
        n = lib().yso_adj_size(h, i)
        a = np.zeros(n, np.float32 if nm.startswith("rest") else np.uint32)
        lib().yso_adj_get(h, i, P(a))
        out[nm] = a
    lib().yso_adj_free(h)
    return out


def analytic_one(shape, pcur, pprev, radius, thickness, rot_margin=0.0):
    """narrow_pt_analytic for one vertex: (hit, normal, d)."""
    sh = np.ascontiguousarray(shape, SHAPE_DTYPE).reshape(1)
    n = np.zeros(3, np.float32)
    d = np.zeros(1, np.float32)
    hit = lib().yso_analytic_one(P(sh), P(np.asarray(pcur, np.float32)), P(np.asarray(pprev, np.float32)),
                                 radius, thickness, rot_margin, P(n), P(d))
    return bool(hit), n, float(d[0])


def rot_margin(shape, radius, thickness) -> float:
    sh = np.ascontiguousarray(shape, SHAPE_DTYPE).reshape(1)
    return float(lib().yso_rot_margin(P(sh), radius, thickness))


def broad_box(shape, inflate):
    sh = np.ascontiguousarray(shape, SHAPE_DTYPE).reshape(1)
    out = np.zeros(6, np.float32)
    fin = lib().yso_broad_box(P(sh), inflate, P(out))
    return bool(fin), out


def narrow_analytic(x, xp, state_off, beh, shapes, pairs, radius, thickness, cap=None):
    """narrowAnalytic over explicit (cloth, collider) pairs: contacts in
    pair-then-vertex order and the total count."""
    x = np.ascontiguousarray(x, np.float32)
    xp = np.ascontiguousarray(xp, np.float32)
    so = np.ascontiguousarray(state_off, np.uint32)
    be = np.ascontiguousarray(beh, np.uint32)
    sh = np.ascontiguousarray(shapes, SHAPE_DTYPE)
    pr = np.ascontiguousarray(pairs, np.uint32).reshape(-1, 2)
    cap = len(x) * max(len(pr), 1) if cap is None else cap
    out = np.zeros(max(cap, 1), CONTACT_DTYPE)
    n = lib().yso_narrow_analytic(P(x), P(xp), P(so), P(be), len(be), P(sh), len(sh), P(pr), len(pr), radius,
                                  thickness, P(out), cap)
    return out[: min(n, cap)], int(n)


class OracleScene:
    """CPU restatement of the packed scene + Simulator::update substeps."""

    def __init__(self, spec, builder: int = 0):
        p = spec.params
        fp = np.array([p.subh, p.kair, p.kd, *p.gravity, p.margin, p.radius], np.float32)
        ip = np.array([p.substeps, p.rebuild_frames, p.self_mode, p.cols_per_point], np.uint32)
        self.h = lib().yso_scene_new(P(fp), P(ip))
        lib().yso_scene_set_builder(self.h, builder)
        self.spec = spec
        self._keep = []
        for m in spec.meshes:
            x = np.ascontiguousarray(m.x, np.float32)
            v = np.ascontiguousarray(m.v if m.v is not None else np.zeros_like(x), np.float32)
            mass = np.ascontiguousarray(m.mass if m.mass is not None else np.ones(m.nV, np.float32), np.float32)
            mask = np.ascontiguousarray(m.mask if m.mask is not None else np.ones(m.nV, np.float32), np.float32)
            F = np.ascontiguousarray(m.facets, np.uint32)
            kp = np.array([m.kstretch, m.kshear, m.kbend, m.thickness], np.float32)
            rest = np.array(m.grid_rest, np.float32)
            idx = lib().yso_scene_add_mesh(self.h, m.behavior, m.flags, m.nV, P(x), P(v), P(mass), P(mask), m.nF,
                                           P(F), P(kp), m.grid_n, P(rest))
            if getattr(m, "collider", None) is not None:
                self.set_collider(idx, *m.collider)
        lib().yso_scene_pack(self.h)
        self.nV = spec.nV

    def __del__(self):
        if getattr(self, "h", None):
            lib().yso_scene_free(self.h)
            self.h = None

    def step(self, n=1):
        lib().yso_scene_step(self.h, n)

    def set_collider(self, mesh, kind, center, half=(0.0, 0.0, 0.0), q=(1.0, 0.0, 0.0, 0.0)):
        c = np.array(center, np.float32)
        h = np.array(half, np.float32)
        r = np.array(q, np.float32)
        if lib().yso_scene_set_collider(self.h, mesh, kind, P(c), P(h), P(r)) != 0:
            raise ValueError("yso_scene_set_collider rejected the collider")

    def set_environment(self, wind, gates):
        """applyEnvironmentForces inputs: the wind vector and, per mesh, its
        (apply_gravity, apply_wind) gates; they act from the next frame
        start."""
        lib().yso_scene_set_wind(self.h, P(np.asarray(wind, np.float32)))
        for m, (g, w) in enumerate(gates):
            if lib().yso_scene_set_mesh_env(self.h, m, int(bool(g)), int(bool(w))) != 0:
                raise ValueError("yso_scene_set_mesh_env rejected the mesh")

    def shapes(self):
        n = lib().yso_scene_shapes(self.h, None)
        out = np.zeros(n, SHAPE_DTYPE)
        lib().yso_scene_shapes(self.h, P(out))
        return out

    def stage(self, which: int):
        lib().yso_scene_stage(self.h, which)

    def get(self, which: str):
        code = {"x": 0, "v": 1, "xprev": 2, "f": 3, "ext": 4}[which]
        out = np.zeros((self.nV, 3), np.float32)
        lib().yso_scene_get(self.h, code, P(out))
        return out

    def set(self, which: str, arr):
        code = {"x": 0, "v": 1, "xprev": 2}[which]
        a = np.ascontiguousarray(arr, np.float32)
        lib().yso_scene_set(self.h, code, P(a))

    def stats(self):
        out = np.zeros(7, np.uint64)
        lib().yso_scene_stats(self.h, P(out))
        keys = ("frame", "cursor", "broad_rows", "contacts_kept", "anomaly", "flags", "contacts")
        return dict(zip(keys, (int(v) for v in out)))

    def rows(self):
        n = lib().yso_scene_nrows(self.h)
        out = np.zeros(n, ROW_DTYPE)
        lib().yso_scene_rows(self.h, P(out))
        return out

    def contacts(self):
        n = lib().yso_scene_ncontacts(self.h)
        off = np.zeros(self.nV + 1, np.uint32)
        out = np.zeros(n, CONTACT_DTYPE)
        lib().yso_scene_contacts(self.h, P(off), P(out))
        return off, out

    def tree(self, mesh: int):
        nn = lib().yso_scene_tree_nodes(self.h, mesh)
        nodes = np.zeros(nn, NODE_DTYPE)
        parent = np.zeros(nn, np.int32)
        n = (nn + 1) // 2
        codes = np.zeros(n, np.uint32)
        idx = np.zeros(n, np.uint32)
        lib().yso_scene_tree(self.h, mesh, P(nodes), P(parent), P(codes), P(idx))
        return nodes, parent, codes, idx


# ---------------------------------------------------------------- adjoint (FP64)
class Rollout:
    """FP64 CPU reference of the differentiable FastGridCloth rollout
    (ys_adjoint_oracle.cpp): forward substeps and the hand-derived adjoint."""

    def __init__(self, spec, k, L, v0=None):
        d = ctypes_double = C.c_double
        L_ = lib()
        for name, res, args in [("yso_roll_new", vp, [vp, vp, vp, vp, vp, vp, vp, vp]),
                                ("yso_roll_free", None, [vp]), ("yso_roll_num_springs", C.c_uint64, [vp]),
                                ("yso_roll_set", None, [vp, vp, vp, vp]),
                                ("yso_roll_forward", C.c_uint64, [vp, C.c_int, C.c_int, vp]),
                                ("yso_roll_backward", None, [vp, C.c_int, vp, vp, vp, vp])]:
            fn = getattr(L_, name)
            fn.restype = res
            fn.argtypes = args
        del d, ctypes_double
        cloth, ob = spec.meshes[0], spec.meshes[1]
        p = spec.params
        self.N = cloth.grid_n
        self.V = cloth.nV
        ip = np.array([cloth.grid_n, ob.nV, ob.nF], np.int32)
        dp = np.array([p.kd, p.kair, p.subh, cloth.thickness, p.margin, p.radius, *p.gravity], np.float64)
        self._arrs = [np.ascontiguousarray(a, np.float64) for a in
                      (cloth.x, cloth.v if v0 is None else v0, cloth.mass, cloth.mask, ob.x)]
        oF = np.ascontiguousarray(ob.facets, np.uint32)
        self.h = L_.yso_roll_new(P(ip), P(dp), *[P(a) for a in self._arrs], P(oF))
        self.S = int(L_.yso_roll_num_springs(self.h))
        self.set(k, L)

    def __del__(self):
        if getattr(self, "h", None):
            lib().yso_roll_free(self.h)
            self.h = None

    def set(self, k=None, L=None, v0=None):
        a = [None if t is None else np.ascontiguousarray(t, np.float64) for t in (k, L, v0)]
        lib().yso_roll_set(self.h, *[P(t) for t in a])

    def forward(self, T, keep=False):
        x = np.zeros((self.V, 3), np.float64)
        n = lib().yso_roll_forward(self.h, T, 1 if keep else 0, P(x))
        return x, int(n)

    def backward(self, T, dLdx):
        gk = np.zeros(self.S, np.float64)
        gL = np.zeros(self.S, np.float64)
        gv = np.zeros((self.V, 3), np.float64)
        lib().yso_roll_backward(self.h, T, P(np.ascontiguousarray(dLdx, np.float64)), P(gk), P(gL), P(gv))
        return gk, gL, gv
