"""ctypes wrapper of oracle/_ref/libysref.so: the reference's own Metal kernels
compiled for the host (see oracle/build_ref.py).  TEST INFRASTRUCTURE ONLY."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import build_ref
from .oracle import CONTACT_DTYPE, NODE_DTYPE, ROW_DTYPE

vp = C.c_void_p
u32 = C.c_uint32
f32 = C.c_float
_lib = None


def available() -> bool:
    return os.path.exists(build_ref.OUT) or build_ref.available()


def lib():
    global _lib
    if _lib is None:
        path = build_ref.build()
        if not path:
            raise FileNotFoundError("reference kernels not built (reference checkout absent)")
        L = C.CDLL(path)
        sig = {
            "yref_fill_mortons": (None, [vp, vp, u32, vp, vp]),
            "yref_build_tree": (None, [vp, vp, u32, vp, vp, vp]),
            "yref_leaves": (None, [vp, vp, u32, vp, vp]),
            "yref_swept_leaves": (None, [vp, vp, vp, u32, f32, vp, vp]),
            "yref_bottom_up": (None, [vp, vp, u32, vp]),
            "yref_agglomerative": (C.c_int32, [vp, vp, u32, vp, vp, vp]),
            "yref_scene_roundtrip": (C.c_int, [C.c_char_p, vp, C.c_size_t, vp]),
            "yref_runconfig_roundtrip": (C.c_int, [C.c_char_p, vp, C.c_size_t]),
            "yref_primitive": (C.c_int, [C.c_int, f32, C.c_int, vp, vp, C.c_size_t, C.c_size_t, vp, vp]),
            "yref_uniform_float": (None, [u32, f32, f32, u32, vp]),
            "yref_profile_paths": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, vp, C.c_size_t]),
            "yref_profiler_csv": (C.c_int, [C.c_char_p, C.c_int, vp, vp, vp, vp, vp, C.c_int, vp, vp, C.c_int]),
            "yref_query_points": (u32, [vp, u32, vp, vp, u32, f32, u32, u32, vp, u32, vp]),
            "yref_narrow": (u32, [vp, u32, vp, vp, vp, vp, vp, vp, f32, f32, vp, vp, u32]),
            "yref_tri_forces": (None, [vp, vp, vp, vp, vp, vp, f32, f32, f32, vp, vp, vp, vp, vp, vp, vp, vp, vp,
                                       u32]),
            "yref_integrate_tri": (None, [vp, vp, vp, vp, vp, vp, vp, vp, u32, f32, vp, u32, vp]),
            "yref_grid_forces": (None, [vp, vp, vp, vp, vp, f32, f32, f32, vp, u32]),
            "yref_integrate_grid": (None, [vp, vp, vp, vp, vp, vp, vp, vp, u32, f32, vp, u32, vp]),
            "yref_bucket": (None, [vp, u32, vp, u32, vp, vp, vp]),
            "yref_sh_detect": (u32, [vp, vp, vp, vp, vp, vp, u32, f32, u32, vp, u32, vp]),
            "yref_narrow_analytic": (u32, [vp, vp, vp, vp, u32, u32, u32, u32, f32, f32, f32, vp, u32]),
        }
        for k, (r, a) in sig.items():
            fn = getattr(L, k)
            fn.restype = r
            fn.argtypes = a
        _lib = L
    return _lib


def P(a):
    return None if a is None else a.ctypes.data_as(vp)


def c32(a, dt=np.float32):
    return np.ascontiguousarray(a, dt)


def fill_mortons(x, F, box6):
    x, F, box6 = c32(x), c32(F, np.uint32), c32(box6)
    m = np.zeros((len(F), 2), np.uint32)
    lib().yref_fill_mortons(P(x), P(F), len(F), P(box6), P(m))
    return m[:, 0].copy(), m[:, 1].copy()


def build_tree(x, F, codes, idx):
    """buildTree_Tri + zeroVisitCounts + bottomUpBoxes on sorted (code, index)."""
    x, F = c32(x), c32(F, np.uint32)
    n = len(F)
    m = np.ascontiguousarray(np.stack([codes, idx], 1), np.uint32)
    nodes = np.zeros(2 * n - 1, NODE_DTYPE)
    parent = np.full(2 * n - 1, -1, np.int32)
    lib().yref_build_tree(P(x), P(F), n, P(m), P(nodes), P(parent))
    visits = np.zeros(2 * n - 1, np.uint32)
    lib().yref_bottom_up(P(nodes), P(parent), n, P(visits))
    return nodes, parent


def refit(nodes, parent, x, v, F, codes, idx, dt, swept):
    nodes = nodes.copy()
    x, F = c32(x), c32(F, np.uint32)
    n = len(F)
    m = np.ascontiguousarray(np.stack([codes, idx], 1), np.uint32)
    if swept:
        lib().yref_swept_leaves(P(x), P(c32(v)), P(F), n, dt, P(m), P(nodes))
    else:
        lib().yref_leaves(P(x), P(F), n, P(m), P(nodes))
    visits = np.zeros(2 * n - 1, np.uint32)
    lib().yref_bottom_up(P(nodes), P(c32(parent, np.int32)), n, P(visits))
    return nodes


def query_points(qx, F, nodes, margin, qobj, tobj, cap=None):
    qx, F = c32(qx), c32(F, np.uint32)
    cap = cap or max(64, len(qx) * 64)
    rows = np.zeros(cap, ROW_DTYPE)
    flags = np.zeros(2, np.uint32)
    n = lib().yref_query_points(P(qx), len(qx), P(F), P(nodes), len(nodes), margin, qobj, tobj, P(rows), cap,
                                P(flags))
    return rows[: min(n, cap)], n, flags


def narrow(rows, x, voff, F, foff, vaf, vaf_off, radius, thickness, xprev, cap=None):
    cap = cap or max(64, len(rows))
    out = np.zeros(cap, CONTACT_DTYPE)
    n = lib().yref_narrow(P(np.ascontiguousarray(rows)), len(rows), P(c32(x)), P(c32(voff, np.uint32)),
                          P(c32(F, np.uint32)), P(c32(foff, np.uint32)), P(c32(vaf, np.uint32)),
                          P(c32(vaf_off, np.uint32)), radius, thickness, P(c32(xprev)), P(out), cap)
    return out[: min(n, cap)]


def agglomerative(x, F, codes, idx):
    """agglomerativeBuild_Tri + agglomerativeSwapRoot over sorted (code, index)
    pairs: (nodes, parent, pre-swap root slot)."""
    n = len(codes)
    mortons = np.ascontiguousarray(np.stack([codes, idx], 1), np.uint32)
    nodes = np.zeros(2 * n - 1, NODE_DTYPE)
    parent = np.full(2 * n - 1, -1, np.int32)
    k = lib().yref_agglomerative(P(c32(x)), P(c32(F, np.uint32)), n, P(mortons), P(nodes), P(parent))
    return nodes, parent, int(k)


def scene_roundtrip(text: str, runconfig: bool = False):
    """scene_format (or sim_config) parseString + toString: (ok, text or error, warnings)."""
    buf = C.create_string_buffer(1 << 22)
    w = np.zeros(1, np.int32)
    if runconfig:
        rc = lib().yref_runconfig_roundtrip(text.encode(), buf, len(buf))
    else:
        rc = lib().yref_scene_roundtrip(text.encode(), buf, len(buf), P(w))
    return rc == 0, buf.value.decode(), int(w[0])


def primitive(kind: str, size: float, tess: int):
    """primitive::sphere / cube / cylinder at the origin: (positions, facets)."""
    k = {"sphere": 0, "cube": 1, "cylinder": 2}[kind]
    nv, nf = np.zeros(1, np.uint32), np.zeros(1, np.uint32)
    lib().yref_primitive(k, size, tess, None, None, 0, 0, P(nv), P(nf))
    pos = np.zeros((int(nv[0]), 3), np.float32)
    fac = np.zeros((int(nf[0]), 3), np.uint32)
    lib().yref_primitive(k, size, tess, P(pos), P(fac), len(pos), len(fac), P(nv), P(nf))
    return pos, fac


def uniform_float(seed: int, lo: float, hi: float, n: int):
    """std::uniform_real_distribution<float>(lo, hi) over std::mt19937(seed)."""
    out = np.zeros(n, np.float32)
    lib().yref_uniform_float(seed, lo, hi, n, P(out))
    return out


def profile_paths(root: str, scene_path: str, frames: int):
    buf = C.create_string_buffer(4096)
    lib().yref_profile_paths(root.encode(), scene_path.encode(), frames, buf, len(buf))
    return tuple(buf.value.decode().split("\n"))


def profiler_csv(path: str, seq, wall, frame_ms, broad, narrow, names, sec_ms, max_frames=240) -> str:
    """FrameProfilerHistory::exportCsv of the given frames; returns the file's text."""
    n = len(seq)
    arr = (C.c_char_p * max(len(names), 1))(*[s.encode() for s in names])
    sec = np.ascontiguousarray(np.asarray(sec_ms, np.float64).reshape(n, len(names)))
    lib().yref_profiler_csv(path.encode(), n, P(np.asarray(seq, np.uint64)), P(np.asarray(wall, np.float64)),
                            P(np.asarray(frame_ms, np.float64)), P(np.asarray(broad, np.uint64)),
                            P(np.asarray(narrow, np.uint64)), len(names), arr, P(sec), max_frames)
    with open(path) as f:
        return f.read()


def narrow_analytic(x, xprev, voff, shapes, oid, shape_index, cloth_beh, radius, thickness, rot_margin, cap=None):
    """narrow_pt_analytic over every vertex of cloth mesh oid against
    shapes[shape_index] (SHAPE_DTYPE records)."""
    voff = c32(voff, np.uint32)
    nv = int(voff[oid + 1] - voff[oid])
    cap = cap or max(64, nv)
    out = np.zeros(cap, CONTACT_DTYPE)
    n = lib().yref_narrow_analytic(P(c32(x)), P(c32(xprev)), P(voff), P(np.ascontiguousarray(shapes)), oid, nv,
                                   shape_index, cloth_beh, radius, thickness, rot_margin, P(out), cap)
    return out[: min(n, cap)]


def tri_forces(x, v, ext, mass3, mask, subh, kair, kd, cp4, adj, F):
    x, v = c32(x), c32(v)
    f = np.zeros_like(x)
    lib().yref_tri_forces(P(x), P(v), P(f), P(c32(mass3)), P(c32(mask)), P(c32(ext)), subh, kair, kd,
                          P(c32(cp4)), P(c32(adj["edges"], np.uint32)), P(c32(F, np.uint32)),
                          P(c32(adj["vae"], np.uint32)), P(c32(adj["vae_off"], np.uint32)), P(c32(adj["rest_edge"])),
                          P(c32(adj["opp"], np.uint32)), P(c32(adj["opp_off"], np.uint32)), P(c32(adj["rest_opp"])),
                          len(x))
    return f


def grid_params(P1, rest6, k3, thickness):
    a = np.zeros(11, np.uint32)
    a[0] = P1
    a[1:7] = np.asarray(rest6, np.float32).view(np.uint32)
    a[7:10] = np.asarray(k3, np.float32).view(np.uint32)
    a[10] = np.asarray([thickness], np.float32).view(np.uint32)[0]
    return a


def grid_forces(x, v, ext, mass3, subh, kair, kd, gp11):
    x, v = c32(x), c32(v)
    f = np.zeros_like(x)
    lib().yref_grid_forces(P(x), P(v), P(f), P(c32(mass3)), P(c32(ext)), subh, kair, kd, P(c32(gp11, np.uint32)),
                           len(x))
    return f


def integrate(kind, x, v, f, mass3, mask, csr, csr_off, voff, oid, subh, params):
    x, v = c32(x).copy(), c32(v).copy()
    an = np.zeros(1, np.uint32)
    fn = lib().yref_integrate_tri if kind == "tri" else lib().yref_integrate_grid
    fn(P(x), P(v), P(c32(f)), P(c32(mass3)), P(c32(mask)), P(np.ascontiguousarray(csr)), P(c32(csr_off, np.uint32)),
       P(c32(voff, np.uint32)), oid, subh, P(c32(params, np.float32 if kind == "tri" else np.uint32)), len(x), P(an))
    return x, v, int(an[0])


def sh_detect(x, so, fo, F, beh, shape, margin, self_rows=True, cap=None):
    """SpatialHashing<METAL>::detectCollisions with the reference's kernels:
    BroadCollision rows (ROW_DTYPE, in kernel emission order) and stats."""
    if cap is None:
        cap = 64 * len(F) + 64
    out = np.zeros(cap, ROW_DTYPE)
    st = np.zeros(6, np.uint32)
    n = lib().yref_sh_detect(P(c32(x)), P(c32(so, np.uint32)), P(c32(F, np.uint32)), P(c32(fo, np.uint32)),
                             P(c32(beh, np.uint32)), P(c32(shape, np.uint32)), len(beh), margin, int(self_rows),
                             P(out), cap, P(st))
    assert n <= cap, "row capacity"
    return out[:n], st
