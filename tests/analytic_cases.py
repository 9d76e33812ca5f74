"""Seeded analytic-collider cases shared by the golden generator and the tests.

Each case is one collider shape (AnalyticShape records, SHAPE_DTYPE) with a
cloud of vertices (x, x_prev) around it: points inside, on and outside the
shape and its contact band, static and moving, short and tunnelling segments,
axis-parallel segments against an unrotated shape, the centre itself.  Cloud i
is cloth mesh i of a packed array (state_off); the pairs are (i, shape i's
mesh index).
"""
from __future__ import annotations

import numpy as np

from ysim_b200 import generators as G

SPHERE, BOX, CYLINDER, PLANE = 1, 2, 3, 4
RADIUS, THICKNESS = np.float32(0.012), np.float32(0.015)


def _quat(rng, angle=None):
    axis = rng.normal(size=3)
    ang = rng.uniform(0, np.pi) if angle is None else angle
    return np.array(G.quat_axis_angle(axis, ang), np.float32)


def _shape(kind, c, h, q, pc, pq, obj, flags=1):
    s = np.zeros((), G.SHAPE_DTYPE)
    s["kind"], s["obj"], s["beh"], s["flags"] = kind, obj, 4, flags
    s["rq"], s["pc"][:3], s["prq"] = q, pc, pq
    s["cr"][:3] = c
    if kind == SPHERE:
        s["cr"][3] = h[0]
        s["he"] = (h[0], h[1], h[2], h[1])
    elif kind == BOX:
        s["he"][:3] = h
    elif kind == CYLINDER:
        s["cr"][3] = max(h[0], h[2])
        s["he"] = (h[0], h[1], h[2], h[1])
    return s


def cases(seed: int = 11, per_shape: int = 1000):
    """(shapes, x, xprev, state_off, behaviors, pairs)."""
    rng = np.random.default_rng(seed)
    ident = np.array([1, 0, 0, 0], np.float32)
    specs = []
    for kind in (SPHERE, BOX, CYLINDER, PLANE):
        for mode in ("identity", "rotated", "moving"):
            specs.append((kind, mode))
    specs.append((SPHERE, "ellipsoid"))
    specs.append((BOX, "disabled"))
    shapes, xs, xps = [], [], []
    for i, (kind, mode) in enumerate(specs):
        c = rng.uniform(-0.5, 0.5, 3).astype(np.float32)
        h = rng.uniform(0.05, 0.3, 3).astype(np.float32)
        if kind == SPHERE and mode != "ellipsoid":
            h[:] = h[0]
        if kind == PLANE:
            h[:] = 0
        q = ident if mode in ("identity", "disabled") else _quat(rng)
        pc, pq = c.copy(), q.copy()
        if mode == "moving":
            pc = (c + rng.normal(0, 0.03, 3)).astype(np.float32)
            pq = (q + rng.normal(0, 0.02, 4)).astype(np.float32)
            pq = (pq / np.linalg.norm(pq.astype(np.float64))).astype(np.float32)
        shapes.append(_shape(kind, c, h, q, pc, pq, obj=len(specs) + i, flags=0 if mode == "disabled" else 1))
        # local points in 1.4x the shape's extent (a slab for a plane)
        ext = np.where(h > 0, h, 0.3).astype(np.float64) * 1.4 + 0.05
        if kind == PLANE:
            ext = np.array([0.4, 0.08, 0.4])
        n = per_shape
        loc = rng.uniform(-1, 1, (n, 3)) * ext
        loc[0] = 0.0                                   # the centre
        vel = rng.normal(0, 0.01, (n, 3))
        k = n // 5
        vel[:k] = rng.normal(0, 0.3, (k, 3))           # long, tunnelling segments
        vel[k:k + 20] = 0.0                            # x == x_prev
        if mode == "identity":
            vel[k + 20:k + 60, 0] = 0.0                # axis-parallel segments
            vel[k + 20:k + 60, 2] = 0.0
        w = G.quat_rotate(q.astype(np.float64), loc) + c
        xs.append(w.astype(np.float32))
        xps.append((w - vel).astype(np.float32))
    shapes = np.array(shapes, G.SHAPE_DTYPE)
    state_off = np.arange(len(specs) + 1, dtype=np.uint32) * per_shape
    # cloth meshes 0..n-1 (FastGridCloth), colliders n..2n-1
    beh = np.concatenate([np.full(len(specs), 1, np.uint32), np.full(len(specs), 4, np.uint32)])
    state_off = np.concatenate([state_off, np.full(len(specs), state_off[-1], np.uint32)])
    pairs = np.stack([np.arange(len(specs)), shapes["obj"]], 1).astype(np.uint32)
    return shapes, np.concatenate(xs), np.concatenate(xps), state_off, beh, pairs


def canon_contacts(c):
    """Contacts sorted by (cloth, vertex, collider)."""
    return c[np.lexsort((c["tobj"], c["point"], c["qobj"]))]
