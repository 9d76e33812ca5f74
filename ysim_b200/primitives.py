"""Triangle meshes of the reference's scene sources, float32 operation for operation.

* sphere / cube / cylinder: primitive::sphere, cube (welded), cylinder
  (include/primitive_geometry.hpp:73-413).  The float trigonometry is the C
  library's sinf / cosf, which the reference's std::sin / std::cos of a
  float call.
* grid: MeshGridInitializer::initialize (include/sim/initializers.hpp:41-120)
  and the pack-time cloth jiggle (applyClothJiggle, initializers.hpp:209-222).
  The jiggle draws std::uniform_real_distribution<float>(0, 1e-4) from
  std::mt19937 as libstdc++ computes them (one 32-bit draw per value, u / 2^32
  in float).  A build against another standard library may draw other
  values; the jiggle is below 1e-4 either way.
* obj: ObjData::loadObject (include/objreader.hpp:116-285): v, f (triangles
  and quads, v, v/t, v//n, v/t/n), other records skipped.  A negative index
  k resolves as the reference resolves it, k - 1 + (vertices so far), one
  below the Wavefront convention (-1 = the last vertex); an index that lands
  outside the mesh is an error.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math
import re
from typing import List, Tuple

import numpy as np

F32 = np.float32

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.sinf.restype = ctypes.c_float
_libm.sinf.argtypes = [ctypes.c_float]
_libm.cosf.restype = ctypes.c_float
_libm.cosf.argtypes = [ctypes.c_float]


def _sinf(x) -> np.float32:
    return F32(_libm.sinf(float(x)))


def _cosf(x) -> np.float32:
    return F32(_libm.cosf(float(x)))


_PI = F32(3.14159265358979323846)


def _offset(pos: List[Tuple], center) -> np.ndarray:
    c = [F32(v) for v in center]
    return np.array([[F32(p[0]) + c[0], F32(p[1]) + c[1], F32(p[2]) + c[2]] for p in pos], F32).reshape(-1, 3)


# ---------------------------------------------------------------- sphere
def sphere(size: float, tessellation: int, center=(0.0, 0.0, 0.0)):
    """UV sphere of diameter `size`: a pole, tess - 1 rings of tess vertices, a pole."""
    t = max(int(tessellation), 3)
    r = F32(size) * F32(0.5)
    pos = [(F32(0), r, F32(0))]
    for i in range(1, t):
        theta = (_PI * F32(i)) / F32(t)
        sy = _cosf(theta) * r
        sr = _sinf(theta) * r
        for j in range(t):
            phi = ((F32(2) * _PI) * F32(j)) / F32(t)
            pos.append((sr * _cosf(phi), sy, sr * _sinf(phi)))
    pos.append((F32(0), -r, F32(0)))
    south = (t - 1) * t + 1

    def inner(i, j):
        return 1 + (i - 1) * t + (j % t)

    fac = [(0, inner(1, j), inner(1, j + 1)) for j in range(t)]
    for i in range(1, t - 1):
        for j in range(t):
            a, b, c, d = inner(i, j), inner(i, j + 1), inner(i + 1, j), inner(i + 1, j + 1)
            fac += [(a, c, d), (a, d, b)]
    fac += [(south, inner(t - 1, j + 1), inner(t - 1, j)) for j in range(t)]
    return _offset(pos, center), np.array(fac, np.uint32)


# ---------------------------------------------------------------- cube
def _llround(x: float) -> int:
    """llround: nearest integer, halves away from zero."""
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


def cube(size: float, tessellation: int, center=(0.0, 0.0, 0.0)):
    """Cube of edge `size`, t x t cells per face, coincident seam vertices
    welded (first occurrence keeps its slot)."""
    t = max(int(tessellation), 1)
    s = F32(size)
    h = s * F32(0.5)
    z = F32(0)
    faces = [((h, -h, -h), (z, s, z), (z, z, s)), ((-h, -h, h), (z, s, z), (z, z, -s)),
             ((-h, h, h), (s, z, z), (z, z, -s)), ((-h, -h, -h), (s, z, z), (z, z, s)),
             ((-h, -h, h), (s, z, z), (z, s, z)), ((h, -h, -h), (-s, z, z), (z, s, z))]
    c = [F32(v) for v in center]
    pos, fac = [], []
    for o, u, v in faces:
        base = len(pos)
        for i in range(t + 1):
            vi = F32(i) / F32(t)
            for j in range(t + 1):
                uj = F32(j) / F32(t)
                pos.append(tuple(((o[k] + uj * u[k]) + vi * v[k]) + c[k] for k in range(3)))
        for i in range(t):
            for j in range(t):
                p00 = base + i * (t + 1) + j
                p10, p01 = p00 + 1, p00 + (t + 1)
                p11 = p01 + 1
                fac += [(p00, p01, p11), (p00, p11, p10)]
    q = F32(1.0) / (s * F32(1e-5) if s > 0 else F32(1e-5))
    qd = float(q)
    seen, out, remap = {}, [], []
    for p in pos:
        key = tuple(_llround(float(x) * qd) for x in p)
        if key in seen:
            remap.append(seen[key])
        else:
            seen[key] = len(out)
            remap.append(len(out))
            out.append(p)
    fac = [(remap[a], remap[b], remap[cc]) for a, b, cc in fac]
    return np.array(out, F32).reshape(-1, 3), np.array(fac, np.uint32)


# ---------------------------------------------------------------- cylinder
def cylinder(size: float, tessellation: int, center=(0.0, 0.0, 0.0)):
    """Closed cylinder (axis +y) of diameter and height `size`: t + 1 rings
    of t vertices and two cap centres."""
    t = max(int(tessellation), 3)
    s = F32(size)
    r = s * F32(0.5)
    hh = s * F32(0.5)
    pos = []
    for i in range(t + 1):
        y = -hh + (s * F32(i)) / F32(t)
        for j in range(t):
            phi = ((F32(2) * _PI) * F32(j)) / F32(t)
            pos.append((r * _cosf(phi), y, r * _sinf(phi)))
    bottom, top = (t + 1) * t, (t + 1) * t + 1
    pos += [(F32(0), -hh, F32(0)), (F32(0), hh, F32(0))]

    def side(i, j):
        return i * t + (j % t)

    fac = []
    for i in range(t):
        for j in range(t):
            a, b, c, d = side(i, j), side(i, j + 1), side(i + 1, j), side(i + 1, j + 1)
            fac += [(a, c, d), (a, d, b)]
    fac += [(bottom, side(0, j + 1), side(0, j)) for j in range(t)]
    fac += [(top, side(t, j), side(t, j + 1)) for j in range(t)]
    return _offset(pos, center), np.array(fac, np.uint32)


# ---------------------------------------------------------------- jiggle RNG
class MT19937:
    """The 32-bit Mersenne Twister (Matsumoto & Nishimura 1998), seeded as
    std::mt19937(seed)."""

    def __init__(self, seed: int):
        mt = [seed & 0xFFFFFFFF]
        for i in range(1, 624):
            mt.append((1812433253 * (mt[-1] ^ (mt[-1] >> 30)) + i) & 0xFFFFFFFF)
        self.mt, self.i = mt, 624

    def _twist(self):
        mt = self.mt
        for k in range(624):
            y = (mt[k] & 0x80000000) | (mt[(k + 1) % 624] & 0x7FFFFFFF)
            mt[k] = mt[(k + 397) % 624] ^ (y >> 1) ^ (0x9908B0DF if y & 1 else 0)
        self.i = 0

    def next_u32(self) -> int:
        if self.i >= 624:
            self._twist()
        y = self.mt[self.i]
        self.i += 1
        y ^= y >> 11
        y ^= (y << 7) & 0x9D2C5680
        y ^= (y << 15) & 0xEFC60000
        y ^= y >> 18
        return y & 0xFFFFFFFF


_ONE_BELOW = np.nextafter(F32(1), F32(0))


def uniform_float(seed: int, lo: float, hi: float, n: int) -> np.ndarray:
    """std::uniform_real_distribution<float>(lo, hi) over std::mt19937(seed):
    u = float(draw) / 2^32 (clamped below 1), value = u * (hi - lo) + lo."""
    g = MT19937(seed)
    a, b = F32(lo), F32(hi)
    span = b - a
    scale = F32(4294967296.0)
    out = np.empty(n, F32)
    for k in range(n):
        u = F32(g.next_u32()) / scale
        if u >= F32(1):
            u = _ONE_BELOW
        out[k] = u * span + a
    return out


# ---------------------------------------------------------------- grid
PLANE_AXIS = {"XYPlane": 2, "YZPlane": 0, "XZPlane": 1}  # the plane normal


def grid(direction: str, center, n: int, size: float, jiggle: bool, seed: int):
    """n x n grid of edge `size` centred at `center` in the given plane, with
    the optional initial jiggle (U[0, 1e-4) on the plane normal, seeded by the
    object id); facets alternate their diagonal with (row + col) parity."""
    n = int(n)
    size = F32(size)
    half = F32(float(size) / 2.0)
    length = size / F32(n - 1)
    cx, cy, cz = (F32(c) for c in center)
    jig = uniform_float(seed, 0.0, 1.0 / 10000.0, n * n) if jiggle else np.zeros(n * n, F32)
    x = np.empty((n * n, 3), F32)
    for row in range(n):
        for col in range(n):
            px = F32(col) * length - half
            py = F32(-row) * length + half
            pz = jig[row * n + col]
            if direction == "XYPlane":
                x[row * n + col] = (px + cx, py + cy, pz + cz)
            elif direction == "YZPlane":
                x[row * n + col] = (pz + cx, px + cy, -py + cz)
            else:  # XZPlane (the default for an unknown name)
                x[row * n + col] = (px + cx, pz + cy, -py + cz)
    fac = []
    for row in range(n - 1):
        for col in range(n - 1):
            p00, p10 = row * n + col, row * n + col + 1
            p01, p11 = (row + 1) * n + col, (row + 1) * n + col + 1
            if ((row + col) & 1) == 0:
                fac += [(p00, p01, p11), (p00, p11, p10)]
            else:
                fac += [(p00, p01, p10), (p10, p01, p11)]
    return x, np.array(fac, np.uint32).reshape(-1, 3)


def cloth_jiggle(x: np.ndarray, direction: str, seed: int) -> np.ndarray:
    """applyClothJiggle: U[0, 1e-4) added to the plane-normal coordinate of
    every vertex (world axes, after the transform), seeded by the object id
    xor the mesh id."""
    axis = PLANE_AXIS.get(direction, 1)
    out = x.copy()
    out[:, axis] = out[:, axis] + uniform_float(seed & 0xFFFFFFFF, 0.0, 1.0 / 10000.0, len(x))
    return out


# ---------------------------------------------------------------- obj
_FACE = re.compile(r"-?\d+(/-?\d+|/)*")


def load_obj(path: str, scale: float, offset):
    """Vertices (scaled, offset) and triangles of a Wavefront .obj file."""
    verts, fac = [], []
    with open(path) as f:
        for line in f:
            parts = line.split(None, 1)
            if not parts:
                continue
            kind, rest = parts[0], (parts[1] if len(parts) > 1 else "")
            if kind == "v":
                v = rest.split()
                verts.append((F32(v[0]), F32(v[1]), F32(v[2])))
            elif kind == "f":
                elem = []
                for m in _FACE.finditer(rest):
                    idx = int(m.group(0).split("/")[0]) - 1
                    if idx < 0:
                        idx += len(verts)
                    elem.append(idx)
                bad = [e for e in elem if not 0 <= e < len(verts)]
                if bad:
                    raise ValueError(f"{path}: face index out of range ({bad[0] + 1} of {len(verts)} vertices)")
                if len(elem) == 4:
                    fac += [(elem[0], elem[1], elem[2]), (elem[0], elem[2], elem[3])]
                elif len(elem) == 3:
                    fac.append(tuple(elem))
                else:
                    raise ValueError(f"{path}: a face with {len(elem)} vertices (3 or 4 supported)")
    s = F32(scale)
    o = [F32(c) for c in offset]
    x = np.array([[v[k] * s + o[k] for k in range(3)] for v in verts], F32).reshape(-1, 3)
    return x, np.array(fac, np.uint32).reshape(-1, 3)
