"""Seeded synthetic inputs for the cloth hot path (numpy, float32 / uint32).

Shapes follow the reference generators where they exist:
  * grid cloth -- MeshGridInitializer (initializers.hpp:41-120): row-major
    P x P grid, alternating diagonal per (row+col)&1, XZ plane, centred;
  * FastGridCloth rest lengths -- recomputeFastGridRest (collision_pod.hpp:415-438).
The icosphere, its gradient-noise displacement, the triangle soup of the
collision microbenchmark and the batched instance sampler are new generators
(the reference has only UV spheres, primitive_geometry.hpp:50).  Every random
draw comes from numpy.random.Generator(PCG64(seed)).
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional

import numpy as np

F32 = np.float32


@dataclasses.dataclass
class Mesh:
    behavior: int
    flags: int
    x: np.ndarray            # (V, 3) float32
    facets: np.ndarray       # (M, 3) uint32
    v: Optional[np.ndarray] = None
    mass: Optional[np.ndarray] = None
    mask: Optional[np.ndarray] = None
    kstretch: float = 0.0
    kshear: float = 0.0
    kbend: float = 0.0
    thickness: float = 0.0
    grid_n: int = 0
    grid_rest: tuple = (0.0,) * 6
    group: int = 0
    # analytic collider: (kind, centre (3), local half extents (3), orientation
    # (w, x, y, z)) or None for a triangle collider
    collider: Optional[tuple] = None

    @property
    def nV(self) -> int:
        return int(self.x.shape[0])

    @property
    def nF(self) -> int:
        return int(self.facets.shape[0])


@dataclasses.dataclass
class Params:
    subh: float
    substeps: int
    kair: float = -0.001        # symplectic_system.hpp:196
    kd: float = 0.5             # symplectic_system.hpp:197
    gravity: tuple = (0.0, -9.81, 0.0)
    margin: float = 0.015       # simulator.hpp:180
    radius: float = 0.012       # simulator.hpp:181
    rebuild_frames: int = 10    # simulator.hpp:3253
    self_mode: int = 0
    cols_per_point: int = 15    # scene.hpp:1139


@dataclasses.dataclass
class SceneSpec:
    name: str
    params: Params
    meshes: List[Mesh]
    seed: int = 0

    @property
    def nV(self) -> int:
        return sum(m.nV for m in self.meshes)


# ---------------------------------------------------------------- grid cloth
def grid_cloth(P: int, size: float, center=(0.0, 0.0, 0.0)):
    """Positions and facets of MeshGridInitializer in the XZ plane (no jiggle)."""
    half = F32(size / 2.0)
    length = F32(F32(size) / F32(P - 1))
    rows, cols = np.meshgrid(np.arange(P), np.arange(P), indexing="ij")
    px = (cols.astype(F32) * length - half).astype(F32)
    py = (-(rows.astype(F32)) * length + half).astype(F32)
    c = np.asarray(center, dtype=F32)
    x = np.empty((P * P, 3), F32)
    x[:, 0] = (px.ravel() + c[0]).astype(F32)
    x[:, 1] = c[1]
    x[:, 2] = (-py.ravel() + c[2]).astype(F32)
    r, q = np.meshgrid(np.arange(P - 1), np.arange(P - 1), indexing="ij")
    r = r.ravel()
    q = q.ravel()
    p00 = r * P + q
    p10 = r * P + q + 1
    p01 = (r + 1) * P + q
    p11 = (r + 1) * P + q + 1
    even = ((r + q) & 1) == 0
    f = np.empty((2 * len(r), 3), np.int64)
    a = np.where(even[:, None], np.stack([p00, p01, p11], 1), np.stack([p00, p01, p10], 1))
    b = np.where(even[:, None], np.stack([p00, p11, p10], 1), np.stack([p10, p01, p11], 1))
    f[0::2] = a
    f[1::2] = b
    return x, f.astype(np.uint32)


def fast_grid_rest(x: np.ndarray, P: int):
    """recomputeFastGridRest (collision_pod.hpp:415-438): 6 directional rests."""
    def dist(a, b):
        d = (x[a] - x[b]).astype(F32)
        return float(np.sqrt(F32(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), dtype=F32))
    return (dist(0, 1), dist(0, P), dist(0, P + 1), dist(1, P), dist(0, 2), dist(0, 2 * P))


# ---------------------------------------------------------------- icosphere
def icosphere(level: int):
    """Unit icosphere: icosahedron subdivided `level` times (edge midpoints
    projected to the sphere).  level L: 10*4^L + 2 vertices, 20*4^L faces."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
                  [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
                  [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    for _ in range(level):
        nv = len(v)
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]], 0)
        key = np.minimum(e[:, 0], e[:, 1]) * nv + np.maximum(e[:, 0], e[:, 1])
        uk, inv = np.unique(key, return_inverse=True)
        a, b = uk // nv, uk % nv
        mid = (v[a] + v[b]) * 0.5
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        m = inv.reshape(3, -1).T + nv          # midpoints of (01, 12, 20)
        v = np.concatenate([v, mid], 0)
        f = np.concatenate([
            np.stack([f[:, 0], m[:, 0], m[:, 2]], 1),
            np.stack([f[:, 1], m[:, 1], m[:, 0]], 1),
            np.stack([f[:, 2], m[:, 2], m[:, 1]], 1),
            np.stack([m[:, 0], m[:, 1], m[:, 2]], 1)], 0)
    return v, f.astype(np.uint32)


def perlin3(p: np.ndarray, seed: int) -> np.ndarray:
    """Improved gradient noise (Perlin 2002) with a seeded permutation; values
    in about [-1, 1]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    perm = rng.permutation(256)
    perm = np.concatenate([perm, perm])
    grads = np.array([[1, 1, 0], [-1, 1, 0], [1, -1, 0], [-1, -1, 0], [1, 0, 1], [-1, 0, 1], [1, 0, -1],
                      [-1, 0, -1], [0, 1, 1], [0, -1, 1], [0, 1, -1], [0, -1, -1]], dtype=np.float64)
    pi = np.floor(p).astype(np.int64)
    pf = p - pi
    pi &= 255

    def fade(t):
        return t * t * t * (t * (t * 6 - 15) + 10)

    u = fade(pf)

    def grad(ix, iy, iz, dx, dy, dz):
        h = perm[perm[perm[ix] + iy] + iz] % 12
        g = grads[h]
        return g[:, 0] * dx + g[:, 1] * dy + g[:, 2] * dz

    out = 0.0
    res = []
    for cx in (0, 1):
        for cy in (0, 1):
            for cz in (0, 1):
                res.append(grad((pi[:, 0] + cx) & 255, (pi[:, 1] + cy) & 255, (pi[:, 2] + cz) & 255,
                                pf[:, 0] - cx, pf[:, 1] - cy, pf[:, 2] - cz))
    def lerp(a, b, t):
        return a + t * (b - a)
    x00 = lerp(res[0], res[4], u[:, 0]); x01 = lerp(res[1], res[5], u[:, 0])
    x10 = lerp(res[2], res[6], u[:, 0]); x11 = lerp(res[3], res[7], u[:, 0])
    y0 = lerp(x00, x10, u[:, 1]); y1 = lerp(x01, x11, u[:, 1])
    out = lerp(y0, y1, u[:, 2])
    return out


def obstacle_sphere(level: int, radius: float, center=(0.0, 0.0, 0.0), amplitude: float = 0.0, seed: int = 0,
                    frequency: float = 4.0) -> Mesh:
    """Static icosphere obstacle (behavior Float: target-only, never integrated,
    tree built once), optionally displaced radially by amplitude * noise."""
    v, f = icosphere(level)
    r = np.full(len(v), radius, np.float64)
    if amplitude:
        r = r + amplitude * perlin3(v * frequency + 17.0, seed)
    x = (v * r[:, None] + np.asarray(center, np.float64)).astype(F32)
    from ._lib import FLOAT, MESH_COLLIDABLE, MESH_STATIC
    return Mesh(behavior=FLOAT, flags=MESH_STATIC | MESH_COLLIDABLE, x=x, facets=f,
                v=np.zeros_like(x), mass=np.zeros(len(x), F32), mask=np.ones(len(x), F32))


# ---------------------------------------------------------------- analytic colliders
# AnalyticShape record (collision_pod.hpp:295-309), the layout of
# ys_analytic_shape.
SHAPE_DTYPE = np.dtype([("cr", "<f4", 4), ("he", "<f4", 4), ("rq", "<f4", 4), ("pc", "<f4", 4), ("prq", "<f4", 4),
                        ("kind", "<u4"), ("obj", "<u4"), ("beh", "<u4"), ("flags", "<u4")])
assert SHAPE_DTYPE.itemsize == 96


def quat_axis_angle(axis, angle: float):
    """(w, x, y, z) of a rotation by angle (radians) about axis."""
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    h = 0.5 * angle
    return (float(np.cos(h)), *(float(c) for c in a * np.sin(h)))


def quat_rotate(q, v: np.ndarray) -> np.ndarray:
    """Rotate rows of v by the unit quaternion q = (w, x, y, z) (float64)."""
    w, qv = q[0], np.asarray(q[1:], np.float64)
    v = np.asarray(v, np.float64)
    t = 2.0 * np.cross(qv, v)
    return v + w * t + np.cross(qv, t)


def fit_local_half(x: np.ndarray, center, q) -> tuple:
    """Scene::fitAnalyticLocalHalf's geometry fit (scene.hpp:622-640): the
    vertices in the collider's frame (inverse rotation about the centre),
    per-axis max |coordinate| -- the smallest origin-centred box holding the
    mesh."""
    qi = (q[0], -q[1], -q[2], -q[3])
    loc = quat_rotate(qi, np.asarray(x, np.float64) - np.asarray(center, np.float64))
    return tuple(float(h) for h in np.abs(loc).max(axis=0))


def analytic_collider(kind: int, center, half=(0.0, 0.0, 0.0), q=(1.0, 0.0, 0.0, 0.0), level: int = 2) -> Mesh:
    """A static analytic collider (behavior Float, collidable) with a coarse
    triangle surface of its shape for display: an ellipsoid from an
    icosphere, a box or cylinder from a scaled icosphere, a plane from a
    2 x 2 quad.  Only the shape (kind, centre, half extents, orientation)
    takes part in the collision path."""
    from ._lib import COLLIDER_PLANE, FLOAT, MESH_COLLIDABLE, MESH_STATIC
    if kind == COLLIDER_PLANE:
        v = np.array([[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], np.float64)
        f = np.array([[0, 2, 1], [0, 3, 2]], np.uint32)
    else:
        v, f = icosphere(level)
        v = v * np.asarray(half, np.float64)
    x = (quat_rotate(q, v) + np.asarray(center, np.float64)).astype(F32)
    return Mesh(behavior=FLOAT, flags=MESH_STATIC | MESH_COLLIDABLE, x=x, facets=np.asarray(f, np.uint32),
                v=np.zeros_like(x), mass=np.zeros(len(x), F32), mask=np.ones(len(x), F32),
                collider=(int(kind), tuple(float(c) for c in center), tuple(float(h) for h in half),
                          tuple(float(c) for c in q)))


# ---------------------------------------------------------------- configs
def config_c1(seed: int = 1, P: int = 64, level: int = 4, height: float = 1.0) -> SceneSpec:
    """Plain FastGridCloth 64x64 over a static level-4 icosphere (r 0.3);
    k 1e3/5e2/1e1, m 1e-3, thickness 1e-3, 10 substeps/frame, reference
    margin/radius, jiggle U[0,1e-4] on the normal axis.  subh is 1/6000
    (h = 1/600 split in 10): the 12-spring stencil's stiffness over m = 1e-3
    puts the explicit integrator's stability limit below 1/600."""
    from ._lib import FAST_GRID_CLOTH, MESH_COLLIDABLE
    rng = np.random.Generator(np.random.PCG64(seed))
    x, f = grid_cloth(P, 1.0, (0.0, height, 0.0))
    x[:, 1] = (x[:, 1] + rng.uniform(0.0, 1e-4, P * P).astype(F32)).astype(F32)
    cloth = Mesh(behavior=FAST_GRID_CLOTH, flags=MESH_COLLIDABLE, x=x, facets=f, v=np.zeros_like(x),
                 mass=np.full(P * P, 1e-3, F32), mask=np.ones(P * P, F32), kstretch=1e3, kshear=5e2, kbend=1e1,
                 thickness=1e-3, grid_n=P, grid_rest=fast_grid_rest(x, P))
    obst = obstacle_sphere(level, 0.3)
    return SceneSpec("c1_fastgrid64_ico4", Params(subh=1.0 / 6000.0, substeps=10), [cloth, obst], seed)


def config_c1_analytic(seed: int = 1, P: int = 64, height: float = 1.0) -> SceneSpec:
    """C1's FastGridCloth falling on analytic colliders instead of a triangle
    obstacle: a sphere (r 0.3) at the origin, a box tilted 30 degrees, a
    cylinder on its side and a floor plane at y = -0.35 (the analytic
    collider path: BroadPhase markers + narrow_pt_analytic)."""
    from ._lib import COLLIDER_BOX, COLLIDER_CYLINDER, COLLIDER_PLANE, COLLIDER_SPHERE
    spec = config_c1(seed=seed, P=P, height=height)
    cloth = spec.meshes[0]
    shapes = [
        analytic_collider(COLLIDER_SPHERE, (0.0, 0.0, 0.0), (0.3, 0.3, 0.3)),
        analytic_collider(COLLIDER_BOX, (0.32, -0.1, 0.2), (0.12, 0.08, 0.1), quat_axis_angle((0, 0, 1), np.pi / 6)),
        analytic_collider(COLLIDER_CYLINDER, (-0.3, -0.15, -0.25), (0.1, 0.15, 0.1),
                          quat_axis_angle((1, 0, 0), np.pi / 2)),
        analytic_collider(COLLIDER_PLANE, (0.0, -0.35, 0.0)),
    ]
    return SceneSpec(f"c1_fastgrid{P}_analytic", spec.params, [cloth] + shapes, seed)


def config_c2(seed: int = 2, P: int = 512, level: int = 7, height: float = 0.37, self_mode: int = 1,
              obstacle: bool = True, size: float = 1.0, kstretch: float = 1e3, kbend: float = 1e1,
              gravity: float = -1.0) -> SceneSpec:
    """Plain TriangularCloth P x P (512: 262,144 v, 522,242 tris), jitter
    U(-0.1s, 0.1s) on all axes, self-collision on, over a static displaced
    level-7 icosphere (radius 0.3 size, radial noise amplitude 0.05 size);
    subh 1/1200, 20 substeps/frame.  Margin, radius and contact thickness are
    the reference defaults (0.015, 0.012) and C1's thickness (1e-3) scaled by
    the grid-spacing ratio so the contact band stays about one edge length, as
    in the reference's 64-grid scenes.  `size` scales the whole scene.
    Gravity is 1 m/s^2: at this resolution and step the explicit integrator's
    stability bound (k/m below about 0.67/subh^2) leaves a 1 m sheet under
    9.81 m/s^2 stretched by several hundred percent under its own weight; it
    then crumples through itself and the reference's self-contact push blows
    it up (measured: every stiffness / damping variant at 9.81 diverges within
    about 10 frames of contact)."""
    from ._lib import MESH_COLLIDABLE, MESH_SELF_COLLIDE, TRIANGULAR_CLOTH
    rng = np.random.Generator(np.random.PCG64(seed))
    s = size / (P - 1)
    x, f = grid_cloth(P, size, (0.0, height * size, 0.0))
    x = (x + rng.uniform(-0.1 * s, 0.1 * s, x.shape).astype(F32)).astype(F32)
    scale = s / (1.0 / 63.0)
    cloth = Mesh(behavior=TRIANGULAR_CLOTH, flags=MESH_COLLIDABLE | MESH_SELF_COLLIDE, x=x, facets=f,
                 v=np.zeros_like(x), mass=np.full(P * P, 1e-2, F32), mask=np.ones(P * P, F32), kstretch=kstretch,
                 kshear=5e2, kbend=kbend, thickness=1e-3 * scale)
    prm = Params(subh=1.0 / 1200.0, substeps=20, margin=0.015 * scale, radius=0.012 * scale, self_mode=self_mode,
                 gravity=(0.0, gravity, 0.0))
    meshes = [cloth]
    if obstacle:
        meshes.append(obstacle_sphere(level, 0.3 * size, amplitude=0.05 * size, seed=seed + 1000))
    return SceneSpec(f"c2_tricloth{P}_ico{level}", prm, meshes, seed)


def soup(n: int, seed: int = 3, nq: Optional[int] = None):
    """Collision microbenchmark soup: centroids U[0,1]^3, per-triangle vertex
    offsets N(0, sigma^2 I) with sigma = exp(N(ln 1e-3, 0.5^2)); nq query
    points U[0,1]^3."""
    rng = np.random.Generator(np.random.PCG64(seed))
    c = rng.uniform(0.0, 1.0, (n, 3))
    sig = np.exp(rng.normal(np.log(1e-3), 0.5, n))
    x = (c[:, None, :] + rng.normal(0.0, 1.0, (n, 3, 3)) * sig[:, None, None]).reshape(-1, 3).astype(F32)
    f = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    q = rng.uniform(0.0, 1.0, (nq if nq is not None else n, 3)).astype(F32)
    return x, f, q


def config_c4(seed: int = 4, instances: int = 256, lo: int = 16, hi: int = 256, level: int = 4,
              drop: float = 0.1) -> SceneSpec:
    """Batched: independent FastGridCloth instances (side U{lo..hi}) each over
    its own level-4 icosphere (random offset, r in [0.2, 0.5]); instances sit
    3 m apart and only collide within their own group; each cloth starts
    `drop` above its obstacle's top.  Cloth physics and step are C1's
    (k 1e3/5e2/1e1, m 1e-3, subh 1/6000, 10 substeps/frame)."""
    from ._lib import FAST_GRID_CLOTH, MESH_COLLIDABLE
    rng = np.random.Generator(np.random.PCG64(seed))
    meshes = []
    cols = int(np.ceil(np.sqrt(instances)))
    for i in range(instances):
        P = int(rng.integers(lo, hi + 1))
        r = float(rng.uniform(0.2, 0.5))
        off = rng.uniform(-0.2, 0.2, 3)
        base = np.array([3.0 * (i % cols), 0.0, 3.0 * (i // cols)])
        x, f = grid_cloth(P, 1.0, tuple(base + np.array([0.0, r + drop, 0.0])))
        x[:, 1] = (x[:, 1] + rng.uniform(0.0, 1e-4, P * P).astype(F32)).astype(F32)
        cloth = Mesh(behavior=FAST_GRID_CLOTH, flags=MESH_COLLIDABLE, x=x, facets=f, v=np.zeros_like(x),
                     mass=np.full(P * P, 1e-3, F32), mask=np.ones(P * P, F32), kstretch=1e3, kshear=5e2, kbend=1e1,
                     thickness=1e-3, grid_n=P, grid_rest=fast_grid_rest(x, P), group=i)
        ob = obstacle_sphere(level, r, center=tuple(base + off * np.array([1.0, 0.0, 1.0])))
        ob.group = i
        meshes += [cloth, ob]
    return SceneSpec(f"c4_batched{instances}", Params(subh=1.0 / 6000.0, substeps=10), meshes, seed)


def split_instances(spec: SceneSpec) -> List[SceneSpec]:
    """The plain per-instance form of a batched scene: one scene per group
    (its cloth and its obstacle), same parameters, group ids reset to 0."""
    groups = {}
    for m in spec.meshes:
        groups.setdefault(m.group, []).append(dataclasses.replace(m, group=0))
    return [SceneSpec(f"{spec.name}_inst{g}", spec.params, ms, spec.seed) for g, ms in sorted(groups.items())]


def shard_instances(spec: SceneSpec, rank: int, world: int) -> SceneSpec:
    """The instances (groups) of a batched scene that rank `rank` of `world`
    runs: largest first, each to the rank with the fewest vertices so far
    (ties to the lower rank), so every rank gets a similar vertex count
    whatever the mix of sizes.  Groups keep their ids; meshes keep their
    order."""
    sizes = {}
    for m in spec.meshes:
        sizes[m.group] = sizes.get(m.group, 0) + m.nV
    load = [0] * world
    owner = {}
    for g in sorted(sizes, key=lambda g: (-sizes[g], g)):
        r = min(range(world), key=lambda k: (load[k], k))
        owner[g] = r
        load[r] += sizes[g]
    mine = [m for m in spec.meshes if owner[m.group] == rank]
    return SceneSpec(f"{spec.name}_shard{rank}of{world}", spec.params, mine, spec.seed)


# ---------------------------------------------------------------- adjoint
def grid_spring_params(N: int, rest6, k3):
    """Per-spring stiffness and rest length of a FastGridCloth in the canonical
    spring order: stretch-x (r,c)-(r,c+1), stretch-y (r,c)-(r+1,c), shear "\\\\"
    (r,c)-(r+1,c+1), shear "/" (r,c+1)-(r+1,c), bend-x (r,c)-(r,c+2), bend-y
    (r,c)-(r+2,c), each row-major.  Uniform values reproduce
    FastGridClothBehaviorParams exactly."""
    fam = [(N * (N - 1), rest6[0], k3[0]), ((N - 1) * N, rest6[1], k3[0]), ((N - 1) ** 2, rest6[2], k3[1]),
           ((N - 1) ** 2, rest6[3], k3[1]), (N * (N - 2), rest6[4], k3[2]), ((N - 2) * N, rest6[5], k3[2])]
    k = np.concatenate([np.full(n, kk, F32) for n, _, kk in fam])
    L = np.concatenate([np.full(n, rr, F32) for n, rr, _ in fam])
    return k, L


def config_c5(seed: int = 5, N: int = 128, level: int = 4, height: float = 0.33) -> SceneSpec:
    """Differentiable rollout: FastGridCloth N x N (size 1) above a static
    level-4 icosphere (r 0.3); subh 1/600, one substep per step; m 1e-2,
    k 1e3/5e2/1e1 (stable at this step), thickness 1e-3."""
    from ._lib import FAST_GRID_CLOTH, MESH_COLLIDABLE
    rng = np.random.Generator(np.random.PCG64(seed))
    x, f = grid_cloth(N, 1.0, (0.0, height, 0.0))
    x[:, 1] = (x[:, 1] + rng.uniform(0.0, 1e-4, N * N).astype(F32)).astype(F32)
    cloth = Mesh(behavior=FAST_GRID_CLOTH, flags=MESH_COLLIDABLE, x=x, facets=f, v=np.zeros_like(x),
                 mass=np.full(N * N, 1e-2, F32), mask=np.ones(N * N, F32), kstretch=1e3, kshear=5e2, kbend=1e1,
                 thickness=1e-3, grid_n=N, grid_rest=fast_grid_rest(x, N))
    obst = obstacle_sphere(level, 0.3)
    return SceneSpec(f"c5_adjoint{N}", Params(subh=1.0 / 600.0, substeps=1, rebuild_frames=10), [cloth, obst], seed)
