"""CPU tests of the oracle: definitions, brute-force equivalences, known
answers, golden vectors and structural invariants.  No GPU needed."""
import os

import numpy as np
import pytest

from helpers import canon_pairs

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("n", [0, 1, 2, 255, 256, 257, 10_000, 70_001])
def test_radix_sort_is_stable_sort(oracle, n):
    rng = np.random.default_rng(n + 7)
    k = rng.integers(0, 1 << 30, n, dtype=np.uint32)
    if n > 4:
        k[::3] = k[1]
    v = np.arange(n, dtype=np.uint32)
    rk, rv = oracle.radix_sort(k, v)
    o = np.argsort(k, kind="stable")
    assert np.array_equal(rk, k[o]) and np.array_equal(rv, v[o])


def _grid_mesh(P=30, jitter=2e-3, seed=0, fold=False):
    from ysim_b200 import generators as G
    x, f = G.grid_cloth(P, 1.0, (0.0, 0.5, 0.0))
    rng = np.random.default_rng(seed)
    x = (x + rng.uniform(-jitter, jitter, x.shape)).astype(np.float32)
    if fold:  # fold the sheet over itself so self rows appear away from the 1-ring
        z = x[:, 2]
        over = z > 0.1
        x[over, 2] = (0.2 - z[over]).astype(np.float32)
        x[over, 1] = (x[over, 1] + 0.004).astype(np.float32)
    return x, f


@pytest.mark.parametrize("case", ["flat", "fold", "big_move", "nan_prev"])
def test_self_hash_equals_brute_force(oracle, case):
    x, f = _grid_mesh(fold=case == "fold", seed=1)
    rng = np.random.default_rng(2)
    xp = (x + rng.normal(0, 1e-3, x.shape)).astype(np.float32)
    if case == "big_move":
        xp[::7] = (xp[::7] + 3.0).astype(np.float32)  # > 1 m: treated as a pin snap
    if case == "nan_prev":
        xp[::11, 1] = np.nan
    m = np.float32(0.05)
    got = canon_pairs(oracle.self_hash(x, xp, f, m))
    want = canon_pairs(oracle.brute_h1(x, xp, f, m))
    assert len(want) > 0 and np.array_equal(got, want)
    # the vertex's own faces are never rows
    own = (f[got[:, 1]] == got[:, [0]]).any(1)
    assert not own.any()


@pytest.mark.parametrize("margin,self_q", [(1e-3, False), (0.02, False), (0.03, True)])
def test_tree_query_equals_brute_force(oracle, margin, self_q):
    from ysim_b200 import generators as G
    if self_q:
        x, f = _grid_mesh(P=25)
        q = x
    else:
        x, f, q = G.soup(4000, seed=3, nq=3000)
    nodes, parent, codes, idx = oracle.build_tree(x, f)
    got = canon_pairs(oracle.query_points(nodes, f, q, margin, self_q))
    want = canon_pairs(oracle.brute_q1(x, f, q, margin, self_q))
    assert np.array_equal(got, want)


def test_tree_invariants(oracle):
    from ysim_b200 import generators as G
    x, f, _ = G.soup(5000, seed=4)
    nodes, parent, codes, idx = oracle.build_tree(x, f)
    n = len(f)
    assert np.all(np.diff(codes.astype(np.int64)) >= 0)
    assert sorted(idx.tolist()) == list(range(n))
    # leaves hold every primitive once, internal children point inside the tree
    assert np.array_equal(np.sort(nodes["b"][n - 1:]), np.arange(n))
    assert np.all(nodes["a"][n - 1:] == -1)
    inner = nodes[: n - 1]
    assert np.all((inner["a"] >= 0) & (inner["a"] < 2 * n - 1) & (inner["b"] >= 0) & (inner["b"] < 2 * n - 1))
    # every non-root node has exactly one parent, and parents contain children
    kids = np.concatenate([inner["a"], inner["b"]])
    assert np.array_equal(np.sort(kids), np.arange(1, 2 * n - 1))
    for c in range(1, 2 * n - 1):
        p = parent[c]
        assert np.all(nodes["mn"][p] <= nodes["mn"][c]) and np.all(nodes["mx"][p] >= nodes["mx"][c])


def test_single_triangle_tree(oracle):
    """N = 1: the root is the leaf (bvh.hpp:1527 block D-029 fix)."""
    from ysim_b200 import generators as G
    x, f, q = G.soup(1, seed=5, nq=10)
    nodes, parent, codes, idx = oracle.build_tree(x, f)
    assert len(nodes) == 1 and nodes["a"][0] == -1 and nodes["b"][0] == 0
    assert np.allclose(nodes["mn"][0], x.min(0), atol=1e-5) and np.allclose(nodes["mx"][0], x.max(0), atol=1e-5)
    hit = oracle.query_points(nodes, f, x.mean(0, keepdims=True).astype(np.float32), 1e-3, False)
    assert len(hit) == 1


def test_adjacency_invariants(oracle):
    from ysim_b200 import generators as G
    P = 17
    x, f = G.grid_cloth(P, 1.0)
    a = oracle.adjacency(x, f)
    E = len(a["edges"]) // 2
    assert E == 3 * (P - 1) ** 2 + 2 * (P - 1)
    e = a["edges"].reshape(-1, 2)
    assert np.all(e[:, 0] < e[:, 1])
    assert np.all(np.diff(e[:, 0].astype(np.int64) * (P * P) + e[:, 1]) > 0)  # sorted unique
    # interior edges (two faces) give one opposite pair each, symmetric
    n_int = E - 4 * (P - 1)
    assert len(a["opp"]) == 2 * n_int
    pairs = set()
    for v in range(P * P):
        for k in range(a["opp_off"][v], a["opp_off"][v + 1]):
            pairs.add((v, int(a["opp"][k])))
    assert all((b, c) in pairs for (c, b) in pairs)
    # rest lengths are the float32 norms of the edges
    d = x[e[:, 1]] - x[e[:, 0]]
    ref = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2], dtype=np.float32)
    assert np.array_equal(a["rest_edge"], ref)
    # every vertex lists the faces that contain it
    for v in (0, P + 1, P * P - 1):
        fv = a["vaf"][a["vaf_off"][v]:a["vaf_off"][v + 1]]
        assert set(fv.tolist()) == set(np.nonzero((f == v).any(1))[0].tolist())


def _narrow(oracle, qcur, qprev, tri, band):
    n = np.zeros(3, np.float32)
    d = np.zeros(1, np.float32)
    arr = [np.asarray(a, np.float32) for a in (qcur, qprev, *tri)]
    hit = oracle.lib().yso_narrow_one(*[oracle.P(a) for a in arr], np.float32(band), oracle.P(n), oracle.P(d))
    return hit, n, float(d[0])


def test_narrow_known_answers(oracle):
    tri = [(0, 0, 0), (1, 0, 0), (0, 0, 1)]
    band = 0.027
    # resting just above the plane inside the triangle: contact, normal +y
    hit, n, d = _narrow(oracle, (0.2, 0.01, 0.2), (0.2, 0.011, 0.2), tri, band)
    assert hit and np.allclose(n, (0, 1, 0)) and abs(d - 0.01) < 1e-7
    # far above: no contact
    hit, _, _ = _narrow(oracle, (0.2, 0.5, 0.2), (0.2, 0.5, 0.2), tri, band)
    assert not hit
    # tunnelled from above to below: contact, normal towards xPrev, d < 0
    hit, n, d = _narrow(oracle, (0.2, -0.05, 0.2), (0.2, 0.05, 0.2), tri, band)
    assert hit and np.allclose(n, (0, 1, 0)) and d < 0
    # outside the triangle: no contact
    hit, _, _ = _narrow(oracle, (0.9, 0.01, 0.9), (0.9, 0.01, 0.9), tri, band)
    assert not hit
    # degenerate triangle: no contact
    hit, _, _ = _narrow(oracle, (0.2, 0.01, 0.2), (0.2, 0.01, 0.2), [(0, 0, 0), (1, 0, 0), (2, 0, 0)], band)
    assert not hit
    # approached from below: normal flips to -y
    hit, n, d = _narrow(oracle, (0.2, -0.01, 0.2), (0.2, -0.011, 0.2), tri, band)
    assert hit and np.allclose(n, (0, -1, 0)) and abs(d - 0.01) < 1e-7


def test_point_tri_sq_matches_float64(oracle):
    rng = np.random.default_rng(8)
    for _ in range(300):
        a, b, c, p = (rng.normal(0, 1, 3).astype(np.float32) for _ in range(4))
        got = oracle.lib().yso_point_tri_sq(*[oracle.P(np.ascontiguousarray(t)) for t in (p, a, b, c)])
        # float64 brute force: minimise over a fine barycentric grid + edges
        best = np.inf
        A, B, C, Pp = (t.astype(np.float64) for t in (a, b, c, p))
        for u in np.linspace(0, 1, 81):
            for v in np.linspace(0, 1 - u, max(2, int(81 * (1 - u)))):
                q = A + u * (B - A) + v * (C - A)
                best = min(best, float(((Pp - q) ** 2).sum()))
        assert got <= best * (1 + 1e-4) + 1e-6


# ---------------------------------------------------------------- golden
def test_oracle_matches_golden_morton_tree(oracle):
    g = np.load(os.path.join(GOLD, "morton_tree.npz"))
    for name in ("soup", "grid"):
        x, f, q, v = g[f"{name}_x"], g[f"{name}_f"], g[f"{name}_q"], g[f"{name}_v"]
        nodes, parent, codes, idx = oracle.build_tree(x, f)
        assert np.array_equal(codes, g[f"{name}_codes"]) and np.array_equal(idx, g[f"{name}_idx"])
        assert np.array_equal(nodes["a"], g[f"{name}_a"]) and np.array_equal(nodes["b"], g[f"{name}_b"])
        assert np.array_equal(parent[1:], g[f"{name}_parent"][1:])
        assert np.array_equal(nodes["mn"], g[f"{name}_mn"]) and np.array_equal(nodes["mx"], g[f"{name}_mx"])
        sw = oracle.refit(nodes, x, v, f, np.float32(1.0 / 1200.0), True)
        assert np.array_equal(sw["mn"], g[f"{name}_swept_mn"]) and np.array_equal(sw["mx"], g[f"{name}_swept_mx"])
        pairs = canon_pairs(oracle.query_points(sw, f, q, float(g[f"{name}_margin"]), bool(g[f"{name}_self"])))
        assert np.array_equal(pairs, g[f"{name}_pairs"]) and len(pairs) > 0
        an, ap, _, _ = oracle.build_tree(x, f, builder=1)
        assert np.array_equal(an["a"], g[f"{name}_agg_a"]) and np.array_equal(an["b"], g[f"{name}_agg_b"])
        assert np.array_equal(ap, g[f"{name}_agg_parent"])
        assert np.array_equal(an["mn"], g[f"{name}_agg_mn"]) and np.array_equal(an["mx"], g[f"{name}_agg_mx"])


@pytest.mark.parametrize("name", ["c1", "c2hash"])
def test_oracle_matches_golden_substep(oracle, name):
    from ysim_b200 import generators as G
    spec = {"c1": lambda: G.config_c1(P=24, level=2, height=0.2999),
            "c2hash": lambda: G.config_c2(P=32, level=3, height=0.315, gravity=-9.81)}[name]()
    g = np.load(os.path.join(GOLD, f"substep_{name}.npz"))
    o = oracle.OracleScene(spec)
    o.set("x", g["x"]); o.set("v", g["v"]); o.set("xprev", g["xprev"])
    o.stage(0)  # frame 0: rebuild from the golden state
    o.stage(1); o.stage(2)
    rows = o.rows()
    t = np.stack([rows["qobj"], rows["point"], rows["tobj"], rows["tri"]], 1).astype(np.uint32)
    t = t[np.lexsort((t[:, 3], t[:, 2], t[:, 1], t[:, 0]))]
    assert np.array_equal(t, g["rows"])
    o.stage(3)
    off, c = o.contacts()
    assert np.array_equal(off, g["csr_off"])
    assert np.array_equal(c["tri"], g["c_tri"]) and np.array_equal(c["tobj"], g["c_tobj"])
    assert np.array_equal(c["n"].view(np.uint32), g["c_n"].view(np.uint32))
    assert np.array_equal(c["d"].view(np.uint32), g["c_d"].view(np.uint32))
    o.stage(4); o.stage(5)
    n0 = spec.meshes[0].nV
    assert np.array_equal(o.get("f")[:n0].view(np.uint32), g["f"].view(np.uint32))
    assert np.array_equal(o.get("x")[:n0].view(np.uint32), g["x_next"].view(np.uint32))
    assert np.array_equal(o.get("v")[:n0].view(np.uint32), g["v_next"].view(np.uint32))
    if name == "c2hash":
        assert len(c) > 0


def test_oracle_matches_golden_analytic(oracle):
    """The oracle's analytic narrow phase reproduces the reference kernel's
    contacts (tests/golden/analytic.npz) bit for bit."""
    from analytic_cases import canon_contacts
    g = np.load(os.path.join(GOLD, "analytic.npz"))
    shapes = g["shapes"].view(oracle.SHAPE_DTYPE)
    ref = g["contacts"].view(oracle.CONTACT_DTYPE)
    for k in range(len(shapes)):
        assert np.float32(oracle.rot_margin(shapes[k], g["radius"], g["thickness"])) == g["rot_margin"][k]
    oc, n = oracle.narrow_analytic(g["x"], g["xprev"], g["state_off"], g["beh"], shapes, g["pairs"], g["radius"],
                                   g["thickness"])
    assert n == len(ref) > 1000
    assert np.array_equal(canon_contacts(oc).view(np.uint8), ref.view(np.uint8))


def test_analytic_margins_and_broad_box(oracle):
    """Rotation margins follow theta = 2 acos|q . q_prev| (bruteforce.hpp:201-240,
    bvh.hpp:2465-2479); the broad box of every shape holds the shape at both
    poses, padded by the inflate band; a half-space has no finite box."""
    from analytic_cases import cases
    from ysim_b200 import generators as G
    shapes, *_ = cases(seed=5, per_shape=10)
    rad, th, inflate = np.float32(0.012), np.float32(0.015), np.float32(0.027)
    rng = np.random.default_rng(0)
    for s in shapes:
        dq = min(abs(float(np.dot(s["rq"].astype(np.float64), s["prq"].astype(np.float64)))), 1.0)
        theta = 2.0 * np.arccos(dq)
        m = oracle.rot_margin(s, rad, th)
        kind = int(s["kind"])
        if theta <= 1e-9 or kind == 4:
            assert m == 0.0
        else:
            he = s["he"].astype(np.float64)
            rmax = {1: he[:3].max(), 2: np.sqrt((he[:3] ** 2).sum()),
                    3: np.sqrt(float(s["cr"][3]) ** 2 + he[3] ** 2)}[kind]
            assert m == np.float32(theta * (rmax + float(rad) + float(th)))
        finite, box = oracle.broad_box(s, inflate)
        assert finite == (kind != 4)
        if not finite:
            continue
        # sample the shape's surface at both poses
        u = rng.normal(size=(2000, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        if kind == 1:
            loc = u * s["he"][:3]
        elif kind == 2:
            loc = np.sign(u) * s["he"][:3] * rng.uniform(0, 1, (2000, 3)) ** 0.01
        else:
            r, hh = float(s["cr"][3]), float(s["he"][3])
            ang = rng.uniform(0, 2 * np.pi, 2000)
            loc = np.stack([r * np.cos(ang), rng.uniform(-hh, hh, 2000), r * np.sin(ang)], 1)
        for c, q in ((s["cr"][:3], s["rq"]), (s["pc"][:3], s["prq"])):
            w = G.quat_rotate(q.astype(np.float64), loc) + c
            assert (w >= box[:3] + inflate - 1e-5).all() and (w <= box[3:] - inflate + 1e-5).all()


def test_analytic_scene_markers_and_roll(oracle):
    """Scene-level analytic path on the oracle: the pack seeds prev = cur, a
    moved collider rolls its old pose into prev at the next frame, a cloth
    under a half-space gets one contact per vertex within the band, and an
    analytic collider emits no triangle rows."""
    from ysim_b200 import generators as G
    spec = G.config_c1(P=12, level=1, height=0.2)
    cloth = spec.meshes[0]
    plane = G.analytic_collider(4, (0.0, 0.19, 0.0))
    sph = G.analytic_collider(1, (2.0, 0.0, 0.0), (0.1, 0.1, 0.1))
    spec = G.SceneSpec("plane", spec.params, [cloth, plane, sph], 0)
    o = oracle.OracleScene(spec)
    sh = o.shapes()
    assert len(sh) == 2 and list(sh["obj"]) == [1, 2]
    assert np.array_equal(sh["pc"][:, :3], sh["cr"][:, :3]) and np.array_equal(sh["prq"], sh["rq"])
    o.step(1)
    assert o.stats()["broad_rows"] == 0
    off, c = o.contacts()
    assert len(c) == cloth.nV and (c["tobj"] == 1).all() and (c["tri"] == 0).all()
    assert np.allclose(c["n"], [0.0, 1.0, 0.0])
    o.set_collider(2, 1, (2.0, 0.05, 0.0), (0.1, 0.1, 0.1), G.quat_axis_angle((0, 1, 0), 0.1))
    o.step(spec.params.substeps)  # through the next frame start
    sh = o.shapes()
    assert np.allclose(sh["pc"][1, :3], [2.0, 0.0, 0.0]) and np.allclose(sh["cr"][1, :3], [2.0, 0.05, 0.0])
    assert sh["prq"][1, 0] == 1.0 and sh["rq"][1, 0] < 1.0
    assert oracle.rot_margin(sh[1], 0.012, 0.015) > 0.0
    o.step(spec.params.substeps)  # unchanged pose: prev catches up
    sh = o.shapes()
    assert np.array_equal(sh["pc"][1, :3], sh["cr"][1, :3]) and np.array_equal(sh["prq"][1], sh["rq"][1])


# ---------------------------------------------------------------- host logic
def test_generator_sizes_and_determinism():
    from ysim_b200 import generators as G
    v, f = G.icosphere(7)
    assert len(v) == 163_842 and len(f) == 327_680
    v, f = G.icosphere(4)
    assert len(v) == 2_562 and len(f) == 5_120
    x, f = G.grid_cloth(512, 1.0)
    assert len(x) == 262_144 and len(f) == 522_242
    a = G.config_c2(P=16, level=2)
    b = G.config_c2(P=16, level=2)
    assert all(np.array_equal(m.x, n.x) for m, n in zip(a.meshes, b.meshes))
    c1 = G.config_c1()
    assert c1.meshes[0].nV == 4096 and c1.meshes[0].nF == 7938 and c1.meshes[1].nF == 5120


def test_c_abi_exports_every_declared_symbol():
    """The library loads on a CPU-only machine and exports every function
    include/ysim_b200.h declares (no compute call is made)."""
    import ctypes
    import re
    from ysim_b200 import _lib, build
    path = build.build()
    hdr = open(os.path.join(os.path.dirname(GOLD), "..", "include", "ysim_b200.h")).read()
    names = set(re.findall(r"^\s*(?:const char\*|ys_status|size_t|void)\s+(ys_[a-z0-9_]+)\s*\(", hdr, re.M))
    assert len(names) > 30
    lib = ctypes.CDLL(path)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert names <= set(_lib.EXPORTED) | {"ys_last_error", "ys_version"}, sorted(names - set(_lib.EXPORTED))
    assert lib.ys_version


def test_scene_uploads_are_ordered_on_the_scene_stream():
    """A scene runs on a non-blocking stream, which does not wait for work on
    the legacy default stream: a plain cudaMemset, or a cudaMemcpy from
    pageable host memory (which may return before its DMA lands), could
    still be in flight when the scene's kernels read the buffer.  Every
    upload and clear in the scene code therefore goes on the scene's stream
    (read-backs after a stream synchronisation may stay synchronous)."""
    import re
    src = open(os.path.join(os.path.dirname(GOLD), "..", "ysim_b200", "csrc", "ys_scene.cu")).read()
    assert not re.search(r"cudaMemset\(", src)
    assert not re.search(r"cudaMemcpy\([^;]*cudaMemcpyHostToDevice\)", src)
