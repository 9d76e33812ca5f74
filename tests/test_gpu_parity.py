"""GPU parity: every stage of the CUDA path against the CPU oracle, through the C ABI.

Bars: bit-exact for Morton codes, sorted keys/indices, LBVH topology, AABBs
and canonically sorted candidate / contact lists; positions, velocities and
forces within 1e-5 relative max-abs per substep (they come out bit-identical
because both sides round every float op once in the same order).
"""
import ctypes as C

import numpy as np
import pytest

from helpers import canon_pairs, canon_rows, reachable, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-5  # relative max-abs per substep (positions, velocities, forces)


def _dev(t_np, dtype=None):
    import torch
    t = torch.from_numpy(np.ascontiguousarray(t_np)).cuda()
    return t


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_morton_bit_exact(cuda_lib, oracle):
    from ysim_b200 import _lib, generators as G
    import torch
    for x, f in [G.soup(100_000, seed=11)[:2], G.grid_cloth(97, 1.0, (0.1, 0.4, -0.2))]:
        dx, df = _dev(x.reshape(-1)), _dev(f.reshape(-1).astype(np.int32))
        n = len(f)
        codes = torch.empty(n, dtype=torch.int32, device="cuda")
        idx = torch.empty(n, dtype=torch.int32, device="cuda")
        _lib.check(cuda_lib.ys_morton_codes(_p(dx), len(x), _p(df), n, _p(codes), _p(idx), None))
        rc, ri = oracle.morton(x, f)
        assert np.array_equal(codes.cpu().numpy().view(np.uint32), rc)
        assert np.array_equal(idx.cpu().numpy().view(np.uint32), ri)


@pytest.mark.parametrize("n", [1, 2, 3, 1000, 4096, 4097, 300_001])
def test_radix_sort_bit_exact(cuda_lib, oracle, n):
    from ysim_b200 import _lib
    import torch
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 1 << 30, n, dtype=np.uint32)
    keys[: n // 3] = keys[0]  # many duplicates: stability matters
    vals = np.arange(n, dtype=np.uint32)
    dk, dv = _dev(keys.view(np.int32)), _dev(vals.view(np.int32))
    scratch = torch.empty(int(cuda_lib.ys_radix_sort_scratch_bytes(n)) + 16, dtype=torch.uint8, device="cuda")
    _lib.check(cuda_lib.ys_radix_sort_pairs(_p(dk), _p(dv), n, _p(scratch), None))
    rk, rv = oracle.radix_sort(keys, vals)
    assert np.array_equal(dk.cpu().numpy().view(np.uint32), rk)
    assert np.array_equal(dv.cpu().numpy().view(np.uint32), rv)
    o = np.argsort(keys, kind="stable")
    assert np.array_equal(rk, keys[o]) and np.array_equal(rv, vals[o])


def _lbvh(cuda_lib, x, f, consistent=False, builder=0):
    from ysim_b200 import _lib
    h = C.c_void_p()
    _lib.check(cuda_lib.ys_lbvh_create(C.byref(h), len(f), 0, None))
    if consistent:
        _lib.check(cuda_lib.ys_lbvh_set_split(h, 1))
    if builder:
        _lib.check(cuda_lib.ys_lbvh_set_builder(h, builder))
    dx, df = _dev(x.reshape(-1)), _dev(f.reshape(-1).astype(np.int32))
    _lib.check(cuda_lib.ys_lbvh_build(h, _p(dx), len(x), _p(df), len(f)))
    return h, dx, df


class _DevView:
    """Expose a raw device allocation to torch via __cuda_array_interface__."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "version": 3}


def _d2h(ptr: int, nbytes: int, dtype) -> np.ndarray:
    import torch
    torch.cuda.synchronize()
    t = torch.as_tensor(_DevView(ptr, nbytes), device="cuda")
    return t.cpu().numpy().view(dtype)


def tree_arrays(cuda_lib, h):
    from ysim_b200 import _lib
    from ysim_b200.scene import NODE_DTYPE
    nodes, parent, codes, idx = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
    n = C.c_uint32()
    _lib.check(cuda_lib.ys_lbvh_arrays(h, C.byref(nodes), C.byref(parent), C.byref(codes), C.byref(idx), C.byref(n)))
    N = n.value
    return (_d2h(nodes.value, (2 * N - 1) * 32, NODE_DTYPE), _d2h(parent.value, (2 * N - 1) * 4, np.int32),
            _d2h(codes.value, N * 4, np.uint32), _d2h(idx.value, N * 4, np.uint32))


def _tree_equal(a_nodes, b_nodes):
    """Topology bit-exact; boxes bit-exact on every node the root reaches."""
    assert np.array_equal(a_nodes["a"], b_nodes["a"])
    assert np.array_equal(a_nodes["b"], b_nodes["b"])
    r = reachable(b_nodes)
    assert np.array_equal(a_nodes["mn"][r].view(np.uint32), b_nodes["mn"][r].view(np.uint32))
    assert np.array_equal(a_nodes["mx"][r].view(np.uint32), b_nodes["mx"][r].view(np.uint32))


@pytest.mark.parametrize("builder", [0, 1], ids=["karras", "apetrei"])
@pytest.mark.parametrize("case", ["soup", "grid", "tiny1", "tiny2", "dups"])
def test_lbvh_build_refit_query(cuda_lib, oracle, case, builder):
    """Karras (buildTree_Tri + bottomUpBoxes) or Apetrei (agglomerativeBuild_Tri
    + agglomerativeSwapRoot) build, swept refit and queries, node for node
    against the oracle."""
    from ysim_b200 import _lib, generators as G
    import torch
    if case == "soup":
        x, f, q = G.soup(50_000, seed=5)
    elif case == "grid":
        x, f = G.grid_cloth(65, 1.0, (0.0, 0.5, 0.0))
        q = x.copy()
    elif case == "tiny1":
        x, f, q = G.soup(1, seed=6, nq=50)
    elif case == "tiny2":
        x, f, q = G.soup(2, seed=7, nq=50)
    else:  # identical centroids -> identical Morton codes, index tie-breaks
        x, f, q = G.soup(3000, seed=8)
        x = np.tile(x[:3], (3000, 1)).astype(np.float32)
    h, dx, df = _lbvh(cuda_lib, x, f, builder=builder)
    try:
        nodes, parent, codes, idx = tree_arrays(cuda_lib, h)
        rn, rp, rc, ri = oracle.build_tree(x, f, builder=builder)
        assert np.array_equal(codes, rc) and np.array_equal(idx, ri)
        if builder:
            assert np.array_equal(parent, rp)
            assert reachable(rn).all()  # consistent: every node reached once
        else:
            assert np.array_equal(parent[1:], rp[1:])
        _tree_equal(nodes, rn)
        # swept refit
        rng = np.random.default_rng(1)
        v = rng.normal(0, 1.0, x.shape).astype(np.float32)
        dv = _dev(v.reshape(-1))
        _lib.check(cuda_lib.ys_lbvh_refit(h, _p(dx), _p(dv), np.float32(1.0 / 1200), 1))
        nodes2, _, _, _ = tree_arrays(cuda_lib, h)
        _tree_equal(nodes2, oracle.refit(rn, x, v, f, np.float32(1.0 / 1200), True))
        # point query, within h = 1e-3 (and the self variant)
        for margin, self_q in [(1e-3, False), (0.02, True)]:
            if self_q and case != "grid":
                continue
            dq = _dev(q.reshape(-1))
            cap = 4_000_000
            pairs = torch.empty(2 * cap, dtype=torch.int32, device="cuda")
            cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
            _lib.check(cuda_lib.ys_lbvh_query(h, _p(dq), len(q), np.float32(margin), int(self_q), _p(pairs), cap,
                                              _p(cnt)))
            n = int(cnt.item())
            assert n <= cap
            got = canon_pairs(pairs[: 2 * n].cpu().numpy().view(np.uint32))
            want = canon_pairs(oracle.query_points(oracle.refit(rn, x, v, f, np.float32(1.0 / 1200), True), f, q,
                                                   margin, self_q))
            assert np.array_equal(got, want)
    finally:
        _lib.check(cuda_lib.ys_lbvh_destroy(h))


def _small_specs():
    from ysim_b200 import generators as G
    return {
        "c1": G.config_c1(P=24, level=2, height=0.2999),
        "c2hash": G.config_c2(P=40, level=3, height=0.33, gravity=-9.81),
        "c2bvh": G.config_c2(P=40, level=3, height=0.33, self_mode=2, gravity=-9.81),
        "edge": _edge_spec(),
    }


def _edge_spec():
    """A FastGridCloth 16x16 (size 0.5) resting 5e-4 above a level-2
    icosphere (r 0.2) and an obstacle mesh built to hit the contact edge
    cases of narrow_pt_tri and integrate_cloth_grid:
      * a flat quad exactly in the cloth's plane (previous and current
        distance both 0: the orientation falls back to d_cur, the contact
        has d = 0 and pushes by the full thickness);
      * a strip 5e-4 below the pinned first row (mask 0: the push is applied
        all the same, physics.metal:291-296), one of its triangles listed
        twice (two contacts with equal n and d push twice);
      * a degenerate (collinear) triangle under the cloth (normal below
        1e-12: no contact);
    and two coincident cloth vertices (spring length below 1e-7: skipped)."""
    from ysim_b200 import _lib, generators as G
    F32 = np.float32
    P, H = 16, F32(0.2005)
    x, f = G.grid_cloth(P, 0.5, (0.0, float(H), 0.0))
    rest = G.fast_grid_rest(x, P)
    x[8 * P + 5] = x[8 * P + 4]
    mask = np.ones(P * P, F32)
    mask[:P] = 0.0
    cloth = G.Mesh(behavior=_lib.FAST_GRID_CLOTH, flags=_lib.MESH_COLLIDABLE, x=x, facets=f, v=np.zeros_like(x),
                   mass=np.full(P * P, 1e-3, F32), mask=mask, kstretch=1e3, kshear=5e2, kbend=1e1,
                   thickness=1e-3, grid_n=P, grid_rest=rest)
    sph = G.obstacle_sphere(2, 0.2)
    zrow = float(x[0, 2])
    low = F32(H - F32(5e-4))
    extra = np.array([[0.1, H, 0.1], [0.3, H, 0.1], [0.3, H, 0.3], [0.1, H, 0.3],          # in-plane quad
                      [-0.3, low, zrow - 0.01], [0.3, low, zrow - 0.01], [0.3, low, zrow + 0.01],
                      [-0.3, low, zrow + 0.01],                                              # strip under row 0
                      [0.0, H - 0.001, 0.0], [0.01, H - 0.001, 0.0], [0.02, H - 0.001, 0.0]],  # collinear
                     F32)
    b = sph.nV
    tris = np.array([[b, b + 1, b + 2], [b, b + 2, b + 3], [b + 4, b + 5, b + 6], [b + 4, b + 6, b + 7],
                     [b + 4, b + 5, b + 6], [b + 8, b + 9, b + 10]], np.uint32)
    ox = np.concatenate([sph.x, extra]).astype(F32)
    ob = G.Mesh(behavior=sph.behavior, flags=sph.flags, x=ox, facets=np.concatenate([sph.facets, tris]),
                v=np.zeros_like(ox), mass=np.zeros(len(ox), F32), mask=np.ones(len(ox), F32))
    return G.SceneSpec("edge_cases", G.Params(subh=1.0 / 6000.0, substeps=10), [cloth, ob], 0)


def _advance_to_contact(spec, frames):
    """Run the oracle a few frames so the stage checks see real contacts."""
    from oracle import oracle as O
    o = O.OracleScene(spec)
    o.step(frames * spec.params.substeps)
    return o


@pytest.mark.parametrize("layout", [0, 1], ids=["reference_tree", "cube_tree"])
@pytest.mark.parametrize("name", ["c1", "c2hash", "c2bvh"])
def test_scene_staged_and_fused_match_oracle(cuda_lib, oracle, name, layout):
    """Rows, contacts and states equal the oracle's (which builds the
    reference's trees) under both tree layouts: the layout changes the descent
    order, never a candidate set."""
    _scene_parity(oracle, name, layout, 0)


@pytest.mark.parametrize("layout", [0, 1], ids=["reference_tree", "cube_tree"])
@pytest.mark.parametrize("name", ["c1", "c2hash"])
def test_scene_apetrei_build_matches_oracle(cuda_lib, oracle, name, layout):
    """The same with every tree built by the Apetrei path (the oracle builds
    the reference's Apetrei trees)."""
    _scene_parity(oracle, name, layout, 1)


@pytest.mark.parametrize("layout", [0, 1], ids=["reference_tree", "cube_tree"])
def test_scene_edge_cases_match_oracle(cuda_lib, oracle, layout):
    """The edge-case scene from its first substep (where the in-plane
    contacts, the pinned pushes and the double push all fire), staged and
    fused, against the oracle."""
    _scene_parity(oracle, "edge", layout, 0, advance=0)


def _scene_parity(oracle, name, layout, builder, advance=3):
    from ysim_b200.scene import Scene
    spec = _small_specs()[name]
    o = _advance_to_contact(spec, advance)
    x0, v0, xp0 = o.get("x"), o.get("v"), o.get("xprev")
    s = Scene(spec, tree_layout=layout, tree_builder=builder)
    try:
        # both sides start at frame 0 from the same mid-drape state, so the
        # frame-0 preamble rebuilds every non-Float tree from x0 on both
        s.set("x", x0); s.set("v", v0); s.set("xprev", xp0)
        o2 = oracle.OracleScene(spec, builder=builder)
        o2.set("x", x0); o2.set("v", v0); o2.set("xprev", xp0)
        for sub in range(spec.params.substeps + 2):
            # ---- oracle stages
            o2.stage(0); o2.stage(1); o2.stage(2)
            orows = o2.rows()
            o2.stage(3)
            ooff, oc = o2.contacts()
            o2.stage(4)
            o2.stage(5)
            # ---- GPU stages
            s.broad_phase.build(); s.broad_phase.refit_swept(); s.broad_phase.detect_collisions()
            grows = s.rows()
            assert np.array_equal(canon_rows(grows), canon_rows(orows)), f"rows differ at substep {sub}"
            s.narrow_phase.narrow_and_sort_by_vertices()
            goff, gc = s.contacts()
            assert np.array_equal(goff, ooff)
            assert np.array_equal(gc["tobj"], oc["tobj"]) and np.array_equal(gc["tri"], oc["tri"])
            assert np.array_equal(np.stack([gc["nx"], gc["ny"], gc["nz"], gc["d"]], 1).view(np.uint32),
                                  np.concatenate([oc["n"], oc["d"][:, None]], 1).view(np.uint32))
            s.system.snapshot_xprev()
            s.system.update()
            assert rel_err(s.get("f"), o2.get("f")) <= TOL
            assert rel_err(s.get("x"), o2.get("x")) <= TOL
            assert rel_err(s.get("v"), o2.get("v")) <= TOL
            assert rel_err(s.get("xprev"), o2.get("xprev")) <= TOL
        st = s.stats()
        assert st["flags"] == 0, st
    finally:
        s.close()
    # fused path from the same state
    s = Scene(spec, tree_layout=layout, tree_builder=builder)
    try:
        s.set("x", x0); s.set("v", v0); s.set("xprev", xp0)
        s.set_record(True)
        o3 = oracle.OracleScene(spec, builder=builder)
        o3.set("x", x0); o3.set("v", v0); o3.set("xprev", xp0)
        for sub in range(2 * spec.params.substeps + 3):
            o3.step(1)
            s.step(1)
            ooff, oc = o3.contacts()
            goff, gc = s.contacts()
            assert np.array_equal(goff, ooff), f"contact offsets differ at substep {sub}"
            assert np.array_equal(gc["tobj"], oc["tobj"]) and np.array_equal(gc["tri"], oc["tri"])
            assert rel_err(s.get("x"), o3.get("x")) <= TOL
            assert rel_err(s.get("v"), o3.get("v")) <= TOL
        assert s.stats()["broad_rows"] == o3.stats()["broad_rows"]
        assert s.stats()["flags"] == 0
    finally:
        s.close()


@pytest.mark.parametrize("builder", [0, 1], ids=["karras", "apetrei"])
def test_scene_tree_matches_oracle(cuda_lib, oracle, builder):
    """With the reference layout the scene's trees are the reference's, node
    for node (codes, order, parents, boxes), from either builder."""
    from ysim_b200 import _lib
    from ysim_b200.scene import Scene
    spec = _small_specs()["c2hash"]
    s = Scene(spec, tree_layout=_lib.TREE_REFERENCE, tree_builder=builder)
    o = oracle.OracleScene(spec, builder=builder)
    o.stage(0)
    try:
        for m in range(len(spec.meshes)):
            gn, gp, gcodes, gidx = s.tree(m)
            on, op, ocodes, oidx = o.tree(m)
            assert np.array_equal(gcodes, ocodes) and np.array_equal(gidx, oidx)
            assert np.array_equal(gp[1:], op[1:])
            _tree_equal(gn, on)
    finally:
        s.close()


@pytest.mark.parametrize("case", ["soup", "sparse", "huge_tri"])
def test_spatial_hash_equals_lbvh_query(cuda_lib, oracle, case):
    """Spatial-hash broad phase == LBVH point query (== brute force) as sets."""
    import torch
    from ysim_b200 import _lib, generators as G
    x, f, q = G.soup(60_000 if case != "sparse" else 20_000, seed=31, nq=40_000)
    if case == "huge_tri":  # a few triangles spanning far more cells than the grid allows
        x = x.copy()
        x[0:9] = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 1]] * 3, np.float32)
    h_margin = np.float32(1e-3 if case != "sparse" else 4e-3)
    cell = np.float32(2 * h_margin)
    dx, df, dq = _dev(x.reshape(-1)), _dev(f.reshape(-1).astype(np.int32)), _dev(q.reshape(-1))
    cap = 1 << 22
    sh = C.c_void_p()
    _lib.check(cuda_lib.ys_shash_create(C.byref(sh), len(f), 64 * len(f), 0, None))
    try:
        _lib.check(cuda_lib.ys_shash_build(sh, _p(dx), _p(df), len(f), cell))
        pairs = torch.empty(2 * cap, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        _lib.check(cuda_lib.ys_shash_query(sh, _p(dq), len(q), h_margin, _p(pairs), cap, _p(cnt)))
        n = int(cnt.item())
        got = canon_pairs(pairs[: 2 * n].cpu().numpy().view(np.uint32))
    finally:
        _lib.check(cuda_lib.ys_shash_destroy(sh))
    h, _, _ = _lbvh(cuda_lib, x, f)
    try:
        pairs = torch.empty(2 * cap, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        _lib.check(cuda_lib.ys_lbvh_query(h, _p(dq), len(q), h_margin, 0, _p(pairs), cap, _p(cnt)))
        n = int(cnt.item())
        bvh = canon_pairs(pairs[: 2 * n].cpu().numpy().view(np.uint32))
    finally:
        _lib.check(cuda_lib.ys_lbvh_destroy(h))
    assert len(got) > 0
    assert np.array_equal(got, bvh)
    assert np.array_equal(got, canon_pairs(oracle.brute_q1(x, f, q, float(h_margin), False)))


def test_large_query_sets_in_morton_order(cuda_lib, oracle):
    """Large query sets run their threads in the points' Morton order (pairs
    still name the input points): from 2^21 points the LBVH query, which then
    equals the oracle's queryPoints over the oracle's own tree, and from 2^23
    the spatial hash, which then equals the LBVH, as sets."""
    import torch
    from ysim_b200 import _lib, generators as G
    x, f, _ = G.soup(60_000, seed=41, nq=1)
    rng = np.random.default_rng(42)
    margin = np.float32(1e-3)
    dx, df = _dev(x.reshape(-1)), _dev(f.reshape(-1).astype(np.int32))
    cap = 1 << 22
    pairs = torch.empty(2 * cap, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")

    def lbvh_pairs(h, dq, nq):
        _lib.check(cuda_lib.ys_lbvh_query(h, _p(dq), nq, margin, 0, _p(pairs), cap, _p(cnt)))
        n = int(cnt.item())
        assert n <= cap
        return canon_pairs(pairs[: 2 * n].cpu().numpy().view(np.uint32))

    q2 = rng.uniform(0, 1, ((1 << 21) + 1000, 3)).astype(np.float32)
    q8 = rng.uniform(0, 1, ((1 << 23) + 1000, 3)).astype(np.float32)
    dq2, dq8 = _dev(q2.reshape(-1)), _dev(q8.reshape(-1))
    h, _, _ = _lbvh(cuda_lib, x, f)
    try:
        rn, _, _, _ = oracle.build_tree(x, f)
        want = canon_pairs(oracle.query_points(rn, f, q2, float(margin)))
        assert len(want) > 5000
        for _ in range(2):  # the second call reuses the order buffers
            assert np.array_equal(lbvh_pairs(h, dq2, len(q2)), want)
        bvh8 = lbvh_pairs(h, dq8, len(q8))
    finally:
        _lib.check(cuda_lib.ys_lbvh_destroy(h))
    sh = C.c_void_p()
    _lib.check(cuda_lib.ys_shash_create(C.byref(sh), len(f), 64 * len(f), 0, None))
    try:
        _lib.check(cuda_lib.ys_shash_build(sh, _p(dx), _p(df), len(f), np.float32(2 * margin)))
        _lib.check(cuda_lib.ys_shash_query(sh, _p(dq8), len(q8), margin, _p(pairs), cap, _p(cnt)))
        n = int(cnt.item())
        assert len(bvh8) > 20000
        assert np.array_equal(canon_pairs(pairs[: 2 * n].cpu().numpy().view(np.uint32)), bvh8)
    finally:
        _lib.check(cuda_lib.ys_shash_destroy(sh))


def _dup_code_soup(seed=7):
    """Triangles in clusters of 20 around 300 centres, each cluster far inside
    one Morton cell (1/1024 of the box): long runs of equal codes."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.05, 0.95, (300, 3))
    c = np.repeat(centres, 20, axis=0) + rng.uniform(-5e-5, 5e-5, (6000, 3))
    x = (c[:, None, :] + rng.normal(0, 1e-4, (6000, 3, 3))).reshape(-1, 3).astype(np.float32)
    # two far corners fix the box so every cluster stays inside its cell
    x = np.concatenate([x, np.array([[0, 0, 0], [1e-6, 0, 0], [0, 1e-6, 0], [1, 1, 1], [1, 1 - 1e-6, 1],
                                     [1 - 1e-6, 1, 1]], np.float32)])
    f = np.arange(len(x), dtype=np.uint32).reshape(-1, 3)
    q = (np.repeat(centres, 10, axis=0) + rng.uniform(-1e-3, 1e-3, (3000, 3))).astype(np.float32)
    return x, f, q


def _query_pairs(cuda_lib, h, q, margin):
    import torch
    from ysim_b200 import _lib
    dq = _dev(q.reshape(-1))
    cap = 1 << 22
    pairs = torch.empty(2 * cap, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    _lib.check(cuda_lib.ys_lbvh_query(h, _p(dq), len(q), margin, 0, _p(pairs), cap, _p(cnt)))
    n = int(cnt.item())
    return canon_pairs(pairs[: 2 * n].cpu().numpy().view(np.uint32))


def test_equal_code_runs_reference_and_consistent_split(cuda_lib, oracle):
    """Runs of equal Morton codes.  The reference's split: the GPU tree and
    its query equal the oracle's (the reference's) node for node and pair for
    pair, leaves reached twice or never included.  The (code, index) split:
    one parent per node, and the query equals brute force and the spatial hash
    exactly (no duplicate, nothing missing)."""
    import torch
    from ysim_b200 import _lib
    x, f, q = _dup_code_soup()
    margin = np.float32(1e-3)
    onodes, oparent, ocodes, oidx = oracle.build_tree(x, f)
    _, counts = np.unique(ocodes, return_counts=True)
    assert (counts >= 3).sum() > 100
    brute = canon_pairs(oracle.brute_q1(x, f, q, float(margin), False))
    # reference split
    h, dx, df = _lbvh(cuda_lib, x, f)
    try:
        nodes, parent, codes, idx = tree_arrays(cuda_lib, h)
        assert np.array_equal(codes, ocodes) and np.array_equal(idx, oidx)
        assert np.array_equal(nodes["a"], onodes["a"]) and np.array_equal(nodes["b"], onodes["b"])
        ref = _query_pairs(cuda_lib, h, q, margin)
        assert np.array_equal(ref, canon_pairs(oracle.query_points(onodes, f, q, float(margin))))
        assert not np.array_equal(ref, brute)  # the inconsistent topology shows
    finally:
        _lib.check(cuda_lib.ys_lbvh_destroy(h))
    # consistent split
    h, dx, df = _lbvh(cuda_lib, x, f, consistent=True)
    try:
        nodes, parent, codes, idx = tree_arrays(cuda_lib, h)
        claims = np.zeros(len(nodes), np.int64)
        inner = nodes["a"] >= 0
        np.add.at(claims, nodes["a"][inner], 1)
        np.add.at(claims, nodes["b"][inner], 1)
        assert claims[0] == 0 and (claims[1:] == 1).all()
        cons = _query_pairs(cuda_lib, h, q, margin)
        assert np.array_equal(cons, brute)
    finally:
        _lib.check(cuda_lib.ys_lbvh_destroy(h))
    sh = C.c_void_p()
    _lib.check(cuda_lib.ys_shash_create(C.byref(sh), len(f), 64 * len(f), 0, None))
    try:
        dq = _dev(q.reshape(-1))
        _lib.check(cuda_lib.ys_shash_build(sh, _p(dx), _p(df), len(f), np.float32(2 * margin)))
        cap = 1 << 22
        pairs = torch.empty(2 * cap, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        _lib.check(cuda_lib.ys_shash_query(sh, _p(dq), len(q), margin, _p(pairs), cap, _p(cnt)))
        n = int(cnt.item())
        assert np.array_equal(canon_pairs(pairs[: 2 * n].cpu().numpy().view(np.uint32)), brute)
    finally:
        _lib.check(cuda_lib.ys_shash_destroy(sh))


def _expand10(v):
    out = 0
    for i in range(10):
        out |= ((v >> i) & 1) << (3 * i)
    return out


def _cell_bucket(x, y, z, mask):
    """The hash's bucket of cell (x, y, z): the cell's Morton code within its
    1024^3 block, xor a Teschner hash of the block (ys_shash.cu)."""
    m = (_expand10(x & 1023) << 2) | (_expand10(y & 1023) << 1) | _expand10(z & 1023)
    blk = (((x >> 10) * 73856093) ^ ((y >> 10) * 19349663) ^ ((z >> 10) * 83492791)) & 0xFFFFFFFF
    return (m ^ blk) & mask


def test_spatial_hash_bucket_collision_inside_one_triangle(cuda_lib):
    """Two cells of one triangle that share a hash bucket, the query probing
    one of them: the pair is reported once (the triangle's entries in one
    bucket are seen once, whichever of its cells they were binned for).  The
    triangle spans 3 x 2 x 2 cells, so the build's table has 32 buckets; cells
    two apart in x can share one."""
    import torch
    from ysim_b200 import _lib
    max_entries = 1024
    mask = 31  # the build's table: 2 x 12 entries rounded up to a power of two
    found = None
    for x in range(100, 400):
        for y in range(100, 140):
            for z in range(100, 110):
                h0 = _cell_bucket(x, y, z, mask)
                if any(_cell_bucket(x + dx, y + dy, z + dz, mask) == h0
                       for dx in (0, 1, 2) for dy in (0, 1) for dz in (0, 1) if (dx, dy, dz) != (0, 0, 0)):
                    found = (x, y, z)
                    break
            if found:
                break
        if found:
            break
    assert found is not None
    c = np.float32(2e-3)
    x0, y0, z0 = found
    lo = np.array([x0, y0, z0], np.float64) * float(c) + 1e-4
    hi = (np.array([x0, y0, z0], np.float64) + np.array([3, 2, 2])) * float(c) - 1e-4
    tri = np.array([[lo[0], lo[1], lo[2]], [hi[0], lo[1], hi[2]], [lo[0], hi[1], hi[2]]], np.float32)
    f = np.arange(3, dtype=np.uint32).reshape(1, 3)
    q = ((np.array([[x0, y0, z0]], np.float64) + 1) * float(c)).astype(np.float32)
    dx, df, dq = _dev(tri.reshape(-1)), _dev(f.reshape(-1).astype(np.int32)), _dev(q.reshape(-1))
    sh = C.c_void_p()
    _lib.check(cuda_lib.ys_shash_create(C.byref(sh), 1, max_entries, 0, None))
    try:
        _lib.check(cuda_lib.ys_shash_build(sh, _p(dx), _p(df), 1, c))
        pairs = torch.zeros(64, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        _lib.check(cuda_lib.ys_shash_query(sh, _p(dq), 1, np.float32(c / 2), _p(pairs), 32, _p(cnt)))
        assert int(cnt.item()) == 1
        assert pairs[:2].cpu().tolist() == [0, 0]
    finally:
        _lib.check(cuda_lib.ys_shash_destroy(sh))


def check_wide_boxes(s, spec, mesh=0):
    """After a refit of the current state: every leaf slot of the mesh's
    4-wide tree holds its face's swept box (x and x + v subh, float32 as the
    reference computes buildSweptLeaf_Tri), and every internal slot the union
    of its child's slots; returns the number of wide nodes checked."""
    s.broad_phase.refit_swept()
    W = s.wide_tree(mesh)
    assert len(W) > 0
    voff = sum(m.nV for m in spec.meshes[:mesh])
    m = spec.meshes[mesh]
    x = s.get("x")[voff:voff + m.nV]
    v = s.get("v")[voff:voff + m.nV]
    dt = np.float32(spec.params.subh)
    p = x[m.facets]
    sp = (p + (v[m.facets] * dt).astype(np.float32)).astype(np.float32)
    leaf_lo = np.minimum(p, sp).min(1)
    leaf_hi = np.maximum(p, sp).max(1)
    child = W["child"]
    lo = W["lo"].transpose(0, 2, 1)  # (node, slot, axis)
    hi = W["hi"].transpose(0, 2, 1)
    leaf = (child < 0)
    f = ~child[leaf]
    assert np.array_equal(lo[leaf], leaf_lo[f]) and np.array_equal(hi[leaf], leaf_hi[f])
    inner = (child >= 0) & (child != 0x7FFFFFFF)
    c = child[inner]
    assert np.array_equal(lo[inner], lo[c].min(1)) and np.array_equal(hi[inner], hi[c].max(1))
    # every face is a leaf exactly once
    assert np.array_equal(np.sort(f), np.arange(m.nF))
    return len(W)


def test_wide_refit_boxes_are_exact(cuda_lib):
    """The 4-wide refit (leaf slots from the swept leaf boxes, internal slots
    as unions over sorted-leaf ranges) gives exactly the boxes a bottom-up
    union gives, after steps and a rebuild."""
    from ysim_b200.scene import Scene
    spec = _small_specs()["c2hash"]
    s = Scene(spec)
    try:
        s.step(2 * spec.params.substeps + 3)
        assert check_wide_boxes(s, spec) > 100
        s.step(10 * spec.params.substeps)  # through the rebuild at frame 10
        check_wide_boxes(s, spec)
        assert s.stats()["flags"] == 0
    finally:
        s.close()


@pytest.mark.parametrize("case", ["soup", "big_soup", "grid", "tiny1", "tiny2", "dups"])
def test_consistent_lbvh_range_refit_is_the_bottom_up_refit(cuda_lib, case):
    """With the (code, index) split the standalone LBVH refits by sorted-leaf
    ranges (leaf pass with block boxes, then the nodes whose range crosses a
    256-leaf block): after the build and after a swept refit, every leaf box is
    its face's box (float32, as buildSweptLeaf_Tri computes it) and every
    internal box the union of its two children's, bit for bit."""
    from ysim_b200 import _lib, generators as G
    if case in ("soup", "big_soup"):
        x, f, _ = G.soup(50_000 if case == "soup" else 300_000, seed=5)
    elif case == "grid":
        x, f = G.grid_cloth(65, 1.0, (0.0, 0.5, 0.0))
    elif case == "tiny1":
        x, f, _ = G.soup(1, seed=6, nq=5)
    elif case == "tiny2":
        x, f, _ = G.soup(2, seed=7, nq=5)
    else:
        x, f, _ = G.soup(3000, seed=8)
        x = np.tile(x[:3], (3000, 1)).astype(np.float32)
    h, dx, df = _lbvh(cuda_lib, x, f, consistent=True)
    try:
        n = len(f)

        def check(v, dt):
            nodes, parent, _, idx = tree_arrays(cuda_lib, h)
            p = x[f[idx]]
            if v is None:
                lo, hi = p.min(1), p.max(1)
            else:
                sp = (p + (v[f[idx]] * np.float32(dt)).astype(np.float32)).astype(np.float32)
                lo, hi = np.minimum(p, sp).min(1), np.maximum(p, sp).max(1)
            leaves = nodes[n - 1:]
            assert np.array_equal(leaves["mn"], lo) and np.array_equal(leaves["mx"], hi)
            inner = nodes[: n - 1]
            a, b = inner["a"], inner["b"]
            assert np.array_equal(inner["mn"], np.minimum(nodes["mn"][a], nodes["mn"][b]))
            assert np.array_equal(inner["mx"], np.maximum(nodes["mx"][a], nodes["mx"][b]))
            assert reachable(nodes).all()

        check(None, 0.0)
        v = np.random.default_rng(1).normal(0, 1.0, x.shape).astype(np.float32)
        dv = _dev(v.reshape(-1))
        _lib.check(cuda_lib.ys_lbvh_refit(h, _p(dx), _p(dv), np.float32(1.0 / 1200), 1))
        check(v, 1.0 / 1200)
    finally:
        _lib.check(cuda_lib.ys_lbvh_destroy(h))
