"""Pin the CPU oracle against the reference's own kernel code.

oracle/_ref is the reference's Metal compute kernels (bvh.metal,
bruteforce.metal, physics.metal) compiled for the host through
oracle/ref_shim (built by oracle/build_ref.py from the reference checkout in
place).  Every restated stage is compared with the kernel it restates on
identical inputs: Morton codes, Karras topology, leaf / swept / bottom-up
boxes, point queries, narrow contacts, spring forces and integration.
The reference's radix sort and CPU spatial hash have no host-runnable form;
they are pinned by definition (numpy stable sort) and by brute-force
enumeration (test_oracle_props.py).
"""
import numpy as np
import pytest

from helpers import canon_pairs, rel_err

refk = pytest.importorskip("oracle.refkernels")
if not refk.available():
    pytest.skip("reference kernels unavailable (no reference checkout)", allow_module_level=True)


def _boxes_equal(a, b):
    # min/max are exact; the reference's fmin/fmax may pick either zero sign
    assert np.array_equal(a["mn"], b["mn"]) and np.array_equal(a["mx"], b["mx"])


def _inputs():
    from ysim_b200 import generators as G
    x1, f1, q1 = G.soup(20_000, seed=21)
    x2, f2 = G.grid_cloth(60, 1.0, (0.0, 0.3, 0.0))
    rng = np.random.default_rng(3)
    x2 = (x2 + rng.uniform(-2e-3, 2e-3, x2.shape)).astype(np.float32)
    x3, f3 = G.icosphere(3)
    x3 = (x3 * 0.3).astype(np.float32)
    return [(x1, f1, q1), (x2, f2, x2.copy()), (x3, f3, (x3 * 1.01).astype(np.float32))]


def test_morton_matches_reference_kernel(oracle):
    for x, f, _ in _inputs():
        box = np.zeros(6, np.float32)
        oracle.lib().yso_scene_box(oracle.P(x), len(x), oracle.P(box))
        rc, ri = refk.fill_mortons(x, f, box)
        oc, oi = oracle.morton(x, f)
        assert np.array_equal(rc, oc) and np.array_equal(ri, oi)


def test_karras_and_bottom_up_match_reference_kernels(oracle):
    for x, f, _ in _inputs():
        on, op, oc, oi = oracle.build_tree(x, f)
        rn, rp = refk.build_tree(x, f, oc, oi)
        assert np.array_equal(rn["a"], on["a"]) and np.array_equal(rn["b"], on["b"])
        assert np.array_equal(rp[1:], op[1:])
        _boxes_equal(rn, on)


def test_swept_refit_matches_reference_kernels(oracle):
    rng = np.random.default_rng(9)
    for x, f, _ in _inputs():
        on, op, oc, oi = oracle.build_tree(x, f)
        v = rng.normal(0, 0.5, x.shape).astype(np.float32)
        dt = np.float32(1.0 / 1200.0)
        _boxes_equal(refk.refit(on, op, x, v, f, oc, oi, dt, True), oracle.refit(on, x, v, f, dt, True))
        _boxes_equal(refk.refit(on, op, x, None, f, oc, oi, dt, False), oracle.refit(on, x, None, f, dt, False))


@pytest.mark.parametrize("margin", [1e-3, 0.015])
def test_query_points_matches_reference_kernel(oracle, margin):
    for k, (x, f, q) in enumerate(_inputs()):
        on, op, oc, oi = oracle.build_tree(x, f)
        self_q = k == 1  # grid cloth queried against itself
        rows, n, flags = refk.query_points(q, f, on, margin, 0, 0 if self_q else 1)
        assert n == len(rows) and flags[0] == 0
        got = canon_pairs(np.stack([rows["point"], rows["tri"]], 1))
        want = canon_pairs(oracle.query_points(on, f, q, margin, self_q))
        assert np.array_equal(got, want)


def _packed(spec):
    """Packed scene arrays (Scene::pack layout, scene.hpp:783-1180)."""
    from oracle import oracle as O
    voff, foff, F, vaf, vaf_off = [0], [0], [], [], [0]
    for m in spec.meshes:
        a = O.adjacency(m.x, m.facets)
        base = vaf_off[-1]
        vaf_off += list(base + a["vaf_off"][1:])
        vaf.append(a["vaf"])
        F.append(m.facets.reshape(-1))
        voff.append(voff[-1] + m.nV)
        foff.append(foff[-1] + m.nF)
    return (np.array(voff, np.uint32), np.array(foff, np.uint32), np.concatenate(F).astype(np.uint32),
            np.concatenate(vaf).astype(np.uint32), np.array(vaf_off, np.uint32))


@pytest.mark.parametrize("name", ["c1", "c2hash", "c2bvh"])
def test_substep_stages_match_reference_kernels(oracle, name):
    from ysim_b200 import generators as G
    spec = {"c1": G.config_c1(P=24, level=2, height=0.2999),
            "c2hash": G.config_c2(P=40, level=3, height=0.33, gravity=-9.81),
            "c2bvh": G.config_c2(P=40, level=3, height=0.33, self_mode=2, gravity=-9.81)}[name]
    o = oracle.OracleScene(spec)
    o.step(3 * spec.params.substeps + 1)  # mid-drape, contacts present
    voff, foff, F, vaf, vaf_off = _packed(spec)
    p = spec.params
    checked_contacts = 0
    for _ in range(3):
        o.stage(0); o.stage(1); o.stage(2)
        x, xp, v = o.get("x"), o.get("xprev"), o.get("v")
        rows = o.rows()
        o.stage(3)
        ooff, oc = o.contacts()
        # narrow_pt_tri on the oracle's rows
        rc = refk.narrow(rows, x, voff, F, foff, vaf, vaf_off, np.float32(p.radius), np.float32(p.margin), xp)
        key = lambda c: np.lexsort((c["tri"], c["tobj"], c["point"], c["qobj"]))
        rc, occ = rc[key(rc)], oc[key(oc)]
        assert len(rc) == len(occ)
        for fld in ("point", "tri", "qobj", "tobj"):
            assert np.array_equal(rc[fld], occ[fld])
        assert np.array_equal(rc["n"].view(np.uint32), occ["n"].view(np.uint32))
        assert np.array_equal(rc["d"].view(np.uint32), occ["d"].view(np.uint32))
        checked_contacts += len(rc)
        o.stage(4)
        # forces + integrate of the cloth with the reference kernels, on the
        # oracle's canonical per-vertex contact CSR
        m = spec.meshes[0]
        n0 = m.nV
        mass3 = np.repeat(m.mass, 3).astype(np.float32)
        ext = (np.asarray(p.gravity, np.float32)[None, :] * m.mass[:, None]).astype(np.float32)
        if m.behavior == 0:
            adj = oracle.adjacency(m.x, m.facets)
            cp4 = np.array([m.kstretch, m.kshear, m.kbend, m.thickness], np.float32)
            rf = refk.tri_forces(x[:n0], v[:n0], ext, mass3, m.mask, np.float32(p.subh), np.float32(p.kair),
                                 np.float32(p.kd), cp4, adj, m.facets.reshape(-1))
            prm, kind = cp4, "tri"
        else:
            gp = refk.grid_params(m.grid_n, m.grid_rest, (m.kstretch, m.kshear, m.kbend), m.thickness)
            rf = refk.grid_forces(x[:n0], v[:n0], ext, mass3, np.float32(p.subh), np.float32(p.kair),
                                  np.float32(p.kd), gp)
            prm, kind = gp, "grid"
        rx, rv, _ = refk.integrate(kind, x[:n0], v[:n0], rf, mass3, m.mask, oc, ooff, voff, 0, np.float32(p.subh),
                                   prm)
        o.stage(5)
        assert np.array_equal(rf.view(np.uint32), o.get("f")[:n0].view(np.uint32))
        assert rel_err(rx, o.get("x")[:n0]) <= 1e-5 and rel_err(rv, o.get("v")[:n0]) <= 1e-5
        assert np.array_equal(rx.view(np.uint32), o.get("x")[:n0].view(np.uint32))
    if name != "c1":
        assert checked_contacts > 0


def test_bucket_kernels_partition_like_oracle(oracle):
    """narrow_bucket_* (GPU CSR, order nondeterministic) == oracle CSR as
    per-vertex multisets."""
    from ysim_b200 import generators as G
    spec = G.config_c2(P=40, level=3, height=0.33, gravity=-9.81)
    o = oracle.OracleScene(spec)
    o.step(3 * spec.params.substeps + 1)
    for k in range(4):
        o.stage(k)
    off, oc = o.contacts()
    voff = np.array([0, spec.meshes[0].nV, spec.nV], np.uint32)
    offsets = np.zeros(spec.nV + 1, np.uint32)
    counter = np.zeros(spec.nV, np.uint32)
    out = np.zeros_like(oc)
    refk.lib().yref_bucket(refk.P(np.ascontiguousarray(oc)), len(oc), refk.P(voff), spec.nV + 1, refk.P(offsets),
                           refk.P(counter), refk.P(out))
    assert np.array_equal(offsets, off)
    for g in range(spec.nV):
        a, b = out[off[g]:off[g + 1]], oc[off[g]:off[g + 1]]
        assert sorted(zip(a["tobj"], a["tri"])) == sorted(zip(b["tobj"], b["tri"]))


def _sh_scenes():
    from ysim_b200 import generators as G
    return [("c1", G.config_c1(P=24, level=2, height=0.2999), 0.015),
            ("c2", G.config_c2(P=40, level=3, height=0.33, gravity=-9.81), 0.01),
            ("c4", G.config_c4(instances=4, lo=8, hi=20, level=2, drop=0.001), 0.015)]


@pytest.mark.parametrize("self_rows", [True, False])
def test_face_face_hash_matches_reference_kernels(oracle, self_rows):
    """H2: the restated face-face hash gives the reference kernels' rows (as a
    multiset) and the same entry / cell / pair counts and grid."""
    from helpers import canon_rows_full
    for name, spec, margin in _sh_scenes():
        x, so, fo, F, beh, shape = oracle.pack_meshes(spec.meshes)
        a, sa = oracle.sh_face_face(x, so, fo, F, beh, shape, margin, self_rows)
        b, sb = refk.sh_detect(x, so, fo, F, beh, shape, margin, self_rows)
        assert len(a) > 0, name
        assert np.array_equal(sa, sb), (name, sa, sb)
        assert np.array_equal(canon_rows_full(a), canon_rows_full(b)), name


def test_analytic_narrow_matches_reference_kernel(oracle):
    """narrow_pt_analytic (bruteforce.metal:236-499) restated: every contact
    of every collider kind -- static, rotated, moving, ellipsoid, disabled --
    bit for bit (normals and distances), none missing or extra."""
    from analytic_cases import RADIUS, THICKNESS, canon_contacts, cases
    shapes, x, xp, so, beh, pairs = cases(seed=23, per_shape=4000)
    oc, n = oracle.narrow_analytic(x, xp, so, beh, shapes, pairs, RADIUS, THICKNESS)
    ref = []
    for k, (cloth, _) in enumerate(pairs):
        if not shapes[k]["flags"] & 1:
            continue
        rm = np.float32(oracle.rot_margin(shapes[k], RADIUS, THICKNESS))
        ref.append(refk.narrow_analytic(x, xp, so, shapes, int(cloth), k, int(beh[cloth]), RADIUS, THICKNESS, rm))
    rc = canon_contacts(np.concatenate(ref))
    oc = canon_contacts(oc)
    assert n == len(oc) == len(rc)
    assert np.array_equal(oc.view(np.uint8), rc.view(np.uint8))
    for kind in (1, 2, 3, 4):
        assert (rc["tshape"] == kind).sum() > 100, kind
    # the disabled collider emits nothing
    off = shapes["obj"][shapes["flags"] == 0]
    assert not np.isin(rc["tobj"], off).any()


def _dup_soup(seed=7):
    """Triangles clustered on 40 points: runs of equal Morton codes."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0, 1, (40, 3))[rng.integers(0, 40, 600)]
    x = (c[:, None, :] + rng.normal(0, 1e-4, (600, 3, 3))).reshape(-1, 3).astype(np.float32)
    return x, np.arange(len(x), dtype=np.uint32).reshape(-1, 3)


def test_apetrei_build_matches_reference_kernel(oracle):
    """agglomerativeBuild_Tri + agglomerativeSwapRoot (bvh.metal:884-1199)
    restated: children, parents and boxes node for node, the root in slot 0,
    one parent per node even over runs of equal codes."""
    cases = [(x, f) for x, f, _ in _inputs()] + [_dup_soup()]
    for x, f in cases:
        nodes, parent, codes, idx = oracle.build_tree(x, f, builder=1)
        rn, rp, k = refk.agglomerative(x, f, codes, idx)
        assert np.array_equal(nodes["a"], rn["a"]) and np.array_equal(nodes["b"], rn["b"])
        assert np.array_equal(parent, rp) and parent[0] == -1
        _boxes_equal(nodes, rn)
        n = len(f)
        claims = np.bincount(np.concatenate([nodes["a"][: n - 1], nodes["b"][: n - 1]]), minlength=2 * n - 1)
        assert claims[0] == 0 and (claims[1:] == 1).all()
    assert len(codes) - len(np.unique(codes)) > 100  # the last case has runs of equal codes
