"""GPU path against the golden vectors produced by the reference's own kernels
(tests/golden/make_golden.py), through the C ABI.  Independent of the oracle:
these run on a machine without the reference checkout."""
import ctypes as C
import os

import numpy as np
import pytest

from helpers import canon_pairs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_gpu_lbvh_matches_golden(cuda_lib):
    import torch
    from ysim_b200 import _lib
    from test_gpu_parity import tree_arrays
    g = np.load(os.path.join(GOLD, "morton_tree.npz"))
    for name in ("soup", "grid"):
        x, f, q, v = g[f"{name}_x"], g[f"{name}_f"], g[f"{name}_q"], g[f"{name}_v"]
        h = C.c_void_p()
        _lib.check(cuda_lib.ys_lbvh_create(C.byref(h), len(f), 0, None))
        try:
            dx, df = _dev(x.reshape(-1)), _dev(f.reshape(-1).astype(np.int32))
            _lib.check(cuda_lib.ys_lbvh_build(h, _p(dx), len(x), _p(df), len(f)))
            nodes, parent, codes, idx = tree_arrays(cuda_lib, h)
            assert np.array_equal(codes, g[f"{name}_codes"]) and np.array_equal(idx, g[f"{name}_idx"])
            assert np.array_equal(nodes["a"], g[f"{name}_a"]) and np.array_equal(nodes["b"], g[f"{name}_b"])
            assert np.array_equal(parent[1:], g[f"{name}_parent"][1:])
            assert np.array_equal(nodes["mn"], g[f"{name}_mn"]) and np.array_equal(nodes["mx"], g[f"{name}_mx"])
            dv = _dev(v.reshape(-1))
            _lib.check(cuda_lib.ys_lbvh_refit(h, _p(dx), _p(dv), np.float32(1.0 / 1200.0), 1))
            nodes, _, _, _ = tree_arrays(cuda_lib, h)
            assert np.array_equal(nodes["mn"], g[f"{name}_swept_mn"])
            assert np.array_equal(nodes["mx"], g[f"{name}_swept_mx"])
            cap = 1 << 20
            pairs = torch.empty(2 * cap, dtype=torch.int32, device="cuda")
            cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
            dq = _dev(q.reshape(-1))
            _lib.check(cuda_lib.ys_lbvh_query(h, _p(dq), len(q), np.float32(g[f"{name}_margin"]),
                                              int(g[f"{name}_self"]), _p(pairs), cap, _p(cnt)))
            n = int(cnt.item())
            got = canon_pairs(pairs[: 2 * n].cpu().numpy().view(np.uint32))
            assert np.array_equal(got, g[f"{name}_pairs"])
        finally:
            _lib.check(cuda_lib.ys_lbvh_destroy(h))


def test_gpu_apetrei_build_matches_golden(cuda_lib):
    """ys_lbvh_set_builder(YS_BUILD_APETREI): the reference's
    agglomerativeBuild_Tri + agglomerativeSwapRoot tree, node for node."""
    from ysim_b200 import _lib
    from test_gpu_parity import tree_arrays
    g = np.load(os.path.join(GOLD, "morton_tree.npz"))
    for name in ("soup", "grid"):
        x, f = g[f"{name}_x"], g[f"{name}_f"]
        h = C.c_void_p()
        _lib.check(cuda_lib.ys_lbvh_create(C.byref(h), len(f), 0, None))
        try:
            _lib.check(cuda_lib.ys_lbvh_set_builder(h, _lib.BUILD_APETREI))
            dx, df = _dev(x.reshape(-1)), _dev(f.reshape(-1).astype(np.int32))
            _lib.check(cuda_lib.ys_lbvh_build(h, _p(dx), len(x), _p(df), len(f)))
            nodes, parent, codes, idx = tree_arrays(cuda_lib, h)
            assert np.array_equal(codes, g[f"{name}_codes"]) and np.array_equal(idx, g[f"{name}_idx"])
            assert np.array_equal(nodes["a"], g[f"{name}_agg_a"]) and np.array_equal(nodes["b"], g[f"{name}_agg_b"])
            assert np.array_equal(parent, g[f"{name}_agg_parent"])
            assert np.array_equal(nodes["mn"], g[f"{name}_agg_mn"])
            assert np.array_equal(nodes["mx"], g[f"{name}_agg_mx"])
        finally:
            _lib.check(cuda_lib.ys_lbvh_destroy(h))


@pytest.mark.parametrize("name", ["c1", "c2hash"])
@pytest.mark.parametrize("fused", [False, True])
def test_gpu_substep_matches_golden(cuda_lib, name, fused):
    from ysim_b200 import generators as G
    from ysim_b200.scene import Scene
    spec = {"c1": lambda: G.config_c1(P=24, level=2, height=0.2999),
            "c2hash": lambda: G.config_c2(P=32, level=3, height=0.315, gravity=-9.81)}[name]()
    g = np.load(os.path.join(GOLD, f"substep_{name}.npz"))
    s = Scene(spec)
    try:
        s.set("x", g["x"]); s.set("v", g["v"]); s.set("xprev", g["xprev"])
        n0 = spec.meshes[0].nV
        if fused:
            s.set_record(True)
            s.step(1)
        else:
            s.broad_phase.build(); s.broad_phase.refit_swept(); s.broad_phase.detect_collisions()
            rows = s.rows()
            t = np.stack([rows["qobj"], rows["point"], rows["tobj"], rows["tri"]], 1).astype(np.uint32)
            t = t[np.lexsort((t[:, 3], t[:, 2], t[:, 1], t[:, 0]))]
            assert np.array_equal(t, g["rows"])
            s.narrow_phase.narrow_and_sort_by_vertices()
        off, c = s.contacts()
        assert np.array_equal(off, g["csr_off"])
        assert np.array_equal(c["tri"], g["c_tri"]) and np.array_equal(c["tobj"], g["c_tobj"])
        n = np.stack([c["nx"], c["ny"], c["nz"]], 1)
        assert np.array_equal(n.view(np.uint32), g["c_n"].view(np.uint32))
        assert np.array_equal(c["d"].view(np.uint32), g["c_d"].view(np.uint32))
        if not fused:
            s.system.snapshot_xprev()
            s.system.update()
            assert np.array_equal(s.get("f")[:n0].view(np.uint32), g["f"].view(np.uint32))
        assert np.array_equal(s.get("x")[:n0].view(np.uint32), g["x_next"].view(np.uint32))
        assert np.array_equal(s.get("v")[:n0].view(np.uint32), g["v_next"].view(np.uint32))
        assert s.stats()["flags"] == 0
    finally:
        s.close()
