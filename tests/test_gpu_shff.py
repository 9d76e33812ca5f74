"""The face-face spatial-hash broad phase (ys_shff_*, the reference's
SpatialHashing<METAL>::detectCollisions) through the C ABI, against the CPU
oracle (itself pinned to the reference's kernels): identical rows as a
multiset, identical entry / cell / pair counts and grid."""
import ctypes as C

import numpy as np
import pytest

from helpers import canon_rows_full

pytestmark = pytest.mark.gpu


def _dev(a, dt):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dt).reshape(-1).view(np.int32 if dt != np.float32 else dt)).cuda()


def _p(t):
    return C.c_void_p(t.data_ptr())


def _run(cuda_lib, x, so, fo, F, beh, shape, margin, self_rows, cap=None):
    import torch
    from ysim_b200 import _lib
    from ysim_b200.scene import ROW_DTYPE
    nF = len(F)
    cap = cap if cap is not None else 64 * nF + 64
    h = C.c_void_p()
    _lib.check(cuda_lib.ys_shff_create(C.byref(h), nF, 0, None))
    try:
        dx, dso, dF, dfo = _dev(x, np.float32), _dev(so, np.uint32), _dev(F, np.uint32), _dev(fo, np.uint32)
        db, ds = _dev(beh, np.uint32), _dev(shape, np.uint32)
        rows = torch.empty(cap * 8, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        for _ in range(2):  # a second detect on the same handle gives the same rows
            _lib.check(cuda_lib.ys_shff_detect(h, _p(dx), len(x), _p(dso), _p(dF), _p(dfo), nF, _p(db), _p(ds),
                                               len(beh), np.float32(margin), int(self_rows), _p(rows), cap, _p(cnt)))
            n = int(cnt.item())
            got = rows[: 8 * min(n, cap)].cpu().numpy().view(np.uint32).view(ROW_DTYPE)
        st = (C.c_uint32 * 6)()
        _lib.check(cuda_lib.ys_shff_stats(h, st))
        return got, n, np.array(list(st), np.uint32)
    finally:
        _lib.check(cuda_lib.ys_shff_destroy(h))


def _scenes():
    from ysim_b200 import generators as G
    return {"c1": (G.config_c1(P=24, level=2, height=0.2999), 0.015),
            "c2": (G.config_c2(P=40, level=3, height=0.33, gravity=-9.81), 0.01),
            "c4": (G.config_c4(instances=4, lo=8, hi=20, level=2, drop=0.001), 0.015)}


@pytest.mark.parametrize("self_rows", [True, False])
@pytest.mark.parametrize("name", ["c1", "c2", "c4"])
def test_face_face_hash_matches_oracle(cuda_lib, oracle, name, self_rows):
    spec, margin = _scenes()[name]
    x, so, fo, F, beh, shape = oracle.pack_meshes(spec.meshes)
    want, wst = oracle.sh_face_face(x, so, fo, F, beh, shape, margin, self_rows)
    got, n, st = _run(cuda_lib, x, so, fo, F, beh, shape, margin, self_rows)
    assert n == len(want) > 0
    assert np.array_equal(st, wst), (st, wst)
    assert np.array_equal(canon_rows_full(got), canon_rows_full(want))


def test_face_face_hash_soup_of_meshes(cuda_lib, oracle):
    """Several meshes of a triangle soup, two of them Float (their pairs are
    dropped), uneven sizes, self rows on; plus a capacity too small: the count
    is exact and the rows written are a subset."""
    from ysim_b200 import generators as G
    from ysim_b200._lib import FLOAT, TRIANGULAR_CLOTH
    x, f, _ = G.soup(30_000, seed=41)
    cuts = [0, 9000, 16000, 16500, 30000]
    meshes = []
    for i in range(4):
        fs = f[cuts[i]:cuts[i + 1]]
        vids = np.unique(fs)
        remap = np.full(len(x), 0, np.uint32)
        remap[vids] = np.arange(len(vids), dtype=np.uint32)
        meshes.append(G.Mesh(behavior=FLOAT if i in (1, 2) else TRIANGULAR_CLOTH, flags=0, x=x[vids],
                             facets=remap[fs]))
    xs, so, fo, F, beh, shape = oracle.pack_meshes(meshes)
    shape = np.array([0, 1, 2, 0], np.uint32)
    want, wst = oracle.sh_face_face(xs, so, fo, F, beh, shape, 2e-3, True)
    got, n, st = _run(cuda_lib, xs, so, fo, F, beh, shape, 2e-3, True)
    assert n == len(want) > 0 and np.array_equal(st, wst)
    assert np.array_equal(canon_rows_full(got), canon_rows_full(want))
    got_s, n_s, _ = _run(cuda_lib, xs, so, fo, F, beh, shape, 2e-3, True, cap=n // 3)
    assert n_s == n and len(got_s) == n // 3
    full = {tuple(r) for r in canon_rows_full(want).tolist()}
    assert all(tuple(r) in full for r in canon_rows_full(got_s).tolist())


def test_face_face_hash_rejects_unaligned_rows(cuda_lib):
    """The broad kernel writes rows as 16-byte stores, so a row buffer that
    is not 16-byte aligned is refused before any launch (YS_ERR_BAD_ARG)."""
    import torch
    from ysim_b200 import _lib
    spec = _scenes()["c1"][0]
    x = np.concatenate([m.x for m in spec.meshes]).astype(np.float32)
    F = np.concatenate([m.facets for m in spec.meshes]).astype(np.uint32)
    so = np.concatenate([[0], np.cumsum([m.nV for m in spec.meshes])]).astype(np.uint32)
    fo = np.concatenate([[0], np.cumsum([m.nF for m in spec.meshes])]).astype(np.uint32)
    beh = np.array([m.behavior for m in spec.meshes], np.uint32)
    shape = np.zeros(len(spec.meshes), np.uint32)
    h = C.c_void_p()
    _lib.check(cuda_lib.ys_shff_create(C.byref(h), len(F), 0, None))
    try:
        dx, dso, dF, dfo = _dev(x, np.float32), _dev(so, np.uint32), _dev(F, np.uint32), _dev(fo, np.uint32)
        db, ds = _dev(beh, np.uint32), _dev(shape, np.uint32)
        rows = torch.empty(64 * 8 + 4, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
        r = cuda_lib.ys_shff_detect(h, _p(dx), len(x), _p(dso), _p(dF), _p(dfo), len(F), _p(db), _p(ds), len(beh),
                                    np.float32(0.015), 1, C.c_void_p(rows.data_ptr() + 4), 64, _p(cnt))
        assert r == _lib.YS_ERR_BAD_ARG
    finally:
        _lib.check(cuda_lib.ys_shff_destroy(h))
