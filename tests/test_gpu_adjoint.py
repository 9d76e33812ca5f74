"""Differentiable rollouts: the CUDA adjoint (ys_adjoint_*) through the C ABI
and its torch.autograd.Function, against the FP64 CPU reference adjoint and
FP64 central finite differences."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small(N=16, level=3, height=0.2995):
    from ysim_b200 import generators as G
    return G.config_c5(N=N, level=level, height=height)


def test_uniform_grid_springs_reproduce_fastgrid(cuda_lib):
    """Per-spring arrays holding FastGridClothBehaviorParams' values give the
    same positions bit for bit as the three-stiffness / six-rest-length form."""
    import torch
    from ysim_b200 import _lib, generators as G
    from ysim_b200.scene import Scene
    spec = _small(N=24, level=2, height=0.2999)
    c = spec.meshes[0]
    k, L = G.grid_spring_params(c.grid_n, c.grid_rest, (c.kstretch, c.kshear, c.kbend))
    a, b = Scene(spec), Scene(spec)
    try:
        dk, dL = torch.from_numpy(k).cuda(), torch.from_numpy(L).cuda()
        torch.cuda.synchronize()
        import ctypes as C
        _lib.check(cuda_lib.ys_scene_set_grid_springs(b.h, 0, C.c_void_p(dk.data_ptr()), C.c_void_p(dL.data_ptr())))
        a.step(40)
        b.step(40)
        assert np.array_equal(a.get("x").view(np.uint32), b.get("x").view(np.uint32))
        assert np.array_equal(a.get("v").view(np.uint32), b.get("v").view(np.uint32))
    finally:
        a.close()
        b.close()


def _problem(spec, seed=0):
    """Uniform FastGrid springs, a random initial velocity and a linear loss
    sum(w * x_T).  The loss is linear so that its gradient (the adjoint seed)
    is the same exact array in FP32 and FP64: a quadratic loss seeded with
    2 (x_T - x*) would carry the FP32 quantisation of x_T (~3e-8 at |x| ~ 0.5)
    into a seed whose entries are themselves ~1e-6, i.e. percent-level noise
    before the adjoint even starts."""
    from ysim_b200 import generators as G
    from oracle import oracle as O
    c = spec.meshes[0]
    k, L = G.grid_spring_params(c.grid_n, c.grid_rest, (c.kstretch, c.kshear, c.kbend))
    rng = np.random.default_rng(seed)
    v0 = rng.normal(0, 0.02, (c.nV, 3)).astype(np.float32)
    w = (rng.normal(0, 1, (c.nV, 3)) / c.nV).astype(np.float32)
    R = O.Rollout(spec, k, L, v0=v0)
    return k, L, v0, w, R


# Windows on which the rollout is a smooth function of the parameters and the
# FP32 and FP64 forwards take the same branch at every step.  The contact
# response pushes a penetrating vertex out to the thickness along the contact
# normal and removes its approaching normal velocity, so on the next step that
# vertex is re-tested `d < thickness` with d on the boundary itself: FP32 and
# FP64 (and any finite-difference perturbation) pick "push again" or "release"
# by round-off, after which the rollouts are different branches of a
# piecewise-smooth map.  The contact window therefore ends at the first step
# with a push (found with the FP32 oracle, whose forward is bit-identical to
# the CUDA one); the contact-free window runs 40 steps of springs and
# integration alone.
WINDOWS = [pytest.param(0.5, False, id="contact_free_40"),
           pytest.param(0.2995, True, id="contacts_to_first_push")]


def _window(spec, v0, contacts):
    if not contacts:
        return 40
    from oracle import oracle as O
    S = O.OracleScene(spec)
    v = S.get("v")
    v[: len(v0)] = v0
    S.set("v", v)
    thickness = spec.meshes[0].thickness
    for t in range(1, 41):
        S.step(1)
        off, c = S.contacts()
        if (c["d"][: int(off[len(v0)])] < thickness).any():
            return t
    raise AssertionError("no contact push within 40 steps")


@pytest.mark.parametrize("height,contacts", WINDOWS)
def test_adjoint_matches_fp64_reference_and_fd(cuda_lib, height, contacts):
    import torch
    from ysim_b200.adjoint import ClothRollout
    spec = _small(height=height)
    k, L, v0, w, R = _problem(spec)
    T = _window(spec, v0, contacts)
    V = spec.meshes[0].nV
    w64 = w.astype(np.float64)
    # FP64 reference adjoint
    x64, ncontacts = R.forward(T, keep=True)
    assert (ncontacts > 0) == contacts
    gk64, gL64, gv64 = R.backward(T, w64)
    # CUDA adjoint through torch.autograd
    roll = ClothRollout(spec, steps=T, checkpoint_every=5)
    try:
        kt = torch.tensor(k, device="cuda", requires_grad=True)
        Lt = torch.tensor(L, device="cuda", requires_grad=True)
        vt = torch.tensor(v0, device="cuda", requires_grad=True)
        xT = roll(kt, Lt, vt)
        loss = (xT * torch.tensor(w, device="cuda")).sum()
        loss.backward()
        gk, gL, gv = kt.grad.cpu().numpy(), Lt.grad.cpu().numpy(), vt.grad.cpu().numpy()
        # FP32 rollout vs the FP64 one: round-off only on a branch-stable window
        assert np.abs(xT.detach().cpu().numpy() - x64).max() < 1e-6
        # FP32 adjoint vs FP64 adjoint, norm-relative per parameter group
        rels = {name: np.linalg.norm(g32 - g64) / max(np.linalg.norm(g64), 1e-30)
                for name, g32, g64 in (("k", gk, gk64), ("L", gL, gL64), ("v0", gv, gv64))}
        print("adjoint rel err", rels)
        assert max(rels.values()) < 1e-3, rels
        # FP64 central differences (step 1e-6 relative for k, 1e-6 absolute for L, v0)
        rng = np.random.default_rng(3)
        loss64 = lambda x: float((x * w64).sum())
        checks = []
        for _ in range(3):
            i = int(rng.integers(len(k)))
            eps = 1e-6 * float(k[i])
            kk = k.astype(np.float64).copy(); kk[i] += eps; R.set(kk, L); lp = loss64(R.forward(T)[0])
            kk[i] -= 2 * eps; R.set(kk, L); lm = loss64(R.forward(T)[0]); R.set(k, L)
            checks.append((gk[i], (lp - lm) / (2 * eps), np.abs(gk64).max()))
            i = int(rng.integers(len(L)))
            eps = 1e-6
            ll = L.astype(np.float64).copy(); ll[i] += eps; R.set(k, ll); lp = loss64(R.forward(T)[0])
            ll[i] -= 2 * eps; R.set(k, ll); lm = loss64(R.forward(T)[0]); R.set(k, L)
            checks.append((gL[i], (lp - lm) / (2 * eps), np.abs(gL64).max()))
            j = int(rng.integers(3 * V))
            vv = v0.reshape(-1).astype(np.float64).copy(); vv[j] += eps; R.set(v0=vv); lp = loss64(R.forward(T)[0])
            vv[j] -= 2 * eps; R.set(v0=vv); lm = loss64(R.forward(T)[0]); R.set(v0=v0.reshape(-1))
            checks.append((gv.reshape(-1)[j], (lp - lm) / (2 * eps), np.abs(gv64).max()))
        for g, fd, scale in checks:
            assert abs(g - fd) <= 1e-3 * scale + 1e-2 * abs(fd), (g, fd, scale)
    finally:
        roll.close()


def test_checkpoint_interval_does_not_change_gradients(cuda_lib):
    import torch
    from ysim_b200.adjoint import ClothRollout
    spec = _small()
    T = 24
    k, L, v0, w, _ = _problem(spec, seed=1)
    out = []
    for K in (1, 5, 24):
        roll = ClothRollout(spec, steps=T, checkpoint_every=K)
        try:
            kt = torch.tensor(k, device="cuda", requires_grad=True)
            Lt = torch.tensor(L, device="cuda", requires_grad=True)
            vt = torch.tensor(v0, device="cuda", requires_grad=True)
            loss = (roll(kt, Lt, vt) * torch.tensor(w, device="cuda")).sum()
            loss.backward()
            out.append((kt.grad.cpu().numpy(), Lt.grad.cpu().numpy(), vt.grad.cpu().numpy()))
        finally:
            roll.close()
    for o in out[1:]:
        for a, b in zip(out[0], o):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


# ---------------------------------------------------------------- 64-bit mode
def _f32_spec(spec):
    """The scene keeps its parameters in binary32; the FP64 reference is given
    the same values, so that both FP64 rollouts solve one problem."""
    import dataclasses
    r = lambda v: float(np.float32(v))
    p = spec.params
    spec.params = dataclasses.replace(p, subh=r(p.subh), kd=r(p.kd), kair=r(p.kair), margin=r(p.margin),
                                      radius=r(p.radius), gravity=tuple(r(g) for g in p.gravity))
    spec.meshes[0].thickness = r(spec.meshes[0].thickness)
    return spec


def _roll64(spec, k, L, v0, T, K=5, tree_layout=None):
    import torch
    from ysim_b200.adjoint import ClothRollout
    roll = ClothRollout(spec, steps=T, checkpoint_every=K, precision=64, tree_layout=tree_layout)
    t = [torch.tensor(np.asarray(a, np.float64), device="cuda", requires_grad=True) for a in (k, L, v0)]
    return roll, t


# Bit-for-bit agreement holds on any window, pushes and releases included:
# both FP64 rollouts take the same branch at every test because they compute
# the same binary64 values.
@pytest.mark.parametrize("height,T,layout", [(0.5, 40, None), (0.2995, 60, None), (0.2995, 25, None),
                                              (0.2995, 60, 0)],
                         ids=["contact_free_40", "contacts_60_pushes", "contacts_25", "contacts_60_reference_tree"])
def test_fp64_adjoint_matches_fp64_reference_bit_for_bit(cuda_lib, height, T, layout):
    """The contact search descends the scene's float tree of the obstacle, in
    the cube layout (default) or the reference's layout."""
    import torch
    spec = _f32_spec(_small(height=height))
    k, L, v0, w, R = _problem(spec)
    w64 = w.astype(np.float64)
    x64, ncontacts = R.forward(T, keep=True)
    assert (ncontacts > 0) == (height < 0.4)
    gk64, gL64, gv64 = R.backward(T, w64)
    roll, (kt, Lt, vt) = _roll64(spec, k, L, v0, T, K=7, tree_layout=layout)
    try:
        xT = roll(kt, Lt, vt)
        assert xT.dtype == torch.float64
        assert np.array_equal(xT.detach().cpu().numpy(), x64)
        (xT * torch.tensor(w64, device="cuda")).sum().backward()
        assert np.array_equal(kt.grad.cpu().numpy(), gk64)
        assert np.array_equal(Lt.grad.cpu().numpy(), gL64)
        assert np.array_equal(vt.grad.cpu().numpy(), gv64)
    finally:
        roll.close()


@pytest.mark.parametrize("height,contacts", WINDOWS)
def test_fp64_adjoint_within_1e4_of_fp64_finite_differences(cuda_lib, height, contacts):
    """Central differences of the GPU's own FP64 rollout, per parameter group
    at the step that balances truncation against round-off (k: 1e-3
    relative; L: 1e-6; v0: 1e-5), on the largest and on random components.
    Each must agree with the adjoint to 1e-4 relative, |g - fd| / |fd|,
    where |fd| is at least 1e-4 of the group's largest gradient and a
    thousand times the difference's own round-off; below either floor the
    error is taken relative to that floor instead."""
    import torch
    spec = _f32_spec(_small(height=height))
    k, L, v0, w, _ = _problem(spec)
    T = _window(spec, v0, contacts)
    w64 = torch.tensor(w.astype(np.float64), device="cuda")
    roll, (kt, Lt, vt) = _roll64(spec, k, L, v0, T)
    try:
        (roll(kt, Lt, vt) * w64).sum().backward()
        grads = [kt.grad.cpu().numpy().reshape(-1), Lt.grad.cpu().numpy().reshape(-1), vt.grad.cpu().numpy().reshape(-1)]
        base = [t.detach().clone().reshape(-1) for t in (kt, Lt, vt)]

        def loss(group, i, delta):
            p = [b.clone() for b in base]
            p[group][i] += delta
            with torch.no_grad():
                return float((roll(p[0], p[1], p[2].reshape(-1, 3)) * w64).sum())

        rng = np.random.default_rng(7)
        worst, n_rel = 0.0, 0
        for group, g in enumerate(grads):
            gmax = float(np.abs(g).max())
            idx = list(np.argsort(-np.abs(g))[:3]) + list(rng.integers(len(g), size=3))
            for i in idx:
                eps = 1e-3 * abs(float(base[0][i])) if group == 0 else (1e-6 if group == 1 else 1e-5)
                lp, lm = loss(group, int(i), eps), loss(group, int(i), -eps)
                fd = (lp - lm) / (2 * eps)
                noise = 64 * np.finfo(np.float64).eps * (abs(lp) + abs(lm)) / (2 * eps)
                floor = max(1e-4 * gmax, 1e3 * noise)
                err = abs(g[i] - fd) / max(abs(fd), floor)
                assert err <= 1e-4, (group, int(i), g[i], fd, floor, err)
                if abs(fd) >= floor:
                    worst = max(worst, err)
                    n_rel += 1
        assert n_rel >= 9  # at least the three largest of each group
        print("fp64 adjoint vs fp64 fd, worst relative error", worst, "over", n_rel, "components")
    finally:
        roll.close()


def test_fp64_mode_float_entry_points_and_checkpoints(cuda_lib):
    """Float tensors through the 64-bit mode give the binary64 results
    rounded; checkpoint intervals leave the binary64 gradients unchanged."""
    import torch
    spec = _f32_spec(_small())
    T = 24
    k, L, v0, w, R = _problem(spec, seed=1)
    x64, _ = R.forward(T, keep=True)
    g64 = R.backward(T, w.astype(np.float64))
    from ysim_b200.adjoint import ClothRollout
    roll = ClothRollout(spec, steps=T, checkpoint_every=5, precision=64)
    try:
        kt, Lt, vt = (torch.tensor(a, device="cuda", requires_grad=True) for a in (k, L, v0))
        xT = roll(kt, Lt, vt)
        assert xT.dtype == torch.float32
        assert np.array_equal(xT.detach().cpu().numpy(), x64.astype(np.float32))
        (xT * torch.tensor(w, device="cuda")).sum().backward()
        for got, want in zip((kt.grad, Lt.grad, vt.grad), g64):
            assert np.array_equal(got.cpu().numpy(), want.astype(np.float32))
    finally:
        roll.close()
    out = []
    for K in (1, 24):
        roll, (kt, Lt, vt) = _roll64(spec, k, L, v0, T, K=K)
        try:
            (roll(kt, Lt, vt) * torch.tensor(w.astype(np.float64), device="cuda")).sum().backward()
            out.append([t.grad.cpu().numpy() for t in (kt, Lt, vt)])
        finally:
            roll.close()
    for a, b, c in zip(out[0], out[1], g64):
        assert np.array_equal(a, b) and np.array_equal(a, c)
