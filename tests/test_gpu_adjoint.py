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


def _problem(spec, T, seed=0):
    import torch
    from ysim_b200 import generators as G
    from oracle import oracle as O
    c = spec.meshes[0]
    k, L = G.grid_spring_params(c.grid_n, c.grid_rest, (c.kstretch, c.kshear, c.kbend))
    rng = np.random.default_rng(seed)
    kt = (k * np.exp(rng.normal(0, 0.3, len(k)))).astype(np.float64)
    v0 = rng.normal(0, 0.02, (c.nV, 3)).astype(np.float32)
    R = O.Rollout(spec, kt, L, v0=v0)
    xstar, _ = R.forward(T)
    R.set(k, L)
    return k, L, v0, xstar, R


def test_adjoint_matches_fp64_reference_and_fd(cuda_lib):
    import torch
    from ysim_b200.adjoint import ClothRollout
    spec = _small()
    T = 40
    k, L, v0, xstar, R = _problem(spec, T)
    V = spec.meshes[0].nV
    # FP64 reference adjoint
    x64, ncontacts = R.forward(T, keep=True)
    assert ncontacts > 0
    gk64, gL64, gv64 = R.backward(T, 2.0 * (x64 - xstar) / V)
    # CUDA adjoint through torch.autograd
    roll = ClothRollout(spec, steps=T, checkpoint_every=10)
    try:
        kt = torch.tensor(k, device="cuda", requires_grad=True)
        Lt = torch.tensor(L, device="cuda", requires_grad=True)
        vt = torch.tensor(v0, device="cuda", requires_grad=True)
        xT = roll(kt, Lt, vt)
        target = torch.tensor(xstar, dtype=torch.float32, device="cuda")
        loss = ((xT - target) ** 2).sum(1).mean()
        loss.backward()
        gk, gL, gv = kt.grad.cpu().numpy(), Lt.grad.cpu().numpy(), vt.grad.cpu().numpy()
        # FP32 rollout vs the FP64 one: round-off only (40 steps, with contacts)
        assert np.abs(xT.detach().cpu().numpy() - x64).max() < 5e-4
        for g32, g64 in ((gk, gk64), (gL, gL64), (gv, gv64)):
            rel = np.linalg.norm(g32 - g64) / max(np.linalg.norm(g64), 1e-30)
            assert rel < 1e-3, rel
        # FP64 central differences on a few parameters (eps 1e-6)
        rng = np.random.default_rng(3)
        loss64 = lambda x: float(((x - xstar) ** 2).sum(1).mean())
        eps = 1e-6
        checks = []
        for _ in range(3):
            i = int(rng.integers(len(k)))
            kk = k.astype(np.float64).copy(); kk[i] += eps; R.set(kk, L); lp = loss64(R.forward(T)[0])
            kk[i] -= 2 * eps; R.set(kk, L); lm = loss64(R.forward(T)[0]); R.set(k, L)
            checks.append((gk[i], (lp - lm) / (2 * eps)))
            j = int(rng.integers(3 * V))
            vv = v0.reshape(-1).astype(np.float64).copy(); vv[j] += eps; R.set(v0=vv); lp = loss64(R.forward(T)[0])
            vv[j] -= 2 * eps; R.set(v0=vv); lm = loss64(R.forward(T)[0]); R.set(v0=v0.reshape(-1))
            checks.append((gv.reshape(-1)[j], (lp - lm) / (2 * eps)))
        scale = max(abs(fd) for _, fd in checks)
        for g, fd in checks:
            assert abs(g - fd) <= 1e-3 * scale + 1e-3 * abs(fd), (g, fd)
    finally:
        roll.close()


def test_checkpoint_interval_does_not_change_gradients(cuda_lib):
    import torch
    from ysim_b200.adjoint import ClothRollout
    spec = _small()
    T = 24
    k, L, v0, xstar, _ = _problem(spec, T, seed=1)
    out = []
    for K in (1, 5, 24):
        roll = ClothRollout(spec, steps=T, checkpoint_every=K)
        try:
            kt = torch.tensor(k, device="cuda", requires_grad=True)
            Lt = torch.tensor(L, device="cuda", requires_grad=True)
            vt = torch.tensor(v0, device="cuda", requires_grad=True)
            loss = ((roll(kt, Lt, vt) - torch.tensor(xstar, dtype=torch.float32, device="cuda")) ** 2).sum(1).mean()
            loss.backward()
            out.append((kt.grad.cpu().numpy(), Lt.grad.cpu().numpy(), vt.grad.cpu().numpy()))
        finally:
            roll.close()
    for o in out[1:]:
        for a, b in zip(out[0], o):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
