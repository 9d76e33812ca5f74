"""The adjoint on the C5 configuration at its full size: FastGridCloth
128x128 (16,384 vertices, 97,026 springs) over a level-4 icosphere, 200 steps
at subh 1/600 with obstacle contact, checkpoints every 20; loss = mean
|x_T - x*|^2, x* the final state of a rollout whose per-spring stiffness is
k exp(N(0, 0.3^2)).

* The 64-bit mode against the FP64 CPU adjoint (oracle/ys_adjoint_oracle.cpp)
  on the whole 200-step problem: trajectory and all three gradients bit for
  bit, pushes and releases included (both compute the same binary64 values,
  so they take the same branch at every contact test).
* The 64-bit mode against FP64 central differences of its own rollout on the
  longest branch-stable prefix (the steps before the first contact push; the
  push re-tests a vertex exactly at the thickness on the next step, where
  any perturbation picks a branch by round-off): 64 random components and the
  three largest of each parameter group.
* The FP32 adjoint against the 64-bit one on that prefix, norm-relative per
  parameter group.
"""
import numpy as np
import pytest

from test_gpu_adjoint import _f32_spec

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

STEPS, EVERY = 200, 20


@pytest.fixture(scope="module")
def c5(cuda_lib, oracle):
    """(spec, k, L, v0, x*_T for T = 200 and for the prefix, prefix length)."""
    from ysim_b200 import generators as G
    spec = _f32_spec(G.config_c5())
    c = spec.meshes[0]
    k, L = G.grid_spring_params(c.grid_n, c.grid_rest, (c.kstretch, c.kshear, c.kbend))
    rng = np.random.default_rng(5)
    kstar = (k * np.exp(rng.normal(0.0, 0.3, k.shape))).astype(np.float32)
    v0 = np.zeros((c.nV, 3), np.float32)
    # first step whose contact response pushes a vertex (FP32 oracle, whose
    # forward is bit-identical to the CUDA one)
    S = oracle.OracleScene(spec)
    push = None
    for t in range(1, STEPS + 1):
        S.step(1)
        off, cc = S.contacts()
        if (cc["d"][: int(off[c.nV])] < c.thickness).any():
            push = t
            break
    assert push is not None and push > 20, push
    prefix = push - 1
    R = oracle.Rollout(spec, kstar, L, v0=v0)
    xs_full = R.forward(STEPS)[0]
    xs_prefix = R.forward(prefix)[0]
    return spec, k, L, v0, xs_full, xs_prefix, prefix


def _mse_seed(xT, xs):
    """d/dx_T of mean_i |x_T,i - x*_i|^2, in binary64."""
    return 2.0 * (np.asarray(xT, np.float64) - xs) / len(xs)


def test_c5_fp64_adjoint_bit_identical_to_fp64_reference(c5, oracle):
    import torch
    from ysim_b200.adjoint import ClothRollout
    spec, k, L, v0, xs, _, _ = c5
    R = oracle.Rollout(spec, k, L, v0=v0)
    x64, ncontacts = R.forward(STEPS, keep=True)
    assert ncontacts > 0
    seed = _mse_seed(x64, xs)
    gk64, gL64, gv64 = R.backward(STEPS, seed)
    roll = ClothRollout(spec, steps=STEPS, checkpoint_every=EVERY, precision=64)
    try:
        kt, Lt, vt = (torch.tensor(np.asarray(a, np.float64), device="cuda", requires_grad=True) for a in (k, L, v0))
        xT = roll(kt, Lt, vt)
        assert np.array_equal(xT.detach().cpu().numpy(), x64)
        xT.backward(torch.tensor(seed, device="cuda"))
        assert np.array_equal(kt.grad.cpu().numpy(), gk64)
        assert np.array_equal(Lt.grad.cpu().numpy(), gL64)
        assert np.array_equal(vt.grad.cpu().numpy(), gv64)
        assert np.abs(gk64).max() > 0 and np.abs(gv64).max() > 0
    finally:
        roll.close()


def test_c5_fp64_adjoint_within_1e4_of_finite_differences(c5):
    """Central differences of the GPU's FP64 rollout on the branch-stable
    prefix, Richardson-extrapolated from steps h and h/2 (truncation error of
    order h^4), h per group balancing truncation against round-off (k: 1e-3
    relative, L: 1e-6, v0: 1e-5).  |g - fd| / |fd| <= 1e-4, where |fd| is at
    least 1e-4 of the group's largest gradient and ten times the difference's
    round-off; below either floor the error is taken relative to that floor.
    The round-off is that of the final positions (each rollout rounds x_T to
    binary64, and the perturbations move it by only a few thousand ulps for
    the smallest components): 64 eps sum_i |dL/dx_i| |x_i| per step h/2."""
    import torch
    from ysim_b200.adjoint import ClothRollout
    spec, k, L, v0, _, xs, T = c5
    xs_t = torch.tensor(xs, device="cuda")
    roll = ClothRollout(spec, steps=T, checkpoint_every=EVERY, precision=64)
    try:
        params = [torch.tensor(np.asarray(a, np.float64), device="cuda", requires_grad=True) for a in (k, L, v0)]
        xT = roll(*params)
        ((xT - xs_t) ** 2).sum(1).mean().backward()
        grads = [p.grad.cpu().numpy().reshape(-1) for p in params]
        xT = xT.detach().cpu().numpy()
        sens = float((np.abs(_mse_seed(xT, xs)) * np.abs(xT)).sum())  # sum_i |dL/dx_i| |x_i|
        base = [p.detach().clone().reshape(-1) for p in params]

        def loss(group, i, delta):
            p = [b.clone() for b in base]
            p[group][i] += delta
            with torch.no_grad():
                return float(((roll(p[0], p[1], p[2].reshape(-1, 3)) - xs_t) ** 2).sum(1).mean())

        rng = np.random.default_rng(11)
        worst, n_rel, n = 0.0, 0, 0
        for group, g in enumerate(grads):
            gmax = float(np.abs(g).max())
            idx = list(np.argsort(-np.abs(g))[:3]) + list(rng.integers(len(g), size=22 if group < 2 else 20))
            for i in idx:
                i = int(i)
                eps = 1e-3 * abs(float(base[0][i])) if group == 0 else (1e-6 if group == 1 else 1e-5)
                lp, lm = loss(group, i, eps), loss(group, i, -eps)
                hp, hm = loss(group, i, eps / 2), loss(group, i, -eps / 2)
                fd = (4.0 * (hp - hm) / eps - (lp - lm) / (2 * eps)) / 3.0
                noise = 64 * np.finfo(np.float64).eps * sens / (eps / 2)
                floor = max(1e-4 * gmax, 10 * noise)
                err = abs(g[i] - fd) / max(abs(fd), floor)
                assert err <= 1e-4, (group, i, g[i], fd, floor, err)
                n += 1
                if abs(fd) >= floor:
                    worst = max(worst, err)
                    n_rel += 1
        assert n == 73 and n_rel >= 9
        print(f"C5 prefix of {T} steps: worst |g - fd| / |fd| {worst:.2e} over {n_rel} of {n} components")
    finally:
        roll.close()


def test_c5_fp32_adjoint_tracks_fp64_on_the_prefix(c5):
    """The FP32 adjoint differentiates the FP32 rollout; on the branch-stable
    prefix its gradients agree with the 64-bit mode's (norm-relative, per
    group) to 1e-4 for v0, 1e-3 for L and 1e-2 for k.  The k gradient is a
    sum of adjoint-weighted strains |d| - L of the FP32 trajectory, whose
    positions differ from the binary64 ones by some 1e-7 while the strains
    are ~1e-5: that, not the reverse pass's own arithmetic, bounds it (the
    64-bit mode meets 1e-4 against finite differences).  Both reverse passes
    take the same seed, the loss gradient of the binary64 rollout (rounded to
    binary32 for the FP32 pass): in the first steps x_T - x* is a few ulps of
    x_T in binary32, so a seed formed from the FP32 state would be mostly its
    rounding."""
    import torch
    from ysim_b200.adjoint import ClothRollout
    spec, k, L, v0, _, xs, T = c5
    out, seed = {}, None
    for prec, dt in ((64, torch.float64), (32, torch.float32)):
        roll = ClothRollout(spec, steps=T, checkpoint_every=EVERY, precision=prec)
        try:
            params = [torch.tensor(np.asarray(a), dtype=dt, device="cuda", requires_grad=True) for a in (k, L, v0)]
            xT = roll(*params)
            if seed is None:
                seed = _mse_seed(xT.detach().cpu().numpy(), xs)
            xT.backward(torch.tensor(seed, dtype=dt, device="cuda"))
            out[prec] = [p.grad.double().cpu().numpy() for p in params]
        finally:
            roll.close()
    rels = {name: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
            for name, a, b in zip(("k", "L", "v0"), out[32], out[64])}
    print("C5 prefix FP32 vs FP64 adjoint, norm-relative:", rels)
    assert rels["v0"] < 1e-4 and rels["L"] < 1e-3 and rels["k"] < 1e-2, rels
