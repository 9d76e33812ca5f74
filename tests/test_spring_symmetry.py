"""The arithmetic behind the tile thread order's shared springs, in IEEE
float32 on the host: the stencil spring of calc_spring (physics.metal:146-153)
evaluated from its second end is the exact negation of its value from the
first end, except in two cases where both ends compute the same bits:

* a component whose dx is exactly zero (the unit vector's component is +0
  from either end, so the product keeps the sign of the scalar factor);
* a degenerate spring (length below 1e-7: +0 from both ends).

The fused kernel's tile table stores one evaluation per spring with flags for
those cases; this test checks the rule on random springs, springs with equal
coordinates, springs at rest with zero relative velocity (a zero scalar
factor: signed-zero forces) and degenerate springs."""
import numpy as np

F32 = np.float32


def _spring(p0, v0, p1, v1, rest, ks, kd):
    """calc_spring in float32, one operation at a time (no fused multiply-add):
    the order of the kernel's f3 helpers."""
    dx = (p1 - p0).astype(F32)
    dv = (v1 - v0).astype(F32)
    d2 = F32(F32(F32(dx[0] * dx[0]) + F32(dx[1] * dx[1])) + F32(dx[2] * dx[2]))
    ln = F32(np.sqrt(d2))
    if ln < F32(1e-7):
        return np.zeros(3, F32)
    nd = (dx / ln).astype(F32)
    dvn = F32(F32(F32(dv[0] * nd[0]) + F32(dv[1] * nd[1])) + F32(dv[2] * nd[2]))
    s = F32(F32(F32(ks) * F32(ln - F32(rest))) + F32(F32(kd) * dvn))
    return (nd * s).astype(F32)


def _shared(fa, p0, p1):
    """The second end's value from the first end's, by the table's rule."""
    dx = (p1 - p0).astype(F32)
    d2 = F32(F32(F32(dx[0] * dx[0]) + F32(dx[1] * dx[1])) + F32(dx[2] * dx[2]))
    if F32(np.sqrt(d2)) < F32(1e-7):
        return fa.copy()
    return np.where(dx == F32(0), fa, -fa).astype(F32)


def _bits(a):
    return np.asarray(a, F32).view(np.uint32)


def test_shared_spring_is_the_second_ends_own_value():
    rng = np.random.default_rng(7)
    cases = 0
    for it in range(4000):
        p0 = rng.uniform(-1, 1, 3).astype(F32)
        p1 = (p0 + rng.normal(0, 0.01, 3)).astype(F32)
        v0 = rng.normal(0, 0.1, 3).astype(F32)
        v1 = rng.normal(0, 0.1, 3).astype(F32)
        kind = it % 5
        if kind == 1:  # equal coordinates: dx exactly zero on some axes
            ax = rng.integers(0, 3, size=rng.integers(1, 3))
            p1[ax] = p0[ax]
        elif kind == 2:  # at rest, no relative velocity: a zero scalar factor, signed-zero forces
            v1 = v0.copy()
            ax = rng.integers(0, 3)
            p1[ax] = p0[ax]
        elif kind == 3:  # degenerate
            p1 = (p0 + rng.normal(0, 1e-9, 3)).astype(F32)
        rest = F32(np.sqrt(np.sum((p1.astype(np.float64) - p0) ** 2))) if kind == 2 else F32(rng.uniform(0, 0.02))
        ks, kd = F32(rng.uniform(1, 1e3)), F32(rng.uniform(0, 1))
        fa = _spring(p0, v0, p1, v1, rest, ks, kd)
        fb = _spring(p1, v1, p0, v0, rest, ks, kd)
        assert np.array_equal(_bits(_shared(fa, p0, p1)), _bits(fb)), (it, fa, fb)
        cases += int(np.any(fa == 0))
    assert cases > 100  # signed zeros were exercised


def test_plain_negation_would_flip_zero_signs():
    """Without the flags, the second end would get the opposite zero sign on
    an axis with dx = 0: visible when its running force sum is -0."""
    p0 = np.array([0.0, 0.5, 0.25], F32)
    p1 = np.array([0.01, 0.5, 0.25], F32)  # dy = dz = 0
    v = np.zeros(3, F32)
    rest = F32(0.005)  # stretched: s > 0
    fa = _spring(p0, v, p1, v, rest, F32(1e3), F32(0.5))
    fb = _spring(p1, v, p0, v, rest, F32(1e3), F32(0.5))
    assert fa[1] == 0 and fb[1] == 0
    assert _bits(fb)[1] == _bits(fa)[1] != _bits(-fa)[1]
    minus0 = np.array([-0.0], F32)
    assert _bits(minus0 + fb[1:2]) != _bits(minus0 + (-fa)[1:2])
