"""The oracle's rollout problem and its transposes (CPU).

The transposes in obl_oracle_adj.c are written as explicit transposed operators; these
tests pin them against the forward operators they transpose:

* the projection P is linear: <P x, y> = <x, P^T y>;
* convec is quadratic and the rollout step F is quadratic in the state, so the central
  difference (F(s+d) - F(s-d))/2 equals the tangent F'(s) d exactly (up to rounding)
  for any d: <(F(s+d) - F(s-d))/2, l> = <d, F'(s)^T l>;
* the rollout gradient of J against central finite differences (eps = 1e-4).
"""
import numpy as np
import pytest

from overlappingbls_b200.fields import DOMAIN, make_fields

NX, NY, NZT = 16, 12, 17


def grid(orc, nx=NX, ny=NY, nzt=NZT, stress_free=False):
    return orc.Grid(nx, ny, nzt, **DOMAIN, ubc_stress_free=stress_free)


def rnd(g, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    f = g.field()
    f[: g.nxt] = scale * rng.standard_normal(f[: g.nxt].shape)
    return f


def dot(g, a, b):
    return sum(float(np.sum(x[: g.nxt] * y[: g.nxt])) for x, y in zip(a, b))


def state(g):
    f = make_fields(g.nxt, g.nyt, g.nzt, lz_tot=DOMAIN["lz_tot"], with_theta=False)
    return [f["u"], f["v"], f["w"]]


@pytest.mark.parametrize("stress_free", [False, True])
def test_projection_transpose(orc, stress_free):
    g = grid(orc, stress_free=stress_free)
    x = [rnd(g, s) for s in (1, 2, 3)]
    y = [rnd(g, s) for s in (4, 5, 6)]
    px = g.projection(*x)
    pty = g.projection_vjp(*y)
    lhs, rhs = dot(g, px, y), dot(g, x, pty)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0), (lhs, rhs)


def test_convec_transpose(orc):
    g = grid(orc)
    s = state(g)
    d = [rnd(g, k, 0.1) for k in (11, 12, 13)]
    lc = [rnd(g, k) for k in (14, 15, 16)]
    for a in lc:
        a[:, :, 0] = 0.0
        a[:, :, g.nz] = 0.0
    cp = g.convec(*[a + b for a, b in zip(s, d)])
    cm = g.convec(*[a - b for a, b in zip(s, d)])
    tang = [0.5 * (p - m) for p, m in zip(cp, cm)]
    adj = g.convec_vjp(*s, *lc)
    lhs, rhs = dot(g, tang, lc), dot(g, d, adj)
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs), (lhs, rhs)


@pytest.mark.parametrize("stress_free", [False, True])
def test_step_transpose(orc, stress_free):
    g = grid(orc, stress_free=stress_free)
    s = state(g)
    d = [rnd(g, k, 0.1) for k in (21, 22, 23)]
    lam = [rnd(g, k) for k in (24, 25, 26)]
    fp = g.rollout_step(*[a + b for a, b in zip(s, d)])
    fm = g.rollout_step(*[a - b for a, b in zip(s, d)])
    tang = [0.5 * (p - m) for p, m in zip(fp, fm)]
    adj = g.rollout_step_vjp(*s, *lam)
    lhs, rhs = dot(g, tang, lam), dot(g, d, adj)
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs), (lhs, rhs)


def test_step_is_not_a_bare_projection(orc):
    g = grid(orc)
    s = state(g)
    a = g.rollout_step(*s)
    b = g.projection(*s)
    diff = max(float(np.abs(x[: g.nxt] - y[: g.nxt]).max()) for x, y in zip(a, b))
    assert diff > 1e-4


def test_ke_band_gradient(orc):
    g = grid(orc)
    s = state(g)
    J, lam = g.ke_band(*s, 0.0, 300.0, grad=True)
    assert J > 0
    d = [rnd(g, k) for k in (31, 32, 33)]
    eps = 1e-3
    Jp = g.ke_band(*[a + eps * b for a, b in zip(s, d)], 0.0, 300.0)
    Jm = g.ke_band(*[a - eps * b for a, b in zip(s, d)], 0.0, 300.0)
    fd = (Jp - Jm) / (2 * eps)
    assert abs(fd - dot(g, lam, d)) <= 1e-9 * abs(fd)


def test_rollout_gradient_fd(orc):
    g = grid(orc)
    s = state(g)
    nsteps, zlo, zhi = 3, 0.0, 300.0
    J, grad = g.rollout_grad(nsteps, *s, zlo, zhi)
    eps = 1e-4
    for k in range(4):
        d = [rnd(g, 100 + 3 * k + i) for i in range(3)]
        Jp = g.rollout_grad(nsteps, *[a + eps * b for a, b in zip(s, d)], zlo, zhi, grad=False)
        Jm = g.rollout_grad(nsteps, *[a - eps * b for a, b in zip(s, d)], zlo, zhi, grad=False)
        fd = (Jp - Jm) / (2 * eps)
        gd = dot(g, grad, d)
        assert abs(fd - gd) <= 1e-6 * abs(gd), (k, fd, gd)
