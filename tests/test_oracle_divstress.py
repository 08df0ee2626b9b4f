"""The oracle's divstress_uv / divstress_w (107_divstress.f90:4-104) against closed forms.

Band-limited trigonometric stresses have exact spectral x and y derivatives, and the
vertical terms are the reference's one-sided differences of the level values, so the
whole divergence has a closed form at every grid point: this pins the restatement
(levels, roles, pads and BOGUS planes) independently of its own ddx/ddy/ddz.
"""
import numpy as np
import pytest

BOGUS = -1234567890.0   # 001_param.f90:40
DOM = dict(lx_tot=2 * np.pi * 1000.0, ly_tot=2 * np.pi * 1000.0, lz_tot=1000.0, z_i=1000.0, dt=0.5)


def _grid(orc, nx, ny, nzt):
    return orc.Grid(nx, ny, nzt, **DOM)


def _case(g):
    x = np.arange(g.ldx)[:, None, None] * (2 * np.pi / g.nxt)
    y = np.arange(g.nyt)[None, :, None] * (2 * np.pi / g.nyt)
    z = np.arange(g.nz + 1)[None, None, :] * g.dz
    kx0, ky0 = 2 * np.pi / g.lx, 2 * np.pi / g.ly
    F = lambda a: np.asfortranarray(np.broadcast_to(a, (g.ldx, g.nyt, g.nz + 1)).copy())
    tx = F(np.sin(3 * x + 0.2) * np.cos(2 * y) * (1 + z / 100))
    ty = F(np.cos(x - 0.4) * np.sin(3 * y + 0.1) * np.exp(-z / 300))
    tz = F((np.sin(2 * x) * np.cos(y) + 0.5) * (z / 50) ** 2)
    dtx = F(3 * kx0 * np.cos(3 * x + 0.2) * np.cos(2 * y) * (1 + z / 100))
    dty = F(3 * ky0 * np.cos(x - 0.4) * np.cos(3 * y + 0.1) * np.exp(-z / 300))
    for a in (tx, ty, tz):
        a[g.nxt:] = 1e3   # the reference reads only x < nxt of its inputs
    return tx, ty, tz, dtx + dty


@pytest.mark.parametrize("nx,ny,nzt", [(16, 12, 9), (32, 48, 17), (24, 16, 5)])
def test_divstress_uv_closed_form(orc, nx, ny, nzt):
    g = _grid(orc, nx, ny, nzt)
    tx, ty, tz, dh = _case(g)
    out = g.divstress_uv(tx, ty, tz)
    nz, n = g.nz, g.nxt
    # levels 1..nz-1 take ddz_w: (tz(k+1) - tz(k))/dz
    exp = dh[:n, :, 1:nz] + (tz[:n, :, 2:nz + 1] - tz[:n, :, 1:nz]) / g.dz
    scale = np.abs(exp).max()
    assert np.abs(out[:n, :, 1:nz] - exp).max() <= 1e-12 * scale
    assert np.all(out[n:, :, 1:nz] == 0.0)
    assert np.all(out[:, :, 0] == BOGUS) and np.all(out[:, :, nz] == BOGUS)


@pytest.mark.parametrize("nx,ny,nzt", [(16, 12, 9), (32, 48, 17), (24, 16, 5)])
def test_divstress_w_closed_form(orc, nx, ny, nzt):
    g = _grid(orc, nx, ny, nzt)
    tx, ty, tz, dh = _case(g)
    out = g.divstress_w(tx, ty, tz)
    nz, n = g.nz, g.nxt
    exp = dh[:n].copy()
    # levels 2..nz-1 take ddz_uv: (tz(k) - tz(k-1))/dz; the wall level 1 and the top
    # level nz none (coordz == 0 and coordz == npz-1 both hold on one rank)
    exp[:, :, 2:nz] += (tz[:n, :, 2:nz] - tz[:n, :, 1:nz - 1]) / g.dz
    scale = np.abs(exp[:, :, 1:]).max()
    assert np.abs(out[:n, :, 1:] - exp[:, :, 1:]).max() <= 1e-12 * scale
    assert np.all(out[n:, :, 1:] == 0.0)
    assert np.all(out[:, :, 0] == BOGUS)


def test_divstress_is_linear(orc):
    g = _grid(orc, 16, 12, 9)
    rng = np.random.default_rng(4)
    a = [np.asfortranarray(rng.standard_normal((g.ldx, g.nyt, g.nz + 1))) for _ in range(6)]
    for op in (g.divstress_uv, g.divstress_w):
        s = op(*[x + 2.0 * y for x, y in zip(a[:3], a[3:])])
        p, q = op(*a[:3]), op(*a[3:])
        lv = slice(1, g.nz) if op == g.divstress_uv else slice(1, g.nz + 1)
        assert np.abs(s[:, :, lv] - (p[:, :, lv] + 2.0 * q[:, :, lv])).max() <= 1e-12 * np.abs(s[:, :, lv]).max()
