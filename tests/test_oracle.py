"""CPU tests of the FP64 oracle: FFT accuracy, analytic known answers and the
reference's own invariants (these pin the oracle; the reference ships no tests)."""
import numpy as np
import pytest

from conftest import rel_l2

DOM = dict(lx_tot=2 * np.pi * 1000.0, ly_tot=2 * np.pi * 1000.0, lz_tot=1000.0, z_i=1000.0, dt=0.5)


@pytest.mark.parametrize("n", [8, 12, 16, 18, 24, 32, 48, 64, 96, 100, 128, 144, 192, 7, 9, 15])
def test_fft_vs_naive_long_double(orc, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for sign in (-1, 1):
        assert rel_l2(orc.fft_c2c(x, sign), orc.dft_naive(x, sign)) < 1e-14
    assert rel_l2(orc.fft_c2c(x, -1), np.fft.fft(x)) < 1e-14
    r = rng.standard_normal(n)
    assert rel_l2(orc.fft_r2c(r), np.fft.rfft(r)) < 1e-14
    if n % 2 == 0:
        assert rel_l2(orc.fft_c2r(np.fft.rfft(r), n), r * n) < 1e-14


def test_c2r_ignores_imag_of_dc_and_nyquist(orc):
    # FFTW's c2r discards Im X[0] and Im X[n/2]; the reference's ifftn relies on it
    rng = np.random.default_rng(3)
    c = rng.standard_normal(9) + 1j * rng.standard_normal(9)
    c2 = c.copy()
    c2[0] = c2[0].real
    c2[-1] = c2[-1].real
    assert np.allclose(orc.fft_c2r(c, 16), orc.fft_c2r(c2, 16), atol=1e-13)


def _grid(orc, nx=16, ny=12, nzt=9, **kw):
    d = dict(DOM)
    d.update(kw)
    return orc.Grid(nx, ny, nzt, **d)


def test_ddx_ddy_known_answer(orc):
    g = _grid(orc)
    x = np.arange(g.ldx)[:, None, None] * (2 * np.pi / g.nxt)
    y = np.arange(g.nyt)[None, :, None] * (2 * np.pi / g.nyt)
    f = np.asfortranarray(np.broadcast_to(np.sin(3 * x) * np.cos(2 * y), (g.ldx, g.nyt, g.nz + 1)).copy())
    kx0, ky0 = 2 * np.pi / g.lx, 2 * np.pi / g.ly
    ex = (3 * kx0 * np.cos(3 * x) * np.cos(2 * y))[: g.nxt]
    ey = (-2 * ky0 * np.sin(3 * x) * np.sin(2 * y))[: g.nxt]
    assert np.abs(g.ddx(f)[: g.nxt] - ex).max() < 1e-12
    assert np.abs(g.ddy(f)[: g.nxt] - ey).max() < 1e-12


def test_ddx_kills_nyquist(orc):
    g = _grid(orc)
    x = np.arange(g.ldx)[:, None, None]
    f = np.asfortranarray(np.broadcast_to(np.cos(np.pi * x) + 0.0, (g.ldx, g.nyt, g.nz + 1)).copy())
    assert np.abs(g.ddx(f)[: g.nxt]).max() < 1e-12


def test_zero_padding_interpolates_band_limited(orc):
    g = _grid(orc)
    X = lambda n: np.arange(n)[:, None] * (2 * np.pi / n)
    Y = lambda n: np.arange(n)[None, :] * (2 * np.pi / n)
    f = lambda xx, yy: 1.0 + np.sin(2 * xx + 0.3) * np.cos(3 * yy) + 0.5 * np.cos(5 * xx - yy)
    var = np.zeros((g.ldx, g.nyt), order="F")
    var[: g.nxt] = f(X(g.nxt), Y(g.nyt))
    big = g.zero_padding(var)
    assert np.abs(big - f(X(g.nxt2), Y(g.nyt2))).max() < 1e-12
    back = g.zero_unpadding(big)
    assert np.abs(back[: g.nxt] - var[: g.nxt]).max() < 1e-12
    assert np.array_equal(back[g.nxt:], back[:2])  # 108_01_padd.f90:195


def test_fftn_ifftn_round_trip_removes_nyquist(orc):
    g = _grid(orc)
    rng = np.random.default_rng(0)
    p = np.asfortranarray(rng.standard_normal((g.ldx, g.nyt)))
    s = g.fftn(p)
    assert np.all(s[-1, :] == 0) and np.all(s[:, g.nyt // 2] == 0)
    back = g.ifftn(s) / (g.nxt * g.nyt)
    ref = np.fft.irfft2(np.where(_nyq_mask(g), np.fft.rfft2(p[: g.nxt].T).T, 0).T, s=(g.nyt, g.nxt)).T
    assert rel_l2(back[: g.nxt], ref) < 1e-13


def _nyq_mask(g):
    m = np.ones((g.lhx, g.nyt), bool)
    m[-1, :] = False
    m[:, g.nyt // 2] = False
    return m


def _fields(g, seed=2):
    rng = np.random.default_rng(seed)
    f = [g.filter_data(np.asfortranarray(rng.standard_normal((g.ldx, g.nyt, g.nz + 1)))) for _ in range(3)]
    f[2][:, :, 1] = 0.0
    f[2][:, :, g.nz] = 0.0
    return f


def _div(g, u, v, w):
    return g.ddx(u) + g.ddy(v) + g.ddz_w(w)


def test_pipelined_thomas_is_rank_independent(orc):
    # the pipelined solve across z-ranks is an exact sequential Thomas sweep
    g = _grid(orc)
    u, v, w = _fields(g)
    r2 = g.press_stag_array(u, v, w, npz=2)
    r4 = g.press_stag_array(u, v, w, npz=4)
    for a, b in zip(r2, r4):
        assert np.array_equal(a[: g.nxt], b[: g.nxt])


def test_projection_is_divergence_free_multi_rank(orc):
    # check_rmsdiv (901_debug.f90:24-62) of the canonical (npz >= 2) projection
    g = _grid(orc)
    u, v, w = _fields(g)
    p, dpx, dpy = g.press_stag_array(u, v, w, npz=2)
    uu, vv, ww = g.project(u, v, w, dpx, dpy, g.dpdz(p))
    d0 = _div(g, u, v, w)[: g.nxt, :, 1 : g.nz]
    d1 = _div(g, uu, vv, ww)[: g.nxt, :, 1 : g.nz]
    assert np.abs(d1).max() < 1e-12 * np.abs(d0).max()


def test_single_rank_top_is_dirichlet(orc):
    # with npz = 1 the top Neumann row is never built and p_hat(nz-1) is forced to 0
    g = _grid(orc)
    u, v, w = _fields(g)
    p, dpx, dpy = g.press_stag_array(u, v, w, npz=1)
    assert np.abs(p[: g.nxt, :, g.nz - 1]).max() < 1e-12
    uu, vv, ww = g.project(u, v, w, dpx, dpy, g.dpdz(p))
    d1 = _div(g, uu, vv, ww)[: g.nxt, :, 1 : g.nz - 2]
    assert np.abs(d1).max() < 1e-11


def test_projection_idempotent(orc):
    g = _grid(orc)
    u, v, w = _fields(g)
    p, dpx, dpy = g.press_stag_array(u, v, w, npz=2)
    u1, v1, w1 = g.project(u, v, w, dpx, dpy, g.dpdz(p))
    p2, dpx2, dpy2 = g.press_stag_array(u1, v1, w1, npz=2)
    u2, v2, w2 = g.project(u1, v1, w1, dpx2, dpy2, g.dpdz(p2))
    for a, b in ((u1, u2), (v1, v2), (w1, w2)):
        assert rel_l2(b, a) < 1e-12


def test_bad_rank_count_rejected(orc):
    g = _grid(orc)
    u, v, w = _fields(g)
    with pytest.raises(ValueError):
        g.press_stag_array(u, v, w, npz=3)
