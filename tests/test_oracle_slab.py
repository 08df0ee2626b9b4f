"""The z-partitioned pressure solve restated in numpy (oracle/slab_ref.py) against the
single sweep, and the single sweep against the C oracle's press_stag_array (npz = 2)."""
import numpy as np
import pytest

from oracle import slab_ref as sr
from overlappingbls_b200.fields import DOMAIN, make_fields

TADV1 = 1.5


def spectra(orc, g, u, v, w):
    """H_x, H_y (levels 1..L) and H_z (0..L+1, boundary planes 0) of press_stag_array."""
    L, S = g.nz - 1, g.lhx * g.nyt
    sc = 1.0 / (g.nxt * g.nyt) / TADV1 / g.dt_nd
    H = [np.zeros((S, L + 2), complex) for _ in range(3)]
    for c, f in enumerate((u, v, w)):
        for j in range(1, L + 1):
            H[c][:, j] = g.fftn(sc * f[:, :, j]).ravel(order="F")
    return H


def tables(g):
    kx, ky, kx2, ky2, k2, nn = g.wavenumbers()
    return sr.column_tables(kx, ky2[0, :] if ky2.ndim == 2 else ky2, g.lhx, g.nyt)


def test_global_solve_matches_oracle(orc):
    g = orc.Grid(32, 24, 17, **DOMAIN)
    f = make_fields(32, 24, 17, with_theta=False)
    H = spectra(orc, g, f["u"], f["v"], f["w"])
    kx, ky, kx2, ky2, k2, nn = g.wavenumbers()
    KX, KY, K2, NN = sr.column_tables(kx, ky2[0], g.lhx, g.nyt)
    assert np.array_equal(NN, nn.ravel(order="F"))
    ph = sr.global_solve(KX, KY, K2, NN, H[0], H[1], H[2], g.dz)
    p, _, _ = g.press_stag_array(f["u"], f["v"], f["w"], npz=2)
    L = g.nz - 1
    for j in range(0, L + 1):
        pj = g.ifftn(ph[:, j].reshape(g.lhx, g.nyt, order="F"))
        np.testing.assert_allclose(pj[: g.nxt], p[: g.nxt, :, j], rtol=0, atol=1e-11 * np.abs(p).max())


@pytest.mark.parametrize("P", [1, 2, 4])
def test_partition_matches_single_sweep(orc, P):
    rng = np.random.default_rng(P)
    g = orc.Grid(16, 12, 17, **DOMAIN)
    kx, ky, kx2, ky2, k2, nn = g.wavenumbers()
    KX, KY, K2, NN = sr.column_tables(kx, ky2[0], g.lhx, g.nyt)
    S, L = g.lhx * g.nyt, 16
    H = [rng.standard_normal((S, L + 2)) + 1j * rng.standard_normal((S, L + 2)) for _ in range(3)]
    for h in H[:2]:
        h[:, 0] = 0.0
        h[:, L + 1] = 0.0
    ref = sr.global_solve(KX, KY, K2, NN, *H, g.dz)
    Lr = L // P
    loc = []
    for r in range(P):
        sl = slice(r * Lr, r * Lr + Lr + 2)
        Hr = [h[:, sl].copy() for h in H]
        loc.append((Hr, sr.local_solve(KX, KY, K2, NN, *Hr, g.dz, r, P)))
    ia = np.stack([l[1][3] for l in loc])
    first, last = sr.reduced_solve(ia)
    for r, (Hr, (y, v, w, _)) in enumerate(loc):
        x, dph = sr.finish(y, v, w, first, last, Hr[2][:, 0], NN, g.dz, r, P)
        np.testing.assert_allclose(x, ref[:, r * Lr: r * Lr + Lr + 1], rtol=0, atol=1e-12 * np.abs(ref).max())
