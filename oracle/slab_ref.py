"""numpy restatement of the z-partitioned pressure solve (test infrastructure only).

The column systems are those of init_coef_press + press_stag_array in the npz >= 2 form
(109_press_stag_array.f90:4-68, 203-225): Neumann rows at the bottom of rank 0 and at the
top of the last rank, the (0,0) mean mode integrated to first order.  Two solvers:

* ``global_solve``: one Thomas sweep over all rows of every column (the single-domain
  solve, what the pipelined multi-rank sweep of the reference computes);
* the partitioned form of the library's z-slab step: ``local_solve`` per rank (particular
  solution y and the spikes v, w of the two couplings to the neighbouring ranks, plus
  the interface coefficients), ``reduced_solve`` (the 2P interface unknowns), and
  ``finish`` (x = y - v x_below - w x_above, p_hat(0), dpdz spectrum).

Spectra are (S, L+2) complex arrays (levels 0..L+1) over the S = lhx*nyt columns of one
rank; H_x, H_y are used at levels 1..L, H_z at 0..L+1.
"""
import numpy as np


def column_tables(kx, ky2, lhx, nyt):
    """k^2 and the not-Nyquist mask of the S = lhx*nyt columns (q = kx + lhx*ky)."""
    KX = np.tile(kx, nyt)
    KY = np.repeat(ky2, lhx)
    ix = np.tile(np.arange(lhx), nyt)
    iy = np.repeat(np.arange(nyt), lhx)
    nn = (ix != lhx - 1) & (iy != nyt // 2)
    return KX, KY, KX * KX + KY * KY, nn


def bands(k2, j, L, dz, bottom, top):
    """a, b, c of global row j (1..L) for every column; bottom/top: the row is the first
    row of rank 0 / the last row of the last rank."""
    idz, idz2 = 1.0 / dz, 1.0 / (dz * dz)
    m00 = k2 == 0.0
    b1 = bottom and j == 1
    tl = top and j == L
    a = np.where(m00, 0.0 if b1 else -idz, 0.0 if b1 else idz2)
    c = np.where(m00, 0.0, 0.0 if tl else idz2)
    b = np.where(m00, idz, -(k2 + idz2) if (b1 or tl) else -(k2 + 2.0 * idz2))
    return a, b, c


def rhs(KX, KY, k2, Hx, Hy, Hz, j, dz, bottom):
    """RHS of local row j from the local spectra (Hz holds levels 0..L+1)."""
    m00 = k2 == 0.0
    b1 = bottom and j == 1
    dh = Hz[:, j + 1] - Hz[:, j] + (Hz[:, 0] if b1 else 0.0)
    r = 1j * (KX * Hx[:, j] + KY * Hy[:, j]) + dh / dz
    r00 = np.zeros_like(r) if b1 else Hz[:, j]
    return np.where(m00, r00, r)


def global_solve(KX, KY, k2, nn, Hx, Hy, Hz, dz):
    """p_hat levels 0..L of one domain."""
    S, L = Hx.shape[0], Hx.shape[1] - 2
    A = np.zeros((S, L + 1)); B = np.zeros((S, L + 1)); C = np.zeros((S, L + 1))
    R = np.zeros((S, L + 1), complex)
    for j in range(1, L + 1):
        A[:, j], B[:, j], C[:, j] = bands(k2, j, L, dz, True, True)
        R[:, j] = rhs(KX, KY, k2, Hx, Hy, Hz, j, dz, True)
    x = np.zeros((S, L + 1), complex)
    cp = np.zeros((S, L + 1)); dp = np.zeros((S, L + 1), complex)
    for j in range(1, L + 1):
        den = B[:, j] - (A[:, j] * cp[:, j - 1] if j > 1 else 0.0)
        cp[:, j] = C[:, j] / den
        dp[:, j] = (R[:, j] - (A[:, j] * dp[:, j - 1] if j > 1 else 0.0)) / den
    x[:, L] = dp[:, L]
    for j in range(L - 1, 0, -1):
        x[:, j] = dp[:, j] - cp[:, j] * x[:, j + 1]
    x[:, 0] = x[:, 1] - dz * Hz[:, 0]
    x[~nn] = 0.0
    return x


def local_solve(KX, KY, k2, nn, Hx, Hy, Hz, dz, rank, nranks):
    """The rank's particular solution y and spikes v, w (levels 1..L) and its interface
    coefficients (S, 8): y1.re, y1.im, ym.re, ym.im, v1, vm, w1, wm."""
    S, L = Hx.shape[0], Hx.shape[1] - 2
    bot, top = rank == 0, rank == nranks - 1
    y = np.zeros((S, L + 1), complex); v = np.zeros((S, L + 1)); w = np.zeros((S, L + 1))
    cp = np.zeros((S, L + 1))
    for j in range(1, L + 1):
        a, b, c = bands(k2, j, L, dz, bot, top)
        r = rhs(KX, KY, k2, Hx, Hy, Hz, j, dz, bot)
        asub = 0.0 if j == 1 else a
        csup = 0.0 if j == L else c
        den = b - asub * cp[:, j - 1]
        cp[:, j] = csup / den
        y[:, j] = (r - asub * y[:, j - 1]) / den
        v[:, j] = ((a if j == 1 else 0.0) - asub * v[:, j - 1]) / den
        w[:, j] = ((c if j == L else 0.0) - asub * w[:, j - 1]) / den
    for j in range(L - 1, 0, -1):
        y[:, j] -= cp[:, j] * y[:, j + 1]
        v[:, j] -= cp[:, j] * v[:, j + 1]
        w[:, j] -= cp[:, j] * w[:, j + 1]
    y[~nn] = 0.0; v[~nn] = 0.0; w[~nn] = 0.0
    iface = np.stack([y[:, 1].real, y[:, 1].imag, y[:, L].real, y[:, L].imag,
                      v[:, 1], v[:, L], w[:, 1], w[:, L]], axis=1)
    return y, v, w, iface


def reduced_solve(iface_all):
    """iface_all (P, S, 8) -> first and last unknowns (P, S) of every rank."""
    P, S = iface_all.shape[:2]
    y1 = iface_all[:, :, 0] + 1j * iface_all[:, :, 1]
    ym = iface_all[:, :, 2] + 1j * iface_all[:, :, 3]
    v1, vm, w1, wm = (iface_all[:, :, k] for k in (4, 5, 6, 7))
    # dense 2P x 2P solve per column: unknowns [f_0, l_0, f_1, l_1, ...]
    M = np.zeros((S, 2 * P, 2 * P)); Y = np.zeros((S, 2 * P), complex)
    for k in range(P):
        M[:, 2 * k, 2 * k] = 1.0
        M[:, 2 * k + 1, 2 * k + 1] = 1.0
        if k > 0:
            M[:, 2 * k, 2 * k - 1] = v1[k]
            M[:, 2 * k + 1, 2 * k - 1] = vm[k]
        if k < P - 1:
            M[:, 2 * k, 2 * k + 2] = w1[k]
            M[:, 2 * k + 1, 2 * k + 2] = wm[k]
        Y[:, 2 * k] = y1[k]
        Y[:, 2 * k + 1] = ym[k]
    X = np.linalg.solve(M.astype(complex), Y[..., None])[..., 0]
    return X[:, 0::2].T, X[:, 1::2].T


def finish(y, v, w, first, last, Hz0, nn, dz, rank, nranks):
    """p_hat levels 0..L and the dpdz spectrum (levels 1..L) of the rank."""
    below = last[rank - 1] if rank > 0 else 0.0
    above = first[rank + 1] if rank < nranks - 1 else 0.0
    x = y - v * (below if np.ndim(below) == 0 else below[:, None]) \
          - w * (above if np.ndim(above) == 0 else above[:, None])
    x[:, 0] = x[:, 1] - dz * Hz0 if rank == 0 else below
    x[~nn] = 0.0
    dph = np.zeros_like(x)
    dph[:, 1:] = (x[:, 1:] - x[:, :-1]) / dz
    return x, dph
