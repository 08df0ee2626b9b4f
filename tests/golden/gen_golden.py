"""Generate the golden fixtures of tests/golden/ from an independent numpy/scipy
restatement of the reference hot path.

    python tests/golden/gen_golden.py

The reference (Fortran + MPI + FFTW) ships no golden vectors and cannot be built
here, so these fixtures come from a second, independent restatement: numpy's
pocketfft in place of FFTW and scipy.linalg.solve_banded in place of the pipelined
Thomas sweep.  tests/test_golden.py checks the C oracle against them, so the oracle
is pinned to two implementations that share nothing but the reference's equations
(the routines and lines each function restates are cited inline).
"""
import os

import numpy as np
from scipy.linalg import solve_banded

HERE = os.path.dirname(os.path.abspath(__file__))
PI = 3.1415926535897932384626433      # 001_param.f90:32
TADV1 = 1.5                           # 001_param.f90:152
BOGUS = -1234567890.0                 # 001_param.f90:40


class G:
    def __init__(self, nxt, nyt, nzt, lx_tot, ly_tot, lz_tot, z_i, dt, u_scale=1.0):
        self.nxt, self.nyt, self.nzt = nxt, nyt, nzt
        self.nz = nzt
        self.L = nzt - 1
        self.lhx, self.lhy = nxt // 2 + 1, nyt // 2 + 1
        self.ldx = 2 * self.lhx
        self.nxt2, self.nyt2 = 3 * nxt // 2, 3 * nyt // 2
        self.lx, self.ly = lx_tot / z_i, ly_tot / z_i
        self.dz = (lz_tot / (nzt - 1)) / z_i
        self.dt = dt * u_scale / z_i
        # init_wavenumber (002_fft.f90:131-167)
        self.kx = np.arange(self.lhx) * 2.0 * PI / self.lx
        self.kx[-1] = 0.0
        self.ky = np.arange(self.lhy) * 2.0 * PI / self.ly
        self.ky[-1] = 0.0
        j = np.arange(nyt)
        ky2 = (((j + nyt // 2) % nyt) - nyt // 2) * 2.0 * PI / self.ly
        self.kx2d = np.repeat(self.kx[:, None], nyt, axis=1)
        self.ky2d = np.repeat(ky2[None, :], self.lhx, axis=0)
        self.ky2d[-1, :] = 0.0
        self.kx2d[:, nyt // 2] = 0.0
        self.ky2d[:, nyt // 2] = 0.0
        self.nn = np.ones((self.lhx, nyt), bool)
        self.nn[-1, :] = False
        self.nn[:, nyt // 2] = False
        self.k2 = self.kx2d ** 2 + self.ky2d ** 2


# FFTW conventions with numpy: r2c = rfft, c2r = irfft * n (unnormalised)
def r2c(x, axis):
    return np.fft.rfft(x, axis=axis)


def c2r(c, n, axis):
    return np.fft.irfft(c, n=n, axis=axis) * n


def ddx(g, f):      # 004_derivatives.f90:18-41
    out = np.zeros_like(f)
    a = r2c(f[:g.nxt] / g.nxt, 0)
    a = 1j * g.kx[:, None, None] * a
    out[:g.nxt] = c2r(a, g.nxt, 0)
    return out


def ddy(g, f):      # 004_derivatives.f90:45-81
    out = np.zeros_like(f)
    a = r2c(f[:g.nxt] / g.nyt, 1)
    a = 1j * g.ky[None, :, None] * a
    out[:g.nxt] = c2r(a, g.nyt, 1)
    return out


def fftn(g, p):     # 203_fftn_mpi.f90:4-35
    hx = r2c(p[:g.nxt], 0)
    hx[-1, :] = 0
    out = np.fft.fft(hx, axis=1)
    out[:, g.nyt // 2] = 0
    return out


def ifftn(g, c):    # 203_fftn_mpi.f90:39-67
    hy = np.fft.ifft(c, axis=1) * g.nyt
    out = np.zeros((g.ldx, g.nyt))
    out[:g.nxt] = c2r(hy, g.nxt, 0)
    return out


def zero_padding(g, var):   # 108_01_padd.f90:73-132
    hx = r2c(var[:g.nxt] / g.nxt, 0)
    hb = np.zeros((g.nxt2 // 2 + 1, g.nyt), complex)
    hb[:g.nxt // 2] = hx[:g.nxt // 2]
    xb = c2r(hb, g.nxt2, 0)
    hy = r2c(xb / g.nyt, 1)
    hyb = np.zeros((g.nxt2, g.nyt2 // 2 + 1), complex)
    hyb[:, :g.nyt // 2] = hy[:, :g.nyt // 2]
    return c2r(hyb, g.nyt2, 1)


def zero_unpadding(g, big):  # 108_01_padd.f90:136-197
    hx = r2c(big / g.nxt2, 0)
    hs = np.zeros((g.lhx, g.nyt2), complex)
    hs[:g.nxt // 2] = hx[:g.nxt // 2]
    xs = c2r(hs, g.nxt, 0)
    hy = r2c(xs / g.nyt2, 1)
    hys = np.zeros((g.nxt, g.lhy), complex)
    hys[:, :g.nyt // 2] = hy[:, :g.nyt // 2]
    var = np.zeros((g.ldx, g.nyt))
    var[:g.nxt] = c2r(hys, g.nyt, 1)
    var[g.nxt:] = var[:2]
    return var


def press(g, u, v, w, dbot, dtop, neumann_top):
    """press_stag_array + tdmaSolver_pipelined (109_press_stag_array.f90), solved with
    a banded LU per column instead of the Thomas sweep."""
    L, S = g.L, (g.lhx, g.nyt)
    cst = 1.0 / (g.nxt * g.nyt)
    H = {}
    for nm, f in (("x", u), ("y", v), ("z", w)):
        H[nm] = np.zeros(S + (L + 2,), complex)
        for jz in range(1, L + 1):
            H[nm][:, :, jz] = fftn(g, cst / TADV1 * (f[:, :, jz] / g.dt))
    H["z"][:, :, 0] = fftn(g, cst * dbot)
    if neumann_top:
        H["z"][:, :, L + 1] = fftn(g, cst * dtop)
    phat = np.zeros(S + (L + 1,), complex)
    idz, idz2 = 1.0 / g.dz, 1.0 / g.dz ** 2
    for i in range(g.lhx):
        for j in range(g.nyt):
            if not g.nn[i, j]:
                continue
            k2 = g.k2[i, j]
            a = np.zeros(L + 1)
            b = np.zeros(L + 1)
            c = np.zeros(L + 1)
            r = np.zeros(L + 1, complex)
            hx, hy, hz = H["x"][i, j], H["y"][i, j], H["z"][i, j]
            for jz in range(1, L + 1):
                if k2 > 0:
                    top = neumann_top and jz == L
                    a[jz] = 0.0 if jz == 1 else idz2
                    b[jz] = -(k2 + idz2) if (jz == 1 or top) else -(k2 + 2 * idz2)
                    c[jz] = 0.0 if top else idz2
                    dh = hz[jz + 1] - hz[jz] + (hz[0] if jz == 1 else 0.0)
                    r[jz] = 1j * (g.kx2d[i, j] * hx[jz] + g.ky2d[i, j] * hy[jz]) + dh / g.dz
                else:
                    a[jz] = 0.0 if jz == 1 else -idz
                    b[jz] = idz
                    r[jz] = 0.0 if jz == 1 else hz[jz]
            n = L if neumann_top else L - 1   # npz = 1: p_hat(L) = 0 (Dirichlet)
            ab = np.zeros((3, n), complex)
            ab[0, 1:] = c[1:n]
            ab[1, :] = b[1:n + 1]
            ab[2, :-1] = a[2:n + 1]
            x = solve_banded((1, 1), ab, r[1:n + 1])
            phat[i, j, 1:n + 1] = x
            phat[i, j, 0] = phat[i, j, 1] - g.dz * hz[0]
    p = np.zeros((g.ldx, g.nyt, g.nz + 1))
    dpdx = np.zeros((g.ldx, g.nyt, g.nz))
    dpdy = np.zeros((g.ldx, g.nyt, g.nz))
    p[:, :, 0] = ifftn(g, phat[:, :, 0])
    for jz in range(1, L + 1):
        dpdx[:, :, jz - 1] = ifftn(g, 1j * g.kx2d * phat[:, :, jz])
        dpdy[:, :, jz - 1] = ifftn(g, 1j * g.ky2d * phat[:, :, jz])
        p[:, :, jz] = ifftn(g, phat[:, :, jz])
    return p, dpdx, dpdy


def dpdz(g, p):     # 103_flosol.f90:174-175
    out = np.zeros((g.ldx, g.nyt, g.nz))
    out[:g.nxt, :, :g.nz - 1] = (p[:g.nxt, :, 1:g.nz] - p[:g.nxt, :, :g.nz - 1]) / g.dz
    return out


def project(g, u, v, w, dpdx, dpdy, dpdz_, stress_free=False):   # 110_project.f90:4-62
    u, v, w = u.copy(), v.copy(), w.copy()
    nx, nz = g.nxt, g.nz
    u[:nx, :, 1:nz] += g.dt * (-TADV1 * dpdx[:nx, :, :nz - 1])
    v[:nx, :, 1:nz] += g.dt * (-TADV1 * dpdy[:nx, :, :nz - 1])
    w[:nx, :, 2:nz] += g.dt * (-TADV1 * dpdz_[:nx, :, 1:nz - 1])
    if stress_free:
        u[:, :, nz - 1] = u[:, :, nz - 2]
        v[:, :, nz - 1] = v[:, :, nz - 2]
    w[:, :, nz] = 0.0
    w[:, :, 1] = 0.0
    return u, v, w


GRIDS = {
    "g16x12x9": (16, 12, 9, 2 * PI * 1000.0, 1.5 * PI * 1000.0, 1000.0, 1000.0, 0.5),
    "g12x16x7": (12, 16, 7, 3000.0, 4000.0, 600.0, 500.0, 0.3),
}


def make_case(name, seed):
    g = G(*GRIDS[name])
    rng = np.random.default_rng(seed)
    shape = (g.ldx, g.nyt, g.nz + 1)
    u, v, w, t = (np.asfortranarray(rng.standard_normal(shape)) for _ in range(4))
    w[:, :, 1] = 0.0
    w[:, :, g.nz] = 0.0
    dbot = rng.standard_normal((g.ldx, g.nyt)) * 0.1
    dtop = rng.standard_normal((g.ldx, g.nyt)) * 0.1
    big = np.asfortranarray(rng.standard_normal((g.nxt2, g.nyt2)))
    out = dict(u=u, v=v, w=w, theta=t, dbot=dbot, dtop=dtop, big_in=big)
    out["ddx_u"] = ddx(g, u)
    out["ddy_u"] = ddy(g, u)
    out["fftn_u5"] = fftn(g, u[:, :, 5 % (g.nz + 1)])
    out["ifftn_f"] = ifftn(g, out["fftn_u5"])
    out["pad_u3"] = zero_padding(g, u[:, :, 3])
    out["unpad_big"] = zero_unpadding(g, big)
    for mode, neu in (("neumann", True), ("single", False)):
        p, dpx, dpy = press(g, u, v, w, dbot, dtop, neu)
        dz_ = dpdz(g, p)
        uu, vv, ww = project(g, u, v, w, dpx, dpy, dz_)
        out[f"p_{mode}"], out[f"dpdx_{mode}"], out[f"dpdy_{mode}"] = p, dpx, dpy
        out[f"dpdz_{mode}"] = dz_
        out[f"uproj_{mode}"], out[f"vproj_{mode}"], out[f"wproj_{mode}"] = uu, vv, ww
    return out


if __name__ == "__main__":
    for i, name in enumerate(GRIDS):
        case = make_case(name, 1000 + i)
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, grid=np.array(GRIDS[name]), **case)
        print(path, os.path.getsize(path))
