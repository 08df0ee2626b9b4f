"""ctypes binding of the FP64 CPU oracle (oracle/libobl_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() (as the
checker) and by bench.py's CPU-baseline leg.  The product library never uses it.
PARITY UNPINNED: see obl_oracle.h.

Arrays are numpy arrays in the reference's Fortran layout (order='F'):
    physical field   (ldx, nyt, nz+1)    float64
    spectral plane   (lhx, nyt)          complex128
    padded plane     (nxt2, nyt2)        float64
    dpdx/dpdy/dpdz   (ldx, nyt, nz)      float64   (level jz in slot jz-1)
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libobl_oracle.so")


class OrcGrid(ctypes.Structure):
    _fields_ = [
        ("nxt", ctypes.c_int), ("nyt", ctypes.c_int), ("nzt", ctypes.c_int),
        ("lx_tot", ctypes.c_double), ("ly_tot", ctypes.c_double),
        ("lz_tot", ctypes.c_double), ("z_i", ctypes.c_double),
        ("dt", ctypes.c_double), ("u_scale", ctypes.c_double),
        ("ubc_stress_free", ctypes.c_int),
        ("nz", ctypes.c_int), ("lhx", ctypes.c_int), ("lhy", ctypes.c_int),
        ("ldx", ctypes.c_int), ("ldy", ctypes.c_int), ("nxt2", ctypes.c_int),
        ("nyt2", ctypes.c_int), ("lhx2", ctypes.c_int), ("lhy2", ctypes.c_int),
        ("ldx2", ctypes.c_int), ("ldy2", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
        ("dz", ctypes.c_double), ("dt_nd", ctypes.c_double),
    ]


def build():
    """Compile the oracle with its Makefile (system gcc)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = ctypes.CDLL(_LIB)
        P = ctypes.c_void_p
        G = ctypes.POINTER(OrcGrid)
        I = ctypes.c_int
        sig = {
            "orc_fft_c2c": (None, [I, P, P, I]),
            "orc_fft_r2c": (None, [I, P, P]),
            "orc_fft_c2r": (None, [I, P, P]),
            "orc_dft_naive": (None, [I, P, P, I]),
            "orc_grid_init": (I, [G]),
            "orc_wavenumbers": (None, [G, P, P, P, P, P, P]),
            "orc_ddx": (None, [G, P, P, I]),
            "orc_ddy": (None, [G, P, P, I]),
            "orc_ddz_uv": (None, [G, P, P]),
            "orc_ddz_w": (None, [G, P, P]),
            "orc_divstress_uv": (None, [G, P, P, P, P]),
            "orc_divstress_w": (None, [G, P, P, P, P]),
            "orc_fftn": (None, [G, P, P]),
            "orc_ifftn": (None, [G, P, P]),
            "orc_zero_padding": (None, [G, P, P]),
            "orc_zero_unpadding": (None, [G, P, P]),
            "orc_filter_data": (None, [G, P, I]),
            "orc_press_stag_array": (I, [G, I, P, P, P, P, P, P, P, P]),
            "orc_dpdz": (None, [G, P, P]),
            "orc_project": (None, [G, P, P, P, P, P, P]),
            "orc_step": (I, [G, I, P, P, P, P, P, P, P, P]),
            "orc_convec": (None, [G, P, P, P, P, P, P]),
            "orc_projection": (I, [G, P, P, P]),
            "orc_rollout_step": (I, [G, P, P, P]),
            "orc_ke_band": (ctypes.c_double, [G, P, P, P, ctypes.c_double, ctypes.c_double, P, P, P]),
            "orc_projection_vjp": (I, [G, P, P, P]),
            "orc_convec_vjp": (None, [G, P, P, P, P, P, P, P, P, P]),
            "orc_rollout_step_vjp": (I, [G, P, P, P, P, P, P]),
            "orc_rollout_grad": (I, [G, I, P, P, P, ctypes.c_double, ctypes.c_double, P, P, P, P]),
            "orc_set_threads": (None, [I]),
            "orc_get_threads": (I, []),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a):
    assert a.flags["F_CONTIGUOUS"] or a.ndim == 1, "arrays must be Fortran ordered"
    return a.ctypes.data_as(ctypes.c_void_p)


def set_threads(n):
    lib().orc_set_threads(int(n))


def get_threads():
    return lib().orc_get_threads()


# ----------------------------------------------------------------------------- FFT
def fft_c2c(x, sign):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    lib().orc_fft_c2c(len(x), _p(x), _p(out), int(sign))
    return out


def fft_r2c(x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(len(x) // 2 + 1, np.complex128)
    lib().orc_fft_r2c(len(x), _p(x), _p(out))
    return out


def fft_c2r(c, n):
    c = np.ascontiguousarray(c, dtype=np.complex128)
    out = np.empty(n, np.float64)
    lib().orc_fft_c2r(n, _p(c), _p(out))
    return out


def dft_naive(x, sign):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    lib().orc_dft_naive(len(x), _p(x), _p(out), int(sign))
    return out


# ---------------------------------------------------------------------------- grid
class Grid:
    """Oracle grid: dimensional inputs as in the reference namelist."""

    def __init__(self, nxt, nyt, nzt, lx_tot, ly_tot, lz_tot, z_i, dt, u_scale=1.0,
                 ubc_stress_free=False):
        g = OrcGrid()
        g.nxt, g.nyt, g.nzt = nxt, nyt, nzt
        g.lx_tot, g.ly_tot, g.lz_tot, g.z_i = lx_tot, ly_tot, lz_tot, z_i
        g.dt, g.u_scale = dt, u_scale
        g.ubc_stress_free = 1 if ubc_stress_free else 0
        if lib().orc_grid_init(ctypes.byref(g)) != 0:
            raise ValueError("bad oracle grid")
        self.g = g

    def __getattr__(self, k):
        return getattr(self.__dict__["g"], k)

    @property
    def ref(self):
        return ctypes.byref(self.g)

    def field(self, nlev=None):
        return np.zeros((self.ldx, self.nyt, (self.nz + 1) if nlev is None else nlev),
                        np.float64, order="F")

    def dfield(self):
        return np.zeros((self.ldx, self.nyt, self.nz), np.float64, order="F")

    def wavenumbers(self):
        g = self.g
        kx = np.zeros(g.lhx)
        ky = np.zeros(g.lhy)
        kx2 = np.zeros((g.lhx, g.nyt), order="F")
        ky2 = np.zeros((g.lhx, g.nyt), order="F")
        k2 = np.zeros((g.lhx, g.nyt), order="F")
        nn = np.zeros((g.lhx, g.nyt), np.int32, order="F")
        lib().orc_wavenumbers(self.ref, _p(kx), _p(ky), _p(kx2), _p(ky2), _p(k2), _p(nn))
        return kx, ky, kx2, ky2, k2, nn.astype(bool)

    # --- operators (all Fortran layout) ---
    def ddx(self, f):
        out = np.zeros_like(f, order="F")
        lib().orc_ddx(self.ref, _p(out), _p(f), f.shape[2])
        return out

    def ddy(self, f):
        out = np.zeros_like(f, order="F")
        lib().orc_ddy(self.ref, _p(out), _p(f), f.shape[2])
        return out

    def ddz_uv(self, f, out=None):
        out = np.zeros_like(f, order="F") if out is None else out
        lib().orc_ddz_uv(self.ref, _p(out), _p(f))
        return out

    def ddz_w(self, f, out=None):
        out = np.zeros_like(f, order="F") if out is None else out
        lib().orc_ddz_w(self.ref, _p(out), _p(f))
        return out

    def divstress_uv(self, tx, ty, tz):
        out = np.zeros_like(tx, order="F")
        lib().orc_divstress_uv(self.ref, _p(out), _p(tx), _p(ty), _p(tz))
        return out

    def divstress_w(self, tx, ty, tz):
        out = np.zeros_like(tx, order="F")
        lib().orc_divstress_w(self.ref, _p(out), _p(tx), _p(ty), _p(tz))
        return out

    def fftn(self, plane):
        out = np.zeros((self.lhx, self.nyt), np.complex128, order="F")
        lib().orc_fftn(self.ref, _p(np.asfortranarray(plane)), _p(out))
        return out

    def ifftn(self, spec):
        out = np.zeros((self.ldx, self.nyt), np.float64, order="F")
        lib().orc_ifftn(self.ref, _p(np.asfortranarray(spec)), _p(out))
        return out

    def zero_padding(self, plane):
        out = np.zeros((self.nxt2, self.nyt2), np.float64, order="F")
        lib().orc_zero_padding(self.ref, _p(np.asfortranarray(plane)), _p(out))
        return out

    def zero_unpadding(self, big):
        out = np.zeros((self.ldx, self.nyt), np.float64, order="F")
        lib().orc_zero_unpadding(self.ref, _p(np.asfortranarray(big)), _p(out))
        return out

    def filter_data(self, f):
        f = np.array(f, order="F", copy=True)
        lib().orc_filter_data(self.ref, _p(f), f.shape[2])
        return f

    def press_stag_array(self, u, v, w, divtz_bot=None, divtz_top=None, npz=1):
        zero = np.zeros((self.ldx, self.nyt), order="F")
        db = zero if divtz_bot is None else np.asfortranarray(divtz_bot)
        dt_ = zero if divtz_top is None else np.asfortranarray(divtz_top)
        p = self.field()
        dpdx = self.dfield()
        dpdy = self.dfield()
        rc = lib().orc_press_stag_array(self.ref, int(npz), _p(u), _p(v), _p(w), _p(db),
                                        _p(dt_), _p(p), _p(dpdx), _p(dpdy))
        if rc:
            raise ValueError("press_stag_array: (nzt-1) must be divisible by npz")
        return p, dpdx, dpdy

    def dpdz(self, p):
        out = self.dfield()
        lib().orc_dpdz(self.ref, _p(p), _p(out))
        return out

    def project(self, u, v, w, dpdx, dpdy, dpdz):
        u, v, w = (np.array(a, order="F", copy=True) for a in (u, v, w))
        lib().orc_project(self.ref, _p(u), _p(v), _p(w), _p(dpdx), _p(dpdy), _p(dpdz))
        return u, v, w

    def step_outputs(self):
        """Output arrays of step(), allocated once so that repeated steps reuse them."""
        return dict(u=self.field(), v=self.field(), w=self.field(), d=[self.field() for _ in range(8)],
                    big=[np.zeros((self.nxt2, self.nyt2, self.nz + 1), order="F") for _ in range(4)],
                    p=self.field(), dpdx=self.dfield(), dpdy=self.dfield(), dpdz=self.dfield())

    def step(self, u, v, w, theta, npz=1, out=None):
        """One step; out (from step_outputs) receives the results instead of new arrays."""
        if out is None:
            out = self.step_outputs()
        for k, a in (("u", u), ("v", v), ("w", w)):
            out[k][...] = a
        u, v, w = out["u"], out["v"], out["w"]
        d, big, p = out["d"], out["big"], out["p"]
        dp = [out["dpdx"], out["dpdy"], out["dpdz"]]
        D = (ctypes.c_void_p * 8)(*[a.ctypes.data for a in d])
        B = (ctypes.c_void_p * 4)(*[a.ctypes.data for a in big])
        DP = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in dp])
        rc = lib().orc_step(self.ref, int(npz), _p(u), _p(v), _p(w),
                            _p(np.asfortranarray(theta)), D, B, _p(p), DP)
        if rc:
            raise ValueError("orc_step failed")
        return dict(u=u, v=v, w=w, d=d, big=big, p=p, dpdx=dp[0], dpdy=dp[1], dpdz=dp[2])

    # --- rollout problem of the adjoint (obl_oracle_adj.c) ---
    def _copies(self, *arrs):
        return [np.array(a, dtype=np.float64, order="F", copy=True) for a in arrs]

    def convec(self, u, v, w):
        u, v, w = self._copies(u, v, w)
        cx, cy, cz = self.field(), self.field(), self.field()
        lib().orc_convec(self.ref, _p(u), _p(v), _p(w), _p(cx), _p(cy), _p(cz))
        return cx, cy, cz

    def projection(self, u, v, w):
        u, v, w = self._copies(u, v, w)
        if lib().orc_projection(self.ref, _p(u), _p(v), _p(w)):
            raise ValueError("projection: (nzt-1) must be even")
        return u, v, w

    def rollout_step(self, u, v, w):
        u, v, w = self._copies(u, v, w)
        if lib().orc_rollout_step(self.ref, _p(u), _p(v), _p(w)):
            raise ValueError("rollout_step: bad size")
        return u, v, w

    def ke_band(self, u, v, w, z_lo, z_hi, grad=False):
        u, v, w = self._copies(u, v, w)
        if grad:
            lu, lv, lw = self.field(), self.field(), self.field()
            J = lib().orc_ke_band(self.ref, _p(u), _p(v), _p(w), float(z_lo), float(z_hi),
                                  _p(lu), _p(lv), _p(lw))
            return J, (lu, lv, lw)
        return lib().orc_ke_band(self.ref, _p(u), _p(v), _p(w), float(z_lo), float(z_hi),
                                 None, None, None)

    def projection_vjp(self, lu, lv, lw):
        lu, lv, lw = self._copies(lu, lv, lw)
        if lib().orc_projection_vjp(self.ref, _p(lu), _p(lv), _p(lw)):
            raise ValueError("projection_vjp: bad size")
        return lu, lv, lw

    def convec_vjp(self, u, v, w, lcx, lcy, lcz):
        u, v, w, lcx, lcy, lcz = self._copies(u, v, w, lcx, lcy, lcz)
        lu, lv, lw = self.field(), self.field(), self.field()
        lib().orc_convec_vjp(self.ref, _p(u), _p(v), _p(w), _p(lcx), _p(lcy), _p(lcz),
                             _p(lu), _p(lv), _p(lw))
        return lu, lv, lw

    def rollout_step_vjp(self, u, v, w, lu, lv, lw):
        u, v, w, lu, lv, lw = self._copies(u, v, w, lu, lv, lw)
        if lib().orc_rollout_step_vjp(self.ref, _p(u), _p(v), _p(w), _p(lu), _p(lv), _p(lw)):
            raise ValueError("rollout_step_vjp: bad size")
        return lu, lv, lw

    def rollout_grad(self, nsteps, u, v, w, z_lo, z_hi, grad=True):
        u, v, w = self._copies(u, v, w)
        J = ctypes.c_double(0.0)
        g = [self.field() for _ in range(3)] if grad else [None, None, None]
        P = [(_p(a) if a is not None else None) for a in g]
        rc = lib().orc_rollout_grad(self.ref, int(nsteps), _p(u), _p(v), _p(w), float(z_lo),
                                    float(z_hi), ctypes.byref(J), *P)
        if rc:
            raise ValueError("rollout_grad: bad size")
        return (J.value, tuple(g)) if grad else J.value
