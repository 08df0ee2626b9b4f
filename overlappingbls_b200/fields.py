"""Seeded synthetic boundary-layer fields (the reference has no public dataset).

Recipe (stands in for a restart file of the reference):
  * domain Lx = Ly = 2*pi*1000 m, Lz = 1000 m, z_i = 1000 m, u_scale = 1 m/s;
  * u(z) = (0.45/0.4) ln(z/z0) log-law mean (z0 = 0.1 m by default) at the
    staggered uvp nodes z = (jz - 0.5) dz (SBL/code/102_initial.f90:275-278);
  * u, v, w fluctuations: on every level, random-phase 2D Fourier modes with
    amplitude |k|^(-4/3) (a k^(-5/3) energy spectrum), no Nyquist and no (0,0) mode,
    scaled to an rms of 0.5 m/s;
  * w = 0 at the wall (level 1) and at the top (level nz); ghost levels 0 and nz of
    u, v, theta copy their neighbours;
  * theta = 300 K + gradient * z + N(0, 0.1 K) noise.
Random numbers come from SplitMix64 (Steele, Lea & Flood 2014) keyed by
(seed, field, level, mode), so any level of any field is reproducible alone.
Arrays are float64 in the reference's Fortran layout (ldx, nyt, nz+1).
"""
import numpy as np

_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_G = np.uint64(0x9E3779B97F4A7C15)


def splitmix64(x):
    with np.errstate(over="ignore"):
        x = np.asarray(x, dtype=np.uint64) + _G
        z = (x ^ (x >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def _key(*parts):
    h = np.uint64(0)
    for p in parts:
        h = splitmix64(h ^ np.uint64(p & 0xFFFFFFFFFFFFFFFF))
    return h


def uniform(key, n):
    """n uniforms in [0,1) from the counter stream of `key`."""
    with np.errstate(over="ignore"):
        h = splitmix64(np.uint64(key) ^ np.arange(n, dtype=np.uint64))
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def fluct_plane(nxt, nyt, key, rms=0.5):
    """One level of k^-5/3 random-phase fluctuations, shape (nyt, nxt)."""
    lhx = nxt // 2 + 1
    ky = np.fft.fftfreq(nyt, 1.0 / nyt)[:, None]
    kx = np.arange(lhx)[None, :].astype(np.float64)
    k = np.sqrt(kx * kx + ky * ky)
    amp = np.zeros_like(k)
    nz = k > 0
    amp[nz] = k[nz] ** (-4.0 / 3.0)
    amp[:, lhx - 1] = 0.0          # x Nyquist
    amp[nyt // 2, :] = 0.0         # y Nyquist
    with np.errstate(over="ignore"):
        ph = 2.0 * np.pi * uniform(key, nyt * lhx).reshape(nyt, lhx)
    c = amp * np.exp(1j * ph)
    f = np.fft.irfft2(c, s=(nyt, nxt))
    s = np.sqrt(np.mean(f * f))
    return f * (rms / s) if s > 0 else f


def make_fields(nxt, nyt, nzt, lz_tot=1000.0, z0=0.1, theta_grad=0.01, seed=2024,
                with_theta=True, u_scale=1.0, rms=0.5):
    """Return dict(u, v, w, theta) in Fortran layout (ldx, nyt, nz+1), float64,
    non-dimensionalised by u_scale (velocities)."""
    ldx = 2 * (nxt // 2 + 1)
    nz = nzt
    L = nzt - 1
    dz = lz_tot / L
    out = {}
    for fi, name in enumerate(("u", "v", "w", "theta")):
        if name == "theta" and not with_theta:
            continue
        a = np.zeros((ldx, nyt, nz + 1), np.float64, order="F")
        for jz in range(1, L + 1):
            z = (jz - 0.5) * dz
            if name == "theta":
                key = int(_key(seed, fi, jz))
                u1 = uniform(key, nxt * nyt)
                u2 = uniform(key ^ 0x5DEECE66D, nxt * nyt)
                g = np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)   # Box-Muller
                plane = 300.0 + theta_grad * z + 0.1 * g.reshape(nyt, nxt)
            else:
                plane = fluct_plane(nxt, nyt, int(_key(seed, fi, jz)), rms) / u_scale
                if name == "u":
                    plane = plane + (0.45 / 0.4) * np.log(z / z0) / u_scale
            a[:nxt, :, jz] = plane.T
        if name == "w":
            a[:, :, 1] = 0.0
            a[:, :, nz] = 0.0
            a[:, :, 0] = 0.0
        else:
            a[:, :, 0] = a[:, :, 1]
            a[:, :, nz] = a[:, :, L]
        out[name] = a
    return out


# default physical constants of the benchmark workloads (dimensional)
DOMAIN = dict(lx_tot=2 * np.pi * 1000.0, ly_tot=2 * np.pi * 1000.0, lz_tot=1000.0, z_i=1000.0,
              dt=0.5, u_scale=1.0)


def ensemble_members(seed=2024):
    """The 48 instances of the ensemble workload: 16 each at 96x96x64, 128x128x96 and
    192x192x128 levels (nzt = levels + 1).  Per instance, from its own seeded stream: a
    theta gradient ~ U[0, 0.03] K/m and a roughness length z0 log-uniform in [0.01, 1] m
    (z0 replaces 0.1 m in the log law)."""
    out = []
    for b, (n, levels) in enumerate(((96, 64), (128, 96), (192, 128))):
        for k in range(16):
            i = 16 * b + k
            r = uniform(int(_key(seed, 7, i)), 2)
            out.append(dict(nxt=n, nyt=n, nzt=levels + 1, seed=seed + 1 + i,
                            theta_grad=0.03 * float(r[0]), z0=10.0 ** (-2.0 + 2.0 * float(r[1]))))
    return out
