"""GPU parity of the rollout step, its transpose and the rollout gradient.

* convec, the rollout step and the KE objective against the FP64 oracle;
* the step transpose: the step is quadratic in the state, so the central difference
  (F(s+d) - F(s-d))/2 is exactly the tangent F'(s) d and <tangent, l> = <d, F'(s)^T l>
  holds to rounding for any d;
* the transpose and the rollout gradient against the oracle's explicit transposes;
* the 128x128x128, 16-step rollout: FP64 gradient against central finite differences
  (eps = 1e-4, 64 seeded directions, gate 1e-6), the FP32 (mixed) gradient against the
  FP64 gradient, and the FP64 gradient against the oracle's.
"""
import numpy as np
import pytest

import overlappingbls_b200 as obl
from overlappingbls_b200 import fields
from conftest import identical_inputs, rel_l2

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-11, "mixed": 1e-5}


def _state(nx, ny, nzt, prec):
    f = identical_inputs(fields.make_fields(nx, ny, nzt, with_theta=False), prec)
    return [np.asfortranarray(f[k]) for k in "uvw"]


def _rnd(shape, nx, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    a = np.zeros(shape, order="F")
    a[:nx] = scale * rng.standard_normal(a[:nx].shape)
    return a


def _dot(nx, a, b):
    return sum(float(np.sum(x[:nx] * y[:nx])) for x, y in zip(a, b))


def _ctx(nx, ny, nzt, prec, stress_free=False):
    return obl.Context(nx, ny, nzt, precision=prec, top_bc="neumann", ubc_stress_free=stress_free,
                       **fields.DOMAIN)


def _grid(orc, nx, ny, nzt, stress_free=False):
    return orc.Grid(nx, ny, nzt, **fields.DOMAIN, ubc_stress_free=stress_free)


SIZES = [(64, 64, 33), (96, 64, 17), (32, 48, 9)]


@pytest.mark.parametrize("prec", ["f64", "mixed"])
@pytest.mark.parametrize("nx,ny,nzt", SIZES)
def test_convec_matches_oracle(orc, prec, nx, ny, nzt):
    ctx = _ctx(nx, ny, nzt, prec)
    g = _grid(orc, nx, ny, nzt)
    s = _state(nx, ny, nzt, prec)
    c = [ctx.field() for _ in range(3)]
    ctx.convec(*c, *s)
    ref = g.convec(*s)
    L = g.nz - 1
    for a, r in zip(c, ref):
        assert rel_l2(a[:nx, :, 1:L + 1], r[:nx, :, 1:L + 1]) < TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "mixed"])
@pytest.mark.parametrize("stress_free", [False, True])
@pytest.mark.parametrize("nx,ny,nzt", SIZES)
def test_rollout_step_matches_oracle(orc, prec, stress_free, nx, ny, nzt):
    ctx = _ctx(nx, ny, nzt, prec, stress_free)
    g = _grid(orc, nx, ny, nzt, stress_free)
    s = _state(nx, ny, nzt, prec)
    ref = g.rollout_step(*s)
    out = [a.copy(order="F") for a in s]
    ctx.rollout_step(*out)
    for a, r in zip(out, ref):
        assert rel_l2(a[:nx], r[:nx]) < TOL[prec]


@pytest.mark.parametrize("stress_free", [False, True])
@pytest.mark.parametrize("nx,ny,nzt", SIZES)
def test_step_vjp_exact_transpose(stress_free, nx, ny, nzt):
    ctx = _ctx(nx, ny, nzt, "f64", stress_free)
    s = _state(nx, ny, nzt, "f64")
    d = [_rnd(s[0].shape, nx, 10 + i, 0.1) for i in range(3)]
    lam = [_rnd(s[0].shape, nx, 20 + i) for i in range(3)]
    fp = [(a + b).copy(order="F") for a, b in zip(s, d)]
    fm = [(a - b).copy(order="F") for a, b in zip(s, d)]
    ctx.rollout_step(*fp)
    ctx.rollout_step(*fm)
    tang = [0.5 * (p - m) for p, m in zip(fp, fm)]
    adj = [a.copy(order="F") for a in lam]
    ctx.rollout_step_vjp(*s, *adj)
    lhs, rhs = _dot(nx, tang, lam), _dot(nx, d, adj)
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


@pytest.mark.parametrize("prec", ["f64", "mixed"])
@pytest.mark.parametrize("stress_free", [False, True])
def test_step_vjp_matches_oracle(orc, prec, stress_free):
    nx, ny, nzt = 64, 64, 33
    ctx = _ctx(nx, ny, nzt, prec, stress_free)
    g = _grid(orc, nx, ny, nzt, stress_free)
    s = _state(nx, ny, nzt, prec)
    lam = [_rnd(s[0].shape, nx, 30 + i) for i in range(3)]
    if prec == "mixed":
        lam = [np.asfortranarray(a.astype(np.float32).astype(np.float64)) for a in lam]
    ref = g.rollout_step_vjp(*s, *lam)
    adj = [a.copy(order="F") for a in lam]
    ctx.rollout_step_vjp(*s, *adj)
    for a, r in zip(adj, ref):
        assert rel_l2(a[:nx], r[:nx]) < TOL[prec]


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_ke_band_matches_oracle(orc, prec):
    nx, ny, nzt = 64, 64, 65
    ctx = _ctx(nx, ny, nzt, prec)
    g = _grid(orc, nx, ny, nzt)
    s = _state(nx, ny, nzt, prec)
    lam = [ctx.field() for _ in range(3)]
    J = ctx.ke_band(*s, 0.0, 100.0, *lam)
    Jr, ref = g.ke_band(*s, 0.0, 100.0, grad=True)
    assert abs(J - Jr) <= 1e-12 * abs(Jr)
    for a, r in zip(lam, ref):   # the seeds are stored in the storage type
        assert rel_l2(a[:nx], r[:nx]) < (1e-15 if prec == "f64" else 1e-7)
    assert ctx.ke_band(*s, 2000.0, 3000.0) == 0.0


def test_rollout_grad_rejects_single_rank_top():
    ctx = obl.Context(32, 32, 17, precision="f64", top_bc="single", **fields.DOMAIN)
    s = _state(32, 32, 17, "f64")
    ctx.rollout_grad(2, *s, 0.0, 100.0)   # forward only: any top mode
    with pytest.raises(obl.OblError, match="UNSUPPORTED"):
        ctx.rollout_grad(2, *s, 0.0, 100.0, *[ctx.field() for _ in range(3)])


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_rollout_grad_matches_oracle(orc, prec):
    nx, ny, nzt, nsteps = 64, 64, 33, 4
    ctx = _ctx(nx, ny, nzt, prec)
    g = _grid(orc, nx, ny, nzt)
    s = _state(nx, ny, nzt, prec)
    gr = [ctx.field() for _ in range(3)]
    J = ctx.rollout_grad(nsteps, *s, 0.0, 100.0, *gr)
    Jr, ref = g.rollout_grad(nsteps, *s, 0.0, 100.0)
    assert abs(J - Jr) <= (1e-12 if prec == "f64" else 1e-6) * abs(Jr)
    tol = 1e-10 if prec == "f64" else 1e-4
    for a, r in zip(gr, ref):
        assert rel_l2(a[:nx], r[:nx]) < tol


# ----------------------------------------------------------------- 128^3, 16 steps
C3 = dict(nx=128, ny=128, nzt=129, nsteps=16, z_lo=0.0, z_hi=100.0)


@pytest.fixture(scope="module")
def config3():
    nx, ny, nzt = C3["nx"], C3["ny"], C3["nzt"]
    ctx = _ctx(nx, ny, nzt, "f64")
    s = _state(nx, ny, nzt, "f64")
    gr = [ctx.field() for _ in range(3)]
    J = ctx.rollout_grad(C3["nsteps"], *s, C3["z_lo"], C3["z_hi"], *gr)
    return ctx, s, J, gr


def test_config3_gradient_vs_finite_differences(config3):
    ctx, s, J, gr = config3
    nx, eps = C3["nx"], 1e-4
    worst = 0.0
    for k in range(64):
        d = [_rnd(s[0].shape, nx, 1000 + 3 * k + i) for i in range(3)]
        Jp = ctx.rollout_grad(C3["nsteps"], *[a + eps * b for a, b in zip(s, d)], C3["z_lo"], C3["z_hi"])
        Jm = ctx.rollout_grad(C3["nsteps"], *[a - eps * b for a, b in zip(s, d)], C3["z_lo"], C3["z_hi"])
        fd = (Jp - Jm) / (2 * eps)
        gd = _dot(nx, gr, d)
        worst = max(worst, abs(fd - gd) / abs(gd))
    print(f"config3 FD: J={J:.10e} worst rel err over 64 directions = {worst:.3e}")
    assert worst <= 1e-6


def test_config3_mixed_gradient_vs_f64(config3):
    _, s, J, gr = config3
    nx, ny, nzt = C3["nx"], C3["ny"], C3["nzt"]
    ctx = _ctx(nx, ny, nzt, "mixed")
    s32 = [np.asfortranarray(a.astype(np.float32).astype(np.float64)) for a in s]
    gm = [ctx.field() for _ in range(3)]
    Jm = ctx.rollout_grad(C3["nsteps"], *s32, C3["z_lo"], C3["z_hi"], *gm)
    errs = [rel_l2(a[:nx], b[:nx]) for a, b in zip(gm, gr)]
    print(f"config3 mixed vs f64: J rel {abs(Jm - J) / abs(J):.3e}, grad rel L2 u,v,w = "
          + ", ".join(f"{e:.3e}" for e in errs))
    assert abs(Jm - J) <= 1e-6 * abs(J)
    assert max(errs) <= 1e-5


def test_config3_gradient_vs_oracle(orc, config3):
    _, s, J, gr = config3
    g = _grid(orc, C3["nx"], C3["ny"], C3["nzt"])
    Jr, ref = g.rollout_grad(C3["nsteps"], *s, C3["z_lo"], C3["z_hi"])
    errs = [rel_l2(a[:C3["nx"]], b[:C3["nx"]]) for a, b in zip(gr, ref)]
    print(f"config3 f64 vs oracle: J rel {abs(J - Jr) / abs(Jr):.3e}, grad rel L2 = "
          + ", ".join(f"{e:.3e}" for e in errs))
    assert abs(J - Jr) <= 1e-12 * abs(Jr)
    assert max(errs) <= 1e-10


@pytest.mark.parametrize("prec", ["mixed", "f64"])
def test_config3_timing(prec):
    """Device time of one forward rollout + gradient (128^3, 16 steps, a checkpoint per
    step), from the state on the device; CUDA events on the library's stream."""
    import torch
    nx, ny, nzt = C3["nx"], C3["ny"], C3["nzt"]
    ctx = _ctx(nx, ny, nzt, prec)
    dt = torch.float64 if prec == "f64" else torch.float32
    s = [torch.from_numpy(a.ravel(order="F")).to("cuda", dt) for a in _state(nx, ny, nzt, prec)]
    g = [torch.zeros_like(s[0]) for _ in range(3)]
    P = lambda t: t.data_ptr()
    run = lambda: ctx.rollout_grad_dev(C3["nsteps"], *[P(t) for t in s], C3["z_lo"], C3["z_hi"], *[P(t) for t in g])
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 5
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    pts = nx * ny * (nzt - 1)
    print(f"config3 {prec}: forward + gradient over {C3['nsteps']} steps {ms:.2f} ms, "
          f"{C3['nsteps'] * pts / ms / 1e3:.0f} Mpts/s per (step + transposed step)")
    ctx.close()
