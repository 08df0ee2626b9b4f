"""GPU z-slab step: a domain split over P ranks (one context each, run in lock-step in one
process on one GPU, so that no kernel waits for another) gives the single-domain step on
every rank's levels."""
import numpy as np
import pytest

import overlappingbls_b200 as obl
from overlappingbls_b200 import fields, slab
from conftest import identical_inputs, rel_l2

pytestmark = pytest.mark.gpu


class Bufs:
    def __init__(self, ctx, f):
        import torch
        dt = torch.float64 if ctx.dtype == np.float64 else torch.float32
        self.shape = (ctx.ldx, ctx.nyt, ctx.nz + 1)
        nf, nd = ctx.ldx * ctx.nyt * (ctx.nz + 1), ctx.ldx * ctx.nyt * ctx.nz
        nb = ctx.nxt2 * ctx.nyt2 * (ctx.nz + 1)
        T = lambda a: torch.from_numpy(np.asarray(a, ctx.dtype).ravel(order="F")).cuda()
        self.f = {k: T(f[k]) for k in ("u", "v", "w", "theta")}
        self.d = [torch.full((nf,), float("nan"), dtype=dt, device="cuda") for _ in range(8)]
        self.big = [torch.full((nb,), float("nan"), dtype=dt, device="cuda") for _ in range(4)]
        self.p = torch.full((nf,), float("nan"), dtype=dt, device="cuda")
        self.dp = [torch.full((nd,), float("nan"), dtype=dt, device="cuda") for _ in range(3)]
        self.ctx = ctx
        torch.cuda.synchronize()

    def io(self):
        P = lambda t: t.data_ptr()
        return obl.stepio_dev(P(self.f["u"]), P(self.f["v"]), P(self.f["w"]), P(self.f["theta"]),
                              [P(t) for t in self.d], [P(t) for t in self.big], P(self.p), [P(t) for t in self.dp])

    def get(self):
        c = self.ctx
        F = lambda t, nl: t.double().cpu().numpy().reshape(c.ldx, c.nyt, nl, order="F")
        B = lambda t: t.double().cpu().numpy().reshape(c.nxt2, c.nyt2, c.nz + 1, order="F")
        return dict(u=F(self.f["u"], c.nz + 1), v=F(self.f["v"], c.nz + 1), w=F(self.f["w"], c.nz + 1),
                    p=F(self.p, c.nz + 1), dp=[F(t, c.nz) for t in self.dp], d=[F(t, c.nz + 1) for t in self.d],
                    big=[B(t) for t in self.big])


@pytest.mark.parametrize("prec", ["f64", "mixed"])
@pytest.mark.parametrize("P,nx,ny,L", [(2, 64, 64, 32), (4, 64, 48, 32), (3, 32, 32, 24)])
def test_slab_split_matches_single_domain(prec, P, nx, ny, L):
    import torch
    nzt = L + 1
    f = identical_inputs(fields.make_fields(nx, ny, nzt), prec)
    # single domain
    one = obl.Context(nx, ny, nzt, precision=prec, top_bc="neumann", **fields.DOMAIN)
    b1 = Bufs(one, f)
    io = b1.io()
    one.step_dev(io.u, io.v, io.w, io.theta, list(io.d), list(io.big), io.p, list(io.dp))
    one.synchronize()
    ref = b1.get()
    # P slabs
    nzt_r, lz_r = slab.slab_grid(nx, ny, nzt, fields.DOMAIN["lz_tot"], P)
    Lr = L // P
    dom = dict(fields.DOMAIN, lz_tot=lz_r)
    ctxs = [obl.Context(nx, ny, nzt_r, precision=prec, top_bc="neumann", **dom) for _ in range(P)]
    bufs = [Bufs(c, {k: np.asfortranarray(v[:, :, r * Lr: r * Lr + Lr + 2]) for k, v in f.items()})
            for r, c in enumerate(ctxs)]
    steps = [slab.SlabStep(slab.LibBackend(c), r, P) for r, c in enumerate(ctxs)]
    slab.step_lockstep(steps, [b.io() for b in bufs])
    torch.cuda.synchronize()
    tol = 1e-11 if prec == "f64" else 2e-6
    for r, b in enumerate(bufs):
        got = b.get()
        g0 = r * Lr                        # global level of local level 0
        lv = slice(1, Lr + 1)              # the rank's own levels
        gl = slice(g0 + 1, g0 + Lr + 1)
        for k in ("u", "v", "w"):
            assert rel_l2(got[k][:nx, :, lv], ref[k][:nx, :, gl]) < tol, (r, k)
        assert rel_l2(got["p"][:nx, :, 0: Lr + 1], ref["p"][:nx, :, g0: g0 + Lr + 1]) < tol, (r, "p")
        for i in range(3):
            assert rel_l2(got["dp"][i][:nx, :, 0:Lr], ref["dp"][i][:nx, :, g0: g0 + Lr]) < tol, (r, "dp", i)
        for i in range(8):
            assert rel_l2(got["d"][i][:nx, :, lv], ref["d"][i][:nx, :, gl]) < tol, (r, "d", i)
        for i in range(4):
            assert rel_l2(got["big"][i][:, :, lv], ref["big"][i][:, :, gl]) < tol, (r, "big", i)


@pytest.mark.parametrize("prec", ["f64", "mixed"])
@pytest.mark.parametrize("stress_free", [False, True])
def test_slab_split_with_divtz_planes(prec, stress_free):
    """divtz(:,:,1) enters on the bottom rank and divtz(:,:,nz) on the top rank, and the
    stress-free copy of project() on the top rank only; the split equals the single-domain
    step with the same planes and top condition."""
    import torch
    P, nx, ny, L = 2, 64, 64, 32
    nzt = L + 1
    f = identical_inputs(fields.make_fields(nx, ny, nzt), prec)
    rng = np.random.default_rng(5)
    dt = torch.float64 if prec == "f64" else torch.float32
    planes = [torch.from_numpy(np.asarray(rng.standard_normal(((nx + 2) * ny,)))).to("cuda", dt)
              for _ in range(2)]
    P_ = lambda t: t.data_ptr()
    one = obl.Context(nx, ny, nzt, precision=prec, top_bc="neumann", ubc_stress_free=stress_free,
                      **fields.DOMAIN)
    b1 = Bufs(one, f)
    io = b1.io()
    one.step_dev(io.u, io.v, io.w, io.theta, list(io.d), list(io.big), io.p, list(io.dp),
                 P_(planes[0]), P_(planes[1]))
    one.synchronize()
    ref = b1.get()
    nzt_r, lz_r = slab.slab_grid(nx, ny, nzt, fields.DOMAIN["lz_tot"], P)
    Lr = L // P
    dom = dict(fields.DOMAIN, lz_tot=lz_r)
    ctxs = [obl.Context(nx, ny, nzt_r, precision=prec, top_bc="neumann", ubc_stress_free=stress_free, **dom)
            for _ in range(P)]
    bufs = [Bufs(c, {k: np.asfortranarray(v[:, :, r * Lr: r * Lr + Lr + 2]) for k, v in f.items()})
            for r, c in enumerate(ctxs)]
    ios = []
    for r, b in enumerate(bufs):
        x = b.io()
        ios.append(obl.stepio_dev(x.u, x.v, x.w, x.theta, list(x.d), list(x.big), x.p, list(x.dp),
                                  P_(planes[0]) if r == 0 else None, P_(planes[1]) if r == P - 1 else None))
    steps = [slab.SlabStep(slab.LibBackend(c), r, P) for r, c in enumerate(ctxs)]
    slab.step_lockstep(steps, ios)
    torch.cuda.synchronize()
    tol = 1e-11 if prec == "f64" else 2e-6
    for r, b in enumerate(bufs):
        got = b.get()
        g0 = r * Lr
        assert rel_l2(got["p"][:nx, :, 0: Lr + 1], ref["p"][:nx, :, g0: g0 + Lr + 1]) < tol, r
        for i in range(3):
            assert rel_l2(got["dp"][i][:nx, :, 0:Lr], ref["dp"][i][:nx, :, g0: g0 + Lr]) < tol, (r, i)
        lv, gl = slice(1, Lr + 1), slice(g0 + 1, g0 + Lr + 1)
        for k in ("u", "v", "w"):
            assert rel_l2(got[k][:nx, :, lv], ref[k][:nx, :, gl]) < tol, (r, k)
