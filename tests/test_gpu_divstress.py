"""GPU parity of divstress_uv / divstress_w (107_divstress.f90:4-104) through the C ABI.

* host entry points against the FP64 oracle: computed levels within the tolerance of the
  other operators (FP64 rel L2 <= 1e-12, mixed <= 1e-5), the x pads exactly 0 and the
  BOGUS levels exactly BOGUS in the storage type; input pad columns are never read;
* device entry points equal the host ones bit for bit on the same storage values;
* divstress_w's wall and top levels fed to press_stag_array as divtz(1), divtz(nz)
  give the oracle's pressure with the oracle's planes;
* at 512x512x256 levels (mixed): the fused result against the separately tested ddx,
  ddy, ddz entry points (a size-independent property), and the device time.
"""
import numpy as np
import pytest

import overlappingbls_b200 as obl
from overlappingbls_b200 import fields
from conftest import identical_inputs, rel_l2

pytestmark = pytest.mark.gpu

BOGUS = -1234567890.0
TOL = {"f64": 1e-12, "mixed": 1e-5}
GRIDS = {"config0": (64, 64, 65), "rect": (96, 64, 33), "rect2": (128, 192, 17), "small": (32, 48, 9)}


def _stress(nx, ny, nzt, prec, seed=0):
    rng = np.random.default_rng(seed)
    ldx = nx + 2
    out = {}
    for k in ("tx", "ty", "tz"):
        a = np.asfortranarray(rng.standard_normal((ldx, ny, nzt + 1)))
        a[nx:] = 1e3   # pad columns: never read
        out[k] = a
    return identical_inputs(out, prec)


def _levels(form, nz):
    return (list(range(1, nz)), [0, nz]) if form == "uv" else (list(range(1, nz + 1)), [0])


@pytest.mark.parametrize("prec", ["f64", "mixed"])
@pytest.mark.parametrize("form", ["uv", "w"])
@pytest.mark.parametrize("name", list(GRIDS))
def test_divstress_matches_oracle(orc, name, form, prec):
    nx, ny, nzt = GRIDS[name]
    ctx = obl.Context(nx, ny, nzt, precision=prec, **fields.DOMAIN)
    g = orc.Grid(nx, ny, nzt, **fields.DOMAIN)
    t = _stress(nx, ny, nzt, prec)
    out = ctx.field() + 5.0
    getattr(ctx, "divstress_" + form)(out, t["tx"], t["ty"], t["tz"])
    ref = getattr(g, "divstress_" + form)(t["tx"], t["ty"], t["tz"])
    lv, bog = _levels(form, g.nz)
    assert rel_l2(out[:nx, :, lv], ref[:nx, :, lv]) < TOL[prec]
    assert np.all(out[nx:, :, lv] == 0.0)
    b = BOGUS if prec == "f64" else float(np.float32(BOGUS))
    assert np.all(out[:, :, bog] == b)
    ctx.close()


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_divstress_dev_equals_host(prec):
    import torch
    nx, ny, nzt = 96, 64, 33
    ctx = obl.Context(nx, ny, nzt, precision=prec, **fields.DOMAIN)
    t = _stress(nx, ny, nzt, prec, seed=3)
    dt = torch.float64 if prec == "f64" else torch.float32
    dev = {k: torch.from_numpy(v.ravel(order="F")).to("cuda", dt) for k, v in t.items()}
    for form in ("uv", "w"):
        host = ctx.field()
        getattr(ctx, "divstress_" + form)(host, t["tx"], t["ty"], t["tz"])
        d = torch.full((host.size,), 5.0, dtype=dt, device="cuda")
        getattr(ctx, "divstress_" + form + "_dev")(d.data_ptr(), dev["tx"].data_ptr(), dev["ty"].data_ptr(),
                                                    dev["tz"].data_ptr())
        ctx.synchronize()
        got = d.double().cpu().numpy().reshape(host.shape, order="F")
        assert np.array_equal(got, host), form
    ctx.close()


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_divstress_w_feeds_press_boundary_rows(orc, prec):
    nx, ny, nzt = GRIDS["config0"]
    ctx = obl.Context(nx, ny, nzt, precision=prec, top_bc="neumann", **fields.DOMAIN)
    g = orc.Grid(nx, ny, nzt, **fields.DOMAIN)
    f = identical_inputs(fields.make_fields(nx, ny, nzt), prec)
    t = {k: 1e-2 * v for k, v in _stress(nx, ny, nzt, prec, seed=7).items()}
    t = identical_inputs(t, prec)
    nz, L = g.nz, g.nz - 1
    divt = ctx.field()
    ctx.divstress_w(divt, t["tx"], t["ty"], t["tz"])
    ref = g.divstress_w(t["tx"], t["ty"], t["tz"])
    p, dpx, dpy = ctx.field(), ctx.dfield(), ctx.dfield()
    ctx.press_stag_array(p, dpx, dpy, f["u"], f["v"], f["w"], np.asfortranarray(divt[:, :, 1]),
                         np.asfortranarray(divt[:, :, nz]))
    rp, rdx, rdy = g.press_stag_array(f["u"], f["v"], f["w"], np.asfortranarray(ref[:, :, 1]),
                                      np.asfortranarray(ref[:, :, nz]), npz=2)
    assert rel_l2(p[:nx, :, :L + 1], rp[:nx, :, :L + 1]) < TOL[prec]
    assert rel_l2(dpx[:nx, :, :L], rdx[:nx, :, :L]) < TOL[prec]
    assert rel_l2(dpy[:nx, :, :L], rdy[:nx, :, :L]) < TOL[prec]
    ctx.close()


def test_divstress_512_full_size():
    """512x512 with 256 computed levels, FP32 storage: the fused passes against ddx + ddy +
    ddz from their own entry points, then the device time of each form."""
    import torch
    nx = ny = 512
    nzt = 257
    ctx = obl.Context(nx, ny, nzt, precision="mixed", **fields.DOMAIN)
    ldx, nz = nx + 2, ctx.nz
    n = ldx * ny * (nz + 1)
    gen = torch.Generator(device="cuda").manual_seed(11)
    tx, ty, tz = (torch.randn(n, device="cuda", generator=gen) for _ in range(3))
    out = torch.empty(n, device="cuda")
    parts = [torch.empty(n, device="cuda") for _ in range(3)]
    P = lambda a: a.data_ptr()
    shp = (nz + 1, ny, ldx)
    ctx.ddx_dev(P(parts[0]), P(tx), nz + 1)
    ctx.ddy_dev(P(parts[1]), P(ty), nz + 1)
    report = []
    for form, ddz in (("uv", ctx.ddz_w_dev), ("w", ctx.ddz_uv_dev)):
        ddz(P(parts[2]), P(tz))
        getattr(ctx, "divstress_" + form + "_dev")(P(out), P(tx), P(ty), P(tz))
        ctx.synchronize()
        o = out.view(shp)
        dx, dy, dzt = (q.view(shp).double() for q in parts)
        ref = dx + dy
        if form == "uv":
            ref[1:nz] += dzt[1:nz]
            lv = slice(1, nz)
        else:
            ref[2:nz] += dzt[2:nz]
            lv = slice(1, nz + 1)
        assert rel_l2(o[lv, :, :nx].double().cpu().numpy(), ref[lv, :, :nx].cpu().numpy()) < 1e-6
        assert bool((o[lv, :, nx:] == 0).all())
        # time: inputs (3 x 270 MB) and output are far larger than L2
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        run = lambda: getattr(ctx, "divstress_" + form + "_dev")(P(out), P(tx), P(ty), P(tz))
        for _ in range(3):
            run()
        torch.cuda.synchronize()
        ev[0].record()
        reps = 10
        for _ in range(reps):
            run()
        ev[1].record()
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1]) / reps
        pts = nx * ny * (nz - 1 if form == "uv" else nz)
        report.append(f"divstress_{form}: {ms:.3f} ms, {pts / ms / 1e3:.0f} Mpts/s, "
                      f"{16 * pts / ms / 1e6:.0f} GB/s algorithmic (16 B/pt)")
    print("; ".join(report))
    ctx.close()


@pytest.mark.parametrize("prec", ["f64", "mixed"])
@pytest.mark.parametrize("form", ["uv", "w"])
def test_divstress_z_ranks_match_whole_domain(prec, form):
    """z-rank roles (107_divstress.f90:81-102): two ranks, each holding its levels with the
    ghost levels 0 and nz from its neighbours, give the whole-domain result on every level
    they compute; rank 0 leaves the wall level without dz(tzz), only the top rank computes
    level nz of divstress_w, and the others leave it BOGUS."""
    import torch
    from overlappingbls_b200 import slab
    nx, ny, P, Lr = 64, 48, 2, 8
    nzt = P * Lr + 1
    whole = obl.Context(nx, ny, nzt, precision=prec, **fields.DOMAIN)
    t = _stress(nx, ny, nzt, prec, seed=11)
    ref = whole.field()
    getattr(whole, "divstress_" + form)(ref, t["tx"], t["ty"], t["tz"])
    whole.close()
    nzt_r, lz_r = slab.slab_grid(nx, ny, nzt, fields.DOMAIN["lz_tot"], P)
    dt = torch.float64 if prec == "f64" else torch.float32
    b = BOGUS if prec == "f64" else float(np.float32(BOGUS))
    tol = 1e-14 if prec == "f64" else 1e-6
    for r in range(P):
        ctx = obl.Context(nx, ny, nzt_r, precision=prec, **dict(fields.DOMAIN, lz_tot=lz_r))
        nz = ctx.nz
        loc = {k: torch.from_numpy(np.asfortranarray(v[:, :, r * Lr: r * Lr + nz + 1]).ravel(order="F")).to("cuda", dt)
               for k, v in t.items()}
        out = torch.full(((nx + 2) * ny * (nz + 1),), 5.0, dtype=dt, device="cuda")
        getattr(ctx, "divstress_" + form + "_slab_dev")(out.data_ptr(), loc["tx"].data_ptr(), loc["ty"].data_ptr(),
                                                        loc["tz"].data_ptr(), r, P)
        ctx.synchronize()
        got = out.double().cpu().numpy().reshape((nx + 2, ny, nz + 1), order="F")
        top = r == P - 1
        lv = list(range(1, nz + 1)) if (form == "w" and top) else list(range(1, nz))
        gl = [r * Lr + k for k in lv]
        assert rel_l2(got[:nx, :, lv], ref[:nx, :, gl]) <= tol, r
        assert np.all(got[nx:, :, lv] == 0.0)
        assert np.all(got[:, :, 0] == b)
        if not (form == "w" and top):
            assert np.all(got[:, :, nz] == b)
        ctx.close()
