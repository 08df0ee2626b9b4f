"""GPU parity of every hot-path entry point against the FP64 oracle, through the
C ABI (host-array variants).  FP64 form: relative L2 <= 1e-12.  Mixed form (FP32
FFTs with FP64 TDMA islands): relative L2 <= 1e-5 per output field."""
import numpy as np
import pytest

import overlappingbls_b200 as obl
from overlappingbls_b200 import fields
from conftest import identical_inputs, rel_l2

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "mixed": 1e-5}
GRIDS = {
    "config0": (64, 64, 65),      # the reference's CPU-runnable case
    "rect": (96, 64, 33),         # nx != ny, radix-3 lengths
    "rect2": (128, 192, 17),
    "radix5": (80, 160, 17),      # lengths with a factor 5 (and their 3/2 partners 120, 240)
    "radix5b": (320, 240, 9),
    "radix5c": (640, 80, 5),
}


@pytest.fixture(params=list(GRIDS))
def grid(request):
    return GRIDS[request.param]


@pytest.fixture(params=["f64", "mixed"])
def prec(request):
    return request.param


def _pair(orc, grid, prec, top="neumann"):
    nx, ny, nzt = grid
    ctx = obl.Context(nx, ny, nzt, precision=prec, top_bc=top, **fields.DOMAIN)
    g = orc.Grid(nx, ny, nzt, **fields.DOMAIN)
    f = identical_inputs(fields.make_fields(nx, ny, nzt), prec)
    return ctx, g, f


def test_ddx_ddy(orc, grid, prec):
    ctx, g, f = _pair(orc, grid, prec)
    nx = g.nxt
    for name in ("u", "w", "theta"):
        for op in ("ddx", "ddy"):
            out = ctx.field()
            out[nx:] = 7.0   # pad columns are not written
            getattr(ctx, op)(out, f[name])
            ref = getattr(g, op)(f[name])
            assert rel_l2(out[:nx], ref[:nx]) < TOL[prec], (name, op)
            assert np.all(out[nx:] == 7.0)


def test_fftn_ifftn(orc, grid, prec):
    ctx, g, f = _pair(orc, grid, prec)
    s = ctx.spectral()
    ctx.fftn(f["u"], s)
    for z in (0, 3, g.nz):
        assert rel_l2(s[:, :, z], g.fftn(f["u"][:, :, z])) < TOL[prec]
    back = ctx.field()
    ctx.ifftn(s, back)
    for z in (0, 3, g.nz):
        assert rel_l2(back[: g.nxt, :, z], g.ifftn(s[:, :, z])[: g.nxt]) < TOL[prec]


def test_zero_padding_unpadding(orc, grid, prec):
    ctx, g, f = _pair(orc, grid, prec)
    big = ctx.big_field()
    ctx.zero_padding(f["v"], big)
    for z in (0, 1, g.nz // 2, g.nz):
        assert rel_l2(big[:, :, z], g.zero_padding(f["v"][:, :, z])) < TOL[prec]
    rng = np.random.default_rng(5)
    big2 = np.asfortranarray(rng.standard_normal(big.shape))
    back = ctx.field()
    ctx.zero_unpadding(big2, back)
    for z in (0, 2, g.nz):
        assert rel_l2(back[:, :, z], g.zero_unpadding(big2[:, :, z])) < TOL[prec]


def test_filter_data(orc, grid, prec):
    ctx, g, f = _pair(orc, grid, prec)
    a = f["w"].copy(order="F")
    a[g.nxt:] = 3.0
    ctx.filter_data(a)
    assert rel_l2(a, g.filter_data(np.where(np.arange(g.ldx)[:, None, None] >= g.nxt, 3.0, f["w"]))) < TOL[prec]


def test_ddz(orc, grid, prec):
    ctx, g, f = _pair(orc, grid, prec)
    for op in ("ddz_uv", "ddz_w"):
        out = ctx.field() + 11.0
        ref = g.field() + 11.0
        getattr(ctx, op)(out, f["u"])
        getattr(g, op)(f["u"], ref)
        assert rel_l2(out, ref) < TOL[prec], op


@pytest.mark.parametrize("top,npz", [("neumann", 2), ("single", 1)])
def test_press_stag_array_and_project(orc, grid, prec, top, npz):
    ctx, g, f = _pair(orc, grid, prec, top)
    nx, L = g.nxt, g.nz - 1
    rng = np.random.default_rng(9)
    dbot = np.asfortranarray(rng.standard_normal((g.ldx, g.nyt)) * 1e-3)
    dtop = np.asfortranarray(rng.standard_normal((g.ldx, g.nyt)) * 1e-3)
    p, dpx, dpy = ctx.field(), ctx.dfield(), ctx.dfield()
    ctx.press_stag_array(p, dpx, dpy, f["u"], f["v"], f["w"], dbot, dtop)
    rp, rdx, rdy = g.press_stag_array(f["u"], f["v"], f["w"], dbot, dtop, npz=npz)
    assert rel_l2(p[:nx, :, : L + 1], rp[:nx, :, : L + 1]) < TOL[prec]
    assert rel_l2(dpx[:nx, :, :L], rdx[:nx, :, :L]) < TOL[prec]
    assert rel_l2(dpy[:nx, :, :L], rdy[:nx, :, :L]) < TOL[prec]
    dz = ctx.dfield()
    ctx.dpdz(dz, p)
    rdz = g.dpdz(rp)
    assert rel_l2(dz[:nx, :, :L], rdz[:nx, :, :L]) < TOL[prec]
    u, v, w = (f[k].copy(order="F") for k in "uvw")
    ctx.project(u, v, w, dpx, dpy, dz)
    ru, rv, rw = g.project(f["u"], f["v"], f["w"], rdx, rdy, rdz)
    for a, b in ((u, ru), (v, rv), (w, rw)):
        assert rel_l2(a, b) < TOL[prec]


@pytest.mark.parametrize("nx,ny,nzt", [(512, 512, 17), (384, 384, 9), (80, 160, 9), (640, 640, 5), (96, 64, 33)])
def test_y_pad_by_tensor_copies(nx, ny, nzt):
    """The FP32 y-pad whose input tiles arrive by tensor-map copies (`pad_tma` = 1) gives the
    results of the load-fed y-pad: through zero_padding and through the step's padded
    fields.  Boxes of 256, 192, 160, 128 and 64 rows; at nxt = 80 the last box of a plane
    row runs past the 120 padded columns and is zero-filled."""
    f = fields.make_fields(nx, ny, nzt)
    f = {k: np.asfortranarray(v.astype(np.float32).astype(np.float64)) for k, v in f.items()}
    ctx = obl.Context(nx, ny, nzt, precision="mixed", **fields.DOMAIN)
    outs = {}
    for tma in (1, 0):
        ctx.set_param("pad_tma", tma)
        big = ctx.big_field()
        ctx.zero_padding(f["u"], big)
        u, v, w = (f[k].copy(order="F") for k in "uvw")
        d = [ctx.field() for _ in range(8)]
        bigs = [ctx.big_field() for _ in range(4)]
        p, dp = ctx.field(), [ctx.dfield() for _ in range(3)]
        ctx.step(u, v, w, f["theta"], d, bigs, p, dp)
        ctx.synchronize()
        outs[tma] = [big] + bigs
    same = all(np.array_equal(a, b) for a, b in zip(outs[1], outs[0]))
    print(f"y-pad {nx}x{ny}: tensor-copy and load-fed results bitwise equal: {same}")
    for a, b in zip(outs[1], outs[0]):
        assert np.isfinite(a).all()
        assert rel_l2(a, b) < 1e-6
    ctx.close()
