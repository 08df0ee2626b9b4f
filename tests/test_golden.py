"""The C oracle against the committed golden fixtures, which come from an
independent numpy/scipy restatement of the reference (tests/golden/gen_golden.py)."""
import os

import numpy as np
import pytest

from conftest import rel_l2

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ["g16x12x9", "g12x16x7"]
TOL = 1e-13


@pytest.fixture(params=CASES)
def case(request, orc):
    z = np.load(os.path.join(HERE, request.param + ".npz"))
    gp = z["grid"]
    g = orc.Grid(int(gp[0]), int(gp[1]), int(gp[2]), *[float(x) for x in gp[3:]])
    return g, {k: np.asfortranarray(z[k]) for k in z.files}


def test_derivatives(case):
    g, z = case
    nx = g.nxt
    assert rel_l2(g.ddx(z["u"])[:nx], z["ddx_u"][:nx]) < TOL
    assert rel_l2(g.ddy(z["u"])[:nx], z["ddy_u"][:nx]) < TOL


def test_fftn_ifftn(case):
    g, z = case
    assert rel_l2(g.fftn(z["u"][:, :, 5]), z["fftn_u5"]) < TOL
    assert rel_l2(g.ifftn(z["fftn_u5"])[: g.nxt], z["ifftn_f"][: g.nxt]) < TOL


def test_padding(case):
    g, z = case
    assert rel_l2(g.zero_padding(z["u"][:, :, 3]), z["pad_u3"]) < TOL
    assert rel_l2(g.zero_unpadding(z["big_in"]), z["unpad_big"]) < TOL


@pytest.mark.parametrize("mode,npz", [("neumann", 2), ("neumann", 4), ("single", 1)])
def test_pressure_and_projection(case, mode, npz):
    g, z = case
    L = g.nz - 1
    if L % npz:
        pytest.skip("levels not divisible by npz")
    nx = g.nxt
    p, dpx, dpy = g.press_stag_array(z["u"], z["v"], z["w"], z["dbot"], z["dtop"], npz=npz)
    dz = g.dpdz(p)
    uu, vv, ww = g.project(z["u"], z["v"], z["w"], dpx, dpy, dz)
    assert rel_l2(p[:nx, :, : L + 1], z["p_" + mode][:nx, :, : L + 1]) < TOL
    assert rel_l2(dpx[:nx, :, :L], z["dpdx_" + mode][:nx, :, :L]) < TOL
    assert rel_l2(dpy[:nx, :, :L], z["dpdy_" + mode][:nx, :, :L]) < TOL
    assert rel_l2(dz[:nx, :, :L], z["dpdz_" + mode][:nx, :, :L]) < TOL
    for a, k in ((uu, "uproj_"), (vv, "vproj_"), (ww, "wproj_")):
        assert rel_l2(a, z[k + mode]) < TOL
