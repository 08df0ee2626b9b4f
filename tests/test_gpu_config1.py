"""256x256x128 levels, FP32-mixed: relative L2 error of every output of the step against
the FP64 oracle (npz >= 2 top), on identical FP32-representable inputs; gate 1e-5.
Prints the per-field report and the number of FP64 solve columns."""
import numpy as np
import pytest

import overlappingbls_b200 as obl
from overlappingbls_b200 import fields
from conftest import identical_inputs, rel_l2

pytestmark = pytest.mark.gpu

NAMES = ["dudx", "dudy", "dvdx", "dvdy", "dwdx", "dwdy", "dTdx", "dTdy"]


def test_config1_per_field_errors(orc):
    nx, ny, nzt = 256, 256, 129
    orc.set_threads(0)
    f = identical_inputs(fields.make_fields(nx, ny, nzt), "mixed")
    ctx = obl.Context(nx, ny, nzt, precision="mixed", top_bc="neumann", **fields.DOMAIN)
    u, v, w = (f[k].copy(order="F") for k in "uvw")
    d = [ctx.field() for _ in range(8)]
    big = [ctx.big_field() for _ in range(4)]
    p, dp = ctx.field(), [ctx.dfield() for _ in range(3)]
    ctx.step(u, v, w, f["theta"], d, big, p, dp)
    g = orc.Grid(nx, ny, nzt, **fields.DOMAIN)
    ref = g.step(f["u"], f["v"], f["w"], f["theta"], npz=2)
    L = g.nz - 1
    errs = {}
    for i, n in enumerate(NAMES):
        errs[n] = rel_l2(d[i][:nx], ref["d"][i][:nx])
    for i, n in enumerate(["u_big", "v_big", "w_big", "T_big"]):
        errs[n] = rel_l2(big[i], ref["big"][i])
    errs["p"] = rel_l2(p[:nx, :, : L + 1], ref["p"][:nx, :, : L + 1])
    for a, n in zip(dp, ("dpdx", "dpdy", "dpdz")):
        errs[n] = rel_l2(a[:nx, :, :L], ref[n][:nx, :, :L])
    for a, n in ((u, "u"), (v, "v"), (w, "w")):
        errs[n] = rel_l2(a[:nx], ref[n][:nx])
    print("config1 256x256x128 mixed vs FP64 oracle: fp64 columns", ctx.info["n_fp64_columns"])
    for n, e in errs.items():
        print(f"config1 {n:6s} {e:.3e}")
    assert max(errs.values()) <= 1e-5, errs
