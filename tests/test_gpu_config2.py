"""The headline workload at its stated size (512 x 512 x 256 levels, Neumann top, the
seeded boundary-layer fields with theta) against the FP64 oracle, every output of the
step: the 8 horizontal derivatives, the 4 padded fields, p, dpdx, dpdy, dpdz and the
projected u, v, w.  Mixed form <= 1e-5 and FP64 form <= 1e-12 relative L2 per field, on
identical FP32-representable inputs.  The oracle's step is the composition of
ddx/ddy (004_derivatives.f90:18-81), zero_padding (108_01_padd.f90:73-132),
press_stag_array with its rank pipeline (109_press_stag_array.f90:107-319, npz = 2),
dpdz (103_flosol.f90:169-175) and project (110_project.f90:4-62)."""
import os

import numpy as np
import pytest

import overlappingbls_b200 as obl
from overlappingbls_b200 import fields
from conftest import identical_inputs

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "mixed": 1e-5}
NX = NY = 512
NZT = 257
NAMES = ["dudx", "dudy", "dvdx", "dvdy", "dwdx", "dwdy", "dtdx", "dtdy",
         "u_big", "v_big", "w_big", "t_big", "p", "dpdx", "dpdy", "dpdz", "u", "v", "w"]


@pytest.fixture(scope="module")
def headline(orc):
    f = identical_inputs(fields.make_fields(NX, NY, NZT), "mixed")
    try:
        threads = len(os.sched_getaffinity(0))
    except Exception:
        threads = os.cpu_count()
    orc.set_threads(threads)
    g = orc.Grid(NX, NY, NZT, **fields.DOMAIN)
    ref = g.step(f["u"], f["v"], f["w"], f["theta"], npz=2)
    refs = [ref["d"][i] for i in range(8)] + [ref["big"][i] for i in range(4)] + \
           [ref["p"], ref["dpdx"], ref["dpdy"], ref["dpdz"], ref["u"], ref["v"], ref["w"]]
    return f, refs


@pytest.mark.parametrize("prec", ["mixed", "f64"])
def test_headline_step_matches_oracle(headline, prec):
    import torch
    f, refs = headline
    ctx = obl.Context(NX, NY, NZT, precision=prec, top_bc="neumann", **fields.DOMAIN)
    inf = ctx.info
    dt = torch.float64 if inf["elem_bytes"] == 8 else torch.float32
    dev = torch.device("cuda", 0)
    ldx, L = inf["ldx"], inf["nz"] - 1
    nf, nd, nb = inf["field_elems"], inf["dfield_elems"], inf["big_elems"]
    t = {k: torch.from_numpy(f[k].ravel(order="F")).to(dev, dt) for k in ("u", "v", "w", "theta")}
    d = [torch.full((nf,), float("nan"), dtype=dt, device=dev) for _ in range(8)]
    big = [torch.full((nb,), float("nan"), dtype=dt, device=dev) for _ in range(4)]
    p = torch.full((nf,), float("nan"), dtype=dt, device=dev)
    dp = [torch.full((nd,), float("nan"), dtype=dt, device=dev) for _ in range(3)]
    P = lambda x: x.data_ptr()
    ctx.step_dev(P(t["u"]), P(t["v"]), P(t["w"]), P(t["theta"]), [P(x) for x in d], [P(x) for x in big],
                 P(p), [P(x) for x in dp])
    ctx.synchronize()
    nd_valid = ldx * NY * L
    outs = [(x, True, None) for x in d] + [(x, False, None) for x in big] + [(p, True, ldx * NY * (L + 1))]
    outs += [(x, True, nd_valid) for x in dp] + [(t[k], False, None) for k in ("u", "v", "w")]
    errs = {}
    for nm, (a, cut, n), r in zip(NAMES, outs, refs):
        b = torch.from_numpy(np.ravel(r, order="F")).to(dev)
        if n is not None:
            a, b = a[:n], b[:n]
        a = a.double()
        if cut:
            a, b = a.view(-1, ldx)[:, :NX], b.view(-1, ldx)[:, :NX]
        assert bool(torch.isfinite(a).all()), nm
        errs[nm] = float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
        del a, b
    print(f"\n512x512x256 levels, {prec} vs the FP64 oracle (relative L2), "
          f"{inf['n_fp64_columns']} FP64 columns:")
    for nm, e in errs.items():
        print(f"  {nm:6s} {e:.3e}")
    worst = max(errs, key=errs.get)
    assert errs[worst] < TOL[prec], (worst, errs[worst])
    ctx.close()
