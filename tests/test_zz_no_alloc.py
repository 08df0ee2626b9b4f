"""GPU test of obl_zero_padding_noalloc_dev, the zero_padding variant that allocates
nothing (for callers that may not allocate device memory when they call: an application
whose device memory all belongs to its own pool, or a latency-critical path where
cudaMalloc/cudaFree would block).  Its scratch is a static device array, so the test
checks, through the C ABI, that two calls in a row give the same result as the
allocating entry point obl_zero_padding_dev, that the calls do not change the free
device memory, and that a request larger than the static scratch is refused.

The file name sorts last so that a run stopping at the first failure has already run
every other test."""
import numpy as np
import pytest

import overlappingbls_b200 as obl
from overlappingbls_b200 import fields
from conftest import identical_inputs, rel_l2

pytestmark = pytest.mark.gpu

TOL = {"f64": 1e-12, "mixed": 1e-5}
SCRATCH = 8 << 20   # OBL_NOALLOC_SCRATCH_BYTES


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_noalloc_matches_allocating_entry_point(prec):
    import torch

    nx, ny, nzt = 512, 512, 9
    ctx = obl.Context(nx, ny, nzt, precision=prec, **fields.DOMAIN)
    es = ctx.info["elem_bytes"]
    dt = torch.float64 if es == 8 else torch.float32
    nlev = SCRATCH // (es * ctx.nxt2 * ny)          # as many levels as the scratch holds
    assert nlev >= 1
    f = identical_inputs(fields.make_fields(nx, ny, nzt), prec)
    dev = torch.device("cuda", 0)
    plane = ctx.ldx * ny
    big_n = ctx.nxt2 * ctx.nyt2 * nlev

    def dfield(name):
        return torch.from_numpy(f[name][:, :, 1:1 + nlev].ravel(order="F").copy()).to(dev, dt)

    inputs = [dfield("u"), dfield("theta")]
    assert inputs[0].numel() == plane * nlev
    ref = [torch.zeros(big_n, dtype=dt, device=dev) for _ in inputs]
    out = [torch.full((big_n,), float("nan"), dtype=dt, device=dev) for _ in inputs]

    # first call on this device looks up the scratch address (not timed, not measured)
    warm = torch.zeros(big_n, dtype=dt, device=dev)
    ctx.zero_padding_noalloc_dev(inputs[0].data_ptr(), warm.data_ptr(), nlev)
    torch.cuda.synchronize()

    free0 = torch.cuda.mem_get_info(0)[0]
    for x, o in zip(inputs, out):                    # two calls in a row
        ctx.zero_padding_noalloc_dev(x.data_ptr(), o.data_ptr(), nlev)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info(0)[0]
    assert free1 == free0, "the no-allocation entry point changed the free device memory"

    for x, r in zip(inputs, ref):
        ctx.zero_padding_dev(x.data_ptr(), r.data_ptr(), nlev)
    torch.cuda.synchronize()
    for o, r in zip(out, ref):
        a = o.double().cpu().numpy()
        b = r.double().cpu().numpy()
        assert np.isfinite(a).all()
        assert rel_l2(a, b) < TOL[prec]

    # a request beyond the static scratch is refused with a clear error
    too_many = nlev + 2
    big_x = torch.zeros(plane * too_many, dtype=dt, device=dev)
    big_o = torch.zeros(ctx.nxt2 * ctx.nyt2 * too_many, dtype=dt, device=dev)
    with pytest.raises(obl.OblError, match="static scratch"):
        ctx.zero_padding_noalloc_dev(big_x.data_ptr(), big_o.data_ptr(), too_many)
    ctx.close()
