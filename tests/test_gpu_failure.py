"""Host-side failure paths (no GPU fault involved).

Device allocations: every allocation the library makes goes through one function whose
n-th call from a given point can be made to fail as cudaMalloc would (the "fail_alloc"
parameter of a context, or OBL_FAIL_ALLOC for the allocations of obl_ctx_create).  Each
entry point must then return OBL_ERR_NOMEM with a message, leave the context usable, and
give the right answer once allocation works again; a context whose creation fails must
clean up after itself.  The reference has no such paths: it stops the run on errors
(102_initial.f90:164-168)."""
import numpy as np
import pytest

import overlappingbls_b200 as obl
from overlappingbls_b200 import fields
from conftest import rel_l2

pytestmark = pytest.mark.gpu

NX, NY, NZT = 64, 48, 17


def test_context_creation_fails_cleanly_at_every_allocation(monkeypatch):
    import torch
    free0 = torch.cuda.mem_get_info(0)[0]
    first_ok = None
    for n in range(1, 64):
        monkeypatch.setenv("OBL_FAIL_ALLOC", str(n))
        try:
            ctx = obl.Context(NX, NY, NZT, precision="mixed", **fields.DOMAIN)
        except obl.OblError as e:
            assert "OBL_ERR_NOMEM" in str(e), str(e)
            continue
        ctx.close()
        first_ok = n
        break
    monkeypatch.delenv("OBL_FAIL_ALLOC")
    # several allocations were each failed in turn, then creation needed no more
    assert first_ok is not None and first_ok > 3, first_ok
    torch.cuda.synchronize()
    # the failed creations freed what they had allocated (allow for allocator granularity)
    assert torch.cuda.mem_get_info(0)[0] >= free0 - (4 << 20)


def _entry_points(ctx, g, f):
    """(name, call, check) triples on host arrays; check compares with the oracle."""
    L = g.nz - 1

    def ddx():
        out = ctx.field()
        ctx.ddx(out, f["u"])
        return rel_l2(out[:NX], g.ddx(f["u"])[:NX])

    def pad():
        big = np.zeros((ctx.nxt2, ctx.nyt2), order="F")
        ctx.zero_padding(f["u"][:, :, 3], big)
        return rel_l2(big, g.zero_padding(f["u"][:, :, 3]))

    def press():
        p, dx, dy = ctx.field(), ctx.dfield(), ctx.dfield()
        ctx.press_stag_array(p, dx, dy, f["u"], f["v"], f["w"])
        rp, _, _ = g.press_stag_array(f["u"], f["v"], f["w"], npz=2)
        return rel_l2(p[:NX, :, :L + 1], rp[:NX, :, :L + 1])

    def step():
        u, v, w = (f[k].copy(order="F") for k in "uvw")
        d = [ctx.field() for _ in range(8)]
        big = [ctx.big_field() for _ in range(4)]
        p, dp = ctx.field(), [ctx.dfield() for _ in range(3)]
        ctx.step(u, v, w, f["theta"], d, big, p, dp)
        ref = g.step(f["u"], f["v"], f["w"], f["theta"], npz=2)
        return max(rel_l2(p[:NX, :, :L + 1], ref["p"][:NX, :, :L + 1]), rel_l2(w, ref["w"]))

    def rollout():
        u, v, w = (f[k].copy(order="F") for k in "uvw")
        ctx.rollout_step(u, v, w)
        ru, rv, rw = g.rollout_step(f["u"], f["v"], f["w"])
        return max(rel_l2(u, ru), rel_l2(w, rw))

    return [("ddx", ddx), ("zero_padding", pad), ("press_stag_array", press), ("step", step),
            ("rollout_step", rollout)]


@pytest.mark.parametrize("which", range(5))
def test_entry_point_allocation_failure_then_recovery(orc, which):
    g = orc.Grid(NX, NY, NZT, **fields.DOMAIN)
    f = fields.make_fields(NX, NY, NZT)
    ctx = obl.Context(NX, NY, NZT, precision="f64", **fields.DOMAIN)
    name, call = _entry_points(ctx, g, f)[which]
    ctx.set_param("fail_alloc", 1)          # the next device allocation fails
    with pytest.raises(obl.OblError) as ei:
        call()
    assert "OBL_ERR_NOMEM" in str(ei.value) and "allocation" in str(ei.value), (name, str(ei.value))
    assert ctx.get_param("fail_alloc") == 0
    # the context is still usable and the answer is right
    assert call() < 1e-12, name
    ctx.close()


def test_staged_solve_wait_gives_up(orc):
    """The staged pressure solve waits for its bulk copies on mbarriers with a bound of
    about a second.  With bytes expected that no copy delivers (the `stage_timeout_test`
    parameter), every wait gives up, the step returns OBL_ERR_TIMEOUT when it synchronizes,
    and the context then steps correctly again."""
    import time
    nx, ny, nzt = 64, 64, 65
    L = nzt - 2
    g = orc.Grid(nx, ny, nzt, **fields.DOMAIN)
    f = fields.make_fields(nx, ny, nzt)
    ctx = obl.Context(nx, ny, nzt, precision="mixed", **fields.DOMAIN)
    ctx.set_param("tdma_segments", 1)   # the whole-column solve (few columns pick the column-segmented one)
    ctx.set_param("tdma_stage", 1)      # its copy-fed form (by default only above 128 levels)

    def step():
        u, v, w = (f[k].copy(order="F") for k in "uvw")
        d = [ctx.field() for _ in range(8)]
        big = [ctx.big_field() for _ in range(4)]
        p, dp = ctx.field(), [ctx.dfield() for _ in range(3)]
        ctx.step(u, v, w, f["theta"], d, big, p, dp)
        return p, w

    ctx.set_param("stage_timeout_test", 1)
    t0 = time.perf_counter()
    with pytest.raises(obl.OblError, match="OBL_ERR_TIMEOUT"):
        step()
    waited = time.perf_counter() - t0
    assert waited < 30.0
    ctx.set_param("stage_timeout_test", 0)
    p, w = step()
    ref = g.step(f["u"], f["v"], f["w"], f["theta"], npz=2)
    assert rel_l2(p[:nx, :, :L + 1], ref["p"][:nx, :, :L + 1]) < 1e-5
    assert rel_l2(w, ref["w"]) < 1e-5
    print(f"staged solve: the waits gave up and the step returned after {waited:.1f} s")
    ctx.close()
