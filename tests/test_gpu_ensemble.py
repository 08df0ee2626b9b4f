"""GPU ensemble: many instances of different sizes through the step together.

Every mode (instance after instance, per-instance streams, one persistent launch) and
its CUDA-graph replay must give the result of the single-instance step on each
instance.  The 48-instance workload (16 each at 96x96x64, 128x128x96, 192x192x128
levels, FP32-mixed) is run in every mode and its aggregate throughput printed.
"""
import numpy as np
import pytest

import overlappingbls_b200 as obl
from overlappingbls_b200 import fields
from conftest import rel_l2

pytestmark = pytest.mark.gpu


class Buffers:
    """Device buffers of one instance's step (torch tensors in the storage type)."""

    def __init__(self, ctx, f):
        import torch
        self.torch = torch
        dt = torch.float64 if ctx.dtype == np.float64 else torch.float32
        nf = ctx.ldx * ctx.nyt * (ctx.nz + 1)
        nd = ctx.ldx * ctx.nyt * ctx.nz
        nb = ctx.nxt2 * ctx.nyt2 * (ctx.nz + 1)
        dev = "cuda"
        self.inputs = {k: torch.from_numpy(np.asarray(f[k], ctx.dtype).ravel(order="F")).to(dev)
                       for k in ("u", "v", "w", "theta")}
        self.f = {k: torch.empty(nf, dtype=dt, device=dev) for k in ("u", "v", "w", "theta")}
        self.d = [torch.empty(nf, dtype=dt, device=dev) for _ in range(8)]
        self.big = [torch.empty(nb, dtype=dt, device=dev) for _ in range(4)]
        self.p = torch.empty(nf, dtype=dt, device=dev)
        self.dp = [torch.empty(nd, dtype=dt, device=dev) for _ in range(3)]
        self.npts = ctx.nxt * ctx.nyt * (ctx.nzt - 1)
        self.nx = ctx.nxt
        self.shape = (ctx.ldx, ctx.nyt, ctx.nz + 1)
        self.reset()

    def reset(self):
        for k in self.f:
            self.f[k].copy_(self.inputs[k])
        for t in self.d + self.big + self.dp + [self.p]:
            t.fill_(float("nan"))
        # the ensemble runs on its own non-blocking stream: the fills must be done first
        self.torch.cuda.synchronize()

    def io(self):
        P = lambda t: t.data_ptr()
        return obl.stepio_dev(P(self.f["u"]), P(self.f["v"]), P(self.f["w"]), P(self.f["theta"]),
                              [P(t) for t in self.d], [P(t) for t in self.big], P(self.p),
                              [P(t) for t in self.dp])

    def outputs(self):
        """u, v, w, p, dpdx..dpdz, d[8], big[4] as float64 numpy (x < nxt where meaningful)."""
        out = [self.f[k] for k in ("u", "v", "w")] + [self.p] + self.dp + self.d + self.big
        return [t.double().cpu().numpy() for t in out]


def _members_small():
    return [dict(nxt=32, nyt=32, nzt=9, seed=1, theta_grad=0.01, z0=0.1),
            dict(nxt=48, nyt=48, nzt=17, seed=2, theta_grad=0.02, z0=0.5),
            dict(nxt=64, nyt=32, nzt=33, seed=3, theta_grad=0.0, z0=0.02),
            dict(nxt=96, nyt=96, nzt=17, seed=4, theta_grad=0.03, z0=1.0)]


def _grids(members):
    return [dict(nxt=m["nxt"], nyt=m["nyt"], nzt=m["nzt"], **fields.DOMAIN) for m in members]


def _fields(m):
    return fields.make_fields(m["nxt"], m["nyt"], m["nzt"], z0=m["z0"], theta_grad=m["theta_grad"],
                              seed=m["seed"])


def _compare(a, b, tol):
    """Worst relative L2 difference over the entries the reference wrote (finite)."""
    worst = 0.0
    for x, y in zip(a, b):
        x, y = x.reshape(-1), y.reshape(-1)
        ok = np.isfinite(y)
        assert np.isfinite(x[ok]).all(), "an entry the single-instance step writes was not written"
        e = rel_l2(x[ok], y[ok])
        worst = e if e > worst else worst
    assert worst <= tol, worst
    return worst


@pytest.mark.parametrize("prec", ["mixed", "f64"])
def test_ensemble_modes_match_single_instance(prec):
    members = _members_small()
    ens = obl.Ensemble(_grids(members), precision=prec)
    bufs = [Buffers(c, _fields(m)) for c, m in zip(ens.contexts, members)]
    ref = []
    for m, b in zip(members, bufs):   # single-instance reference: its own context
        ctx = obl.Context(m["nxt"], m["nyt"], m["nzt"], precision=prec, **fields.DOMAIN)
        b.reset()
        io = b.io()
        ctx.step_dev(io.u, io.v, io.w, io.theta, list(io.d), list(io.big), io.p, list(io.dp))
        ctx.synchronize()
        ref.append(b.outputs())
        ctx.close()
    for mode in ("sequential", "concurrent", "persistent", "persistent_split", "persistent_flow"):
        for graph in (False, True):
            ens.set_mode(mode)
            for b in bufs:
                b.reset()
            ios = [b.io() for b in bufs]
            if graph:
                ens.capture_dev(ios)   # runs one uncaptured step first
                for b in bufs:
                    b.reset()
                ens.replay()
            else:
                ens.step_dev(ios)
            ens.synchronize()
            for b, r in zip(bufs, ref):
                _compare(b.outputs(), r, 1e-6 if prec == "mixed" else 1e-13)
    ens.close()


def test_ensemble_rejects_unsupported_lengths():
    ens = obl.Ensemble(_grids([dict(nxt=384, nyt=384, nzt=9)]), precision="mixed")
    with pytest.raises(obl.OblError, match="UNSUPPORTED"):
        ens.set_mode("persistent")
    ens.close()


def test_config4_ensemble_48():
    members = fields.ensemble_members()
    assert len(members) == 48
    ens = obl.Ensemble(_grids(members), precision="mixed")
    bufs = [Buffers(c, _fields(m)) for c, m in zip(ens.contexts, members)]
    npts = sum(b.npts for b in bufs)
    ios = [b.io() for b in bufs]
    ens.set_mode("sequential")
    ens.step_dev(ios)
    ens.synchronize()
    ref = [b.outputs()[:8] for b in bufs]
    report = {}
    for mode in ("sequential", "concurrent", "persistent", "persistent_split", "persistent_flow"):
        ens.set_mode(mode)
        for graph in (False, True):
            ms = ens.time_dev(ios, use_graph=graph, warmup=3, reps=10)
            report[(mode, graph)] = ms
    ens.set_mode("persistent")
    for b in bufs:
        b.reset()
    ens.capture_dev(ios)
    for b in bufs:
        b.reset()
    ens.replay()
    ens.synchronize()
    worst = max(_compare(b.outputs()[:8], r, 1e-6) for b, r in zip(bufs, ref))
    base = report[("sequential", False)]
    for (mode, graph), ms in report.items():
        print(f"config4 {mode:18s} graph={int(graph)}: {ms:8.3f} ms/step  "
              f"{npts / ms / 1e3:9.1f} Mpts/s  x{base / ms:5.2f} vs sequential")
    print(f"config4 persistent+graph vs sequential: max rel L2 {worst:.2e}; mode {ens.get_mode()}")
    ens.close()


def test_autotune_ensemble_and_step(tmp_path):
    from overlappingbls_b200 import tune
    path = str(tmp_path / "tune.json")
    members = _members_small()
    ens = obl.Ensemble(_grids(members), precision="mixed")
    bufs = [Buffers(c, _fields(m)) for c, m in zip(ens.contexts, members)]
    ios = [b.io() for b in bufs]
    shapes = [(m["nxt"], m["nyt"], m["nzt"]) for m in members]
    best, ms = tune.tune_ensemble(ens, ios, shapes, path=path, reps=3)
    assert ms is not None and best in [dict(c) for c in tune.ENSEMBLE_CANDIDATES]
    again, ms2 = tune.tune_ensemble(ens, ios, shapes, path=path)
    assert again == best and ms2 is None            # from the cache
    # the tuned mode gives the single-instance results
    ens.set_mode("sequential")
    for b in bufs:
        b.reset()
    ens.step_dev(ios)
    ens.synchronize()
    ref = [b.outputs() for b in bufs]
    tune.apply_ensemble(ens, best)
    for b in bufs:
        b.reset()
    ens.step_dev(ios)
    ens.synchronize()
    for b, r in zip(bufs, ref):
        _compare(b.outputs(), r, 1e-6)
    # per-instance step variant of one grid
    ctx = ens.contexts[3]
    p, t = tune.tune_step(ctx, bufs[3], path=path, reps=3)
    assert t is not None and p in tune.step_candidates(ctx.nxt, ctx.nyt)
    print("autotune:", best, ms, "step", p, t)
    ens.close()


def test_grid_barrier_wait_gives_up():
    """The persistent kernel's grid barrier, run by one CTA: it releases when it should;
    with no other CTA ever arriving, its bounded wait gives up, the host reads
    OBL_ERR_TIMEOUT, and the context keeps working."""
    import time
    ctx = obl.Context(32, 32, 9, precision="mixed", **fields.DOMAIN)
    ctx.selftest_grid_barrier(False)
    t0 = time.perf_counter()
    with pytest.raises(obl.OblError, match="OBL_ERR_TIMEOUT"):
        ctx.selftest_grid_barrier(True)
    waited = time.perf_counter() - t0
    assert waited < 60.0
    ctx.selftest_grid_barrier(False)
    f = fields.make_fields(32, 32, 9)
    out = ctx.field()
    ctx.ddx(out, f["u"])
    assert np.isfinite(out[:32]).all()
    print(f"grid barrier: the never-released wait gave up after {waited:.1f} s")
    ctx.close()
