#!/usr/bin/env python
"""Benchmark: Mpts/s of the projection-plus-derivative step (mixed vs FP64) on B200.

One "step" is one pass of the hot path over one instance: ddx/ddy and 3/2-rule
zero_padding of u, v, w, theta on every level, press_stag_array (forward 2D FFT of
the divergence RHS per level, batched tridiagonal solve per (kx,ky), inverse FFTs),
dpdz and project -- obl_step_dev through the C ABI.  Mpts/s = nx*ny*(nzt-1)/t/1e6.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Default workload: 512 x 512 x 256 levels, FP32-mixed (the headline configuration).
Multi-GPU (torchrun), --mode slab (default): one domain of 512 x 512 x (256 N) levels split
in z, each rank holding a 512 x 512 x 256-level slab (weak scaling); the step is the
z-slab step of overlappingbls_b200.slab (partitioned pressure solve, two all-gathers over
NCCL per step).  --mode replicas: every rank advances its own independent instance.  The
time is the max over ranks.
--impl reference times the FP64 CPU restatement of the reference path (the oracle)
on the host cores, on a bounded sample of the same workload.
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (nxt, nyt, nzt)
    "512x512x256": (512, 512, 257),
    "512x512x64": (512, 512, 65),     # small case of the headline planes, for ncu captures
    "256x256x128": (256, 256, 129),
    "128x128x128": (128, 128, 129),
    "64x64x64": (64, 64, 65),
}
METRIC = "Mpts/s per projection step, mixed vs FP64 on 1 B200 at <=1e-5 rel err; %HBM"
BYTES_PER_PT = 28   # reals moved per point by the step (4 in, 24 out), algorithmic


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ----------------------------------------------------------------------------- clocks
class Clocks:
    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                c = [x.strip() for x in line.split(",")]
                if len(c) < 9 or (self.uuid and c[0] != self.uuid):
                    continue
                rows.append(c)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- helpers
def algorithmic_bytes(name, info, s):
    """Compulsory bytes of one launch of a library kernel (its own inputs read once,
    outputs written once); intermediates of other kernels are not counted."""
    nx, ny, nz = info["nxt"], info["nyt"], info["nz"]
    nx2, ny2, lhx = info["nxt2"], info["nyt2"], info["lhx"]
    L, nlev = nz - 1, nz + 1
    c = 2 * s
    table = {
        "ddx_rows": 2 * nx * ny * nlev * s,
        "ddy_cols": 2 * nx * ny * nlev * s,
        "pad_rows": (nx + nx2) * ny * nlev * s,
        "pad_cols": (nx2 * ny + nx2 * ny2) * nlev * s,
        "press_fwd_rows": nx * ny * L * s + lhx * ny * L * c,
        "press_fwd_cols": 2 * lhx * ny * L * c,
        "tdma": 5 * lhx * ny * L * c,
        "tdma_mixed": 5 * lhx * ny * L * c,
        # one launch per field: field in, ddx and the x-padded rows out, and on u, v, w the
        # RHS x-spectrum of levels 1..L out (mean over the 4 launches of a step)
        "rows_fwd3": ((2 * nx + nx2) * ny * nlev * s * 4 + 3 * lhx * ny * L * c) / 4,
        # p_hat (0..L) and the dpdz spectrum in; y-inverses of p, dpdx, dpdy, dpdz out
        "pinv_cols": (2 * L + 1) * lhx * ny * c + (4 * L + 1) * lhx * ny * c,
        # the four y-inverses and u, v, w in; p, dpdx, dpdy, dpdz and u, v, w out
        "pinv_rows_project": (4 * L + 1) * lhx * ny * c + 3 * nx * ny * L * s + (4 * L + 1) * nx * ny * s
                             + 3 * nx * ny * L * s,
    }
    return table.get(name)


def run_ours(args, rank, local, world):
    import torch
    import overlappingbls_b200 as obl
    from overlappingbls_b200 import fields, slab

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    nx, ny, nzt = WORKLOADS[args.workload]
    L = nzt - 1
    pts = nx * ny * L
    hbm, peak_kind = peaks()
    f64 = fields.make_fields(nx, ny, nzt, seed=2024 + rank)
    if args.prec != "f64":
        # identical inputs for the mixed and FP64 forms: FP32-representable values, so the
        # mixed-vs-FP64 error measures the computation rather than the input rounding
        f64 = {k: v.astype(np.float32).astype(np.float64) for k, v in f64.items()}
    stream = torch.cuda.current_stream(dev)
    slab_mode = world > 1 and args.mode == "slab"
    comm = slab.TorchComm() if slab_mode else None
    slabs = {}

    def make_ctx(prec):
        c = obl.Context(nx, ny, nzt, precision=prec, top_bc="neumann", device=local,
                        fp64_k2_max=args.fp64_k2_max, **fields.DOMAIN)
        c.set_stream(stream.cuda_stream)
        for kv in args.param:
            k, v = kv.split("=")
            c.set_param(k, int(v))
        if slab_mode:
            slabs[id(c)] = slab.SlabStep(slab.LibBackend(c), rank, world, comm)
        return c

    def dev_set(ctx, dtype):
        inf = ctx.info
        nf, nd, nb = inf["field_elems"], inf["dfield_elems"], inf["big_elems"]
        t = {k: torch.from_numpy(f64[k].ravel(order="F")).to(dev, dtype) for k in ("u", "v", "w", "theta")}
        t0 = {k: v.clone() for k, v in t.items()}
        d = [torch.zeros(nf, dtype=dtype, device=dev) for _ in range(8)]
        big = [torch.zeros(nb, dtype=dtype, device=dev) for _ in range(4)]
        p = torch.zeros(nf, dtype=dtype, device=dev)
        dp = [torch.zeros(nd, dtype=dtype, device=dev) for _ in range(3)]
        return t, t0, d, big, p, dp

    def step(ctx, S):
        t, _, d, big, p, dp = S
        if slab_mode:
            io = obl.stepio_dev(t["u"].data_ptr(), t["v"].data_ptr(), t["w"].data_ptr(), t["theta"].data_ptr(),
                                [x.data_ptr() for x in d], [x.data_ptr() for x in big], p.data_ptr(),
                                [x.data_ptr() for x in dp])
            slabs[id(ctx)].step(io)
            return
        ctx.step_dev(t["u"].data_ptr(), t["v"].data_ptr(), t["w"].data_ptr(), t["theta"].data_ptr(),
                     [x.data_ptr() for x in d], [x.data_ptr() for x in big], p.data_ptr(),
                     [x.data_ptr() for x in dp])

    def restore(S):
        for k in ("u", "v", "w"):
            S[0][k].copy_(S[1][k])

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def timed(ctx, S, K, W):
        for _ in range(W):
            step(ctx, S)
        torch.cuda.synchronize()
        n0 = ctx.launch_count()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            step(ctx, S)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms = e0.elapsed_time(e1)
        if world > 1:
            x = torch.tensor([ms], device=dev)
            torch.distributed.all_reduce(x, op=torch.distributed.ReduceOp.MAX)
            ms = float(x.item())
        return ms / K, ctx.launch_count() - n0

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass

    # ---- mixed (headline) ----
    ctx = make_ctx(args.prec)
    es = ctx.info["elem_bytes"]
    dtype = torch.float32 if es == 4 else torch.float64
    S = dev_set(ctx, dtype)
    clk = Clocks(uuid) if rank == 0 else None
    ms, launches = timed(ctx, S, args.steps, args.warmup)
    clocks = clk.stop() if clk else None
    value = pts * world / (ms * 1e-3) / 1e6

    # per-kernel device time (separate, untimed pass)
    restore(S)
    ctx.timing(True)
    step(ctx, S)
    kt = ctx.timing_report()
    ctx.timing(False)
    dom = max(kt.items(), key=lambda kv: kv[1][1])
    dom_name, (dom_n, dom_ms) = dom[0], dom[1]
    ab = algorithmic_bytes(dom_name, ctx.info, es)
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            traffic = json.load(fh).get(args.workload, {}).get(args.prec, {}).get(dom_name)
    except Exception:
        pass
    roof = None
    if ab:
        ach = ab / (dom_ms / dom_n * 1e-3) / 1e9
        roof = {"bound": "hbm", "kernel": dom_name, "achieved": round(ach, 1), "peak": hbm,
                "unit": "GB/s", "frac": round(ach / hbm, 4), "peak_kind": peak_kind,
                "traffic": traffic, "launches_per_step": dom_n}
    step_bytes = BYTES_PER_PT * pts * es
    step_gbs = step_bytes / (ms * 1e-3) / 1e9

    # ---- FP64 form and the mixed-vs-FP64 error ----
    fp64 = None
    err = None
    if args.prec != "f64" and not args.skip_fp64:
        restore(S)
        step(ctx, S)   # one fresh mixed step from the pristine inputs
        ctx64 = make_ctx("f64")
        S64 = dev_set(ctx64, torch.float64)
        ms64, _ = timed(ctx64, S64, max(3, args.steps // 2), args.warmup)
        restore(S64)
        step(ctx64, S64)
        torch.cuda.synchronize()
        v64 = pts * world / (ms64 * 1e-3) / 1e6
        fp64 = {"value": round(v64, 1), "ms_per_step": round(ms64, 4),
                "hbm_frac_step": round(BYTES_PER_PT * pts * 8 / (ms64 * 1e-3) / 1e9 / hbm, 4),
                "mixed_over_fp64": round(value / v64, 3)}
        # relative L2 error of every output of the mixed step against the FP64 GPU form
        inf = ctx.info
        nxw, ldx = inf["nxt"], inf["ldx"]

        def rl(a, b, cut=True):
            a, b = a.double(), b
            if cut:
                a = a.view(-1, ldx)[:, :nxw]
                b = b.view(-1, ldx)[:, :nxw]
            return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))
        errs = {}
        for i, nm in enumerate(["dudx", "dudy", "dvdx", "dvdy", "dwdx", "dwdy", "dtdx", "dtdy"]):
            errs[nm] = rl(S[2][i], S64[2][i])
        for i, nm in enumerate(["u_big", "v_big", "w_big", "t_big"]):
            errs[nm] = rl(S[3][i], S64[3][i], cut=False)
        nd_valid = inf["ldx"] * inf["nyt"] * L
        errs["p"] = rl(S[4][: inf["ldx"] * inf["nyt"] * (L + 1)], S64[4][: inf["ldx"] * inf["nyt"] * (L + 1)])
        for i, nm in enumerate(["dpdx", "dpdy", "dpdz"]):
            errs[nm] = rl(S[5][i][:nd_valid], S64[5][i][:nd_valid])
        for nm in ("u", "v", "w"):
            errs[nm] = rl(S[0][nm], S64[0][nm], cut=False)
        err = {"max": max(errs.values()), "fields": {k: float(f"{v:.3e}") for k, v in errs.items()}}
        del S64
        ctx64.close()

    # ---- end to end through the host C ABI (pinned host buffers) ----
    e2e = None
    if not args.skip_e2e:
        inf = ctx.info
        nf, nd, nb = inf["field_elems"], inf["dfield_elems"], inf["big_elems"]
        hd = np.float32 if es == 4 else np.float64
        tdt = torch.float32 if es == 4 else torch.float64

        def pin(n, src=None):
            t = torch.empty(n, dtype=tdt, pin_memory=True)
            if src is not None:
                t.copy_(torch.from_numpy(src.ravel(order="F").astype(hd)))
            return t.numpy()
        u, v, w, th = (pin(nf, f64[k]) for k in ("u", "v", "w", "theta"))
        shp = lambda a, s: a.reshape(s, order="F")
        fs = (inf["ldx"], inf["nyt"], inf["nz"] + 1)
        bs = (inf["nxt2"], inf["nyt2"], inf["nz"] + 1)
        ds = (inf["ldx"], inf["nyt"], inf["nz"])
        H = dict(u=shp(u, fs), v=shp(v, fs), w=shp(w, fs), th=shp(th, fs),
                 d=[shp(pin(nf), fs) for _ in range(8)], big=[shp(pin(nb), bs) for _ in range(4)],
                 p=shp(pin(nf), fs), dp=[shp(pin(nd), ds) for _ in range(3)])
        ke = max(2, min(5, args.steps))

        def host_step():
            if not slab_mode:
                ctx.step(H["u"], H["v"], H["w"], H["th"], H["d"], H["big"], H["p"], H["dp"])
                return
            # the slab step has no host variant: pinned host -> device, step, device -> host
            t = S[0]
            for k, hk in (("u", u), ("v", v), ("w", w), ("theta", th)):
                t[k].copy_(torch.from_numpy(hk), non_blocking=True)
            step(ctx, S)
            outs = [(S[2][i], H["d"][i]) for i in range(8)] + [(S[3][i], H["big"][i]) for i in range(4)]
            outs += [(S[4], H["p"])] + [(S[5][i], H["dp"][i]) for i in range(3)]
            outs += [(t["u"], H["u"]), (t["v"], H["v"]), (t["w"], H["w"])]
            for dsrc, hdst in outs:
                torch.from_numpy(hdst.reshape(-1, order="F")).copy_(dsrc, non_blocking=True)
            torch.cuda.synchronize()
        host_step()   # warm-up
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ke):
            host_step()
        torch.cuda.synchronize()
        sec = (time.perf_counter() - t0) / ke
        if world > 1:
            x = torch.tensor([sec], device=dev)
            torch.distributed.all_reduce(x, op=torch.distributed.ReduceOp.MAX)
            sec = float(x.item())
        L1 = inf["nz"] - 1
        h2d = 4 * nf * es
        d2h = (8 * nx * ny * (inf["nz"] + 1) + 4 * nb + nx * ny * (L1 + 1) + 3 * nx * ny * L1 + 3 * nf) * es
        e2e = {"value": round(pts * world / sec / 1e6, 2), "unit": "Mpts/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": ke, "timing": "wall clock around the synchronous C-ABI call"}

    # ---- CPU baseline: the FP64 oracle on a bounded sample (rank 0, N = 1) ----
    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        cpu = cpu_baseline(nx, ny, sample_levels=8)

    res = {
        "metric": METRIC, "value": round(value, 1), "unit": "Mpts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if args.prec == "mixed" else args.prec, "data": "synthetic",
        "config": {"workload": f"{args.workload} ({nx}x{ny}x{L} levels), {args.prec}",
                   "nxt": nx, "nyt": ny, "nzt": nzt, "points_per_instance": pts, "instances": world,
                   "precision": args.prec, "top_bc": "neumann",
                   "fp64_columns": ctx.info["n_fp64_columns"],
                   "l2": "inputs larger than L2 (one field = %.0f MB)" % (ctx.info["field_elems"] * es / 1e6),
                   "parallelism": (f"z-slabs x{world}: one {nx}x{ny}x{L * world}-level domain, "
                                   "partitioned pressure solve, 2 all-gathers per step") if slab_mode
                                  else f"replicas x{world}"},
        "step_roofline": {"bound": "hbm", "bytes_per_step": step_bytes, "achieved": round(step_gbs, 1),
                          "peak": hbm, "unit": "GB/s", "frac": round(step_gbs / hbm, 4),
                          "peak_kind": peak_kind},
        "roofline": roof, "kernel_ms": {k: [v[0], round(v[1], 4)] for k, v in kt.items()},
        "fp64_form": fp64, "rel_err_vs_fp64": err, "e2e": e2e, "cpu_baseline": cpu,
        "clocks": clocks, "gpu_launches": int(launches),
    }
    ctx.close()
    return res


def cpu_baseline(nx, ny, sample_levels=8, threads=None):
    """The oracle's full step on a bounded sample (nx x ny x sample_levels)."""
    from oracle import orc
    from overlappingbls_b200 import fields
    threads = threads or os.cpu_count()
    orc.set_threads(threads)
    nzt = sample_levels + 1
    f = fields.make_fields(nx, ny, nzt)
    g = orc.Grid(nx, ny, nzt, **fields.DOMAIN)
    t0 = time.perf_counter()
    g.step(f["u"], f["v"], f["w"], f["theta"], npz=2)
    sec = time.perf_counter() - t0
    return {"value": round(nx * ny * sample_levels / sec / 1e6, 3), "unit": "Mpts/s", "cores": threads,
            "kind": "port", "sample": f"one full step of the FP64 oracle on {nx}x{ny}x{sample_levels} levels "
            f"({sec:.2f} s, {threads} threads)"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    nx, ny, nzt = WORKLOADS[args.workload]
    from oracle import orc
    from overlappingbls_b200 import fields
    threads = os.cpu_count()
    orc.set_threads(threads)
    lev = 8
    f = fields.make_fields(nx, ny, lev + 1)
    g = orc.Grid(nx, ny, lev + 1, **fields.DOMAIN)
    for _ in range(min(args.warmup, 1)):
        g.step(f["u"], f["v"], f["w"], f["theta"], npz=2)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        g.step(f["u"], f["v"], f["w"], f["theta"], npz=2)
    sec = (time.perf_counter() - t0) / args.steps
    v = nx * ny * lev / sec / 1e6
    return {"metric": METRIC, "value": round(v, 3), "unit": "Mpts/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(sec * 1e3 * (nzt - 1) / lev, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": f"{args.workload} ({nx}x{ny}x{nzt - 1} levels)", "nxt": nx, "nyt": ny,
                       "nzt": nzt, "sample_levels": lev},
            "cpu_baseline": {"value": round(v, 3), "unit": "Mpts/s", "cores": threads, "kind": "port",
                             "sample": f"full step on {nx}x{ny}x{lev} levels per timed step (FP64 C restatement "
                                       "of the reference; the Fortran/MPI/FFTW reference is not buildable here)"},
            "e2e": {"value": round(v, 3), "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOADS), default="512x512x256")
    ap.add_argument("--prec", choices=["mixed", "f64", "f32"], default="mixed")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--fp64-k2-max", type=float, default=-1.0,
                    help="mixed mode: k^2 bound of the FP64 TDMA columns (-1 = library default)")
    ap.add_argument("--mode", choices=["slab", "replicas"], default="slab",
                    help="N > 1: one z-split domain (slab) or independent instances (replicas)")
    ap.add_argument("--param", action="append", default=[],
                    help="execution tuning name=value passed to obl_set_param (e.g. fused=0)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, local, world = env_rank()
    if world > 1:
        import torch
        if args.impl == "ours":
            torch.cuda.set_device(local)
            torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                                 device_id=torch.device("cuda", local))
        else:
            torch.distributed.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            res = run_reference(args, rank, world)
        else:
            res = run_ours(args, rank, local, world)
        if rank == 0 and res is not None:
            print(json.dumps(res), flush=True)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
