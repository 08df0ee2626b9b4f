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

--impl reference times the FP64 CPU restatement of the reference path (the oracle) on
every host core, one full step of the same workload per timed step.

--profile-step runs the warm-up steps and then exactly one step inside the NVTX range
"profiled_step", for profiler captures of every kernel of one step
(ncu --nvtx --nvtx-include "profiled_step/" ...); it prints no bench line.
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (nxt, nyt, nzt)
    "512x512x256": (512, 512, 257),
    "512x512x128": (512, 512, 129),   # one field (136 MB FP32) still exceeds L2: profiler captures
    "512x512x64": (512, 512, 65),
    "256x256x128": (256, 256, 129),
    "128x128x128": (128, 128, 129),
    "64x64x64": (64, 64, 65),
}
METRIC = "Mpts/s per projection step, mixed vs FP64 on 1 B200 at <=1e-5 rel err; %HBM"
BYTES_PER_PT = 28   # reals moved per point by the step (4 in, 24 out), algorithmic
OUT_NAMES = ["dudx", "dudy", "dvdx", "dvdy", "dwdx", "dwdy", "dtdx", "dtdy",
             "u_big", "v_big", "w_big", "t_big", "p", "dpdx", "dpdy", "dpdz", "u", "v", "w"]


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


def workload_config(args, world, slab_mode):
    """The bench line's config: a function of the command line only, so that the GPU arm
    and the reference arm print the same dict for the same workload."""
    nx, ny, nzt = WORKLOADS[args.workload]
    L = nzt - 1
    es = 8 if args.prec == "f64" else 4
    field_mb = (nx + 2) * ny * (nzt + 1) * es / 1e6
    return {"workload": f"{args.workload} ({nx}x{ny}x{L} levels), {args.prec}",
            "nxt": nx, "nyt": ny, "nzt": nzt, "points_per_instance": nx * ny * L, "instances": world,
            "precision": args.prec, "top_bc": "neumann",
            "l2": ("inputs larger than L2 (one field = %.0f MB)" if field_mb > 126 else
                   "inputs smaller than L2 (one field = %.1f MB): not a throughput workload") % field_mb,
            "parallelism": (f"z-slabs x{world}: one {nx}x{ny}x{L * world}-level domain, "
                            "partitioned pressure solve, 2 all-gathers per step") if slab_mode
                           else f"replicas x{world}"}


def cpu_info():
    model = None
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except Exception:
        pass
    try:
        usable = len(os.sched_getaffinity(0))
    except Exception:
        usable = os.cpu_count()
    return {"cpu_model": model, "nproc": os.cpu_count(), "usable_cpus": usable}


# ----------------------------------------------------------------------------- clocks
class Clocks:
    """SM clock, power and clock-event reasons of one GPU, read (never set) every 10 ms
    through NVML while the timed region runs; nvidia-smi at 200 ms if NVML is missing."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))
    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid, index):
        self.rows, self.p, self.nv = [], None, None
        self.done = threading.Event()
        try:
            import pynvml as nv
            nv.nvmlInit()
            try:
                h = nv.nvmlDeviceGetHandleByUUID(uuid)
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(index)
            self.nv, self.h = nv, h
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nv = None
        self.uuid = uuid
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def _poll(self):
        nv, h = self.nv, self.h
        while not self.done.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                self.rows.append((sm, r, pw))
            except Exception:
                pass
            self.done.wait(0.01)

    def stop(self):
        if self.nv is not None:
            self.done.set()
            self.t.join(2)
            if not self.rows:
                return None
            sm = [r[0] for r in self.rows]
            reasons = sorted({n for n, c in self.REASONS for r in self.rows
                              if hasattr(self.nv, c) and r[1] & getattr(self.nv, c)})
            return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(self.rows), "power_w_max": round(max(r[2] for r in self.rows), 1),
                    "source": "NVML, 10 ms"}
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
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows),
                "source": "nvidia-smi, 200 ms"}


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
        "tdma_reg": 5 * lhx * ny * L * c,
        "tdma_staged": 5 * lhx * ny * L * c,
        # levels 1..L of H_x and 0..L+1 of H_z in, the y-transform of G over H_x out (2 launches)
        "press_gform_cols": ((L + (L + 2) + L) * lhx * ny * c) / 2,
        # one launch per field: field in, ddx and the x-padded rows out, and on u, v, w the
        # RHS x-spectrum of levels 1..L out (mean over the 4 launches of a step)
        "rows_fwd3": ((2 * nx + nx2) * ny * nlev * s * 4 + 3 * lhx * ny * L * c) / 4,
        # p_hat (0..L) and the dpdz spectrum in; y-inverses of p, dpdy, dpdz out (dpdx's is
        # i*kx times that of p, formed by the row pass)
        "pinv_cols": (2 * L + 1) * lhx * ny * c + (3 * L + 1) * lhx * ny * c,
        # the three y-inverses and u, v, w in; p, dpdx, dpdy, dpdz and u, v, w out
        "pinv_rows_project": (3 * L + 1) * lhx * ny * c + 3 * nx * ny * L * s + (4 * L + 1) * nx * ny * s
                             + 3 * nx * ny * L * s,
    }
    return table.get(name)


def oracle_step(nx, ny, nzt, f, threads, out=None):
    """One full step of the FP64 oracle (rank-emulating solve, Neumann top) on `threads`
    host threads; returns (seconds, outputs)."""
    from oracle import orc
    from overlappingbls_b200 import fields
    orc.set_threads(threads)
    g = orc.Grid(nx, ny, nzt, **fields.DOMAIN)
    if out is None:
        out = g.step_outputs()
    t0 = time.perf_counter()
    g.step(f["u"], f["v"], f["w"], f["theta"], npz=2, out=out)
    return time.perf_counter() - t0, out


def identical(f64):
    """FP32-representable values: the mixed and FP64 forms and the oracle all get the same
    inputs, so errors measure the computation rather than the rounding to FP32 storage."""
    return {k: np.asfortranarray(v.astype(np.float32).astype(np.float64)) for k, v in f64.items()}


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
        f64 = identical(f64)
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

    # ---- one step for profiler captures ----
    if args.profile_step:
        ctx = make_ctx(args.prec)
        es = ctx.info["elem_bytes"]
        S = dev_set(ctx, torch.float32 if es == 4 else torch.float64)
        for _ in range(args.warmup):
            step(ctx, S)
        torch.cuda.synchronize()
        n0 = ctx.launch_count()
        torch.cuda.nvtx.range_push("profiled_step")
        step(ctx, S)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        print(json.dumps({"profile_step": args.workload, "precision": args.prec,
                          "launches": ctx.launch_count() - n0, "warmup": args.warmup}), flush=True)
        ctx.close()
        return None

    # ---- mixed (headline) ----
    ctx = make_ctx(args.prec)
    es = ctx.info["elem_bytes"]
    dtype = torch.float32 if es == 4 else torch.float64
    S = dev_set(ctx, dtype)
    clk = Clocks(uuid, local) if rank == 0 else None
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

    inf = ctx.info
    ldx = inf["ldx"]

    def outputs(S):
        """(name, device tensor, x-cut, element count) of every step output, in OUT_NAMES order."""
        t, _, d, big, p, dp = S
        nd_valid = ldx * ny * L
        o = [(OUT_NAMES[i], d[i], True, None) for i in range(8)]
        o += [(OUT_NAMES[8 + i], big[i], False, None) for i in range(4)]
        o += [("p", p, True, ldx * ny * (L + 1))]
        o += [(OUT_NAMES[13 + i], dp[i], True, nd_valid) for i in range(3)]
        o += [(k, t[k], False, None) for k in ("u", "v", "w")]
        return o

    def rel(a, b, cut, n):
        """relative L2 error of device tensor a against device tensor b (float64)"""
        if n is not None:
            a, b = a[:n], b[:n]
        a = a.double()
        if cut:
            a = a.view(-1, ldx)[:, :nx]
            b = b.view(-1, ldx)[:, :nx]
        return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))

    # ---- FP64 form and the mixed-vs-FP64 error ----
    fp64 = None
    err = None
    S64 = ctx64 = None
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
        errs = {nm: rel(a, b, cut, n) for (nm, a, cut, n), (_, b, _, _) in zip(outputs(S), outputs(S64))}
        err = {"max": max(errs.values()), "fields": {k: float(f"{v:.3e}") for k, v in errs.items()}}
    else:
        restore(S)
        step(ctx, S)
        torch.cuda.synchronize()

    # ---- CPU baseline and the error against the FP64 oracle (rank 0, N = 1) ----
    cpu = None
    err_orc = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        info = cpu_info()
        threads = info["usable_cpus"]
        sec, ref = oracle_step(nx, ny, nzt, f64, threads)
        # one thread, on a bounded sample: the same grid with 8 levels
        sl = 8
        fs = identical(fields.make_fields(nx, ny, sl + 1, seed=2024))
        sec1, _ = oracle_step(nx, ny, sl + 1, fs, 1)
        del fs
        cpu = {"value": round(pts / sec / 1e6, 3), "unit": "Mpts/s", "cores": threads, "kind": "port",
               "sample": f"one full step of the FP64 oracle on the whole {nx}x{ny}x{L}-level workload "
                         f"({sec:.2f} s, {threads} threads, OpenMP over planes and columns)",
               "single_thread": {"value": round(nx * ny * sl / sec1 / 1e6, 3), "unit": "Mpts/s",
                                 "sample": f"one full step on {nx}x{ny}x{sl} levels ({sec1:.2f} s, 1 thread)"},
               **info}
        refs = [ref["d"][i] for i in range(8)] + [ref["big"][i] for i in range(4)] + \
               [ref["p"], ref["dpdx"], ref["dpdy"], ref["dpdz"], ref["u"], ref["v"], ref["w"]]
        err_orc = {}
        for form, SS in (("mixed", S if args.prec != "f64" else None), ("f64", S64 if args.prec != "f64" else S)):
            if SS is None:
                continue
            e = {}
            for (nm, a, cut, n), r in zip(outputs(SS), refs):
                b = torch.from_numpy(np.ravel(r, order="F")).to(dev)
                e[nm] = rel(a, b, cut, n)
                del b
            err_orc[form] = {"max": max(e.values()), "fields": {k: float(f"{v:.3e}") for k, v in e.items()}}
        err_orc["oracle"] = "FP64 C restatement of the reference (rank-emulating solve, npz = 2), same inputs"
        del ref, refs
    if S64 is not None:
        del S64
        ctx64.close()

    # ---- end to end through the host C ABI (pinned host buffers) ----
    def e2e_run(host_dtype):
        nf, nd, nb = inf["field_elems"], inf["dfield_elems"], inf["big_elems"]
        tdt = torch.float64 if host_dtype == np.float64 else torch.float32
        hb = 8 if host_dtype == np.float64 else 4
        keep = []

        def pin(n, src=None):
            t = torch.empty(n, dtype=tdt, pin_memory=True)
            keep.append(t)
            if src is not None:
                t.copy_(torch.from_numpy(src.ravel(order="F").astype(host_dtype)))
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
        h2d = 4 * nf * hb
        d2h = (8 * nx * ny * (inf["nz"] + 1) + 4 * nb + nx * ny * (L1 + 1) + 3 * nx * ny * L1 + 3 * nf) * hb
        del keep, H
        return {"value": round(pts * world / sec / 1e6, 2), "unit": "Mpts/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": ke,
                "host_arrays": "float64" if hb == 8 else "float32",
                "timing": "wall clock around the synchronous C-ABI call"}

    e2e = e2e32 = None
    if not args.skip_e2e:
        if slab_mode:
            e2e = e2e_run(np.float32 if es == 4 else np.float64)
        else:
            # the drop-in caller's arrays are real(8) (rprec = kind(1.d0)): obl_step
            e2e = e2e_run(np.float64)
            e2e["call"] = "obl_step (float64 host arrays, the reference's real(8) fields)"
            if es == 4:
                e2e32 = e2e_run(np.float32)
                e2e32["call"] = "obl_step_f32 (float32 host arrays)"

    res = {
        "metric": METRIC, "value": round(value, 1), "unit": "Mpts/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if args.prec == "mixed" else args.prec, "data": "synthetic",
        "config": workload_config(args, world, slab_mode),
        "fp64_columns": ctx.info["n_fp64_columns"],
        "step_roofline": {"bound": "hbm", "bytes_per_step": step_bytes, "achieved": round(step_gbs, 1),
                          "peak": hbm, "unit": "GB/s", "frac": round(step_gbs / hbm, 4),
                          "peak_kind": peak_kind},
        "roofline": roof, "kernel_ms": {k: [v[0], round(v[1], 4)] for k, v in kt.items()},
        "fp64_form": fp64, "rel_err_vs_fp64": err, "rel_err_vs_oracle": err_orc,
        "e2e": e2e, "e2e_f32": e2e32, "cpu_baseline": cpu,
        "clocks": clocks, "gpu_launches": int(launches),
    }
    ctx.close()
    return res


def run_reference(args, rank, world):
    """The reference arm: the FP64 oracle (the CPU restatement of the reference path; the
    Fortran/MPI/FFTW reference cannot be built in this image) on every usable host core,
    one full step of the whole workload per timed step."""
    if rank != 0:
        return None
    from overlappingbls_b200 import fields
    from oracle import orc
    nx, ny, nzt = WORKLOADS[args.workload]
    L = nzt - 1
    info = cpu_info()
    threads = info["usable_cpus"]
    f = fields.make_fields(nx, ny, nzt, seed=2024)
    if args.prec != "f64":
        f = identical(f)
    g = orc.Grid(nx, ny, nzt, **fields.DOMAIN)
    out = g.step_outputs()
    orc.set_threads(threads)
    # every step is the whole workload (seconds of CPU work): at most 5 timed steps and 2
    # warm-up steps, so that the run ends within minutes; the line reports the counts used
    nsteps, nwarm = max(1, min(args.steps, 5)), min(args.warmup, 2)
    for _ in range(nwarm):
        g.step(f["u"], f["v"], f["w"], f["theta"], npz=2, out=out)
    t0 = time.perf_counter()
    for _ in range(nsteps):
        g.step(f["u"], f["v"], f["w"], f["theta"], npz=2, out=out)
    sec = (time.perf_counter() - t0) / nsteps
    v = nx * ny * L / sec / 1e6
    sample = (f"one full step of the whole {nx}x{ny}x{L}-level workload per timed step ({nsteps} timed after "
              f"{nwarm} warm-up; the run's --steps/--warmup capped at 5/2), FP64 C restatement "
              "of the reference path (the Fortran/MPI/FFTW reference cannot be built here), "
              f"{threads} threads")
    return {"metric": METRIC, "value": round(v, 3), "unit": "Mpts/s", "n_gpus": world, "steps": nsteps,
            "warmup": nwarm, "ms_per_step": round(sec * 1e3, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            # the same workload as the GPU arm at N = 1 (one domain; rank 0 alone runs)
            "config": workload_config(args, 1, False),
            "cpu_baseline": {"value": round(v, 3), "unit": "Mpts/s", "cores": threads, "kind": "port",
                             "sample": sample, **info},
            "e2e": {"value": round(v, 3), "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)   # about 1 s of timed device work at 512^3/2
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOADS), default="512x512x256")
    ap.add_argument("--prec", choices=["mixed", "f64", "f32"], default="mixed")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--profile-step", action="store_true",
                    help="warm-up steps, then one step in the NVTX range 'profiled_step'; no bench line")
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
