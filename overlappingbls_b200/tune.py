"""Autotuner of the step's execution choices, cached per device in a JSON file.

Three kinds of entries:

* ``step``: per (nxt, nyt, nzt, precision) the single-instance step variant: ``fused``
  0 (multi-output line kernels), 1 (cluster-fused forward plane kernel, square grids; with
  its cluster size and cluster count) or 2 (one kernel per reference routine).
* ``ensemble``: per ensemble signature (the multiset of instance shapes and the
  precision) the ensemble mode (sequential, concurrent streams, one persistent launch,
  the register-class split of it, the dataflow form), whether to replay a CUDA graph, and
  the persistent kernel's CTAs per SM.  ``python -m overlappingbls_b200.tune ensemble
  --mode MODE`` times the 48-instance ensemble in one mode.
* ``build``: per bench workload the compile-time schedule of the kernels: CTA shapes of
  the column FFT kernels (warps and lines per CTA, resident warps per SM), the persistent
  prefetching column form, the y-pad's L2 look-ahead, the scratch padding of the row FFT
  kernels.
  Each candidate is a set of -D definitions; ``build_variants`` compiles one library per
  candidate, ``tune_build`` times each through ``bench.py`` (a subprocess with $OBL_LIB),
  and ``python -m overlappingbls_b200.build --tuned`` compiles the chosen schedule.

The step entries also search the pressure solve's schedule (register-segmented or one
sweep per column; column segments) next to the forward-pass variant.

Each candidate is timed with CUDA events over ``reps`` steps after ``warmup`` steps; the
fastest wins.  Results do not depend on any of these choices (the tests check every
variant against the oracle), so a cached choice is only a speed decision.

The cache path is ``path``, else $OBL_TUNE_CACHE, else
~/.cache/overlappingbls_b200/tune.json.
"""
import json
import os

import numpy as np

CACHE_VERSION = 1


def cache_path(path=None):
    if path:
        return path
    env = os.environ.get("OBL_TUNE_CACHE")
    if env:
        return env
    return os.path.join(os.path.expanduser("~"), ".cache", "overlappingbls_b200", "tune.json")


def load_cache(path=None):
    p = cache_path(path)
    try:
        with open(p) as f:
            c = json.load(f)
        if c.get("version") != CACHE_VERSION:
            return {"version": CACHE_VERSION, "devices": {}}
        return c
    except (OSError, ValueError):
        return {"version": CACHE_VERSION, "devices": {}}


def save_cache(cache, path=None):
    p = cache_path(path)
    d = os.path.dirname(p)
    if d:
        os.makedirs(d, exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def step_key(nxt, nyt, nzt, precision):
    return f"{nxt}x{nyt}x{nzt}:{precision}"


def ensemble_key(shapes, precision):
    """shapes: iterable of (nxt, nyt, nzt)."""
    counts = {}
    for s in shapes:
        k = "x".join(str(int(v)) for v in s)
        counts[k] = counts.get(k, 0) + 1
    return ";".join(f"{k}*{counts[k]}" for k in sorted(counts)) + ":" + precision


def step_candidates(nxt, nyt):
    """The variants of the single-instance step worth timing for this grid: the forward
    pass (multi-output line kernels, one kernel per routine, cluster-fused planes) and,
    with the line kernels, the pressure solve's schedule."""
    cands = [{"fused": 0, "tdma_reg": 1, "tdma_segments": 0}, {"fused": 0, "tdma_reg": 0, "tdma_segments": 0},
             {"fused": 0, "tdma_reg": 1, "tdma_segments": 4}, {"fused": 0, "tdma_reg": 1, "tdma_segments": 16},
             {"fused": 2}]
    if nxt == nyt:
        for csize in (4, 8):
            for ncl in (0, 16):
                cands.append({"fused": 1, "fwd_cluster_size": csize, "fwd_clusters": ncl})
    return cands


# Compile-time schedules searched by tune_build (name -> -D definitions).  "default" is the
# library as built without definitions.
BUILD_CANDIDATES = {
    "default": [],
    "cols_4w4l": ["OBL_PAD_NW=4", "OBL_PAD_WB=4", "OBL_COLS_NW=4", "OBL_COLS_WB=4"],
    "cols_16w_32sm": ["OBL_PAD_NW=16", "OBL_COLS_NW=16"],
    "cols_16w_48sm": ["OBL_PAD_NW=16", "OBL_COLS_NW=16", "OBL_COL_WARPS_SM=48"],
    "cols_pipelined": ["OBL_COL_PIPE=1"],
    "rows_pad16": ["OBL_SIDX_SHIFT=4"],
    "pad_prefetch_off": ["OBL_COL_PF=0"],
}


def variant_path(out_dir, name):
    return os.path.join(out_dir, f"libobl_{name}.so")


def build_variants(out_dir, names=None, jobs=None):
    """Compile one library per build candidate into out_dir (skips existing ones)."""
    from . import build as b
    os.makedirs(out_dir, exist_ok=True)
    done = {}
    for name in names or BUILD_CANDIDATES:
        if name == "default":   # timed with the library as built
            continue
        lib = variant_path(out_dir, name)
        if not os.path.exists(lib):
            b.build(jobs=jobs, defines=BUILD_CANDIDATES[name], out=lib)
        done[name] = lib
    return done


def bench_ms(lib, workload, steps, warmup, timeout=900):
    """ms per step of bench.py's step on workload with library lib (None: the default)."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    env = dict(os.environ)
    if lib:
        env["OBL_LIB"] = os.path.abspath(lib)
    cmd = [sys.executable, os.path.join(root, "bench.py"), "--workload", workload, "--steps", str(steps),
           "--warmup", str(warmup), "--skip-fp64", "--skip-e2e", "--skip-cpu"]
    r = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=timeout)
    if r.returncode != 0:
        return None
    for line in r.stdout.splitlines():
        if line.startswith("{"):
            return float(json.loads(line)["ms_per_step"])
    return None


def tune_build(workload, out_dir, names=None, steps=20, warmup=5, path=None, device=None):
    """Time every built variant on workload, cache all timings and the fastest schedule
    under ``build``/workload.  Returns (name, defines, ms)."""
    device = device or _device_name()
    timings = []
    for name in names or BUILD_CANDIDATES:
        lib = variant_path(out_dir, name) if name != "default" else None
        if lib and not os.path.exists(lib):
            timings.append(({"name": name, "defines": BUILD_CANDIDATES[name]}, None))
            continue
        timings.append(({"name": name, "defines": BUILD_CANDIDATES[name]}, bench_ms(lib, workload, steps, warmup)))
    cache = load_cache(path)
    ent = _entry(cache, device, "build")
    # sweeps may run in parts: timings of candidates not timed now are kept
    now = {p["name"] for p, _ in timings}
    old = [(p, t) for p, t in ent.get(workload, {}).get("timings", []) if p["name"] not in now]
    timings = old + timings
    best, ms = pick(timings)
    ent[workload] = {"params": best, "ms": ms, "timings": [[p, t] for p, t in timings]}
    save_cache(cache, path)
    return best["name"], best["defines"], ms


# The schedule sweep's record on this project's B200s, shipped with the package: what
# ``build --tuned`` uses when the user's cache has no entry for the workload.
PACKAGED_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_b200.json")


def tuned_defines(workload="512x512x256", path=None, device=None):
    """The -D definitions of the cached fastest schedule for workload ([] if none); the
    user's cache first, then the packaged record."""
    if path is None and not any(workload in d.get("build", {}) for d in load_cache().get("devices", {}).values()):
        path = PACKAGED_CACHE
    cache = load_cache(path)
    devs = cache.get("devices", {})
    if device is None:
        device = next((d for d in devs if workload in devs[d].get("build", {})), None)
    ent = devs.get(device, {}).get("build", {}).get(workload)
    return list(ent["params"]["defines"]) if ent else []


ENSEMBLE_CANDIDATES = (
    {"mode": "sequential", "graph": False, "bps": 0},
    {"mode": "sequential", "graph": True, "bps": 0},
    {"mode": "concurrent", "graph": False, "bps": 0},
    {"mode": "concurrent", "graph": True, "bps": 0},
    {"mode": "persistent", "graph": True, "bps": 0},
    {"mode": "persistent", "graph": True, "bps": 1},
    {"mode": "persistent_split", "graph": True, "bps": 0},
    {"mode": "persistent_flow", "graph": True, "bps": 0},
)


def pick(timings):
    """The candidate with the smallest time; timings: list of (params, ms or None)."""
    ok = [(p, t) for p, t in timings if t is not None and np.isfinite(t)]
    if not ok:
        raise RuntimeError("no candidate ran")
    return min(ok, key=lambda pt: pt[1])


def _device_name():
    import torch
    return torch.cuda.get_device_name(0) if torch.cuda.is_available() else "cpu"


def _entry(cache, device, kind):
    return cache.setdefault("devices", {}).setdefault(device, {}).setdefault(kind, {})


def apply_step(ctx, params):
    for k, v in params.items():
        ctx.set_param(k, int(v))


def _time_step(ctx, bufs, warmup, reps):
    """CUDA-event time of obl_step_dev on the context's (legacy default) stream."""
    import torch
    io = bufs.io()
    # the events are recorded on torch's current stream: run the context there
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    run = lambda: ctx.step_dev(io.u, io.v, io.w, io.theta, list(io.d), list(io.big), io.p, list(io.dp))
    for _ in range(warmup):
        run()
    ctx.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        run()
    b.record()
    b.synchronize()
    return a.elapsed_time(b) / reps


def tune_step(ctx, bufs, path=None, warmup=3, reps=10, retune=False):
    """Choose the fastest step variant for ctx's grid (bufs: device buffers with .io()),
    apply it to ctx and cache it.  Returns (params, ms or None when taken from the cache)."""
    cache = load_cache(path)
    ent = _entry(cache, _device_name(), "step")
    key = step_key(ctx.nxt, ctx.nyt, ctx.nzt, ctx.precision)
    if key in ent and not retune:
        apply_step(ctx, ent[key]["params"])
        return ent[key]["params"], None
    timings = []
    for p in step_candidates(ctx.nxt, ctx.nyt):
        try:
            apply_step(ctx, p)
            timings.append((p, _time_step(ctx, bufs, warmup, reps)))
        except Exception:
            timings.append((p, None))
    best, ms = pick(timings)
    apply_step(ctx, best)
    ent[key] = {"params": best, "ms": ms, "timings": [[p, t] for p, t in timings]}
    save_cache(cache, path)
    return best, ms


def apply_ensemble(ens, params):
    ens.set_mode(params["mode"], params.get("bps", 0))


def tune_ensemble(ens, ios, shapes, path=None, warmup=3, reps=10, retune=False):
    """Choose the fastest ensemble mode for these buffers, apply it and cache it.
    Returns (params, ms or None when taken from the cache)."""
    cache = load_cache(path)
    ent = _entry(cache, _device_name(), "ensemble")
    key = ensemble_key(shapes, ens.precision)
    if key in ent and not retune:
        apply_ensemble(ens, ent[key]["params"])
        return ent[key]["params"], None
    timings = []
    for p in ENSEMBLE_CANDIDATES:
        try:
            apply_ensemble(ens, p)
            timings.append((dict(p), ens.time_dev(ios, use_graph=p["graph"], warmup=warmup, reps=reps)))
        except Exception:
            timings.append((dict(p), None))
    best, ms = pick(timings)
    apply_ensemble(ens, best)
    ent[key] = {"params": best, "ms": ms, "timings": [[p, t] for p, t in timings]}
    save_cache(cache, path)
    return best, ms


def ensemble48(mode, steps=10, warmup=3, graph=False, blocks_per_sm=0):
    """Device time per step of the 48-instance ensemble (16 each at 96x96x64, 128x128x96,
    192x192x128 levels, FP32-mixed) in one mode: (ms, Mpts/s).  Inputs and outputs are
    device buffers (torch tensors in the storage type)."""
    import torch
    import overlappingbls_b200 as obl
    from overlappingbls_b200 import fields
    members = fields.ensemble_members()
    ens = obl.Ensemble([dict(nxt=m["nxt"], nyt=m["nyt"], nzt=m["nzt"], **fields.DOMAIN) for m in members],
                       precision="mixed")
    keep, ios, npts = [], [], 0
    for c, m in zip(ens.contexts, members):
        f = fields.make_fields(m["nxt"], m["nyt"], m["nzt"], z0=m["z0"], theta_grad=m["theta_grad"], seed=m["seed"])
        nf = c.ldx * c.nyt * (c.nz + 1)
        nd = c.ldx * c.nyt * c.nz
        nb = c.nxt2 * c.nyt2 * (c.nz + 1)
        dev = lambda n: torch.empty(n, dtype=torch.float32, device="cuda")
        inp = [torch.from_numpy(np.asarray(f[k], np.float32).ravel(order="F")).cuda() for k in ("u", "v", "w", "theta")]
        d, big, p, dp = [dev(nf) for _ in range(8)], [dev(nb) for _ in range(4)], dev(nf), [dev(nd) for _ in range(3)]
        keep += inp + d + big + [p] + dp
        P = lambda t: t.data_ptr()
        ios.append(obl.stepio_dev(*(P(t) for t in inp), [P(t) for t in d], [P(t) for t in big], P(p),
                                  [P(t) for t in dp]))
        npts += c.nxt * c.nyt * (c.nzt - 1)
    torch.cuda.synchronize()
    ens.set_mode(mode, blocks_per_sm)
    ms = ens.time_dev(ios, use_graph=graph, warmup=warmup, reps=steps)
    ens.close()
    return ms, npts / ms / 1e3


def main():
    import argparse
    import overlappingbls_b200 as obl
    ap = argparse.ArgumentParser(description="compile-time schedule sweep of the step's kernels; "
                                             "ensemble mode timing")
    sub = ap.add_subparsers(dest="cmd", required=True)
    e = sub.add_parser("ensemble", help="time the 48-instance ensemble in one mode")
    e.add_argument("--mode", default="persistent", choices=sorted(obl.ENS_MODES))
    e.add_argument("--steps", type=int, default=10)
    e.add_argument("--warmup", type=int, default=3)
    e.add_argument("--graph", action="store_true")
    e.add_argument("--bps", type=int, default=0)
    b = sub.add_parser("build-variants", help="compile one library per schedule candidate")
    b.add_argument("--out", required=True)
    b.add_argument("--only", nargs="*")
    t = sub.add_parser("sweep", help="time the built variants on a workload and cache the choice")
    t.add_argument("--out", required=True)
    t.add_argument("--only", nargs="*")
    t.add_argument("--workload", default="512x512x256")
    t.add_argument("--steps", type=int, default=20)
    t.add_argument("--warmup", type=int, default=5)
    t.add_argument("--cache", default=None)
    a = ap.parse_args()
    if a.cmd == "ensemble":
        ms, mpts = ensemble48(a.mode, a.steps, a.warmup, a.graph, a.bps)
        print(json.dumps({"ensemble": "48 instances", "mode": a.mode, "graph": a.graph, "ms_per_step": round(ms, 4),
                          "Mpts_per_s": round(mpts, 1)}))
    elif a.cmd == "build-variants":
        for name, lib in build_variants(a.out, a.only).items():
            print(name, lib)
    else:
        name, defines, ms = tune_build(a.workload, a.out, a.only, a.steps, a.warmup, a.cache)
        print(json.dumps({"workload": a.workload, "best": name, "defines": defines, "ms": ms,
                          "cache": cache_path(a.cache)}))


if __name__ == "__main__":
    main()
