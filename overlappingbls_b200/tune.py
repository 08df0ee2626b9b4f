"""Autotuner of the step's execution choices, cached per device in a JSON file.

Two kinds of entries:

* ``step``: per (nxt, nyt, nzt, precision) the single-instance step variant: ``fused``
  0 (multi-output line kernels), 1 (cluster-fused forward plane kernel, square grids; with
  its cluster size and cluster count) or 2 (one kernel per reference routine).
* ``ensemble``: per ensemble signature (the multiset of instance shapes and the
  precision) the ensemble mode (sequential, concurrent streams, one persistent launch,
  the register-class split of it), whether to replay a CUDA graph, and the persistent
  kernel's CTAs per SM.

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
    """The variants of the single-instance step worth timing for this grid."""
    cands = [{"fused": 0}, {"fused": 2}]
    if nxt == nyt:
        for csize in (4, 8):
            for ncl in (0, 16):
                cands.append({"fused": 1, "fwd_cluster_size": csize, "fwd_clusters": ncl})
    return cands


ENSEMBLE_CANDIDATES = (
    {"mode": "sequential", "graph": False, "bps": 0},
    {"mode": "sequential", "graph": True, "bps": 0},
    {"mode": "concurrent", "graph": False, "bps": 0},
    {"mode": "concurrent", "graph": True, "bps": 0},
    {"mode": "persistent", "graph": True, "bps": 0},
    {"mode": "persistent", "graph": True, "bps": 1},
    {"mode": "persistent_split", "graph": True, "bps": 0},
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
