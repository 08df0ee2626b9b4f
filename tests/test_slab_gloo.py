"""The z-slab driver over torch.distributed with 2 gloo ranks on the host: the
partitioned solve assembled by the driver's collectives equals the single sweep."""
import json
import os
import socket
import time

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_gloo_slab_solve(tmp_path):
    import torch.multiprocessing as mp
    import slab_worker as sw
    from oracle import slab_ref as sr
    out = str(tmp_path / "ph.npy")
    world = 2
    mp.start_processes(sw.run, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    allp = np.load(out).view(np.complex128)
    g, tables, H = sw.problem()
    ref = sr.global_solve(*tables, *H, g.dz)
    L = H[0].shape[1] - 2
    Lr = L // world
    for r in range(world):
        np.testing.assert_allclose(allp[r], ref[:, r * Lr: r * Lr + Lr + 1], rtol=0,
                                   atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("how", ["exit", "stall"])
def test_survivor_gives_up_when_a_rank_leaves(tmp_path, how):
    """Rank 1 leaves between the two all-gathers of a slab step (its process exits, or it
    stops taking part).  Rank 0 must not hang: its second all-gather ends with an error
    within the process group's short timeout, and the driver's message names the
    exchange.  Failure made on the host; no GPU involved."""
    import torch.multiprocessing as mp
    import slab_worker as sw
    out = str(tmp_path / "rec")
    timeout_s = 5
    ctx = mp.start_processes(sw.run_leaving, args=(2, _free_port(), out, how, timeout_s), nprocs=2,
                             start_method="spawn", join=False)
    # rank 0 writes its record and exits; a stalling rank 1 is ended here once it has
    t0 = time.monotonic()
    while not os.path.exists(out + ".0.json") and time.monotonic() - t0 < 120:
        time.sleep(0.5)
    for p in ctx.processes:
        if p.is_alive():
            p.terminate()
        p.join(10)
    with open(out + ".0.json") as fh:
        rec = json.load(fh)
    assert rec["error"] is not None, rec
    assert "interface coefficients" in rec["error"], rec["error"]
    assert rec["seconds"] < 6 * timeout_s, rec
