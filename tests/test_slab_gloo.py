"""The z-slab driver over torch.distributed with 2 gloo ranks on the host: the
partitioned solve assembled by the driver's collectives equals the single sweep."""
import os
import socket

import numpy as np


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
