"""Worker of the 2-rank gloo test of the z-slab driver (tests/test_slab_gloo.py).

The per-rank compute is the numpy restatement (oracle/slab_ref.py) behind the same
backend interface as the CUDA library; the driver (overlappingbls_b200/slab.py) and its
collectives run unchanged over torch.distributed with the gloo backend.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


class NumpyBackend:
    def __init__(self, tables, dz):
        self.KX, self.KY, self.K2, self.NN = tables
        self.dz = dz
        S = self.KX.shape[0]
        self.S = S
        self.plane_bytes = 16 * S
        self.iface_bytes = 64 * S

    def alloc(self, nbytes, torch):
        return torch.zeros(nbytes, dtype=torch.uint8)

    def begin(self, io, rank, nranks, plane_out):
        plane_out.numpy().view(np.complex128)[:] = io["H"][2][:, 1]

    def solve(self, plane_above, rank, nranks, iface_out):
        H = self.io["H"]
        if plane_above is not None:
            H[2][:, -1] = plane_above.numpy().view(np.complex128)
        from oracle import slab_ref as sr
        self.y, self.v, self.w, iface = sr.local_solve(self.KX, self.KY, self.K2, self.NN, *H, self.dz, rank, nranks)
        iface_out.numpy().view(np.float64)[:] = iface.ravel()

    def finish(self, io, iface_all, rank, nranks):
        from oracle import slab_ref as sr
        ia = iface_all.numpy().view(np.float64).reshape(nranks, self.S, 8)
        first, last = sr.reduced_solve(ia)
        io["ph"], io["dph"] = sr.finish(self.y, self.v, self.w, first, last, io["H"][2][:, 0], self.NN, self.dz,
                                         rank, nranks)


def problem(seed=5, nx=16, ny=12, L=16):
    from oracle import orc
    from oracle import slab_ref as sr
    from overlappingbls_b200.fields import DOMAIN
    g = orc.Grid(nx, ny, L + 1, **DOMAIN)
    kx, ky, kx2, ky2, k2, nn = g.wavenumbers()
    tables = sr.column_tables(kx, ky2[0], g.lhx, g.nyt)
    rng = np.random.default_rng(seed)
    S = g.lhx * g.nyt
    H = [rng.standard_normal((S, L + 2)) + 1j * rng.standard_normal((S, L + 2)) for _ in range(3)]
    return g, tables, H


def run(rank, world, port, out_path):
    import torch
    import torch.distributed as dist
    from overlappingbls_b200 import slab
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        g, tables, H = problem()
        L = H[0].shape[1] - 2
        Lr = L // world
        sl = slice(rank * Lr, rank * Lr + Lr + 2)
        io = {"H": [h[:, sl].copy() for h in H]}
        if rank < world - 1:
            io["H"][2][:, -1] = 0.0       # must come from the rank above through the gather
        b = NumpyBackend(tables, g.dz)
        b.io = io
        step = slab.SlabStep(b, rank, world, slab.TorchComm())
        step.step(io)
        mine = torch.from_numpy(np.ascontiguousarray(io["ph"]).view(np.float64).copy())
        allp = torch.zeros((world,) + tuple(mine.shape), dtype=mine.dtype)
        dist.all_gather(list(allp.unbind(0)), mine)
        if rank == 0:
            np.save(out_path, allp.numpy())
    finally:
        dist.destroy_process_group()


class LeavingComm:
    """TorchComm whose rank `who` leaves before its second all-gather: it exits the
    process abruptly ("exit"), or stops taking part and sleeps ("stall")."""

    def __init__(self, comm, who, how, stall_s):
        self.c, self.who, self.how, self.stall_s, self.calls = comm, who, how, stall_s, 0

    def all_gather(self, out, inp):
        self.calls += 1
        if self.calls == 2 and self.c.rank == self.who:
            if self.how == "exit":
                os._exit(0)
            import time
            time.sleep(self.stall_s)
            os._exit(0)
        self.c.all_gather(out, inp)


def run_leaving(rank, world, port, out_path, how, timeout_s):
    """One slab step with rank world-1 leaving before the second all-gather; every other
    rank records (error message, seconds spent in the step) in out_path.<rank>.json."""
    import datetime
    import json
    import time
    import torch.distributed as dist
    from overlappingbls_b200 import slab
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))
    g, tables, H = problem()
    L = H[0].shape[1] - 2
    Lr = L // world
    sl = slice(rank * Lr, rank * Lr + Lr + 2)
    io = {"H": [h[:, sl].copy() for h in H]}
    b = NumpyBackend(tables, g.dz)
    b.io = io
    comm = LeavingComm(slab.TorchComm(), world - 1, how, stall_s=3 * timeout_s + 10)
    step = slab.SlabStep(b, rank, world, comm)
    t0 = time.monotonic()
    err = None
    try:
        step.step(io)
    except Exception as e:
        err = str(e)
    rec = {"error": err, "seconds": time.monotonic() - t0}
    with open(f"{out_path}.{rank}.json", "w") as fh:
        json.dump(rec, fh)
    os._exit(0)   # the group is broken: leave without its teardown collective
