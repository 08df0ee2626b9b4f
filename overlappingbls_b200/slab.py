"""The step on a domain split in z over several ranks (one GPU each).

Each rank owns a z-slab: nzt_global - 1 = L levels split into nranks blocks of L/nranks
levels, the rank's arrays holding its levels plus the planes it shares with the ranks
below and above (levels 0 and nz of the slab), as the reference's npz z-ranks do
(102_initial.f90:119, nz = (nzt-1)/npz + 1).  One step is

    begin  (rank-local: forward pass, divtz planes, the rank's H_z(1) plane)
    all-gather of the H_z(1) planes        (each rank takes the plane of rank+1)
    solve  (rank-local: partitioned Thomas elimination of the rank's rows, in FP64)
    all-gather of the interface coefficients
    finish (rank-local: reduced system, the rank's p_hat, inverse transforms, project)

The collectives are the only communication; they carry one spectral plane and 64 bytes
per (kx,ky) column per rank.  ``SlabStep`` runs one rank with a collective object
(``TorchComm``: torch.distributed, NCCL between GPUs or gloo on the host);
``step_lockstep`` runs several slabs of one process in lock-step (each phase on every
slab, then the exchange), e.g. to check the split against a single-domain step.

``backend`` is the per-rank compute: ``LibBackend`` (the CUDA library, the product), or
any object with the same methods (the tests use a numpy restatement for the host-only
collective tests).
"""
import numpy as np


class TorchComm:
    """all_gather over torch.distributed (the default group unless one is given)."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)

    def all_gather(self, out, inp):
        """out: (size, *inp.shape) tensor; row k receives rank k's inp."""
        self.dist.all_gather(list(out.unbind(0)), inp, group=self.group)


class LibBackend:
    """The CUDA library as the per-rank compute of a slab (Context of the rank's slab)."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.plane_bytes, self.iface_bytes = ctx.slab_sizes()

    def alloc(self, nbytes, torch):
        return torch.empty(nbytes, dtype=torch.uint8, device="cuda")

    def begin(self, io, rank, nranks, plane_out):
        self.ctx.slab_begin_dev(io, rank, nranks, plane_out.data_ptr())

    def solve(self, plane_above, rank, nranks, iface_out):
        self.ctx.slab_solve_dev(None if plane_above is None else plane_above.data_ptr(), rank, nranks,
                                iface_out.data_ptr())

    def finish(self, io, iface_all, rank, nranks):
        self.ctx.slab_finish_dev(io, iface_all.data_ptr(), rank, nranks)


def slab_grid(nxt, nyt, nzt_global, lz_tot, nranks):
    """(nzt, lz_tot) of one rank's slab context; raises if the levels do not split."""
    L = nzt_global - 1
    if L % nranks or L // nranks < 2:
        raise ValueError(f"{L} levels do not split into {nranks} slabs of >= 2 levels")
    return L // nranks + 1, lz_tot * (L // nranks) / L


class SlabStep:
    """One rank's step of a z-split domain (see the module docstring)."""

    def __init__(self, backend, rank, nranks, comm=None):
        import torch
        self.b, self.rank, self.nranks, self.comm = backend, rank, nranks, comm
        self.plane = backend.alloc(backend.plane_bytes, torch)
        self.planes = torch.stack([backend.alloc(backend.plane_bytes, torch) for _ in range(nranks)])
        self.iface = backend.alloc(backend.iface_bytes, torch)
        self.ifaces = torch.stack([backend.alloc(backend.iface_bytes, torch) for _ in range(nranks)])

    def above(self):
        return self.planes[self.rank + 1] if self.rank < self.nranks - 1 else None

    def _gather(self, what, out, inp):
        # a rank that left or stalls ends the survivors' collective with the process
        # group's timeout or a closed connection; say which exchange of the step it was
        try:
            self.comm.all_gather(out, inp)
        except Exception as e:
            raise RuntimeError(f"slab step, rank {self.rank} of {self.nranks}: the all-gather of the {what} "
                               f"failed ({type(e).__name__}: {e})") from e

    def step(self, io):
        self.b.begin(io, self.rank, self.nranks, self.plane)
        self._gather("H_z(1) planes", self.planes, self.plane)
        self.b.solve(self.above(), self.rank, self.nranks, self.iface)
        self._gather("interface coefficients", self.ifaces, self.iface)
        self.b.finish(io, self.ifaces, self.rank, self.nranks)


def step_lockstep(slabs, ios):
    """The step of all slabs of one process: every phase on every rank, then the
    exchange (a copy into every rank's gather buffer)."""
    for s, io in zip(slabs, ios):
        s.b.begin(io, s.rank, s.nranks, s.plane)
    for s in slabs:
        for t in slabs:
            s.planes[t.rank].copy_(t.plane)
    for s in slabs:
        s.b.solve(s.above(), s.rank, s.nranks, s.iface)
    for s in slabs:
        for t in slabs:
            s.ifaces[t.rank].copy_(t.iface)
    for s, io in zip(slabs, ios):
        s.b.finish(io, s.ifaces, s.rank, s.nranks)
