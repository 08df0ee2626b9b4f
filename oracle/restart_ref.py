"""restart_ref.py -- numpy restatement of the reference's restart files.

TEST INFRASTRUCTURE ONLY: the checker of the library's restart-file entry points.

* write_file_mpi_3d / read_file_mpi_3d (202_parallel.f90:1084-1120, 1211-1250): one
  field is the global FP64 array (nxt, nyt, nzt-1) in Fortran order ('native'
  representation, no record markers) at byte offset disp0; rank (coordy, coordz) owns
  the subarray of shape (nxt, nynpy, nz-1) at start (0, nynpy*coordy, (nz-1)*coordz)
  (102_initial.f90:154-162).  Here npy = 1, so a z-rank's block is one contiguous run;
* checkpoint_final (012_io.f90:496-546) / read_flow_field (102_01_ic.f90:682-734): the
  fields u, v, w, RHSx, RHSy, RHSz, Cs_opt2, F_LM, F_MM, F_QN, F_NN one after the other,
  disp3d = np * sizeof(local block) = the bytes of one global field apart, in
  path_restart // 'vel_tt' // i8.8 // '.out';
* total_time.dat (012_io.f90:485-490, 102_01_ic.f90:697-705): the step number as one
  list-directed integer; a missing file means step 0.

Fields are numpy arrays (ldx, nyt, nz+1) in Fortran order; levels 1..nz-1 go to the file.
"""
import os

import numpy as np

VEL_TT_FIELDS = ("u", "v", "w", "RHSx", "RHSy", "RHSz", "Cs_opt2", "F_LM", "F_MM", "F_QN", "F_NN")


def field_bytes(nxt, nyt, nz, nzranks=1):
    """disp3d: one global field, (nxt, nyt, nzranks*(nz-1)) doubles (012_io.f90:519)."""
    return 8 * nxt * nyt * (nz - 1) * nzranks


def rank_offset(nxt, nyt, nz, zrank):
    """Byte offset of z-rank zrank's block inside a field (start(3) = (nz-1)*coordz)."""
    return 8 * nxt * nyt * (nz - 1) * zrank


def _open_rw(fn):
    # MPI_MODE_WRONLY + MPI_MODE_CREATE: created when missing, never truncated
    return open(fn, "r+b") if os.path.exists(fn) else open(fn, "w+b")


def write_file_3d(fn, var, nxt, disp0=0, zrank=0, nzranks=1):
    nz = var.shape[2] - 1
    block = np.asarray(var[:nxt, :, 1:nz], dtype="=f8")
    with _open_rw(fn) as f:
        f.seek(disp0 + rank_offset(nxt, var.shape[1], nz, zrank))
        f.write(block.tobytes(order="F"))


def read_file_3d(fn, var, nxt, disp0=0, zrank=0, nzranks=1):
    if not os.path.exists(fn):
        raise FileNotFoundError("FILE DOES NOT EXIST")   # 202_parallel.f90:1244-1246
    nyt, nz = var.shape[1], var.shape[2] - 1
    n = nxt * nyt * (nz - 1)
    with open(fn, "rb") as f:
        f.seek(disp0 + rank_offset(nxt, nyt, nz, zrank))
        raw = f.read(8 * n)
    if len(raw) != 8 * n:
        raise EOFError("restart file too short")
    var[:nxt, :, 1:nz] = np.frombuffer(raw, dtype="=f8").reshape((nxt, nyt, nz - 1), order="F")


def vel_tt_name(path_restart, nums):
    return f"{path_restart}vel_tt{nums:08d}.out"


def checkpoint_final(path_restart, nums, fields, nxt, zrank=0, nzranks=1):
    """fields: dict by VEL_TT_FIELDS name; a missing field is written as zeros."""
    if path_restart and not os.path.isdir(path_restart):
        os.mkdir(path_restart)                        # 012_io.f90:514-518
    ref = next(v for v in fields.values() if v is not None)
    nyt, nz = ref.shape[1], ref.shape[2] - 1
    d3 = field_bytes(nxt, nyt, nz, nzranks)
    fn = vel_tt_name(path_restart, nums)
    for k, name in enumerate(VEL_TT_FIELDS):
        v = fields.get(name)
        if v is None:
            v = np.zeros_like(ref)
        write_file_3d(fn, v, nxt, k * d3, zrank, nzranks)
    return fn


def read_flow_field(path_restart, nums, fields, nxt, zrank=0, nzranks=1):
    ref = next(v for v in fields.values() if v is not None)
    nyt, nz = ref.shape[1], ref.shape[2] - 1
    d3 = field_bytes(nxt, nyt, nz, nzranks)
    fn = vel_tt_name(path_restart, nums)
    for k, name in enumerate(VEL_TT_FIELDS):
        if fields.get(name) is not None:
            read_file_3d(fn, fields[name], nxt, k * d3, zrank, nzranks)


def read_total_time(fn):
    if not os.path.exists(fn):
        return 0                                     # "Restart file NOT found"
    with open(fn) as f:
        return int(f.read().split()[0])


def write_total_time(fn, nums):
    with open(fn, "w") as f:
        f.write(f"{nums:12d}\n")                     # list-directed default integer
