"""Restart-file format (CPU): the oracle's restatement and the library's host-only
total_time entry points.

* total_time.dat: the reference's own file (tests/golden/total_time.dat, copied from
  SBL/readin by tests/golden/gen_total_time.py) reads as its step number, and writing
  that number back reproduces the file byte for byte, through the oracle and through
  obl_read_total_time / obl_write_total_time; a missing file means step 0;
* the field layout: one field is the Fortran-order FP64 interior (x < nxt, levels
  1..nz-1); z-ranks writing their own blocks into one file give exactly the file of a
  single rank holding the whole column; vel_tt holds 11 fields one global field apart.
"""
import os

import numpy as np
import pytest

from oracle import restart_ref as rr

GOLD = os.path.join(os.path.dirname(__file__), "golden", "total_time.dat")


def test_total_time_golden_oracle(tmp_path):
    n = rr.read_total_time(GOLD)
    assert n == 4000000
    out = tmp_path / "total_time.dat"
    rr.write_total_time(str(out), n)
    assert out.read_bytes() == open(GOLD, "rb").read()
    assert rr.read_total_time(str(tmp_path / "missing.dat")) == 0


def test_total_time_golden_library(tmp_path):
    import overlappingbls_b200 as obl
    assert obl.read_total_time(GOLD) == 4000000
    out = tmp_path / "total_time.dat"
    obl.write_total_time(str(out), 4000000)
    assert out.read_bytes() == open(GOLD, "rb").read()
    assert obl.read_total_time(str(tmp_path / "missing.dat")) == 0
    obl.write_total_time(str(out), 7)
    assert obl.read_total_time(str(out)) == 7


def _field(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    return np.asfortranarray(rng.standard_normal((nx + 2, ny, nz + 1)))


def test_field_layout(tmp_path):
    nx, ny, nz = 8, 6, 5
    f = _field(nx, ny, nz, 1)
    fn = str(tmp_path / "one.out")
    rr.write_file_3d(fn, f, nx, disp0=16)
    raw = open(fn, "rb").read()
    assert len(raw) == 16 + 8 * nx * ny * (nz - 1)
    got = np.frombuffer(raw[16:], "=f8").reshape((nx, ny, nz - 1), order="F")
    assert np.array_equal(got, f[:nx, :, 1:nz])
    back = np.full_like(f, 3.0)
    rr.read_file_3d(fn, back, nx, disp0=16)
    assert np.array_equal(back[:nx, :, 1:nz], f[:nx, :, 1:nz])
    assert np.all(back[nx:] == 3.0) and np.all(back[:, :, 0] == 3.0) and np.all(back[:, :, nz] == 3.0)


@pytest.mark.parametrize("P", [2, 3])
def test_rank_blocks_tile_the_global_field(tmp_path, P):
    nx, ny, Lr = 8, 6, 4
    g = _field(nx, ny, P * Lr + 1, 2)          # the whole column: levels 0..P*Lr+1
    whole = str(tmp_path / "whole.out")
    rr.write_file_3d(whole, g, nx, disp0=0)
    split = str(tmp_path / "split.out")
    for r in reversed(range(P)):               # any order
        loc = np.asfortranarray(g[:, :, r * Lr: r * Lr + Lr + 2])   # rank r: levels 0..Lr+1
        rr.write_file_3d(split, loc, nx, disp0=0, zrank=r, nzranks=P)
    assert open(whole, "rb").read() == open(split, "rb").read()


def test_vel_tt_fields_and_zeros(tmp_path):
    nx, ny, nz = 8, 6, 5
    fields = {k: _field(nx, ny, nz, 10 + i) for i, k in enumerate(rr.VEL_TT_FIELDS[:6])}
    path = str(tmp_path / "restart") + "/"
    fn = rr.checkpoint_final(path, 1234, fields, nx)
    assert os.path.basename(fn) == "vel_tt00001234.out"
    d3 = rr.field_bytes(nx, ny, nz)
    raw = open(fn, "rb").read()
    assert len(raw) == 11 * d3
    for k, name in enumerate(rr.VEL_TT_FIELDS):
        blk = np.frombuffer(raw[k * d3:(k + 1) * d3], "=f8").reshape((nx, ny, nz - 1), order="F")
        exp = fields[name][:nx, :, 1:nz] if name in fields else 0.0
        assert np.array_equal(blk, np.broadcast_to(exp, blk.shape))
    back = {k: np.zeros_like(v) for k, v in fields.items()}
    rr.read_flow_field(path, 1234, back, nx)
    for k in fields:
        assert np.array_equal(back[k][:nx, :, 1:nz], fields[k][:nx, :, 1:nz])
