"""GPU restart files through the C ABI against the oracle's restatement of the format
(oracle/restart_ref.py: write_file_mpi_3d / read_file_mpi_3d, checkpoint_final,
read_flow_field).  Integer/byte work, so every comparison is exact:

* checkpoint_final_dev writes exactly the oracle's file for the same field values
  (FP32 storage widens exactly), NULL fields as zeros;
* read_flow_field_dev reads an oracle-written file into the interior of each field
  (FP64 exactly, FP32 as the rounded value), leaving the pads, levels 0 and nz and the
  NULL fields untouched;
* two z-ranks (two contexts) writing their blocks give the single-rank file;
* multi-chunk transfers (levels > one 64 MiB chunk) and a missing or short file;
* the transfer rate of one 512x512x256-level field each way.
"""
import os

import numpy as np
import pytest

import overlappingbls_b200 as obl
from overlappingbls_b200 import fields as F
from oracle import restart_ref as rr

pytestmark = pytest.mark.gpu


def _dt(prec):
    import torch
    return torch.float64 if prec == "f64" else torch.float32


def _dev(a, prec):
    import torch
    return torch.from_numpy(np.asarray(a).ravel(order="F")).to("cuda", _dt(prec))


def _host(t, shape):
    return t.double().cpu().numpy().reshape(shape, order="F")


def _rand(shape, seed, prec):
    a = np.asfortranarray(np.random.default_rng(seed).standard_normal(shape))
    return a.astype(np.float32).astype(np.float64) if prec != "f64" else a


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_checkpoint_final_matches_oracle(tmp_path, prec):
    nx, ny, nzt = 64, 48, 33
    ctx = obl.Context(nx, ny, nzt, precision=prec, **F.DOMAIN)
    shape = (ctx.ldx, ny, ctx.nz + 1)
    host = {k: _rand(shape, i, prec) for i, k in enumerate(obl.VEL_TT_FIELDS[:6])}
    dev = {k: _dev(v, prec) for k, v in host.items()}
    gpu_dir, ref_dir = str(tmp_path / "gpu") + "/", str(tmp_path / "ref") + "/"
    ctx.checkpoint_final_dev(gpu_dir, 77, {k: t.data_ptr() for k, t in dev.items()})
    rr.checkpoint_final(ref_dir, 77, host, nx)
    a = open(rr.vel_tt_name(gpu_dir, 77), "rb").read()
    b = open(rr.vel_tt_name(ref_dir, 77), "rb").read()
    assert len(a) == 11 * rr.field_bytes(nx, ny, ctx.nz) and a == b
    ctx.close()


@pytest.mark.parametrize("prec", ["f64", "mixed"])
def test_read_flow_field_matches_oracle(tmp_path, prec):
    nx, ny, nzt = 64, 48, 33
    ctx = obl.Context(nx, ny, nzt, precision=prec, **F.DOMAIN)
    shape = (ctx.ldx, ny, ctx.nz + 1)
    src = {k: _rand(shape, 20 + i, "f64") for i, k in enumerate(obl.VEL_TT_FIELDS)}
    path = str(tmp_path) + "/"
    rr.checkpoint_final(path, 5, src, nx)
    names = [k for k in obl.VEL_TT_FIELDS if k not in ("RHSy", "F_QN")]   # two left NULL
    dev = {k: _dev(np.full(shape, 9.0), prec) for k in names}
    ctx.read_flow_field_dev(path, 5, {k: t.data_ptr() for k, t in dev.items()})
    ctx.synchronize()
    n, nz = nx, ctx.nz
    for k in names:
        got = _host(dev[k], shape)
        exp = src[k][:n, :, 1:nz]
        if prec != "f64":
            exp = exp.astype(np.float32).astype(np.float64)
        assert np.array_equal(got[:n, :, 1:nz], exp), k
        assert np.all(got[n:] == 9.0) and np.all(got[:, :, 0] == 9.0) and np.all(got[:, :, nz] == 9.0), k
    ctx.close()


def test_two_z_ranks_write_the_single_rank_file(tmp_path):
    nx, ny, Lr, P = 32, 32, 8, 2
    whole = obl.Context(nx, ny, P * Lr + 1, precision="f64", **F.DOMAIN)
    g = _rand((whole.ldx, ny, whole.nz + 1), 3, "f64")
    fw, fs = str(tmp_path / "whole.out"), str(tmp_path / "split.out")
    tw = _dev(g, "f64")
    whole.write_file_3d_dev(tw.data_ptr(), fw, disp0=8)
    ranks = [obl.Context(nx, ny, Lr + 1, precision="f64", **F.DOMAIN) for _ in range(P)]
    for r, c in enumerate(ranks):
        t = _dev(np.asfortranarray(g[:, :, r * Lr: r * Lr + Lr + 2]), "f64")
        c.write_file_3d_dev(t.data_ptr(), fs, disp0=8, zrank=r, nzranks=P)
        back = _dev(np.zeros((c.ldx, ny, c.nz + 1)), "f64")
        c.read_file_3d_dev(back.data_ptr(), fw, disp0=8, zrank=r, nzranks=P)
        c.synchronize()
        assert np.array_equal(_host(back, (c.ldx, ny, c.nz + 1))[:nx, :, 1:Lr + 1], g[:nx, :, r * Lr + 1: r * Lr + Lr + 1])
    assert open(fw, "rb").read() == open(fs, "rb").read()
    for c in ranks + [whole]:
        c.close()


def test_multi_chunk_round_trip_and_errors(tmp_path):
    nx = ny = 512
    nzt = 71                        # 70 levels of 2 MiB: chunks of 32, 32 and 6 planes
    ctx = obl.Context(nx, ny, nzt, precision="mixed", **F.DOMAIN)
    shape = (ctx.ldx, ny, ctx.nz + 1)
    a = _rand(shape, 4, "mixed")
    t = _dev(a, "mixed")
    fn = str(tmp_path / "big.out")
    ctx.write_file_3d_dev(t.data_ptr(), fn)
    raw = np.fromfile(fn, "=f8").reshape((nx, ny, ctx.nz - 1), order="F")
    assert np.array_equal(raw, a[:nx, :, 1:ctx.nz])
    back = _dev(np.zeros(shape), "mixed")
    ctx.read_file_3d_dev(back.data_ptr(), fn)
    ctx.synchronize()
    assert np.array_equal(_host(back, shape)[:nx, :, 1:ctx.nz], a[:nx, :, 1:ctx.nz])
    with pytest.raises(obl.OblError, match="OBL_ERR_IO"):
        ctx.read_file_3d_dev(back.data_ptr(), str(tmp_path / "missing.out"))
    with pytest.raises(obl.OblError, match="OBL_ERR_IO"):
        ctx.read_file_3d_dev(back.data_ptr(), fn, disp0=8)   # one double short
    ctx.close()


def test_transfer_rate_512(tmp_path):
    import time
    import torch
    nx = ny = 512
    ctx = obl.Context(nx, ny, 257, precision="mixed", **F.DOMAIN)
    n = ctx.ldx * ny * (ctx.nz + 1)
    t = torch.randn(n, device="cuda")
    back = torch.zeros(n, device="cuda")
    fn = str(tmp_path / "rate.out")
    ctx.write_file_3d_dev(t.data_ptr(), fn)   # first call: staging allocation, file creation
    nbytes = 8 * nx * ny * (ctx.nz - 1)
    t0 = time.perf_counter()
    ctx.write_file_3d_dev(t.data_ptr(), fn)
    t1 = time.perf_counter()
    ctx.read_file_3d_dev(back.data_ptr(), fn)
    t2 = time.perf_counter()
    v = t.view(ctx.nz + 1, ny, ctx.ldx)[1:ctx.nz, :, :nx]
    w = back.view(ctx.nz + 1, ny, ctx.ldx)[1:ctx.nz, :, :nx]
    assert bool((v == w).all())
    # the oracle's restatement on host arrays beside it (one thread, numpy + write/read)
    h = np.asfortranarray(np.zeros((ctx.ldx, ny, ctx.nz + 1)))
    t3 = time.perf_counter()
    rr.write_file_3d(fn, h, nx)
    t4 = time.perf_counter()
    rr.read_file_3d(fn, h, nx)
    t5 = time.perf_counter()
    print(f"restart field 512x512x256 ({nbytes / 1e6:.0f} MB FP64): write {nbytes / (t1 - t0) / 1e9:.2f} GB/s, "
          f"read {nbytes / (t2 - t1) / 1e9:.2f} GB/s from/to HBM; oracle on host arrays: write "
          f"{nbytes / (t4 - t3) / 1e9:.2f} GB/s, read {nbytes / (t5 - t4) / 1e9:.2f} GB/s (wall clock, page cache)")
    os.remove(fn)
    ctx.close()
