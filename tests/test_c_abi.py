"""The C ABI from a plain C program (tests/c/obl_c_check.c): compiled with gcc against
include/obl.h and linked with libobl_b200.so, as a C or Fortran host of the reference
would link it.  On the CPU it must build, link and report that no device is present; on
a GPU its known-answer checks (derivatives, 3/2 padding, a divergence-free projection)
must pass."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "overlappingbls_b200")


def _build(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc is not installed")
    if not os.path.exists(os.path.join(LIBDIR, "libobl_b200.so")):
        pytest.skip("libobl_b200.so is not built")
    exe = str(tmp_path / "obl_c_check")
    cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-Werror", os.path.join(ROOT, "tests", "c", "obl_c_check.c"),
           "-I", os.path.join(ROOT, "include"), "-L", LIBDIR, "-lobl_b200", "-Wl,-rpath," + LIBDIR, "-lm",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_c_program_builds_links_and_runs(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    # 3: no CUDA device (this host); 0: every check passed (a GPU host)
    assert r.returncode in (0, 3), r.stdout + r.stderr


@pytest.mark.gpu
def test_c_program_checks_pass_on_gpu(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "C ABI check passed" in r.stdout


def _build_dropin(tmp_path):
    if shutil.which("gcc") is None:
        pytest.skip("gcc is not installed")
    if not os.path.exists(os.path.join(LIBDIR, "libobl_b200.so")):
        pytest.skip("libobl_b200.so is not built")
    exe = str(tmp_path / "obl_dropin_check")
    cmd = ["gcc", "-std=c11", "-O2", "-Wall", "-Werror", os.path.join(ROOT, "tests", "c", "obl_dropin_check.c"),
           "-I", os.path.join(ROOT, "include"), "-L", LIBDIR, "-lobl_b200", "-Wl,-rpath," + LIBDIR, "-lm",
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_dropin_mirror_builds(tmp_path):
    _build_dropin(tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("top,npz", [("single", 1), ("neumann", 2)])
@pytest.mark.parametrize("theta", [0, 1])
def test_dropin_time_loop_slice_matches_oracle(tmp_path, orc, top, npz, theta):
    """press_stag_array(p, dpdx, dpdy), the flosol dpdz lines and project() through the
    drop-in routines (C restatement of fortran/obl_dropin.f90, real(8) module arrays, the
    reference's interfaces) against the oracle's press_stag_array (npz ranks), dpdz and
    project on the same inputs, with divtz boundary planes and, with theta on, the
    surface-temperature term folded into the bottom plane (109_press_stag_array.f90:187-192)."""
    import numpy as np
    from overlappingbls_b200 import fields
    from conftest import rel_l2

    exe = _build_dropin(tmp_path)
    nx, ny, nzt = 64, 48, 17
    D = fields.DOMAIN
    g = orc.Grid(nx, ny, nzt, **D)
    f = fields.make_fields(nx, ny, nzt)
    rng = np.random.default_rng(31)
    divtz = np.asfortranarray(rng.standard_normal(f["u"].shape) * 0.1)
    T_s = np.asfortranarray(290.0 + rng.standard_normal((nx, ny)))
    zi, us = D["z_i"], D["u_scale"]
    hdr = np.array([nx, ny, nzt, theta], np.int32).tobytes()
    dz = (D["lz_tot"] / (nzt - 1)) / zi
    dh = np.array([D["lx_tot"] / zi, D["ly_tot"] / zi, D["lz_tot"] / zi, D["dt"] * us / zi, zi, us, dz]).tobytes()
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(fin, "wb") as fh:
        fh.write(hdr + dh)
        for a in (f["u"], f["v"], f["w"], divtz, T_s):
            fh.write(np.ravel(a, order="F").tobytes())
    r = subprocess.run([exe, fin, fout, top], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    ldx, nz = g.ldx, g.nz
    nf, nd = ldx * ny * (nz + 1), ldx * ny * nz
    out = np.fromfile(fout, np.float64)
    sizes = [nf, nd, nd, nd, nf, nf, nf]
    parts = np.split(out, np.cumsum(sizes)[:-1])
    shp = lambda a, n: a.reshape((ldx, ny, n), order="F")
    p, dpdx, dpdy, dpdz = shp(parts[0], nz + 1), shp(parts[1], nz), shp(parts[2], nz), shp(parts[3], nz)
    u, v, w = (shp(parts[i], nz + 1) for i in (4, 5, 6))

    # the oracle: bottom plane with the folded surface term, as press_stag_array forms it
    bot = divtz[:, :, 1].copy(order="F")
    if theta:
        bot[:nx] = divtz[:nx, :, 1] - 9.81 * (zi / us ** 2) * (T_s - T_s.mean())
    top_plane = np.asfortranarray(divtz[:, :, nz])
    rp, rdx, rdy = g.press_stag_array(f["u"], f["v"], f["w"], bot, top_plane, npz=npz)
    rdz = g.dpdz(rp)
    ru, rv, rw = g.project(f["u"], f["v"], f["w"], rdx, rdy, rdz)
    L = nz - 1
    assert rel_l2(p[:nx, :, :L + 1], rp[:nx, :, :L + 1]) < 1e-12
    for a, b in ((dpdx, rdx), (dpdy, rdy), (dpdz, rdz)):
        assert rel_l2(a[:nx, :, :L], b[:nx, :, :L]) < 1e-12
    for a, b in ((u, ru), (v, rv), (w, rw)):
        assert rel_l2(a, b) < 1e-12
