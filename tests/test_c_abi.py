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
