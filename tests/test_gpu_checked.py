"""The GPU parity subset under the bounds-checked build.

libobl_b200_check.so (`python -m overlappingbls_b200.build --checked`, -DOBL_CHECK=1) tests
each checked global index of the hot-path kernels against the extents the kernel's
arguments give (column loads and stores, the row units' pairs, the solve's rows and bulk
copies, the pressure inverse's lines) and records a failure instead of making the access
(csrc/check.cuh).  This module runs a subset of the GPU tests in a child process with that
library loaded ($OBL_LIB); the conftest fixture then fails any test that leaves a failed
check behind.  The checks themselves are exercised by obl_check_selftest, which fails one
check without a wrong index in any kernel.  Outputs are also poisoned with NaN before a step
so that an element the kernels fail to write shows up."""
import os
import subprocess
import sys

import numpy as np
import pytest

import overlappingbls_b200 as obl
from overlappingbls_b200 import build, fields
from conftest import ROOT, rel_l2

pytestmark = pytest.mark.gpu

SUBSET = [
    "tests/test_gpu_step.py::test_step_matches_oracle",
    "tests/test_gpu_step.py::test_register_segmented_solve",
    "tests/test_gpu_step.py::test_step_factor5_lengths",
    "tests/test_gpu_checked.py::test_outputs_fully_written",
    "tests/test_gpu_checked.py::test_check_records",
]


def _checked_lib_loaded():
    return os.environ.get("OBL_CHECKED_RUN") == "1"


def test_parity_subset_under_index_checks():
    if _checked_lib_loaded():
        pytest.skip("already the child run")
    if not os.path.exists(build.LIB_CHECK):
        pytest.fail(f"{build.LIB_CHECK} is missing: python -m overlappingbls_b200.build --checked")
    env = dict(os.environ, OBL_LIB=build.LIB_CHECK, OBL_CHECKED_RUN="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-p", "no:cacheprovider", *SUBSET],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=2400)
    tail = "\n".join(r.stdout.splitlines()[-25:])
    print(tail)
    assert r.returncode == 0, tail


def test_check_records():
    """The record path: one failed check is counted with its site, then cleared."""
    if not _checked_lib_loaded():
        pytest.skip("runs in the checked child process")
    assert obl.check_report()[0] == 0
    obl.check_selftest()
    n, first = obl.check_report()
    assert n == 1 and first == "check site 12, index 1", (n, first)
    assert obl.check_report() == (0, "")


@pytest.mark.parametrize("prec", ["mixed", "f64"])
def test_outputs_fully_written(orc, prec):
    """Every output element the parity tests compare is written: outputs start as NaN, and
    after the step the derivatives (x < nxt, every level), the padded fields, p (levels
    0..L) and its gradient (1..L) are finite and match the oracle (128 x 96 x 33)."""
    nx, ny, nzt = 128, 96, 33
    L = nzt - 2
    ctx = obl.Context(nx, ny, nzt, precision=prec, **fields.DOMAIN)
    f = fields.make_fields(nx, ny, nzt)
    if prec == "mixed":
        f = {k: np.asfortranarray(v.astype(np.float32).astype(np.float64)) for k, v in f.items()}
    u, v, w = (f[k].copy(order="F") for k in "uvw")
    d = [ctx.field() for _ in range(8)]
    big = [ctx.big_field() for _ in range(4)]
    p, dp = ctx.field(), [ctx.dfield() for _ in range(3)]
    for a in d + big + [p] + dp:
        a.fill(np.nan)
    ctx.step(u, v, w, f["theta"], d, big, p, dp)
    g = orc.Grid(nx, ny, nzt, **fields.DOMAIN)
    ref = g.step(f["u"], f["v"], f["w"], f["theta"], npz=2)
    tol = 1e-12 if prec == "f64" else 1e-5
    for i in range(8):   # derivatives of u, v, w, theta at every stored level, x < nxt
        assert np.isfinite(d[i][:nx]).all(), i
        assert rel_l2(d[i][:nx], ref["d"][i][:nx]) < tol, i
    for i in range(4):
        assert np.isfinite(big[i]).all(), i
        assert rel_l2(big[i], ref["big"][i]) < tol, i
    assert np.isfinite(p[:nx, :, :L + 1]).all()
    assert rel_l2(p[:nx, :, :L + 1], ref["p"][:nx, :, :L + 1]) < tol
    for a, k in zip(dp, ("dpdx", "dpdy", "dpdz")):
        assert np.isfinite(a[:nx, :, :L]).all(), k
        assert rel_l2(a[:nx, :, :L], ref[k][:nx, :, :L]) < tol, k
    ctx.close()
