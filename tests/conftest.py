"""pytest configuration: the `gpu` marker and shared fixtures.

CPU tests (``-m "not gpu"``) exercise the FP64 oracle, its golden fixtures and the
C-ABI library's loading and argument checks.  GPU tests (``-m gpu``) compare the
CUDA path of libobl_b200.so with the oracle through the C ABI.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libobl_b200.so")


def gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_present():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(autouse=True)
def _index_checks(request):
    """Under the bounds-checked build (tests/test_gpu_checked.py runs a subset of the GPU
    tests with $OBL_LIB = libobl_b200_check.so and $OBL_CHECKED_RUN = 1), every GPU test
    must leave no failed index check behind."""
    yield
    if os.environ.get("OBL_CHECKED_RUN") != "1" or "gpu" not in request.keywords:
        return
    import overlappingbls_b200 as obl
    n, first = obl.check_report()
    assert n != -1, "OBL_CHECKED_RUN is set but the loaded library has no index checks"
    assert n == 0, f"{n} failed index checks, the first: {first}"


@pytest.fixture(scope="session")
def orc():
    from oracle import orc as _orc
    _orc.lib()
    return _orc


def identical_inputs(f, prec):
    """The mixed form stores fields in FP32; the oracle gets the identical (FP32-
    representable) values so that the comparison measures the computation, not the
    rounding of FP64 inputs to FP32 storage."""
    if prec == "f64":
        return f
    return {k: np.asfortranarray(v.astype(np.float32).astype(np.float64)) for k, v in f.items()}


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128 if np.iscomplexobj(a) or np.iscomplexobj(b) else np.float64)
    nb = np.linalg.norm(np.asarray(b).ravel())
    d = np.linalg.norm((a - b).ravel())
    return d / nb if nb > 0 else d
