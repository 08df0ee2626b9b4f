"""CPU tests of the C-ABI boundary: the library builds, loads, exports every symbol
that include/obl.h declares, and rejects bad arguments with status codes (no GPU
needed; no compute is launched)."""
import ctypes
import os
import re

import pytest

import overlappingbls_b200 as obl
from conftest import ROOT, gpu_present

HEADER = os.path.join(ROOT, "include", "obl.h")


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|long long)\s+(obl_\w+)\s*\(", txt, re.M)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(obl.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = obl.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_null_context_is_rejected():
    lib = obl.load_library()
    assert lib.obl_ddx(None, None, None, 1) == 1          # OBL_ERR_ARG
    assert lib.obl_press_stag_array_dev(None, *([None] * 8)) == 1
    assert lib.obl_launch_count(None) == -1
    assert lib.obl_ctx_destroy(None) == 0


def test_bad_grid_rejected_before_touching_the_gpu():
    lib = obl.load_library()
    h = ctypes.c_void_p()
    g = obl.Grid(64, 64, 2, 1.0, 1.0, 1.0, 1.0, 0.1, 1.0)      # nzt too small
    assert lib.obl_ctx_create(ctypes.byref(g), None, ctypes.byref(h)) == 1
    g = obl.Grid(100, 64, 65, 1.0, 1.0, 1.0, 1.0, 0.1, 1.0)    # no FFT plan for 100
    assert lib.obl_ctx_create(ctypes.byref(g), None, ctypes.byref(h)) == 5
    assert not h.value


@pytest.mark.parametrize("n,ok", [(80, True), (160, True), (240, True), (320, True), (640, True),
                                  (512, True), (72, False), (100, False), (1024, False)])
def test_line_lengths_with_plans(n, ok):
    """Lengths with a compiled plan (radix 2, 3, 4, 5 chains and their 3/2 partners) pass the
    length check, which runs before any device call; others give OBL_ERR_UNSUPPORTED."""
    lib = obl.load_library()
    h = ctypes.c_void_p()
    g = obl.Grid(n, 64, 9, 1.0, 1.0, 1.0, 1.0, 0.1, 1.0)
    rc = lib.obl_ctx_create(ctypes.byref(g), None, ctypes.byref(h))
    if ok:
        assert rc != 5
        if rc == 0:
            lib.obl_ctx_destroy(h)
    else:
        assert rc == 5


@pytest.mark.skipif(gpu_present(), reason="checks the no-device path")
def test_no_device_fails_loudly():
    with pytest.raises(obl.OblError, match="NODEV"):
        obl.Context(64, 64, 65, 1.0, 1.0, 1.0, 1.0, 0.1)


def test_every_run_time_parameter_is_documented():
    """Each name obl_set_param accepts (its table in csrc/api.cu) is described in the
    obl_set_param comment of include/obl.h, and the comment names no other."""
    src = open(os.path.join(ROOT, "overlappingbls_b200", "csrc", "api.cu")).read()
    accepted = set(re.findall(r'std::strcmp\(name, "(\w+)"\)', src))
    hdr = open(HEADER).read()
    block = hdr[hdr.index("/* execution tuning"):hdr.index("int obl_set_param")]
    documented = set(re.findall(r'^\s*"(\w+)"\s', block.replace("/*", " "), re.M))
    assert accepted and accepted == documented, (sorted(accepted - documented), sorted(documented - accepted))
