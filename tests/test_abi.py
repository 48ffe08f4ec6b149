"""The C-ABI library builds for sm_100a, loads without a GPU and exports every
entry point include/fdtd_b200.h declares (no compute calls here)."""
import ctypes
import os
import re
import subprocess

from conftest import ROOT, load_package

pkg = load_package()
from special_topics_b200 import _native as N  # noqa: E402


def header_functions():
    src = open(os.path.join(ROOT, "include", "fdtd_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fdtd_\w+)\s*\(", src)))


def test_library_builds_and_loads():
    path = N.build()
    assert os.path.exists(path)
    N.lib()


def test_every_declared_symbol_is_exported():
    L = N.lib()
    names = header_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(L, name), name
    assert sorted(N.EXPORTS) == names


def test_exports_are_plain_c_symbols():
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (fdtd_\w+)$", out, flags=re.M))
    assert set(header_functions()) <= exported


def test_device_count_without_gpu_is_not_an_error():
    n = ctypes.c_int(-1)
    assert N.lib().fdtd_device_count(ctypes.byref(n)) == 0
    assert n.value >= 0


def test_bad_arguments_are_rejected_with_a_message():
    L = N.lib()
    cfg = N.FdtdConfig(1, 1, 1, 1e-3, 1e-3, 1e-3, 1e-12, 10, 0, 0)
    h = ctypes.c_void_p()
    rc = L.fdtd_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == N.FDTD_ERR_BADARG
    assert b"too small" in L.fdtd_last_error()
    assert L.fdtd_run_batch(0, 1, None, None) == N.FDTD_ERR_STATE
