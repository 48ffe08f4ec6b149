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


HANDLE_TYPES = ("fdtd_ctx", "fdtd_batch", "fdtd_es")


def _handle_functions():
    """Header entry points whose first parameter is a handle (or the member
    list of fdtd_batch_create), with their return types."""
    src = open(os.path.join(ROOT, "include", "fdtd_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    out = {}
    for ret, name, args in re.findall(r"\b(int|void|double)\s+(fdtd_\w+)\s*\(([^)]*)\)", src):
        first = args.split(",")[0]
        if any(t in first for t in HANDLE_TYPES):
            out[name] = ret
    return out


def _null_args(fn):
    args = []
    for t in fn.argtypes or []:
        if t in (ctypes.c_int, ctypes.c_long, ctypes.c_longlong, ctypes.c_uint, ctypes.c_size_t):
            args.append(0)
        elif t in (ctypes.c_float, ctypes.c_double):
            args.append(0.0)
        else:
            args.append(None)       # every pointer, the handle included
    return args


def test_null_handles_are_rejected_with_a_message():
    """Every entry point that takes a handle answers a NULL handle (and NULL
    pointers) with an error code and a message, as the reference's ABI does
    (FDTD_OK / FDTD_ERR, fdtd_last_error: fdtd_cuda.h:12-13, fdtd_cuda.cu:40-41),
    before any device work: no GPU is needed for any of these calls."""
    L = N.lib()
    funcs = _handle_functions()
    assert len(funcs) >= 50
    for name, ret in sorted(funcs.items()):
        fn = getattr(L, name)
        assert fn.argtypes is not None, f"{name} has no argtypes in _native"
        rc = fn(*_null_args(fn))
        if ret == "void":
            continue                                   # the free functions accept NULL
        if name in ("fdtd_ctx_step", "fdtd_batch_size"):
            assert rc == -1, name
            continue
        assert rc == N.FDTD_ERR_BADARG, f"{name} returned {rc}"
        assert L.fdtd_last_error(), name
