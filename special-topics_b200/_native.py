"""ctypes binding of libfdtd_b200.so (the C ABI in include/fdtd_b200.h) and its build recipe."""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)
BUILD_DIR = os.path.join(PKG_DIR, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "libfdtd_b200.so")
SOURCES = [os.path.join(PKG_DIR, "csrc", f) for f in
           ("fdtd_b200.cu", "es_net.cu", "fdtd_common.cuh", "fdtd_step.cuh", "fdtd_material.cuh",
            "fdtd_batch.cuh", "fdtd_internal.h", "fdtd_ffpost.cuh")]
CU_SOURCES = [p for p in SOURCES if p.endswith(".cu")]
HEADER = os.path.join(ROOT, "include", "fdtd_b200.h")

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-shared"]

FDTD_OK, FDTD_ERR, FDTD_ERR_BADARG, FDTD_ERR_OOM, FDTD_ERR_CUDA, FDTD_ERR_NONFINITE, FDTD_ERR_STATE = range(7)
PREC_F64, PREC_F32, PREC_F32_TABLE = 0, 1, 2

# Every symbol the header declares (checked by the CPU test suite).
EXPORTS = (
    "fdtd_last_error", "fdtd_device_count", "fdtd_init", "fdtd_upload_coeff", "fdtd_upload_cpml",
    "fdtd_upload_vsource", "fdtd_upload_svoltage", "fdtd_upload_scurrent", "fdtd_run_batch",
    "fdtd_read_field", "fdtd_destroy", "fdtd_create", "fdtd_free", "fdtd_ctx_upload_coeff",
    "fdtd_ctx_upload_cpml", "fdtd_ctx_add_vsource", "fdtd_ctx_add_svoltage", "fdtd_ctx_add_scurrent",
    "fdtd_ctx_setup_farfield", "fdtd_ctx_upload_material", "fdtd_ctx_build_material",
    "fdtd_ctx_override_material", "fdtd_ctx_read_material", "fdtd_ctx_run", "fdtd_ctx_run_timed",
    "fdtd_ctx_profile_kernels", "fdtd_ctx_set_tiling", "fdtd_ctx_get_tiling", "fdtd_ctx_set_prefetch", "fdtd_ctx_step", "fdtd_status",
    "fdtd_ctx_read_trace", "fdtd_ctx_read_field", "fdtd_ctx_read_psi", "fdtd_ctx_read_farfield", "fdtd_dft",
    "fdtd_dft_noalloc", "fdtd_batch_create", "fdtd_batch_free", "fdtd_batch_size", "fdtd_batch_set_tiling",
    "fdtd_batch_get_tiling", "fdtd_batch_run", "fdtd_batch_run_timed", "fdtd_batch_profile_kernels",
    "fdtd_es_create", "fdtd_es_free", "fdtd_es_param_count", "fdtd_es_init_params", "fdtd_es_set_params",
    "fdtd_es_get_params", "fdtd_es_forward", "fdtd_es_loss_grad", "fdtd_es_set_data", "fdtd_es_train",
    "fdtd_es_member_inputs", "fdtd_es_predict_members", "fdtd_ctx_farfield_post",
    "fdtd_ctx_set_dft_accumulator", "fdtd_ctx_state_size", "fdtd_ctx_save_state", "fdtd_ctx_load_state",
    "fdtd_ctx_set_dft_block", "fdtd_batch_set_streams", "fdtd_batch_get_streams",
    "fdtd_ctx_set_block_width", "fdtd_ctx_get_block_width", "fdtd_batch_set_block_width",
    "fdtd_batch_get_block_width", "fdtd_ctx_set_x_wall", "fdtd_ctx_get_x_wall",
    "fdtd_batch_set_members_per_launch", "fdtd_batch_get_members_per_launch",
)


class FdtdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class FdtdConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
                ("numberOfTimeSteps", C.c_int), ("precision", C.c_int), ("device", C.c_int)]


class FdtdEsConfig(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("in_channels", "in_length", "conv_layers", "channels", "kernel", "stride",
                                       "mlp_layers", "mlp_width", "out_dim", "max_batch", "device")]


class FdtdDims(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float), ("dt", C.c_float),
                ("numberOfTimeSteps", C.c_int)]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def build(force: bool = False) -> str:
    """Compiles the engine for sm_100a into the package's _build folder."""
    newest = max(os.path.getmtime(p) for p in SOURCES + [HEADER])
    if not force and os.path.exists(LIB_PATH) and os.path.getmtime(LIB_PATH) >= newest:
        return LIB_PATH
    os.makedirs(BUILD_DIR, exist_ok=True)
    tmp = LIB_PATH + ".tmp"
    cmd = [nvcc(), *NVCC_FLAGS, "-o", tmp, *CU_SOURCES]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


_lib = None


def lib() -> C.CDLL:
    """Loads the engine.  There is no fallback: a missing library is an error."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: build it with special_topics_b200.build()")
    L = C.CDLL(LIB_PATH)
    i, d, v, P = C.c_int, C.c_double, C.c_void_p, C.POINTER
    dp, ip, fp, lp = P(C.c_double), P(C.c_int), P(C.c_float), C.c_long
    L.fdtd_last_error.restype = C.c_char_p
    L.fdtd_device_count.argtypes = [ip]
    L.fdtd_create.argtypes = [P(FdtdConfig), P(v)]
    L.fdtd_free.argtypes = [v]
    L.fdtd_free.restype = None
    L.fdtd_ctx_upload_coeff.argtypes = [v, i, dp, lp]
    L.fdtd_ctx_upload_cpml.argtypes = [v, i, i, dp, dp, dp, dp, dp, dp, dp, lp, dp, lp, dp, lp, dp, lp, i, i]
    L.fdtd_ctx_add_vsource.argtypes = [v, i, ip, dp, i, dp, i]
    L.fdtd_ctx_add_svoltage.argtypes = [v, i, ip, i, d]
    L.fdtd_ctx_add_scurrent.argtypes = [v, ip, ip, dp, i]
    L.fdtd_ctx_setup_farfield.argtypes = [v, i, dp, i, i, i, i, i, i]
    L.fdtd_ctx_upload_material.argtypes = [v, i, P(C.c_ubyte), lp, dp, i]
    ub = P(C.c_ubyte)
    L.fdtd_ctx_build_material.argtypes = [v, ub, lp, i, dp, i, ip, dp]
    L.fdtd_ctx_override_material.argtypes = [v, i, ip, dp, i]
    L.fdtd_ctx_read_material.argtypes = [v, i, ub, lp, dp, ip]
    L.fdtd_ctx_run_timed.argtypes = [v, i, fp]
    L.fdtd_ctx_profile_kernels.argtypes = [v, i, dp]
    L.fdtd_ctx_set_tiling.argtypes = [v, i, i]
    L.fdtd_ctx_get_tiling.argtypes = [v, ip, ip]
    L.fdtd_ctx_set_prefetch.argtypes = [v, i]
    L.fdtd_ctx_run.argtypes = [v, i]
    L.fdtd_ctx_step.argtypes = [v]
    L.fdtd_status.argtypes = [v, ip, ip]
    L.fdtd_ctx_read_trace.argtypes = [v, i, i, dp, i]
    L.fdtd_ctx_read_field.argtypes = [v, i, dp, lp]
    L.fdtd_ctx_read_psi.argtypes = [v, i, i, dp, lp]
    L.fdtd_ctx_read_farfield.argtypes = [v, i, dp, dp, lp]
    L.fdtd_dft.argtypes = [dp, i, d, dp, i, d, dp, dp]
    L.fdtd_ctx_farfield_post.argtypes = [v, dp, dp, i, dp, dp, dp]
    L.fdtd_ctx_set_dft_accumulator.argtypes = [v, i]
    L.fdtd_ctx_set_dft_block.argtypes = [v, i]
    L.fdtd_ctx_set_x_wall.argtypes = [v, i]
    L.fdtd_batch_set_members_per_launch.argtypes = [v, i]
    L.fdtd_batch_get_members_per_launch.argtypes = [v, ip]
    L.fdtd_ctx_get_x_wall.argtypes = [v, ip]
    L.fdtd_ctx_state_size.argtypes = [v, P(C.c_longlong)]
    L.fdtd_ctx_save_state.argtypes = [v, v, C.c_longlong]
    L.fdtd_ctx_load_state.argtypes = [v, v, C.c_longlong]
    L.fdtd_dft_noalloc.argtypes = [dp, i, d, dp, i, d, dp, dp]
    L.fdtd_batch_create.argtypes = [P(v), i, P(v)]
    L.fdtd_batch_free.argtypes = [v]
    L.fdtd_batch_free.restype = None
    L.fdtd_batch_size.argtypes = [v]
    L.fdtd_batch_set_tiling.argtypes = [v, i, i, i, i]
    L.fdtd_batch_get_tiling.argtypes = [v, ip, ip, ip, ip]
    L.fdtd_batch_set_streams.argtypes = [v, i]
    L.fdtd_batch_get_streams.argtypes = [v, ip]
    L.fdtd_ctx_set_block_width.argtypes = [v, i]
    L.fdtd_ctx_get_block_width.argtypes = [v, ip]
    L.fdtd_batch_set_block_width.argtypes = [v, i]
    L.fdtd_batch_get_block_width.argtypes = [v, ip]
    L.fdtd_batch_run.argtypes = [v, i]
    L.fdtd_batch_run_timed.argtypes = [v, i, fp]
    L.fdtd_batch_profile_kernels.argtypes = [v, i, dp]
    L.fdtd_es_create.argtypes = [P(FdtdEsConfig), P(v)]
    L.fdtd_es_free.argtypes = [v]
    L.fdtd_es_free.restype = None
    L.fdtd_es_param_count.argtypes = [v, P(C.c_long)]
    L.fdtd_es_init_params.argtypes = [v, C.c_ulonglong]
    L.fdtd_es_set_params.argtypes = [v, fp, lp]
    L.fdtd_es_get_params.argtypes = [v, fp, lp]
    L.fdtd_es_forward.argtypes = [v, fp, i, fp]
    L.fdtd_es_loss_grad.argtypes = [v, fp, fp, fp, i, fp, fp, lp]
    L.fdtd_es_set_data.argtypes = [v, fp, fp, lp]
    L.fdtd_es_train.argtypes = [v, i, i, fp, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_ulonglong,
                                fp]
    L.fdtd_es_member_inputs.argtypes = [v, P(v), i, i, fp, fp]
    L.fdtd_es_predict_members.argtypes = [v, P(v), i, i, fp, fp]
    L.fdtd_init.argtypes = [P(FdtdDims)]
    L.fdtd_upload_coeff.argtypes = [i, fp, i]
    L.fdtd_upload_cpml.argtypes = [i, i, fp, fp, fp, fp, fp, i, fp, i, fp, i, fp, i, i, i, i]
    L.fdtd_upload_vsource.argtypes = [i, ip, fp, i, fp, i]
    L.fdtd_upload_svoltage.argtypes = [i, ip, i, C.c_float]
    L.fdtd_upload_scurrent.argtypes = [ip, fp, i, ip, fp, i, ip, fp, i]
    L.fdtd_run_batch.argtypes = [i, i, fp, fp]
    L.fdtd_read_field.argtypes = [i, fp, i]
    L.fdtd_destroy.restype = None
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != FDTD_OK:
        raise FdtdError(rc, lib().fdtd_last_error().decode(errors="replace"))


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int))


def fptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


def device_count() -> int:
    n = C.c_int(0)
    check(lib().fdtd_device_count(C.byref(n)))
    return n.value
