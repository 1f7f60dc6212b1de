"""ctypes binding of libscpgpu.so (the C ABI of include/scp_gpu.h).

The library is built in-tree (``python -m scp_b200.build``) and loaded from
the package directory.  There is no fallback: if the shared object is missing
or does not export the ABI, importing the product fails loudly.
"""
from __future__ import annotations

import ctypes
import os

from .params import CParams

LIB_NAME = "libscpgpu.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

# every symbol declared in include/scp_gpu.h
EXPORTS = (
    "scp_gpu_init", "scp_gpu_init_device", "scp_gpu_step", "scp_gpu_sync", "scp_gpu_diag",
    "scp_gpu_snapshot", "scp_gpu_get_info", "scp_gpu_time_steps", "scp_gpu_stream",
    "scp_gpu_free", "scp_gpu_errstr", "scp_gpu_last_cuda_error", "scp_gpu_abi_version",
    "scp_gpu_diag_noalloc", "scp_gpu_check_trig",
)

DIAG_NSLOTS = 40


class DiagOut(ctypes.Structure):
    _fields_ = [("v", ctypes.c_double * DIAG_NSLOTS)]


class Info(ctypes.Structure):
    _fields_ = [
        ("steps_done", ctypes.c_int64),
        ("time", ctypes.c_double),
        ("G_offset", ctypes.c_double),
        ("cg_iterations", ctypes.c_int32),
        ("precision_mode", ctypes.c_int32),
        ("device_bytes", ctypes.c_int64),
        ("state_bytes_per_site", ctypes.c_double),
        ("step_bytes_per_site", ctypes.c_double),
        ("tile_x", ctypes.c_int32),
        ("tile_y", ctypes.c_int32),
        ("seg_len", ctypes.c_int32),
    ]


class ScpError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        super().__init__(what)


_lib = None


def lib() -> ctypes.CDLL:
    """Load the CUDA library once; raises if it is missing or incomplete."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m scp_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    for sym in EXPORTS:
        if not hasattr(L, sym):
            raise ImportError(f"{LIB_PATH} does not export {sym}")
    vp = ctypes.c_void_p
    L.scp_gpu_init.argtypes = [ctypes.POINTER(CParams), ctypes.POINTER(vp), ctypes.POINTER(vp)]
    L.scp_gpu_init_device.argtypes = [ctypes.POINTER(CParams), ctypes.POINTER(vp), ctypes.POINTER(vp)]
    L.scp_gpu_step.argtypes = [vp, ctypes.c_int]
    L.scp_gpu_sync.argtypes = [vp]
    L.scp_gpu_diag.argtypes = [vp, ctypes.POINTER(DiagOut)]
    L.scp_gpu_snapshot.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp)]
    L.scp_gpu_get_info.argtypes = [vp, ctypes.POINTER(Info)]
    L.scp_gpu_time_steps.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.scp_gpu_stream.argtypes = [vp]
    L.scp_gpu_stream.restype = vp
    L.scp_gpu_free.argtypes = [vp]
    L.scp_gpu_free.restype = None
    L.scp_gpu_errstr.argtypes = [ctypes.c_int]
    L.scp_gpu_errstr.restype = ctypes.c_char_p
    L.scp_gpu_last_cuda_error.restype = ctypes.c_char_p
    L.scp_gpu_check_trig.argtypes = [ctypes.c_int, vp, vp]
    L.scp_gpu_diag_noalloc.argtypes = [ctypes.POINTER(CParams), ctypes.POINTER(vp), ctypes.c_double, vp,
                                       ctypes.POINTER(DiagOut)]
    _lib = L
    return L


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        L = lib()
        msg = L.scp_gpu_errstr(rc).decode()
        cuda = L.scp_gpu_last_cuda_error().decode()
        raise ScpError(rc, f"{what}: {msg} ({rc})" + (f" [{cuda}]" if cuda else ""))
