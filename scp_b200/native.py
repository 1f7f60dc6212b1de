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
    "scp_gpu_snapshot", "scp_gpu_snapshot_async", "scp_gpu_snapshot_wait", "scp_gpu_host_alloc",
    "scp_gpu_host_free", "scp_gpu_get_info", "scp_gpu_time_steps", "scp_gpu_stream",
    "scp_gpu_free", "scp_gpu_errstr", "scp_gpu_last_cuda_error", "scp_gpu_abi_version",
    "scp_gpu_diag_noalloc", "scp_gpu_check_trig",
    "scp_srv_create", "scp_srv_submit", "scp_srv_submit_borrowed", "scp_srv_poll", "scp_srv_status", "scp_srv_result",
    "scp_srv_stats", "scp_srv_free",
)

DIAG_NSLOTS = 40

# status codes (include/scp_gpu.h)
SCP_OK = 0
SCP_EINVAL = -1
SCP_ENOMEM = -2
SCP_ECUDA = -3
SCP_ENETCHARGE = -4
SCP_EGAUSS = -5
SCP_ENONFINITE = -6
SCP_EUNSUPPORTED = -7
SCP_ENODEV = -8
SCP_EBUSY = -9
SCP_ETIMEOUT = -10


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
        ("sites_per_thread", ctypes.c_int32),
        ("tma_staging", ctypes.c_int32),
    ]


class SrvConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int32),
        ("max_active", ctypes.c_int32),
        ("mem_budget_bytes", ctypes.c_int64),
        ("chunk_steps", ctypes.c_int32),
        ("use_graph", ctypes.c_int32),
        ("autotune", ctypes.c_int32),
        ("admit_per_poll", ctypes.c_int32),
        ("loader_threads", ctypes.c_int32),
    ]


class SrvRequestInfo(ctypes.Structure):
    _fields_ = [
        ("state", ctypes.c_int32), ("rc", ctypes.c_int32),
        ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double),
        ("nsteps", ctypes.c_int64), ("N", ctypes.c_int32), ("tile_variant", ctypes.c_int32),
    ]


class SrvStats(ctypes.Structure):
    _fields_ = [
        ("step", ctypes.c_int64), ("chunks", ctypes.c_int64), ("mem_in_use", ctypes.c_int64),
        ("n_active", ctypes.c_int32), ("n_queued", ctypes.c_int32), ("n_groups", ctypes.c_int32),
        ("t_admit", ctypes.c_double), ("t_autotune", ctypes.c_double), ("t_run", ctypes.c_double),
        ("t_retire", ctypes.c_double), ("t_wait", ctypes.c_double),
        ("t_launch", ctypes.c_double), ("t_gpu", ctypes.c_double),
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
    L.scp_gpu_snapshot_async.argtypes = [vp, ctypes.c_int, ctypes.POINTER(vp)]
    L.scp_gpu_snapshot_wait.argtypes = [vp]
    L.scp_gpu_host_alloc.argtypes = [ctypes.c_size_t]
    L.scp_gpu_host_alloc.restype = vp
    L.scp_gpu_host_free.argtypes = [vp]
    L.scp_gpu_host_free.restype = None
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
    ip = ctypes.POINTER(ctypes.c_int)
    L.scp_srv_create.argtypes = [ctypes.POINTER(SrvConfig), ctypes.POINTER(vp)]
    L.scp_srv_submit.argtypes = [vp, ctypes.POINTER(CParams), ctypes.POINTER(vp), ctypes.c_int64,
                                 ctypes.POINTER(vp), ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
    L.scp_srv_submit_borrowed.argtypes = L.scp_srv_submit.argtypes
    L.scp_srv_poll.argtypes = [vp, ip, ip]
    L.scp_srv_status.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(SrvRequestInfo)]
    L.scp_srv_result.argtypes = [vp, ctypes.c_int64, ctypes.POINTER(DiagOut)]
    L.scp_srv_stats.argtypes = [vp, ctypes.POINTER(SrvStats)]
    L.scp_srv_free.argtypes = [vp]
    L.scp_srv_free.restype = None
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
