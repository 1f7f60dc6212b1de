"""Python face of the C ABI: one ``Simulation`` per ``scp_gpu`` handle.

Mirrors the reference driver's use of its GPU host functions
(sfa/sim/scp_sim.cu:5175-5597): initialise from host columns, step, read
diagnostics, take snapshots, free.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import native
from .params import DIAG_NAMES, Params

DTYPE_F16, DTYPE_F32, DTYPE_F64 = 0, 1, 2
_NP_DTYPE = {DTYPE_F16: np.uint16, DTYPE_F32: np.float32, DTYPE_F64: np.float64}


class Simulation:
    """A lattice state resident on one GPU, advanced by the fused sm_100a step."""

    def __init__(self, params: Params, cols: Sequence[np.ndarray]):
        L = native.lib()
        self.params = params
        n3 = params.N ** 3
        if len(cols) != params.ncols:
            raise ValueError(f"expected {params.ncols} columns, got {len(cols)}")
        self._keep = [np.ascontiguousarray(c, dtype=np.float64).reshape(-1) for c in cols]
        for c in self._keep:
            if c.size != n3:
                raise ValueError("column size does not match N^3")
        arr = (ctypes.c_void_p * params.ncols)(*[c.ctypes.data for c in self._keep])
        self._cp = params.to_c()
        h = ctypes.c_void_p()
        native.check(L.scp_gpu_init(ctypes.byref(self._cp), arr, ctypes.byref(h)), "scp_gpu_init")
        self._h = h
        self._keep = None

    # ------------------------------------------------------------ stepping
    def step(self, nsteps: int = 1) -> None:
        native.check(native.lib().scp_gpu_step(self._h, int(nsteps)), "scp_gpu_step")

    def sync(self) -> None:
        native.check(native.lib().scp_gpu_sync(self._h), "scp_gpu_sync")

    def time_steps(self, nsteps: int) -> float:
        """Device time in ms of nsteps, CUDA events on the handle's stream."""
        ms = ctypes.c_double()
        native.check(native.lib().scp_gpu_time_steps(self._h, int(nsteps), ctypes.byref(ms)), "time_steps")
        return ms.value

    # ------------------------------------------------------------ readback
    def diag(self) -> dict:
        out = native.DiagOut()
        rc = native.lib().scp_gpu_diag(self._h, ctypes.byref(out))
        vals = {name: out.v[i] for i, name in enumerate(DIAG_NAMES)}
        native.check(rc, "scp_gpu_diag")
        return vals

    def diag_vector(self) -> np.ndarray:
        out = native.DiagOut()
        native.check(native.lib().scp_gpu_diag(self._h, ctypes.byref(out)), "scp_gpu_diag")
        return np.array(out.v[: len(DIAG_NAMES)])

    def snapshot(self, dtype: int = DTYPE_F64, out: list[np.ndarray] | None = None) -> list[np.ndarray]:
        """Current state as host columns (SFA order) in dtype; into `out`
        (ncols arrays of N^3 values of the dtype) when given."""
        p = self.params
        nc = p.snap_ncols
        if out is not None:
            if len(out) < nc or any(c.dtype != _NP_DTYPE[dtype] or c.size != p.N ** 3 or not c.flags.c_contiguous
                                         for c in out[:nc]):
                raise ValueError("snapshot: out needs ncols contiguous arrays of N^3 values of the dtype")
            cols = list(out[:nc])
        else:
            cols = [np.empty(p.N ** 3, dtype=_NP_DTYPE[dtype]) for _ in range(nc)]
        arr = (ctypes.c_void_p * nc)(*[c.ctypes.data for c in cols])
        native.check(native.lib().scp_gpu_snapshot(self._h, int(dtype), arr), "scp_gpu_snapshot")
        return cols

    def snapshot_async(self, cols: list[np.ndarray], dtype: int = DTYPE_F64) -> None:
        """Start a snapshot into caller-owned arrays (N^3 each, of the dtype's
        numpy type); they must stay alive until snapshot_wait() returns."""
        p = self.params
        nc = p.snap_ncols
        if len(cols) < nc or any(c.dtype != _NP_DTYPE[dtype] or c.size != p.N ** 3 for c in cols[:nc]):
            raise ValueError("snapshot_async: need ncols arrays of N^3 values of the dtype")
        arr = (ctypes.c_void_p * nc)(*[c.ctypes.data for c in cols[:nc]])
        native.check(native.lib().scp_gpu_snapshot_async(self._h, int(dtype), arr), "scp_gpu_snapshot_async")

    def snapshot_wait(self) -> None:
        native.check(native.lib().scp_gpu_snapshot_wait(self._h), "scp_gpu_snapshot_wait")

    def snapshot_dict(self, dtype: int = DTYPE_F64) -> dict:
        return dict(zip(self.params.snap_names, self.snapshot(dtype)))

    def info(self) -> native.Info:
        inf = native.Info()
        native.check(native.lib().scp_gpu_get_info(self._h, ctypes.byref(inf)), "scp_gpu_get_info")
        return inf

    @property
    def stream(self) -> int:
        return native.lib().scp_gpu_stream(self._h) or 0

    def close(self) -> None:
        if getattr(self, "_h", None):
            native.lib().scp_gpu_free(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pinned_empty(n: int, dtype=np.float64) -> np.ndarray:
    """A 1-D numpy array of n values in page-locked host memory
    (scp_gpu_host_alloc), released when the array is garbage collected."""
    import weakref
    L = native.lib()
    nbytes = int(n) * np.dtype(dtype).itemsize
    ptr = L.scp_gpu_host_alloc(max(nbytes, 1))
    if not ptr:
        raise MemoryError(f"scp_gpu_host_alloc({nbytes}) failed")
    base = np.frombuffer((ctypes.c_char * max(nbytes, 1)).from_address(ptr), dtype=np.uint8)
    weakref.finalize(base, L.scp_gpu_host_free, ptr)
    return base[:nbytes].view(dtype)
