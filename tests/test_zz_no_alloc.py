"""GPU test of scp_gpu_diag_noalloc, the diagnostics entry point for callers
that cannot allocate device memory while they run (graph replay, memory owned
by another framework, allocation-free real-time loops).  It must give the
same numbers as the handle-based scp_gpu_diag, call after call, although its
reduction scratch is a fixed array inside the library.  Kept in a file of its
own that sorts last, so a failure here never hides the other tests."""
import ctypes

import numpy as np
import pytest

from scp_b200 import native, seeds
from scp_b200.api import Simulation

pytestmark = pytest.mark.gpu


def _noalloc_diag(params, dev_ptrs, g_offset):
    out = native.DiagOut()
    arr = (ctypes.c_void_p * len(dev_ptrs))(*dev_ptrs)
    cp = params.to_c()
    rc = native.lib().scp_gpu_diag_noalloc(ctypes.byref(cp), arr, g_offset, None, ctypes.byref(out))
    native.check(rc, "scp_gpu_diag_noalloc")
    return np.array(out.v[:34])


@pytest.mark.parametrize("gauged", [True, False])
def test_noalloc_diag_matches_handle_diag(gpu, gauged):
    import torch

    st = seeds.small_state(28, gauged, seed=21)
    with Simulation(st.params, st.cols()) as sim:
        sim.step(7)
        want = sim.diag_vector()
        cols = sim.snapshot()
        g_off = sim.info().G_offset
    dev = [torch.from_numpy(c).to("cuda:0") for c in cols]
    torch.cuda.synchronize()
    ptrs = [t.data_ptr() for t in dev]
    got1 = _noalloc_diag(st.params, ptrs, g_off)
    got2 = _noalloc_diag(st.params, ptrs, g_off)
    for got in (got1, got2):
        for q in range(31):
            tol = 1e-11 * max(abs(want[q]), 1e-300) if q not in (7, 13, 14, 15, 19, 24, 25, 27, 28, 29, 30) \
                else 1e-9 * max(abs(want[q]), 1.0)
            assert abs(got[q] - want[q]) <= tol, (q, got[q], want[q])
    assert np.array_equal(got1, got2)


def test_noalloc_diag_rejects_oversize_grid(gpu):
    p = seeds.small_state(8, False).params
    p.N = 4096
    arr = (ctypes.c_void_p * 24)(*([1] * 24))
    out = native.DiagOut()
    rc = native.lib().scp_gpu_diag_noalloc(ctypes.byref(p.to_c()), arr, 0.0, None, ctypes.byref(out))
    assert rc == -1
