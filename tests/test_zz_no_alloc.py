"""GPU tests of scp_gpu_diag_noalloc, the diagnostics entry point for callers
that cannot allocate device memory while they run: a process whose device
memory belongs to another framework's allocator, or a real-time loop for
which an allocation (and the device synchronisation it implies) is a failure.
It must give the same numbers as the handle-based scp_gpu_diag, call after
call, although its reduction scratch is a fixed array inside the library.
Kept in a file of its own that sorts last, so a failure here never hides the
other tests."""
import ctypes

import numpy as np
import pytest

from scp_b200 import native, seeds
from scp_b200.api import Simulation

pytestmark = pytest.mark.gpu

# slots compared with an absolute floor: sums that cancel to near zero
_CANCELLING = (7, 13, 14, 15, 19, 24, 25, 27, 28, 29, 30)


def _call(params, dev_ptrs, g_offset, stream=None):
    out = native.DiagOut()
    arr = (ctypes.c_void_p * len(dev_ptrs))(*dev_ptrs)
    cp = params.to_c()
    rc = native.lib().scp_gpu_diag_noalloc(ctypes.byref(cp), arr, g_offset, stream, ctypes.byref(out))
    return rc, np.array(out.v[:34])


def _noalloc_diag(params, dev_ptrs, g_offset):
    rc, v = _call(params, dev_ptrs, g_offset)
    native.check(rc, "scp_gpu_diag_noalloc")
    return v


CASES = {
    "gauged_periodic": dict(gauged=True),
    "ungauged_periodic": dict(gauged=False),
    # sponge boundary: the interior-radius (Rint) branch of the Gauss sums
    "gauged_sponge": dict(gauged=True, bc_type=0, damp_width=3.0, damp_rate=0.01),
    # links present but g = 0: the ungauged dynamics with th / E carried
    "links_g0": dict(gauged=True, g_gauge=0.0),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_noalloc_diag_matches_handle_diag(gpu, case):
    import torch

    kw = dict(CASES[case])
    gauged = kw.pop("gauged")
    st = seeds.small_state(28, gauged, seed=21, **kw)
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
            tol = 1e-9 * max(abs(want[q]), 1.0) if q in _CANCELLING else 1e-11 * max(abs(want[q]), 1e-300)
            assert abs(got[q] - want[q]) <= tol, (case, q, got[q], want[q])
    assert np.array_equal(got1, got2)


def test_noalloc_diag_rejects_oversize_grid(gpu):
    """A grid beyond the static scratch's limit is refused by the entry
    point's own check, whose message names the limit; no pointer is read."""
    p = seeds.small_state(8, False).params
    p.N = 4096
    rc, _ = _call(p, [None] * 24, 0.0)
    assert rc == native.SCP_EINVAL
    assert "SCP_DIAG_STATIC_MAX_N" in native.lib().scp_gpu_last_cuda_error().decode()


def test_noalloc_diag_refuses_capturing_stream(gpu):
    """On a stream that is capturing a graph the call returns
    SCP_EUNSUPPORTED before it enqueues anything, and the capture stays
    valid."""
    import torch

    st = seeds.small_state(12, True, seed=3)
    with Simulation(st.params, st.cols()) as sim:
        cols = sim.snapshot()
        g_off = sim.info().G_offset
    dev = [torch.from_numpy(c).to("cuda:0") for c in cols]
    ptrs = [t.data_ptr() for t in dev]
    x = torch.zeros(16, device="cuda:0")
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        x.add_(1.0)
        rc, _ = _call(st.params, ptrs, g_off, stream=ctypes.c_void_p(s.cuda_stream))
        x.add_(1.0)
    assert rc == native.SCP_EUNSUPPORTED
    g.replay()
    torch.cuda.synchronize()
    assert float(x[0]) == 2.0
    # and the same columns outside capture still give a result
    v = _noalloc_diag(st.params, ptrs, g_off)
    assert np.isfinite(v[8])
