"""Continuous-batching server: every request's result is the same in the
mix as alone, admission respects slots and the HBM budget, and a small
served mix completes."""
import dataclasses

import numpy as np
import pytest

from scp_b200 import PREC_FP32C, PREC_FP64, serve
from scp_b200.api import Simulation

pytestmark = pytest.mark.gpu


def _requests(prec, seed=4):
    rng = np.random.default_rng(seed)
    out = []
    for N, steps in ((16, 37), (20, 52), (24, 29), (16, 61), (24, 45)):
        p, st, _ = serve.make_request(rng, N, prec, (10, 20))
        out.append((p, st, steps))
    return out


def _run_mix(reqs, staggered=True):
    with serve.Server(chunk_steps=8, autotune=False) as srv:
        first = reqs[:3] if staggered else reqs
        ids = [srv.submit(p, st.cols(), n, snapshot=True) for p, st, n in first]
        if staggered:
            srv.poll()                                       # the first three are running...
            ids += [srv.submit(p, st.cols(), n, snapshot=True) for p, st, n in reqs[3:]]   # ...when two more arrive
        while sum(srv.poll()):
            pass
        return [(srv.snapshot(i), srv.result(i), srv.status(i)) for i in ids]


@pytest.mark.parametrize("prec", [PREC_FP32C, PREC_FP64])
def test_mix_equals_alone(gpu, prec):
    """Each request's final state in the mix is bitwise the state it reaches
    served alone (same kernels, same per-site arithmetic), and matches the
    single-grid scp_gpu_step path within the mode's tolerance."""
    reqs = _requests(prec)
    assert any(p.complex_gauge for p, _, _ in reqs) and any(not p.complex_gauge for p, _, _ in reqs)
    mixed = _run_mix(reqs)
    tol = 1e-11 if prec == PREC_FP64 else 1e-5
    for r, (snap, diag, info) in zip(reqs, mixed):
        assert info.state == serve.DONE
        (snap1, diag1, _), = _run_mix([r], staggered=False)
        for a, b in zip(snap, snap1):
            assert np.array_equal(a, b)
        assert np.array_equal(diag[:31], diag1[:31])
        p, st, n = r
        with Simulation(dataclasses.replace(p, tile_variant=info.tile_variant), st.cols()) as sim:
            sim.step(n)
            alone = sim.snapshot()
        for a, b in zip(snap, alone):
            nb = np.linalg.norm(b)
            assert np.linalg.norm(a - b) <= tol * max(nb, 1e-30)


@pytest.mark.parametrize("prec", [PREC_FP32C, PREC_FP64])
def test_damped_and_zero_coupling_requests(gpu, prec):
    """Requests with the absorbing sponge (their own damped group) and with
    complex_gauge=1, g_gauge=0 (ungauged dynamics, links carried) in one mix:
    each matches the single-grid path within the mode's tolerance."""
    rng = np.random.default_rng(21)
    reqs = []
    for k, N in enumerate((16, 20, 24, 18)):
        p, st, _ = serve.make_request(rng, N, prec, (10, 20))
        if k % 2 == 0:
            p = dataclasses.replace(p, bc_type=0, damp_width=2.0, damp_rate=0.05)
        reqs.append((p, st, 30 + 7 * k))
    p, st, _ = serve.make_request(rng, 16, prec, (10, 20))
    while not p.complex_gauge:
        p, st, _ = serve.make_request(rng, 16, prec, (10, 20))
    reqs.append((dataclasses.replace(p, g_gauge=0.0), st, 33))
    mixed = _run_mix(reqs)
    tol = 1e-11 if prec == PREC_FP64 else 1e-5
    for (p, st, n), (snap, diag, info) in zip(reqs, mixed):
        assert info.state == serve.DONE
        assert len(snap) == p.ncols
        with Simulation(dataclasses.replace(p, tile_variant=info.tile_variant), st.cols()) as sim:
            sim.step(n)
            alone = sim.snapshot()
        for a, b in zip(snap, alone):
            nb = np.linalg.norm(b)
            assert np.linalg.norm(a - b) <= tol * max(nb, 1e-30)


def test_budget_limits_admission(gpu):
    reqs = _requests(PREC_FP32C, seed=9)
    with serve.Server(chunk_steps=10, autotune=False, mem_budget_bytes=1) as srv:   # room for one at a time
        ids = [srv.submit(p, st.cols(), n) for p, st, n in reqs]
        peak = 0
        while True:
            a, q = srv.poll()
            peak = max(peak, srv.stats().n_active, a)
            if a == 0 and q == 0:
                break
        assert peak == 1
        assert all(srv.status(i).state == serve.DONE for i in ids)


def test_slot_limit_and_autotune(gpu):
    reqs = _requests(PREC_FP32C, seed=11)
    with serve.Server(chunk_steps=16, max_active=2, autotune=True) as srv:
        ids = [srv.submit(p, st.cols(), n) for p, st, n in reqs]
        peak = 0
        while True:
            a, q = srv.poll()
            peak = max(peak, a)
            if a == 0 and q == 0:
                break
        assert peak <= 2
        infos = [srv.status(i) for i in ids]
        assert all(i.state == serve.DONE and 1 <= i.tile_variant <= 4 for i in infos)


def test_small_served_mix(gpu):
    reqs = serve.served_mix(n=24, seed=2, rate=1e9, sizes=(16, 24, 32), weights=(0.5, 0.3, 0.2), steps=(20, 80))
    with serve.Server(chunk_steps=10) as srv:
        ids, makespan, lat = serve.run_served(reqs, srv, realtime=False)
        assert all(srv.status(i).state == serve.DONE for i in ids)
        for i in ids:
            d = srv.result(i)
            assert np.isfinite(d[8])
    assert np.all(lat > 0) and makespan > 0


def test_free_with_requests_in_flight(gpu):
    """Closing the server while requests are queued, loading, running and
    retiring returns cleanly (loader and retire threads are joined, every
    handle freed) and the device stays usable."""
    reqs = _requests(PREC_FP64, seed=31) + _requests(PREC_FP32C, seed=32)
    srv = serve.Server(chunk_steps=4, autotune=False, loader_threads=2)
    for p, st, n in reqs:
        srv.submit(p, st.cols(), n)
    srv.poll()
    srv.poll()
    srv.close()
    p, st, n = reqs[0]
    with Simulation(p, st.cols()) as sim:
        sim.step(3)
        assert np.isfinite(sim.diag()["E_total"])

