"""Python face of the continuous-batching server (scp_srv_* in
include/scp_gpu.h) and the served-mix workload: many independent Q-ball
simulations of different grid sizes arriving as a Poisson process.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import time
from typing import Sequence

import numpy as np

from . import native
from .params import Params, PREC_FP32C, PREC_FP64
from .seeds import Ball, State, add_balls, add_noise, THETA_COLS

QUEUED, ACTIVE, DONE, FAILED = 0, 1, 2, 3


class Server:
    """One scp_srv instance on one device."""

    def __init__(self, device: int = 0, max_active: int = 64, mem_budget_bytes: int = 0, chunk_steps: int = 25,
                 use_graph: bool = True, autotune: bool = True, admit_per_poll: int = 0, loader_threads: int = 4):
        L = native.lib()
        cfg = native.SrvConfig(device, max_active, mem_budget_bytes, chunk_steps, 1 if use_graph else 0,
                               1 if autotune else 0, admit_per_poll, loader_threads)
        h = ctypes.c_void_p()
        native.check(L.scp_srv_create(ctypes.byref(cfg), ctypes.byref(h)), "scp_srv_create")
        self._h = h
        self._keep = {}
        self.chunk_steps = chunk_steps

    def submit(self, params: Params, cols: Sequence[np.ndarray], nsteps: int, snapshot: bool = False,
               dtype: int = 2) -> int:
        src = [np.ascontiguousarray(c, dtype=np.float64).reshape(-1) for c in cols]
        arr = (ctypes.c_void_p * len(src))(*[c.ctypes.data for c in src])
        out = None
        outs = None
        if snapshot:
            npd = {0: np.uint16, 1: np.float32, 2: np.float64}[dtype]
            outs = [np.empty(params.N ** 3, dtype=npd) for _ in src]
            out = (ctypes.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
        rid = ctypes.c_int64()
        # borrowed: the server reads these arrays at admission; they are kept here until then
        native.check(native.lib().scp_srv_submit_borrowed(self._h, ctypes.byref(params.to_c()), arr, int(nsteps),
                                                          out, int(dtype), ctypes.byref(rid)), "scp_srv_submit")
        self._keep[rid.value] = (outs, out, src, arr)
        return rid.value

    def poll(self) -> tuple[int, int]:
        a, q = ctypes.c_int(), ctypes.c_int()
        native.check(native.lib().scp_srv_poll(self._h, ctypes.byref(a), ctypes.byref(q)), "scp_srv_poll")
        return a.value, q.value

    def status(self, rid: int) -> native.SrvRequestInfo:
        inf = native.SrvRequestInfo()
        native.check(native.lib().scp_srv_status(self._h, int(rid), ctypes.byref(inf)), "scp_srv_status")
        return inf

    def result(self, rid: int) -> np.ndarray:
        d = native.DiagOut()
        native.check(native.lib().scp_srv_result(self._h, int(rid), ctypes.byref(d)), "scp_srv_result")
        return np.array(d.v[:34])

    def snapshot(self, rid: int):
        return self._keep[rid][0]

    def stats(self) -> native.SrvStats:
        st = native.SrvStats()
        native.check(native.lib().scp_srv_stats(self._h, ctypes.byref(st)), "scp_srv_stats")
        return st

    def close(self):
        if getattr(self, "_h", None):
            native.lib().scp_srv_free(self._h)
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


# ---------------------------------------------------------------- served-mix workload

@dataclasses.dataclass
class Request:
    arrival: float
    params: Params
    state: State
    nsteps: int

    @property
    def site_updates(self) -> int:
        return self.params.N ** 3 * self.nsteps


SIZES = (32, 48, 64, 96, 128)
WEIGHTS = (0.35, 0.25, 0.20, 0.12, 0.08)


def make_request(rng: np.random.Generator, N: int, precision: int, steps: tuple[int, int], sigma_max: float = 3.0):
    """One served request: dx = 0.5, 1-4 balls at random positions at least
    8 sigma apart (sigma shrinks on small boxes so one fits), omega ~
    U(0.6, 0.95), random phase triplets, e in {0, 0.05, 0.1}; theta noise
    N(0, 1e-3).  Gauged requests carry net charge and run with bc_type = 0 and
    no sponge (frozen Gauss offset); ungauged ones are periodic."""
    L = (N - 1) / 4.0
    e = float(rng.choice([0.0, 0.05, 0.1]))
    gauged = e > 0
    p = Params(N=N, L=L, dt_factor=0.2, complex_gauge=1 if gauged else 0, g_gauge=e if gauged else 0.05,
               bc_type=0 if gauged else 2, damp_rate=0.0, precision=precision)
    sigma = min(sigma_max, L / 5.0)
    want = int(rng.integers(1, 5))
    period = N * p.dx
    centres = []
    for _ in range(200):
        if len(centres) == want:
            break
        c = rng.uniform(-L, L, size=3)
        ok = True
        for o in centres:
            d = np.abs(c - o)
            d = np.minimum(d, period - d)
            if np.sqrt((d ** 2).sum()) < 8 * sigma:
                ok = False
                break
        if ok:
            centres.append(c)
    st = State(p)
    balls = [Ball(x0=float(c[0]), y0=float(c[1]), z0=float(c[2]), omega=float(rng.uniform(0.6, 0.95)),
                  sigma=sigma, phases=tuple(float(x) for x in rng.uniform(0, 2 * math.pi, 3))) for c in centres]
    add_balls(st, balls)
    add_noise(st, THETA_COLS, 1e-3, seed=int(rng.integers(0, 2 ** 31)))
    nsteps = int(rng.integers(steps[0], steps[1] + 1))
    return p, st, nsteps


def served_mix(n: int = 512, seed: int = 2, rate: float = 10.0, precision: int = PREC_FP32C,
               sizes: Sequence[int] = SIZES, weights: Sequence[float] = WEIGHTS,
               steps: tuple[int, int] = (500, 5000)) -> list[Request]:
    """The served-mix workload: n requests with Poisson arrivals at `rate`
    per second (seed 2 by default), grid sizes drawn from `sizes` with
    `weights` (small grids favoured)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    w = np.asarray(weights, dtype=float)
    w = w / w.sum()
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        N = int(rng.choice(sizes, p=w))
        p, st, ns = make_request(rng, N, precision, steps)
        out.append(Request(t, p, st, ns))
    return out


def run_served(reqs: Sequence[Request], server: Server, realtime: bool = True, snapshot: bool = False):
    """Submit each request at its arrival time (all at once when realtime is
    False) and poll until all are done.  Returns (ids, makespan_s, latencies_s)
    with latency = completion - submission."""
    t0 = time.perf_counter()
    ids = []
    while True:
        now = time.perf_counter() - t0
        while len(ids) < len(reqs) and (not realtime or reqs[len(ids)].arrival <= now):
            r = reqs[len(ids)]
            ids.append(server.submit(r.params, r.state.cols(), r.nsteps, snapshot=snapshot))
        active, queued = server.poll()
        if active == 0 and queued == 0:
            if len(ids) == len(reqs):
                break
            if realtime:
                time.sleep(max(0.0, reqs[len(ids)].arrival - (time.perf_counter() - t0)))
    makespan = time.perf_counter() - t0
    lat = []
    for i in ids:
        s = server.status(i)
        lat.append(s.t_done - s.t_submit)
    return ids, makespan, np.array(lat)


def run_sequential(reqs: Sequence[Request], precision: int = PREC_FP64):
    """The same requests one after another through scp_gpu_* handles."""
    from .api import Simulation
    t0 = time.perf_counter()
    for r in reqs:
        p = dataclasses.replace(r.params, precision=precision)
        with Simulation(p, r.state.cols()) as sim:
            sim.step(r.nsteps)
            sim.diag_vector()
    return time.perf_counter() - t0
