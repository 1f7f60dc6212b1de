"""Benchmark of the B200 lattice stepper.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c1|c0|c2|c2f|c4f|c3]

One step = one leapfrog step over the whole grid of the workload.  The
default workload is the gauged FP64 128^3 two-ball run (e = 0.1, dx = 0.5,
dt = 0.1).  Under torchrun (N > 1) every rank runs an independent replica
(the stepper does not shard); the reported value is the sum over ranks
divided by the slowest rank's time.

Roofline accounting: the algorithmic bytes of one site-update are every
persistent state word read once and written once (FP64 gauged 2 x 30 x 8 =
480 B, ungauged 384 B; FP32-compensated gauged 2 x 156 = 312 B, ungauged
240 B), as reported by scp_gpu_get_info; achieved GB/s = those bytes x sites
x steps / device time of the timed steps (CUDA events on the stepping
stream).

Workload c3 is the served mixed queue: R requests (default 512) of grid
sizes 32..128 arriving as a Poisson process, run through the
continuous-batching server in FP32-compensated mode, against the same
requests run one after another in FP64 through scp_gpu handles.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (seed workload, precision, description)
    "c1": ("c1", 0, "gauged FP64 128^3, e=0.1, two balls omega=+-0.8 20 sites apart"),
    "c0": ("c0", 0, "ungauged complex FP64 64^3, one ball omega=0.8"),
    "c2": ("c2", 0, "gauged FP64 256^3 + N(0,0.01) thermal noise"),
    "c2f": ("c2", 1, "gauged FP32-compensated 256^3 + N(0,0.01) thermal noise"),
    "c4f": ("c4", 1, "gauged FP32-compensated 512^3, eight co-phase balls"),
    "c3": (None, 1, "served mixed queue, FP32-compensated, Poisson arrivals, N in 32..128 (seed 2)"),
    "c2acc": ("c2", 1, "gauged 256^3 + N(0,0.01) thermal noise: FP32-compensated against FP64, side by side"),
    "c4acc": ("c4", 1, "gauged 512^3, eight co-phase balls: FP32-compensated against FP64 at full size, "
                       "diagnostics every 50 steps"),
    "snap": (None, 1, "host driver scp_sim_b200, gauged FP32C two-ball qball init, f32 SFA snapshots: "
                      "none / synchronous / pipelined"),
    "c1x": ("c1", 0, "gauged FP64 128^3 two balls + Higgs condensate (v=1, lambda=1, kappa_H=2, cavity r=4) "
                     "+ second U(1) gauge (g2=0.1, charges 1,1,-2): per-site FP64 kernels"),
}
WORKLOADS["c1m"] = ("c1", 0, "gauged FP64 128^3, three fabrics: C = the two balls, Q locked to C, L = C's "
                            "matter moved 8 sites along y; charges 0, 1, -1: per-site FP64 kernels")
# parameters a workload adds to its seed's
WORKLOAD_OVER = {"c1x": dict(higgs_v=1.0, higgs_rvoid=4.0, g_gauge2=0.1), "c1m": dict(n_fabrics=3)}


def workload_state(name: str, params):
    """Initial state of a bench workload: its seed's, with fabric L filled for c1m."""
    from scp_b200 import seeds
    from scp_b200.params import COLUMN_NAMES, L_COLUMN_NAMES
    st = seeds.make_state(WORKLOADS[name][0], params)
    if name == "c1m":
        for dst, src in zip(L_COLUMN_NAMES, COLUMN_NAMES[:24]):
            st[dst] = np.roll(st[src], 8, axis=1)
    return st
METRIC = "site-updates/s"


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(x: float, dist, device: str) -> float:
    """The largest x over all ranks (the slowest replica's time); x itself
    without a process group."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank: float, world: int, seconds_max: float) -> float:
    """Whole-job rate of N independent replicas: every rank did the same work,
    and the job took as long as the slowest rank."""
    return units_per_rank * world / seconds_max


def measured_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d.get("hbm_gbs"), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled_traffic(workload: str):
    """DRAM bytes per site-update of the step kernel from the committed ncu
    summary (profiles/step_kernel_<workload>.md, line 'traffic_bytes_per_site: X')."""
    p = os.path.join(ROOT, "profiles", f"step_kernel_{workload}.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_site:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def host_cpus() -> tuple[int, int]:
    """(physical cores, logical threads) of this host."""
    logical = os.cpu_count() or 1
    try:
        import psutil
        phys = psutil.cpu_count(logical=False) or logical
    except ImportError:
        phys = logical
    return phys, logical


def cpu_baseline(params, cols, nsteps: int) -> dict:
    """The reference's own OpenMP CPU stepper on this host, every hardware
    thread in use; `cores` is the thread count used, `physical_cores` the
    host's physical core count."""
    import oracle
    if not oracle.reference_available():
        return {"value": None, "unit": METRIC, "cores": 0, "kind": "reference",
                "sample": "reference binary not built"}
    phys, threads = host_cpus()
    r = oracle.run_reference(params, cols, nsteps, diag_every=nsteps, threads=threads, read_final=False)
    ms = r["wall_ms_per_step"]
    n3 = params.N ** 3
    return {"value": n3 / (ms * 1e-3), "unit": METRIC, "cores": threads, "physical_cores": phys,
            "kind": "reference",
            "sample": f"{nsteps} steps of the same workload, reference scp_sim (OpenMP, {threads} threads on "
                      f"{phys} physical cores), loop wall time {ms:.2f} ms/step"}


L2_BYTES = 126e6


def l2_label(state_bytes: float) -> str:
    """How the timed steps relate to the 126 MB L2: the state is read and
    written once per step, so a state well above L2 needs no flush."""
    mb = state_bytes / 1e6
    if state_bytes > 2 * L2_BYTES:
        return f"state {mb:.0f} MB > 2 x L2 (126 MB): every step streams from HBM, no flush needed"
    return f"state {mb:.0f} MB is within ~2x L2 (126 MB): steps are L2-aided, not an HBM roofline figure"


def reference_gpu(params, cols, lengths=(50, 1050, 2050, 3050)) -> dict:
    """The reference's own CUDA stepper (sfa/sim/scp_sim.cu, recompiled
    unmodified for sm_100a into oracle/_ref/scp_sim_cuda) on the same
    workload.  Its Wall line starts its clock before the t=0 diagnostics and
    snapshot (scp_sim.cu:5405-5457), about 10 s of host work at 128^3 that
    varies by tens of ms from run to run, so the per-step time is the
    least-squares slope of the total over runs of several lengths (3000
    steps apart at the ends, well above that jitter).  The first run of a
    process is slower by most of a second (device and module set-up), so one
    untimed run comes first."""
    import oracle
    if not os.path.exists(oracle.REF_GPU_BIN):
        return {"value": None, "unit": METRIC, "note": "reference CUDA binary not built"}
    oracle.run_reference(params, cols, lengths[0], diag_every=lengths[0], read_final=False,
                         binary=oracle.REF_GPU_BIN)
    tot = {}
    for n in lengths:
        r = oracle.run_reference(params, cols, n, diag_every=n, read_final=False, binary=oracle.REF_GPU_BIN)
        tot[n] = r["wall_ms_per_step"] * n
    xs = np.array(list(tot), dtype=float)
    ys = np.array([tot[n] for n in tot])
    ms, b = np.polyfit(xs, ys, 1)
    resid = float(np.max(np.abs(ys - (ms * xs + b))))
    return {"value": params.N ** 3 / (ms * 1e-3), "unit": METRIC, "ms_per_step": float(ms),
            "runs_ms_total": {str(k): v for k, v in tot.items()}, "fit_max_residual_ms": resid,
            "kind": "reference sfa/sim/scp_sim.cu recompiled for sm_100a, FP64, its own loop clock, "
                    "slope of the loop time over runs of " + ", ".join(str(n) for n in lengths) + " steps"}


def short_rate(workload: str, steps: int = 20, warmup: int = 5) -> dict:
    """Device-timed site-updates/s and HBM roofline fraction of one workload,
    a short run (the 256^3 target configurations of the FP64 and FP32C modes)."""
    from scp_b200 import seeds
    from scp_b200.api import Simulation
    seed, prec, desc = WORKLOADS[workload]
    params = seeds.params_for(seed, precision=prec)
    st = workload_state(workload, params)
    cols = st.cols()
    del st
    n3 = params.N ** 3
    with Simulation(params, cols) as sim:
        del cols
        sim.step(warmup)
        sim.sync()
        clk = Clocks(params.device)
        clk.start()
        ms = sim.time_steps(steps)
        sim.sync()
        clocks = clk.stop()
        info = sim.info()
    peaks = measured_peaks()
    achieved = info.step_bytes_per_site * n3 / (ms / steps * 1e-3) / 1e9
    return {"workload": desc, "N": params.N, "value": n3 * steps / (ms * 1e-3), "unit": METRIC,
            "ms_per_step": ms / steps, "steps": steps, "bytes_per_site": info.step_bytes_per_site,
            "roofline_frac": achieved / peaks["hbm_gbs"], "achieved_gbs": achieved,
            "tma_staging": int(info.tma_staging), "sites_per_thread": int(info.sites_per_thread),
            "clocks": {"sm_mhz": clocks.get("sm_mhz"), "reasons": clocks.get("reasons")}}


def run_reference_arm(args, rank, world):
    from scp_b200 import seeds
    seed, prec, desc = WORKLOADS[args.workload]
    params = seeds.params_for(seed, **WORKLOAD_OVER.get(args.workload, {}))
    cfg = {"workload": desc, "N": params.N, "steps_sample": args.warmup + args.steps,
           "parallelism": "cpu-openmp"}
    if rank != 0:
        return None
    st = workload_state(args.workload, params)
    cb = cpu_baseline(params, st.cols(), args.warmup + args.steps)
    val = cb["value"]
    line = {"metric": METRIC, "value": val, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": (params.N ** 3 / val * 1e3) if val else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg, "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    return line


def step_bytes(params) -> float:
    """Algorithmic bytes per site-update of the layout params select (the
    figure scp_gpu_get_info reports)."""
    nf = 15 if params.complex_gauge else 12
    if params.precision == 0:
        return 2.0 * 8.0 * nf
    return 2.0 * (4.0 * nf + 24.0 + (12.0 if params.complex_gauge else 0.0) + 4.0 * nf)


def request_lines(reqs, ids, srv) -> list[dict]:
    """One record per served request: grid, steps, sites, and its times on the
    server's clock (submission, admission, completion)."""
    out = []
    for r, i in zip(reqs, ids):
        s = srv.status(i)
        out.append({"id": int(i), "N": r.params.N, "steps": r.nsteps, "sites": r.params.N ** 3,
                    "site_updates": r.site_updates, "gauged": int(r.params.complex_gauge),
                    "e": r.params.g_gauge if r.params.complex_gauge else 0.0,
                    "latency_s": s.t_done - s.t_submit, "queue_s": s.t_admit - s.t_submit,
                    "service_s": s.t_done - s.t_admit, "state": int(s.state)})
    return out


def served_once(reqs, args, rate_label: float, log_path: str | None):
    from scp_b200 import serve
    with serve.Server(device=0, max_active=args.max_active, chunk_steps=25) as srv:
        clk = Clocks(0)
        clk.start()
        ids, makespan, lat = serve.run_served(reqs, srv, realtime=True)
        clocks = clk.stop()
        st = srv.stats()
        bad = [(i, r) for i, r in zip(ids, reqs) if srv.status(i).state != serve.DONE]
        bad_info = [f"id {i}: state {srv.status(i).state} rc {srv.status(i).rc} N {r.params.N} "
                    f"e {r.params.g_gauge if r.params.complex_gauge else 0.0} steps {r.nsteps}" for i, r in bad]
        recs = request_lines(reqs, ids, srv)
    if bad:
        raise RuntimeError(f"{len(bad)} served requests failed: " + "; ".join(bad_info[:8]))
    if log_path:
        with open(log_path, "a") as f:
            for rec in recs:
                f.write(json.dumps({"rate_per_s": rate_label, **rec}) + "\n")
    return ids, makespan, lat, clocks, st, recs


def run_served_mix(args) -> dict:
    """Served mixed queue (c3): aggregate site-updates/s of the server over
    the whole makespan (submission of the first request to completion of the
    last), per-request latency percentiles, and the same requests one after
    another through scp_gpu handles in FP64 and in FP32C (so the batching gain
    and the precision gain are reported apart).  A second served run at
    --load (default 0.75) of the capacity the first run measured gives the
    latency below saturation."""
    from scp_b200 import serve, PREC_FP32C
    reqs = serve.served_mix(n=args.requests, seed=2, rate=args.rate)
    total = sum(r.site_updates for r in reqs)
    algo = sum(step_bytes(r.params) * r.site_updates for r in reqs)
    log_path = args.request_log or None
    if log_path and os.path.exists(log_path):
        os.remove(log_path)
    ids, makespan, lat, clocks, st, recs = served_once(reqs, args, args.rate, log_path)
    value = total / makespan
    # service capacity in requests per second of device time
    capacity = len(reqs) / max(st.t_gpu, 1e-9)
    below = None
    if args.load > 0:
        rate2 = args.load * capacity
        reqs2 = serve.served_mix(n=args.requests, seed=2, rate=rate2)
        _, makespan2, lat2, _, _, _ = served_once(reqs2, args, rate2, log_path)
        below = {"rate_per_s": rate2, "load": args.load, "makespan_s": makespan2,
                 "latency_s": {"p50": float(np.percentile(lat2, 50)), "p99": float(np.percentile(lat2, 99)),
                               "max": float(lat2.max())},
                 "value": sum(r.site_updates for r in reqs2) / makespan2}
    seq = {}
    if not args.no_sequential:
        nseq = len(reqs) if args.seq_sample <= 0 else min(args.seq_sample, len(reqs))
        sub = reqs[:nseq]
        for name, prec in (("fp64", 0), ("fp32c", PREC_FP32C)):
            t = serve.run_sequential(sub, precision=prec)
            seq[name] = {"value": sum(r.site_updates for r in sub) / t, "unit": METRIC, "requests": nseq,
                         "precision": name, "wall_s": t}
    peaks = measured_peaks()
    achieved = algo / makespan / 1e9
    sizes = {}
    for r in reqs:
        sizes[r.params.N] = sizes.get(r.params.N, 0) + 1
    return {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": 1, "steps": len(reqs), "warmup": 0,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32c", "data": "synthetic",
        "config": {"workload": WORKLOADS["c3"][2], "requests": len(reqs), "rate_per_s": args.rate,
                   "sizes": sizes, "site_updates": total, "max_active": args.max_active, "chunk_steps": 25,
                   "parallelism": "single-gpu", "l2": "mixed sizes; makespan-level timing"},
        "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                      "max": float(lat.max())},
        "latency_below_capacity": below,
        "capacity_requests_per_s": capacity,
        "makespan_s": makespan,
        "sequential": seq or None,
        "served_over_sequential_fp64": (value / seq["fp64"]["value"]) if seq else None,
        "served_over_sequential_fp32c": (value / seq["fp32c"]["value"]) if seq else None,
        "server_phases_s": {"load": st.t_admit, "autotune": st.t_autotune, "run_wait": st.t_run,
                            "retire": st.t_retire, "idle_wait": st.t_wait, "launch": st.t_launch,
                            "gpu_chunks": st.t_gpu, "chunks": st.chunks},
        "request_log": log_path,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"], "traffic": None,
                     "note": "algorithmic bytes of all requests / makespan (host phases included)"},
        "gpu_launches": int(st.chunks) * 25,
        "clocks": clocks,
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "h2d_bytes_total": int(sum(sum(c.nbytes for c in r.state.cols()) for r in reqs)),
                "includes": "submission from host columns, load, steps, final diagnostics"},
    }


def _half_centroids(cols, params) -> np.ndarray:
    """rho^2-weighted centroids of the x < 0 and x >= 0 halves of the box
    (the two opposite-charge balls of the c1/c2 seeds), rho the Noether
    charge density u*dv - v*du + tu*dtv - tv*dtu summed over components."""
    from scp_b200 import COLUMN_NAMES
    N = params.N
    c = {k: np.asarray(v).reshape(-1) for k, v in zip(COLUMN_NAMES, cols)}
    rho = np.zeros(N ** 3)
    for a in "xyz":
        rho += c[f"phi_{a}"] * c[f"phiim_v{a}"] - c[f"phiim_{a}"] * c[f"phi_v{a}"]
        rho += c[f"theta_{a}"] * c[f"thetaim_v{a}"] - c[f"thetaim_{a}"] * c[f"theta_v{a}"]
    w = (rho * rho).reshape(N, N, N)
    x = -params.L + np.arange(N) * params.dx
    out = []
    for half in (slice(0, N // 2), slice(N // 2, N)):
        wh = w[half]
        tot = wh.sum()
        xi = x[half]
        out.append([float((wh.sum(axis=(1, 2)) * xi).sum() / tot), float((wh.sum(axis=(0, 2)) * x).sum() / tot),
                    float((wh.sum(axis=(0, 1)) * x).sum() / tot)])
    return np.array(out)


def run_precision_compare(args, name: str = "c2acc") -> dict:
    """c2acc: the c2 seed (gauged, thermal background, 256^3) stepped in FP64
    and in FP32-compensated mode side by side; per-observable error of the
    FP32C run against the FP64 run: energy drift, Noether charge, Gauss
    residual, per-field relative L2 and the two half-box charge centroids.
    c4acc: the same comparison for the c4 seed (eight co-phase balls, 512^3,
    FP64 at full size as the reference run) on the diagnostics alone (a
    512^3 snapshot is 32 GB of host memory per run)."""
    import dataclasses
    from scp_b200 import seeds, PREC_FP32C
    from scp_b200.api import Simulation
    seed = "c2" if name == "c2acc" else "c4"
    snapshots = name == "c2acc"
    over = dict(N=args.n, L=(args.n - 1) / 4.0) if args.n else {}
    p64 = seeds.params_for(seed, **over)
    p32 = dataclasses.replace(p64, precision=PREC_FP32C)
    st = seeds.make_state(seed, p64)
    cols = st.cols()
    del st
    total = args.steps
    every, snap_every = 50, max(50, total // 4)
    series = {"fp64": [], "fp32c": []}
    cent = {"fp64": [], "fp32c": []}
    field_l2 = []
    walls = {"fp64": 0.0, "fp32c": 0.0}
    with Simulation(p64, cols) as a, Simulation(p32, cols) as b:
        del cols
        sims = {"fp64": a, "fp32c": b}
        for k, sim in sims.items():
            series[k].append(sim.diag_vector())
        done = 0
        while done < total:
            n = min(every, total - done)
            for k, sim in sims.items():
                t0 = time.perf_counter()
                sim.step(n)
                sim.sync()
                walls[k] += time.perf_counter() - t0
                series[k].append(sim.diag_vector())
            done += n
            if snapshots and (done % snap_every == 0 or done == total):
                snaps = {k: sim.snapshot() for k, sim in sims.items()}
                for k in sims:
                    cent[k].append(_half_centroids(snaps[k], p64))
                l2 = []
                for ca, cb in zip(snaps["fp64"], snaps["fp32c"]):
                    na = np.linalg.norm(ca)
                    if na > 1e-3 * np.sqrt(len(ca)):
                        l2.append(float(np.linalg.norm(cb - ca) / na))
                field_l2.append((done, max(l2)))
                del snaps
    from scp_b200 import DIAG_NAMES
    ix = {n: i for i, n in enumerate(DIAG_NAMES)}
    A, B = np.array(series["fp64"]), np.array(series["fp32c"])
    e0a = A[0, ix["E_total"]]
    drift_a = (A[:, ix["E_total"]] - e0a) / abs(e0a)
    drift_b = (B[:, ix["E_total"]] - B[0, ix["E_total"]]) / abs(B[0, ix["E_total"]])
    q = ix["Q_total"]
    if snapshots:
        ca, cb = np.array(cent["fp64"]), np.array(cent["fp32c"])
        csteps = [s for s, _ in field_l2]
    else:   # the rho^2-weighted centroid of the diagnostics, every diag step
        cols3 = [ix["centroid_x"], ix["centroid_y"], ix["centroid_z"]]
        ca, cb = A[:, cols3], B[:, cols3]
        csteps = list(range(0, total + 1, every))
    n3 = p64.N ** 3
    return {
        "metric": "FP32-compensated error vs FP64", "workload": WORKLOADS[name][2], "N": p64.N, "steps": total,
        "diag_every": every, "data": "synthetic",
        "energy": {"rel_drift_fp64_end": float(drift_a[-1]), "rel_drift_fp32c_end": float(drift_b[-1]),
                   "max_abs_drift_difference": float(np.max(np.abs(drift_b - drift_a))),
                   "rel_E_total_difference_end": float(abs(B[-1, ix["E_total"]] - A[-1, ix["E_total"]]) / abs(e0a))},
        "energy_terms_rel_difference_end": {
            n: float(abs(B[-1, ix[n]] - A[-1, ix[n]]) / abs(e0a))
            for n in ("E_phi_kin", "E_theta_kin", "E_grad", "E_mass", "E_pot", "E_tgrad", "E_tmass", "E_coupling",
                      "E_em")},
        "energy_difference_series": [float(x) for x in (B[::8, ix["E_total"]] - A[::8, ix["E_total"]]) / abs(e0a)],
        "charge": {"Q_total_fp64_end": float(A[-1, q]), "Q_total_fp32c_end": float(B[-1, q]),
                   "sum_abs_Q_phi_fp64_end": float(abs(A[-1, ix["Q_phi"]])),
                   "max_abs_difference": float(np.max(np.abs(B[:, q] - A[:, q])))},
        "gauss": {"gauss_max_fp64_max": float(A[:, ix["gauss_max"]].max()),
                  "gauss_max_fp32c_max": float(B[:, ix["gauss_max"]].max())},
        "field_rel_l2_max_over_columns": field_l2,
        "centroids": {"steps": csteps[:: max(1, len(csteps) // 8)],
                      "fp64": ca[:: max(1, len(csteps) // 8)].tolist(),
                      "max_abs_difference": float(np.max(np.abs(cb - ca)))},
        "other_diagnostics_max_rel_difference": {
            n: float(np.max(np.abs(B[:, ix[n]] - A[:, ix[n]])) / max(np.max(np.abs(A[:, ix[n]])), 1e-300))
            for n in ("phi_max", "P_max", "s_max", "r_core", "Q_core", "E_em")},
        "throughput_incl_diag": {k: n3 * total / walls[k] for k in walls},
    }


def run_snapshot_pipeline(args) -> dict:
    """snap: the config-driven host driver (scp_b200/host/scp_sim_b200) on a
    gauged FP32C run initialised by the reference's own qball init (two
    opposite balls from a Gaussian radial profile), writing f32 SFA frames
    every --snap-every steps: wall ms/step without snapshots, with the
    synchronous snapshot path and with the pipelined one (device
    down-conversion, copy stream, writer thread)."""
    import tempfile
    driver = os.path.join(ROOT, "scp_b200", "host", "scp_sim_b200")
    if not os.path.exists(driver):
        raise SystemExit("scp_b200/host/scp_sim_b200 is not built")
    N = args.n or 128
    L = (N - 1) / 4.0
    dx = 2 * L / (N - 1)
    dt = 0.2 * dx
    steps, every = args.steps, args.snap_every
    out = {}
    with tempfile.TemporaryDirectory() as d:
        prof = os.path.join(d, "profile.txt")
        with open(prof, "w") as f:
            for r in np.arange(0.0, 4 * L, 0.05):
                f.write(f"{r:.4f} {np.exp(-r * r / 18.0):.12e}\n")
        base = {"N": N, "L": L, "dt_factor": 0.2, "complex_phi": 1, "complex_gauge": 1, "g_gauge": 0.1,
                "bc_type": 2, "init": "qball", "qball_profile": prof, "qball_omega": 1.45, "qball_x0": -L / 3,
                "qball_y0": 0.0, "qball_z0": 0.0, "qball2_x0": L / 3, "qball2_y0": 0.0, "qball2_z0": 0.0,
                "qball2_sign": -1, "precision": "f32", "T": steps * dt, "diag_dt": every * dt}
        for name, snap_dt, asyn in (("no_snapshots", 10 * steps * dt, 1), ("synchronous", every * dt, 0),
                                    ("pipelined", every * dt, 1)):
            cfg = os.path.join(d, f"{name}.cfg")
            kv = dict(base, snap_dt=snap_dt, output=os.path.join(d, f"{name}.sfa"),
                      diag_file=os.path.join(d, f"{name}.tsv"))
            with open(cfg, "w") as f:
                f.write("".join(f"{k} = {v}\n" for k, v in kv.items()))
            t0 = time.perf_counter()
            r = subprocess.run([driver, cfg, "-gpu_precision", "fp32c", "-gpu_async_snap", str(asyn)],
                               capture_output=True, text=True, cwd=d)
            wall = time.perf_counter() - t0
            if r.returncode != 0:
                raise RuntimeError(f"driver failed ({name}): {r.stderr[-800:]}")
            m = re.search(r"Wall: ([0-9.]+)s .* ([0-9.]+)ms/step", r.stdout)
            m2 = re.search(r"SFA: .* \((\d+) frames\)", r.stdout)
            out[name] = {"loop_ms_per_step": float(m.group(2)), "loop_s": float(m.group(1)),
                         "process_s": wall, "frames": int(m2.group(1)) if m2 else None,
                         "sfa_bytes": os.path.getsize(kv["output"])}
    frame_bytes = 30 * N ** 3 * 4
    nframes = steps // every
    extra = {k: (out[k]["loop_s"] - out["no_snapshots"]["loop_s"]) / max(nframes, 1)
             for k in ("synchronous", "pipelined")}
    return {"metric": "driver loop ms/step with f32 snapshots", "workload": WORKLOADS["snap"][2], "N": N,
            "steps": steps, "snapshot_every": every, "frame_bytes": frame_bytes, "runs": out,
            "snapshot_cost_s_per_frame": extra, "data": "synthetic"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c1", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--n", type=int, default=0, help="override the grid edge (profiling a smaller case)")
    ap.add_argument("--tile", type=int, default=0, help="tile_variant (0 = library default)")
    ap.add_argument("--requests", type=int, default=512, help="c3: number of requests")
    ap.add_argument("--rate", type=float, default=50.0, help="c3: Poisson arrival rate per second")
    ap.add_argument("--max-active", type=int, default=128, help="c3: server slots")
    ap.add_argument("--no-sequential", action="store_true", help="c3: skip the one-after-another FP64 run")
    ap.add_argument("--seq-sample", type=int, default=0, help="c3: run only the first R requests sequentially")
    ap.add_argument("--load", type=float, default=0.75,
                    help="c3: second served run at this fraction of the measured capacity (0: skip)")
    ap.add_argument("--request-log", default="", help="c3: write one JSON line per served request to this file")
    ap.add_argument("--snap-every", type=int, default=100, help="snap: steps between SFA frames")
    ap.add_argument("--ref-gpu", action="store_true",
                    help="also time the reference's own CUDA stepper on the same FP64 workload (always on for c1)")
    ap.add_argument("--no-targets", action="store_true",
                    help="c1: skip the short 256^3 FP64 / FP32C runs of the performance targets")
    ap.add_argument("--no-ref-gpu", action="store_true", help="c1: skip the reference CUDA stepper")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = env_rank()
    if args.impl == "reference":
        # the reference's stepper runs on the host cores: rank 0 alone times it,
        # the other ranks leave at once (no process group, no GPU needed)
        if args.workload in ("c3", "c2acc", "c4acc", "snap"):
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "this workload exercises the library's "
                                  "server or its two precisions, which the reference does not have; its CPU "
                                  "stepper is timed on the single-run workloads"}))
            return
        line = run_reference_arm(args, rank, world)
        if rank == 0 and line:
            print(json.dumps(line))
        return

    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist_mod
        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
        dist = dist_mod

    if args.workload == "c3":
        if world > 1:
            raise SystemExit("c3 runs on one GPU")
        print(json.dumps(run_served_mix(args)))
        return
    if args.workload == "snap":
        print(json.dumps(run_snapshot_pipeline(args)))
        return
    if args.workload in ("c2acc", "c4acc"):
        if world > 1:
            raise SystemExit(f"{args.workload} runs on one GPU")
        print(json.dumps(run_precision_compare(args, args.workload)))
        return

    from scp_b200 import seeds
    from scp_b200.api import Simulation
    seed, prec, desc = WORKLOADS[args.workload]
    over = dict(N=args.n, L=(args.n - 1) / 4.0) if args.n else {}
    params = seeds.params_for(seed, precision=prec, device=local, tile_variant=args.tile, **over,
                              **WORKLOAD_OVER.get(args.workload, {}))
    # kernels per step: one fused launch (the Higgs / second-gauge stepper
    # too); with three fabrics one per moving fabric plus the link update
    fab = params.complex_gauge and params.n_fabrics == 3
    launches_per_step = ((3 if params.mf_lock_CQ else 4) if fab else 1)
    st = workload_state(args.workload, params)
    cols = st.cols()
    n3 = params.N ** 3

    def barrier():
        if dist:
            import torch
            torch.cuda.synchronize()
            dist.barrier()

    sim = Simulation(params, cols)
    sim.step(args.warmup)
    sim.sync()
    barrier()
    clk = Clocks(local)
    clk.start()
    ms = sim.time_steps(args.steps)
    sim.sync()
    clocks = clk.stop()
    barrier()
    info = sim.info()
    ms_max = max_over_ranks(ms, dist, f"cuda:{local}")
    ms_step = ms_max / args.steps
    # diagnostics as the reference's loop uses them: 10 steps, then one
    # diagnostics call (reductions, point values, copy to the host), timed on
    # the host; what the cycle takes beyond 10 device-timed steps is the cost
    # of a diagnostic (the synchronous launch's own sums included).  A repeat
    # call on an unchanged state times the call alone.
    for _ in range(3):
        sim.step(10)
        sim.diag_vector()
    t0 = time.perf_counter()
    for _ in range(10):
        sim.step(10)
        sim.diag_vector()
    cycle_ms = (time.perf_counter() - t0) / 10 * 1e3
    t0 = time.perf_counter()
    for _ in range(10):
        sim.diag_vector()
    diag_ms = (time.perf_counter() - t0) / 10 * 1e3
    value = replica_throughput(n3 * args.steps, world, ms_max * 1e-3)
    bytes_site = info.step_bytes_per_site
    achieved = bytes_site * n3 / (ms / args.steps * 1e-3) / 1e9
    peaks = measured_peaks()
    sim.close()

    e2e = None
    if not args.no_e2e:
        # end to end through the C ABI: host columns in (H2D inside init),
        # Gauss projection and first force, K steps with diagnostics every
        # 10 steps (D2H), final FP64 snapshot back to host
        # inputs and the result live in page-locked host memory
        from scp_b200.api import pinned_empty
        pin_in = [pinned_empty(n3) for _ in cols]
        for dst, src in zip(pin_in, cols):
            dst[:] = np.asarray(src).reshape(-1)
        snap = [pinned_empty(n3) for _ in range(params.snap_ncols)]   # + th2, E2 with the second gauge
        barrier()
        nd = 0
        t0 = time.perf_counter()
        sim2 = Simulation(params, pin_in)
        t_init = time.perf_counter()
        done = 0
        while done < args.steps:
            k = min(10, args.steps - done)
            sim2.step(k)
            done += k
            sim2.diag_vector()
            nd += 1
        t_steps = time.perf_counter()
        sim2.snapshot(out=snap)
        t1 = time.perf_counter()
        cg_iters = sim2.info().cg_iterations
        sim2.close()
        wall = max_over_ranks(t1 - t0, dist, f"cuda:{local}")
        h2d = sum(c.nbytes for c in cols)
        d2h = sum(c.nbytes for c in snap) + nd * 8 * 53
        e2e = {"value": replica_throughput(n3 * args.steps, world, wall), "unit": METRIC,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "wall_s": wall, "includes": "init upload from page-locked host columns, Gauss projection, "
                                           "steps, diag every 10 steps, final f64 snapshot into page-locked "
                                           "host columns",
               "split_s": {"init": t_init - t0, "steps_and_diag": t_steps - t_init, "snapshot": t1 - t_steps},
               "cg_iterations": cg_iters}

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if prec == 0 else "f32c",
        "data": "synthetic",
        "config": {"workload": desc, "N": params.N, "precision": "fp64" if prec == 0 else "fp32-compensated",
                   "parallelism": f"replicas x{world}" if world > 1 else "single-gpu",
                   "l2": l2_label(info.state_bytes_per_site * n3),
                   "tile": [info.tile_x, info.tile_y, info.seg_len]},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                     "bytes_per_site": bytes_site,
                     "traffic": (lambda t: t * n3 if t else None)(profiled_traffic(args.workload))},
        "gpu_launches": args.steps * launches_per_step,
        "diag": {"ms_per_call": diag_ms, "cycle_10_steps_ms": cycle_ms,
                 "step_equivalents": (cycle_ms - 10 * ms_step) / ms_step,
                 "includes": "energies, charges, Gauss residual, point values, copy to the host"},
        "clocks": clocks,
        "e2e": e2e,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(params, cols, 10 if params.N <= 128 else 3)
    default_c1 = args.workload == "c1" and not args.n
    if rank == 0 and world == 1 and prec == 0 and (args.ref_gpu or (default_c1 and not args.no_ref_gpu)):
        rg = reference_gpu(params, cols)
        if rg.get("value"):
            rg["ours_over_reference_gpu"] = value / rg["value"]
        line["reference_gpu"] = rg
    if rank == 0 and world == 1 and default_c1 and not args.no_targets:
        # the performance targets: FP64 >= 70% of HBM at 256^3, FP32C >= 1.8x FP64
        t64 = short_rate("c2")
        t32 = short_rate("c2f")
        line["targets"] = {"fp64_256": t64, "fp32c_256": t32,
                           "fp32c_over_fp64": t32["value"] / t64["value"],
                           "goals": {"fp64_roofline_frac": 0.70, "fp32c_over_fp64": 1.8}}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
