"""Regenerate the golden fixtures of tests/golden/ by running the reference
CPU stepper itself (oracle/_ref/scp_sim, built from kardianos/scp
sfa/sim/scp_sim.c by oracle/Makefile) on seeded inputs.

Run in a checkout that has the reference tree:  python tests/golden/make_golden.py
Each fixture stores the seed recipe, the reference's final FP64 frame (small
grids) or a fixed sample of its sites (64^3), and its diag TSV rows.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from scp_b200 import seeds  # noqa: E402

SAMPLE_SEED = 12345


def sample_sites(n3: int, k: int = 2048) -> np.ndarray:
    rng = np.random.default_rng(SAMPLE_SEED)
    return np.sort(rng.choice(n3, size=k, replace=False))


def small_case(name: str, N: int, gauged: bool, nsteps: int, diag_every: int, **over):
    st = seeds.small_state(N, gauged, **over)
    p = st.params
    r = oracle.run_reference(p, st.cols(), nsteps, diag_every=diag_every, threads=os.cpu_count())
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        N=N, gauged=int(gauged), nsteps=nsteps, diag_every=diag_every, L=p.L,
        bc_type=p.bc_type, damp_rate=p.damp_rate, damp_width=p.damp_width,
        final=np.stack(r["cols"]), diag=r["diag"], diag_header=np.array(r["diag_header"]),
        names=np.array(r["names"]))
    print(name, "written", r["wall_ms_per_step"], "ms/step")


def gext_case(name: str, N: int, nsteps: int, diag_every: int, **over):
    """Gauged run with the Higgs condensate and / or the second gauge: the
    36-column final frame (th2 and E2 appended) and the diag rows."""
    st = seeds.small_state(N, True, **over)
    p = st.params
    r = oracle.run_reference(p, st.cols(), nsteps, diag_every=diag_every, threads=os.cpu_count())
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        N=N, nsteps=nsteps, diag_every=diag_every, over=json.dumps(over),
        final=np.stack(r["cols"]), diag=r["diag"], diag_header=np.array(r["diag_header"]),
        names=np.array(r["names"]))
    print(name, "written", r["wall_ms_per_step"], "ms/step")


def mf_case(name: str, N: int, nsteps: int, diag_every: int, **kw):
    """Three matter fabrics (n_fabrics = 3) from seeds.mf_state: the 54-column
    final frame (C with the links, then L) and the diag rows."""
    st = seeds.mf_state(N, **kw)
    p = st.params
    r = oracle.run_reference(p, st.cols(), nsteps, diag_every=diag_every, threads=os.cpu_count())
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        N=N, nsteps=nsteps, diag_every=diag_every, kw=json.dumps(kw),
        final=np.stack(r["cols"]), diag=r["diag"], diag_header=np.array(r["diag_header"]),
        names=np.array(r["names"]))
    print(name, "written", r["wall_ms_per_step"], "ms/step")


def real_case(name: str, N: int, nsteps: int, diag_every: int, **over):
    """The real 6-field mode (complex_phi = 0), with optional terms when given:
    the 12-column final frame and the diag rows."""
    st = seeds.real_state(N, **over)
    p = st.params
    r = oracle.run_reference(p, st.cols(), nsteps, diag_every=diag_every, threads=os.cpu_count())
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        N=N, nsteps=nsteps, diag_every=diag_every, over=json.dumps(over),
        final=np.stack(r["cols"]), diag=r["diag"], diag_header=np.array(r["diag_header"]),
        names=np.array(r["names"]))
    print(name, "written", r["wall_ms_per_step"], "ms/step")


def workload_case(name: str, wl: str, nsteps: int, diag_every: int, **over):
    st = seeds.make_state(wl, seeds.params_for(wl, **over) if over else None)
    p = st.params
    r = oracle.run_reference(p, st.cols(), nsteps, diag_every=diag_every, threads=os.cpu_count())
    idx = sample_sites(p.N ** 3)
    fin = np.stack(r["cols"])
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"),
        workload=wl, over=json.dumps(over), nsteps=nsteps, diag_every=diag_every, sites=idx,
        sample=fin[:, idx], col_l2=np.linalg.norm(fin, axis=1), col_sum=fin.sum(axis=1),
        diag=r["diag"], diag_header=np.array(r["diag_header"]), names=np.array(r["names"]))
    print(name, "written", r["wall_ms_per_step"], "ms/step")


CASES = {
    "ref_c1_64_1000": lambda: workload_case("ref_c1_64_1000", "c1", 1000, 10, N=64, L=15.75),
}

if __name__ == "__main__":
    only = sys.argv[1:]
    if only:   # regenerate the named fixtures only
        for name in only:
            CASES[name]()
        sys.exit(0)
    small_case("ref_complex_n12", 12, False, 60, 10)
    small_case("ref_gauged_n12", 12, True, 60, 10)
    small_case("ref_gauged_n10_damped", 10, True, 40, 10, bc_type=0, damp_width=2.0, damp_rate=0.05)
    small_case("ref_complex_n13_damped", 13, False, 40, 10, bc_type=0, damp_width=2.0, damp_rate=0.05)
    workload_case("ref_c0_64_1000", "c0", 1000, 10)
    CASES["ref_c1_64_1000"]()
    gext_case("ref_higgs_gauge2_n12", 12, 60, 10, seed=41, higgs_v=1.0, higgs_rvoid=2.0, g_gauge2=0.2)
    gext_case("ref_higgs_gauge2_n11_damped", 11, 40, 10, seed=43, higgs_v=0.8, higgs_lam=0.5, higgs_kap=1.5,
              g_gauge2=-0.15, gauge2_q0=1.0, gauge2_q1=-1.0, gauge2_q2=0.5,
              bc_type=0, damp_width=2.0, damp_rate=0.05)
    real_case("ref_real_n12", 12, 60, 10, seed=91)
    real_case("ref_real_terms_n11_damped", 11, 40, 10, seed=92, mode=3, alpha_cs=0.2, beta_h=0.3, kappa_h=0.1,
              bc_type=0, damp_width=2.0, damp_rate=0.05)
    mf_case("ref_mf_lock_n12", 12, 40, 10, seed=81, shift=1.5)
    mf_case("ref_mf_free_n11_damped", 11, 40, 10, seed=83, shift=-1.0, l_charge=0.05, mf_lock_CQ=0,
            q_C=0.5, q_Q=1.0, q_L=-1.5, bc_type=0, damp_width=2.0, damp_rate=0.05)
