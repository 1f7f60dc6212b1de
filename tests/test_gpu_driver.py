"""The config-driven host driver (scp_b200/host/scp_sim_b200, the reference's
main flow on top of the C ABI) against the reference binary on the same
config file and seed: same SFA schema, same frames, same diag TSV."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from scp_b200 import seeds

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "scp_b200", "host", "scp_sim_b200")


def _run(binary, cfg, cwd, extra=()):
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
    r = subprocess.run([binary, cfg, *extra], capture_output=True, text=True, cwd=cwd, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


@pytest.mark.parametrize("gauged", [False, True, "g0", "sync", "real", "real_terms", "gext", "gext_sync", "mf",
                                    "mf_free"])
def test_driver_matches_reference_binary(gpu, reference, tmp_path, gauged):
    """gauged="g0": complex_gauge=1 with g_gauge=0, the reference's ungauged
    dispatch with the link columns carried; "sync": gauged with the
    synchronous snapshot path (gpu_async_snap = 0) instead of the pipelined one;
    "real": the real 6-field mode (complex_phi = 0); "real_terms": with optional terms;
    "gext": gauged with the Higgs condensate and the second gauge (36 SFA columns),
    "gext_sync" the same through the synchronous snapshot path; "mf": three
    fabrics with Q locked to C and an L seed file; "mf_free": Q free with its
    own seed file, custom charges, a charged L and the sponge."""
    assert os.path.exists(DRIVER), "host driver not built (make -C scp_b200/host)"
    if gauged == "g0":
        st = seeds.small_state(16, True, seed=13, g_gauge=0.0)
    elif gauged == "real":
        st = seeds.real_state(16, seed=13)
    elif gauged == "real_terms":
        st = seeds.real_state(16, seed=13, mode=3, alpha_cs=0.2, kappa_h=0.1)
    elif gauged in ("gext", "gext_sync"):
        st = seeds.small_state(16, True, seed=13, higgs_v=1.0, higgs_rvoid=2.0, g_gauge2=0.2)
    elif gauged == "mf":
        st = seeds.mf_state(16, seed=13, shift=1.5)
    elif gauged == "mf_free":
        st = seeds.mf_state(15, seed=13, shift=-1.0, mf_lock_CQ=0, l_charge=0.05, q_C=0.5, q_Q=1.0, q_L=-1.5,
                            bc_type=0, damp_width=2.5, damp_rate=0.03)
    else:
        st = seeds.small_state(16, bool(gauged), seed=13)
    p = st.params
    seed = str(tmp_path / "seed.sfa")
    fabric_keys = {}
    if p.n_fabrics == 3:   # fabric C with the links, and the L / Q seed files
        cols = st.cols()
        oracle.write_seed(seed, p, cols[:30])
        fabric_keys["init_sfa_L"] = str(tmp_path / "seed_L.sfa")
        oracle.write_seed(fabric_keys["init_sfa_L"], p, cols[54:78])
        if not p.mf_lock_CQ:
            fabric_keys["init_sfa_Q"] = str(tmp_path / "seed_Q.sfa")
            oracle.write_seed(fabric_keys["init_sfa_Q"], p, cols[30:54])
    else:
        oracle.write_seed(seed, p, st.cols())
    nsteps = 40
    outs = {}
    for name, binary in (("ref", oracle.REF_BIN), ("b200", DRIVER)):
        d = tmp_path / name
        d.mkdir()
        cfg = d / "run.cfg"
        cfg.write_text(p.to_cfg(init="sfa", init_sfa=seed, init_frame=0, T=repr(nsteps * p.dt), precision="f64",
                                output=str(d / "out.sfa"), diag_file=str(d / "diag.tsv"),
                                snap_dt=repr(nsteps // 2 * p.dt), diag_dt=repr(10 * p.dt), **fabric_keys))
        extra = ("-gpu_async_snap", "0") if (name == "b200" and gauged in ("sync", "gext_sync")) else ()
        _run(binary, str(cfg), str(d), extra)
        hdr, rows = oracle.read_diag(str(d / "diag.tsv"))
        frames = [oracle.read_frame(str(d / "out.sfa"), f, p.N ** 3) for f in (0, 1, 2)]
        outs[name] = (hdr, rows, frames)
    (hr, rr, fr), (hb, rb, fb) = outs["ref"], outs["b200"]
    tol = 1e-10 if str(gauged).startswith(("gext", "mf")) else 1e-11
    assert hr == hb and rr.shape == rb.shape
    for f in range(3):
        assert fr[f][0] == fb[f][0]                                   # column names and order
        for a, b in zip(fr[f][1], fb[f][1]):
            nb = np.linalg.norm(a)
            assert np.linalg.norm(a - b) <= tol * max(nb, 1e-30) + 1e-300
    for ci, h in enumerate(hr):
        ref, got = rr[:, ci], rb[:, ci]
        scale = np.maximum(np.abs(ref), 1e-9)
        if h in ("gauss_max", "gauss_l2", "Q_flux", "Q_phi", "Q_theta", "Q_total", "Q_core", "Q_p0", "Q_p1",
                 "Q_p2", "E_coupling", "Q_C", "Q_Q", "Q_L", "Q_em"):
            # roundoff-level sums (Q_flux ~ 1e-13 in a periodic box): the floor is
            # 1e-11, well above the summation-order noise and far below O(1) values
            assert np.all(np.abs(got - ref) <= np.maximum(1e-5 * scale, 1e-11)), h
        else:
            assert np.all(np.abs(got - ref) <= 2e-6 * scale), h


def test_driver_restarts_from_its_snapshot(gpu, tmp_path):
    st = seeds.small_state(12, True, seed=3)
    p = st.params
    seed = str(tmp_path / "seed.sfa")
    oracle.write_seed(seed, p, st.cols())
    cfg = tmp_path / "run.cfg"
    cfg.write_text(p.to_cfg(init="sfa", init_sfa=seed, init_frame=0, T=repr(20 * p.dt), precision="f64",
                            output=str(tmp_path / "a.sfa"), diag_file=str(tmp_path / "a.tsv"),
                            snap_dt=repr(20 * p.dt), diag_dt=repr(10 * p.dt)))
    _run(DRIVER, str(cfg), str(tmp_path))
    r = subprocess.run([DRIVER, str(tmp_path / "a.sfa"), "-T", repr(10 * p.dt), "-output", str(tmp_path / "b.sfa"),
                        "-diag_file", str(tmp_path / "b.tsv")], capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    names, cols = oracle.read_frame(str(tmp_path / "b.sfa"), -1, p.N ** 3)
    assert len(names) == 30 and all(np.all(np.isfinite(c)) for c in cols)
