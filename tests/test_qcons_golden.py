"""The reference's recorded Q-conservation run (v66/cfg/qcons.cfg and
v66/results/qcons_harness2.out): a radial Q-ball (omega = 1.39, the profile
written by the reference's own solver v66/radial_qball.c) at 64^3, eta = 0,
periodic, 1680 steps of dt = 0.0119.  The reference logged Q_total,
Q_phi, Q_theta, s_max, E_total and r_core at every diag step; the fixtures
(tests/golden/make_qcons.py) hold that series and the regenerated profile.

CPU: the fixtures are what the reference's tools produce here (when they are
built).  GPU: the host driver on top of the C ABI reproduces the series."""
import os
import subprocess

import numpy as np
import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
PROFILE = os.path.join(GOLD, "profile_omega1.3900.txt")
DRIVER = os.path.join(ROOT, "scp_b200", "host", "scp_sim_b200")
SOLVER = os.path.join(ROOT, "oracle", "_ref", "radial_qball")


def qcons_cfg(workdir: str, T: float) -> str:
    """The keys of the reference's v66/cfg/qcons.cfg, with this run's paths."""
    kv = dict(N=64, L=15, T=T, dt_factor=0.025, complex_phi=1, init="qball", qball_profile=PROFILE,
              qball_omega=1.39, eta=0, bc_type=2, diag_dt=0.5, snap_dt=1000,
              diag_file=os.path.join(workdir, "diag.tsv"), output=os.path.join(workdir, "out.sfa"),
              precision="f32")
    path = os.path.join(workdir, "qcons.cfg")
    with open(path, "w") as f:
        f.write("".join(f"{k} = {v}\n" for k, v in kv.items()))
    return path


def golden():
    f = np.load(os.path.join(GOLD, "ref_qcons_v66.npz"))
    return [str(c) for c in f["columns"]], f["series"]


def compare(tsv_header, tsv_rows, nrows):
    """The driver / reference TSV against the recorded series: Q to 1e-11
    (the TSV prints it with 13 digits, the series drifts by 7e-14), the others
    to the TSV's 7 printed digits."""
    cols, series = golden()
    ix = {h: i for i, h in enumerate(tsv_header)}
    assert len(tsv_rows) >= nrows
    for c, name in enumerate(cols):
        if name == "t":
            assert np.allclose(tsv_rows[:nrows, 0], series[:nrows, 0])
            continue
        got, want = tsv_rows[:nrows, ix[name]], series[:nrows, c]
        tol = 1e-11 if name.startswith("Q_") else 1e-6
        assert np.all(np.abs(got - want) <= tol * np.maximum(np.abs(want), 1e-300) + 1e-300), name


def test_qcons_fixtures():
    cols, series = golden()
    assert cols == ["t", "Q_total", "Q_phi", "Q_theta", "s_max", "E_total", "r_core"]
    assert series.shape == (41, 7) and series[-1, 0] == 20.0
    assert abs(series[0, 1] - 482.18324185573556) < 1e-12
    assert np.max(np.abs(series[:, 1] / series[0, 1] - 1)) < 1e-13   # the recorded conservation
    lines = open(PROFILE).read().splitlines()
    assert lines[0].startswith("# radial_qball profile: omega=1.390000") and len(lines) == 3 + 3001


@pytest.mark.skipif(not os.path.exists(SOLVER), reason="reference solver not built (make -C oracle ref)")
def test_profile_is_the_reference_solvers(tmp_path):
    out = tmp_path / "p.txt"
    subprocess.run([SOLVER, "-omega", "1.39", "-profile", str(out), "-scan", str(tmp_path / "s.tsv")],
                   check=True, capture_output=True, cwd=str(tmp_path))
    assert out.read_bytes() == open(PROFILE, "rb").read()


@pytest.mark.skipif(not oracle.reference_available(), reason="reference binary not built (make -C oracle ref)")
def test_reference_binary_reproduces_its_record(tmp_path):
    """The reference CPU stepper of this tree, on the regenerated profile,
    reproduces the first 2 time units of its recorded series."""
    cfg = qcons_cfg(str(tmp_path), 2.0)
    env = dict(os.environ, OMP_NUM_THREADS=str(os.cpu_count() or 1))
    subprocess.run([oracle.REF_BIN, cfg], check=True, capture_output=True, cwd=str(tmp_path), env=env)
    hdr, rows = oracle.read_diag(str(tmp_path / "diag.tsv"))
    compare(hdr, rows, 5)


@pytest.mark.gpu
def test_driver_reproduces_qcons_record(gpu, tmp_path):
    """The host driver (the reference's main flow on libscpgpu.so) runs the
    recorded configuration for all 1680 steps and matches every logged row."""
    assert os.path.exists(DRIVER), "host driver not built (make -C scp_b200/host)"
    cfg = qcons_cfg(str(tmp_path), 20.0)
    r = subprocess.run([DRIVER, cfg], capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    hdr, rows = oracle.read_diag(str(tmp_path / "diag.tsv"))
    compare(hdr, rows, 41)
