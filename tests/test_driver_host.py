"""Host-side logic of the config-driven driver (scp_b200/host/scp_sim_b200)
that runs before any GPU call: refusals of configurations outside the
implemented set, and the three-fabric seed loader (placement by column
semantic and component, grid check).  No GPU needed."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from scp_b200 import seeds

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "scp_b200", "host", "scp_sim_b200")

pytestmark = pytest.mark.skipif(not os.path.exists(DRIVER), reason="host driver not built (make -C scp_b200/host)")


def run(tmp_path, **kv):
    base = dict(N=12, L=5.5, T=0.2, dt_factor=0.2, init="oscillon", complex_phi=1, bc_type=2,
                output=str(tmp_path / "out.sfa"), diag_file=str(tmp_path / "diag.tsv"), snap_dt=1000, diag_dt=1)
    base.update(kv)
    cfg = tmp_path / "run.cfg"
    cfg.write_text("".join(f"{k} = {v}\n" for k, v in base.items()))
    return subprocess.run([DRIVER, str(cfg)], capture_output=True, text=True, cwd=str(tmp_path), timeout=120)


@pytest.mark.parametrize("kv,msg", [
    (dict(bc_type=1), "bc_type=1 is not supported"),
    (dict(n_locks=1, complex_gauge=1, g_gauge=0.1), "locks and test_gauge_xform are not supported"),
    (dict(n_fabrics=3, complex_gauge=1, g_gauge=0.0), "n_fabrics=3 needs g_gauge != 0"),
    (dict(higgs_v=1.0, complex_gauge=1, g_gauge=0.0), "higgs_v / g_gauge2 need g_gauge != 0"),
    (dict(g_gauge2=0.2, complex_gauge=1, g_gauge=0.0), "higgs_v / g_gauge2 need g_gauge != 0"),
])
def test_driver_refuses(tmp_path, kv, msg):
    r = run(tmp_path, **kv)
    assert r.returncode == 1 and msg in r.stderr, r.stderr[-500:]


@pytest.mark.skipif(not oracle.reference_available(), reason="needs the SFA writer (make -C oracle ref)")
def test_fabric_seed_grid_must_match(tmp_path):
    small = seeds.small_state(10, False, seed=1)
    path = str(tmp_path / "L10.sfa")
    oracle.write_seed(path, small.params, small.cols())
    r = run(tmp_path, n_fabrics=3, complex_gauge=1, g_gauge=0.1, init_sfa_L=path)
    assert r.returncode == 1 and "SFA grid 10x10x10 != sim 12^3" in r.stderr, r.stderr[-500:]


@pytest.mark.skipif(not oracle.reference_available(), reason="needs the SFA writer (make -C oracle ref)")
def test_fabric_seed_loads_every_column(tmp_path):
    """A 24-column complex seed fills all 24 columns of fabric L; then the
    driver goes on to the device (which a CPU-only machine does not have)."""
    st = seeds.small_state(12, False, seed=2, L=5.5)
    path = str(tmp_path / "L12.sfa")
    oracle.write_seed(path, st.params, st.cols())
    r = run(tmp_path, n_fabrics=3, complex_gauge=1, g_gauge=0.1, init_sfa_L=path)
    assert "Loaded 24 columns into fabric" in r.stdout, r.stdout[-500:] + r.stderr[-500:]
    assert r.returncode == 0 or "no CUDA device" in r.stderr, r.stderr[-500:]
