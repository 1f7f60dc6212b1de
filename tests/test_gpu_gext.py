"""The gauged stepper's extensions -- Higgs condensate and second compact U(1)
gauge (compute_forces_complex_gauge pass C, sfa/sim/scp_sim.c:1112-1262;
verlet_step :1583-1716; init_gauss2_project :2414-2458) -- through the C ABI,
against the reference CPU stepper's own output."""
import ctypes
import json
import os

import numpy as np
import pytest

import oracle
from scp_b200 import PREC_FP32C, Params, native, seeds
from scp_b200.api import DTYPE_F32, DTYPE_F64, Simulation
from scp_b200.params import COLUMN_NAMES

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL_FRAME = 1e-10      # relative L2 per column


def rel_l2(a, b):
    a, b = np.asarray(a).reshape(-1), np.asarray(b).reshape(-1)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


def check_diag(have_rows, want_rows, header):
    """have: diag vectors (slot order); want: the reference TSV rows (t first).
    The TSV prints %.6e; roundoff-level sums get an absolute floor."""
    want = np.asarray(want_rows)[:, 1:]
    have = np.array(have_rows)[:, :want.shape[1]]
    for ci, h in enumerate(header[1:]):
        ref, got = want[:, ci], have[:, ci]
        scale = np.maximum(np.abs(ref), 1e-9)
        if h in ("gauss_max", "gauss_l2", "Q_flux", "Q_phi", "Q_theta", "Q_total", "Q_core", "Q_p0", "Q_p1",
                 "Q_p2", "E_coupling"):
            assert np.all(np.abs(got - ref) <= np.maximum(1e-5 * scale, 1e-11)), h
        else:
            assert np.all(np.abs(got - ref) <= 2e-6 * scale), h


def run_rows(p, cols, nsteps, every):
    rows = []
    with Simulation(p, cols) as sim:
        rows.append(sim.diag_vector())
        for _ in range(nsteps // every):
            sim.step(every)
            rows.append(sim.diag_vector())
        got = sim.snapshot()
    return rows, got


@pytest.mark.parametrize("name", ["ref_higgs_gauge2_n12", "ref_higgs_gauge2_n11_damped"])
def test_gext_matches_golden(gpu, name):
    f = np.load(os.path.join(GOLD, name + ".npz"))
    over = json.loads(str(f["over"]))
    st = seeds.small_state(int(f["N"]), True, **over)
    p = st.params
    rows, got = run_rows(p, st.cols(), int(f["nsteps"]), int(f["diag_every"]))
    assert len(got) == 36 and list(f["names"]) == list(COLUMN_NAMES)
    for c in range(36):
        assert rel_l2(got[c], f["final"][c]) < TOL_FRAME, COLUMN_NAMES[c]
    check_diag(rows, f["diag"], [str(h) for h in f["diag_header"]])


GEXT = [dict(higgs_v=1.0),
        dict(higgs_v=1.2, higgs_rvoid=2.5, higgs_lam=0.7, higgs_kap=3.0),
        dict(g_gauge2=0.2),
        dict(g_gauge2=0.3, gauge2_q0=2.0, gauge2_q1=-1.0, gauge2_q2=-1.0, eta=0.0),
        dict(higgs_v=1.0, higgs_rvoid=2.0, g_gauge2=0.2, bc_type=0, damp_width=2.5, damp_rate=0.03)]


@pytest.mark.parametrize("over", GEXT, ids=lambda t: "-".join(f"{k}{v}" for k, v in t.items()))
@pytest.mark.parametrize("N", [16, 17])
def test_gext_matches_reference_binary(gpu, reference, N, over):
    """Each extension alone and together, even and odd N, periodic and with
    the sponge, against the reference CPU binary on the same seed."""
    st = seeds.small_state(N, True, seed=50 + N, **over)
    p = st.params
    ref = oracle.run_reference(p, st.cols(), 40, diag_every=10)
    rows, got = run_rows(p, st.cols(), 40, 10)
    assert len(got) == len(ref["cols"]) == p.snap_ncols
    for c in range(len(got)):
        assert rel_l2(got[c], ref["cols"][c]) < TOL_FRAME, COLUMN_NAMES[c]
    check_diag(rows, ref["diag"], ref["diag_header"])


def gauss2_residual(p, cols):
    """div E2 - g2 sum_a q_a rho_a per site (gauss2_residual_at, scp_sim.c:2402-2412)."""
    N = p.N
    c = {n: np.asarray(a).reshape(N, N, N) for n, a in zip(COLUMN_NAMES, cols)}
    div = sum(c[f"E2_{ax}"] - np.roll(c[f"E2_{ax}"], 1, axis=d) for d, ax in enumerate("xyz")) / p.dx
    q = (p.gauge2_q0, p.gauge2_q1, p.gauge2_q2)
    rho = 0.0
    for a, ax in enumerate("xyz"):
        rho = rho + q[a] * (c[f"phi_{ax}"] * c[f"phiim_v{ax}"] - c[f"phiim_{ax}"] * c[f"phi_v{ax}"]
                            + c[f"theta_{ax}"] * c[f"thetaim_v{ax}"] - c[f"thetaim_{ax}"] * c[f"theta_v{ax}"])
    return div - p.g_gauge2 * rho


def test_gext_gauss2_projection(gpu):
    """After start-up the second Gauss law holds to the CG tolerance (less its
    mean, which a periodic projection cannot remove), and the second-gauge
    links start at zero."""
    st = seeds.small_state(20, True, seed=61, g_gauge2=0.25)
    p = st.params
    with Simulation(p, st.cols()) as sim:
        cols = sim.snapshot()
    G = gauss2_residual(p, cols)
    G0 = gauss2_residual(p, st.cols() + [np.zeros(p.N ** 3)] * 6)
    assert np.abs(G0 - G0.mean()).max() > 1e-3
    assert np.abs(G - G.mean()).max() < 1e-11 * max(1.0, np.abs(G0).max())
    assert all(np.all(cols[c] == 0) for c in range(30, 33))


def test_gext_ignored_without_complex_gauge(gpu):
    """higgs_v and g_gauge2 without complex_gauge change nothing (the reference
    ignores them with a warning, scp_sim.c:229-238)."""
    st = seeds.small_state(14, False, seed=62)
    p0 = st.params
    p1 = Params(**{**p0.__dict__, "higgs_v": 1.0, "g_gauge2": 0.3})
    with Simulation(p0, st.cols()) as a, Simulation(p1, st.cols()) as b:
        a.step(7)
        b.step(7)
        A, B = a.snapshot(), b.snapshot()
    assert len(A) == len(B) == 24
    assert all(np.array_equal(x, y) for x, y in zip(A, B))


@pytest.mark.parametrize("over,prec", [(dict(higgs_v=1.0, g_gauge=0.0), 0), (dict(g_gauge2=0.2, g_gauge=0.0), 0),
                                       (dict(higgs_v=1.0), PREC_FP32C), (dict(g_gauge2=0.2), PREC_FP32C)])
def test_gext_refused(gpu, over, prec):
    """With g_gauge = 0 (the reference's ungauged dispatch never evolves the
    extensions) and in FP32C: refused at init with SCP_EUNSUPPORTED."""
    st = seeds.small_state(8, True, seed=63)
    p = Params(**{**st.params.__dict__, **over, "precision": prec})
    cols = st.cols()
    arr = (ctypes.c_void_p * 30)(*[c.ctypes.data for c in cols])
    cp = p.to_c()
    h = ctypes.c_void_p()
    assert native.lib().scp_gpu_init(ctypes.byref(cp), arr, ctypes.byref(h)) == -7


def test_gext_snapshots(gpu):
    """f32 snapshots of th2 / E2 are the f64 values rounded; the asynchronous
    snapshot carries the same 36 columns."""
    st = seeds.small_state(12, True, seed=64, g_gauge2=0.2, higgs_v=1.0)
    p = st.params
    with Simulation(p, st.cols()) as sim:
        sim.step(9)
        s64 = sim.snapshot(DTYPE_F64)
        s32 = sim.snapshot(DTYPE_F32)
        bufs = [np.empty(p.N ** 3) for _ in range(36)]
        sim.snapshot_async(bufs, DTYPE_F64)
        sim.snapshot_wait()
    assert len(s64) == len(s32) == 36
    assert np.abs(s64[33]).max() > 0
    for c in range(36):
        assert np.array_equal(s32[c], s64[c].astype(np.float32)), c
        assert np.array_equal(bufs[c], s64[c]), c


def test_gext_matches_reference_binary_48(gpu, reference):
    """Both extensions at 48^3 for 100 steps against the reference CPU binary."""
    st = seeds.small_state(48, True, seed=77, higgs_v=1.0, higgs_rvoid=4.0, g_gauge2=0.15)
    p = st.params
    ref = oracle.run_reference(p, st.cols(), 100, diag_every=25)
    rows, got = run_rows(p, st.cols(), 100, 25)
    assert len(got) == 36
    for c in range(36):
        assert rel_l2(got[c], ref["cols"][c]) < TOL_FRAME, COLUMN_NAMES[c]
    check_diag(rows, ref["diag"], ref["diag_header"])


def test_gext_chunking_is_bitwise(gpu):
    """A step's closing kick and sponge run inside the next step's first sweep
    within one call and on their own at the end of a call, in the same
    operation order: 1 + 3 + 36 steps equal 40 steps in one call, bit for bit."""
    st = seeds.small_state(15, True, seed=79, higgs_v=1.0, higgs_rvoid=2.0, g_gauge2=0.2,
                           bc_type=0, damp_width=2.5, damp_rate=0.03)
    p = st.params
    with Simulation(p, st.cols()) as a, Simulation(p, st.cols()) as b:
        a.step(40)
        for k in (1, 3, 36):
            b.step(k)
        A, B = a.snapshot(), b.snapshot()
    assert all(np.array_equal(x, y) for x, y in zip(A, B))
