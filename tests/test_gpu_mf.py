"""Three matter fabrics C, Q, L under one shared U(1) (force_fabric_gauged_accum
and compute_forces_complex_gauge_mf, sfa/sim/scp_sim.c:1274-1433; verlet_step's
multi-fabric branch :1583-1716; em_rho_at :184-197; compute_mf_charges
:2247-2261) through the C ABI, against the reference CPU stepper's own output."""
import ctypes
import json
import os

import numpy as np
import pytest

import oracle
from scp_b200 import PREC_FP32C, Params, native, seeds
from scp_b200.api import DTYPE_F32, DTYPE_F64, Simulation
from scp_b200.params import DIAG_NAMES

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL_FRAME = 1e-10      # relative L2 per column
ROUNDOFF = ("gauss_max", "gauss_l2", "Q_flux", "Q_phi", "Q_theta", "Q_total", "Q_core", "Q_p0", "Q_p1", "Q_p2",
            "E_coupling", "Q_C", "Q_Q", "Q_L", "Q_em")


def rel_l2(a, b):
    a, b = np.asarray(a).reshape(-1), np.asarray(b).reshape(-1)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


def check_diag(have_rows, want_rows, header):
    """have: diag vectors (slot order); want: the reference TSV rows (t first),
    matched by column name.  The TSV prints %.6e / %.12e; roundoff-level sums
    get an absolute floor."""
    want = np.asarray(want_rows)
    have = np.array(have_rows)
    for ci, h in enumerate(header):
        if h == "t":
            continue
        ref, got = want[:, ci], have[:, DIAG_NAMES.index(h)]
        scale = np.maximum(np.abs(ref), 1e-9)
        if h in ROUNDOFF:
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


@pytest.mark.parametrize("name", ["ref_mf_lock_n12", "ref_mf_free_n11_damped"])
def test_mf_matches_golden(gpu, name):
    f = np.load(os.path.join(GOLD, name + ".npz"))
    kw = json.loads(str(f["kw"]))
    st = seeds.mf_state(int(f["N"]), **kw)
    p = st.params
    rows, got = run_rows(p, st.cols(), int(f["nsteps"]), int(f["diag_every"]))
    assert len(got) == 54 and list(f["names"]) == list(p.snap_names)
    for c in range(54):
        assert rel_l2(got[c], f["final"][c]) < TOL_FRAME, p.snap_names[c]
    check_diag(rows, f["diag"], [str(h) for h in f["diag_header"]])


MF = [dict(),
      dict(mf_lock_CQ=0),
      dict(mf_lock_CQ=0, mf_seed_copy=True),
      dict(q_C=0.5, q_Q=1.0, q_L=-1.5, eta=0.0),
      dict(mf_lock_CQ=0, l_charge=0.05, q_C=-0.3, q_Q=0.7, q_L=2.0, bc_type=0, damp_width=2.5, damp_rate=0.03),
      dict(l_charge=0.05, bc_type=0, damp_width=2.5, damp_rate=0.03)]


@pytest.mark.parametrize("kw", MF, ids=lambda t: "-".join(f"{k}{v}" for k, v in t.items()) or "lock")
@pytest.mark.parametrize("N", [16, 15])
def test_mf_matches_reference_binary(gpu, reference, N, kw):
    """Locked and free Q (free Q seeded from its own state or as a copy of C),
    custom charges with eta = 0, a charged L fabric under the sponge; even and
    odd N; against the reference CPU binary on the same seeds."""
    kw = dict(kw)
    copy = kw.pop("mf_seed_copy", False)
    st = seeds.mf_state(N, seed=90 + N, shift=1.5, **kw)
    p = st.params
    if copy:   # Q starts as C (what mf_seed_Q = 1 does in the reference)
        from scp_b200.params import COLUMN_NAMES, Q_COLUMN_NAMES
        for q, c in zip(Q_COLUMN_NAMES, COLUMN_NAMES[:24]):
            st[q] = st[c].copy()
    ref = oracle.run_reference(p, st.cols(), 40, diag_every=10)
    rows, got = run_rows(p, st.cols(), 40, 10)
    assert len(got) == len(ref["cols"]) == 54
    for c in range(54):
        assert rel_l2(got[c], ref["cols"][c]) < TOL_FRAME, p.snap_names[c]
    check_diag(rows, ref["diag"], ref["diag_header"])


def test_mf_lock_with_empty_L_is_one_fabric(gpu):
    """Locked Q with charges (0, 1, *) and an empty L fabric: the C fabric and
    the links evolve exactly as the single-fabric gauged stepper (fused
    kernel) evolves them."""
    st = seeds.mf_state(16, seed=95)
    for k in list(st):
        if k.startswith("l"):
            st[k][:] = 0.0
    p = st.params
    one = seeds.small_state(16, True, seed=95)
    assert all(np.array_equal(a, b) for a, b in zip(st.cols()[:30], one.cols()))
    with Simulation(p, st.cols()) as a, Simulation(one.params, one.cols()) as b:
        a.step(25)
        b.step(25)
        A, B = a.snapshot(), b.snapshot()
        da, db = a.diag_vector(), b.diag_vector()
    for c in range(30):
        assert rel_l2(A[c], B[c]) < 1e-10, c
    assert all(np.all(A[c] == 0) for c in range(30, 54))
    for q in (0, 1, 2, 3, 4, 5, 6, 8, 9, 10, 12, 26):
        assert abs(da[q] - db[q]) <= 1e-10 * max(abs(db[q]), 1.0), DIAG_NAMES[q]
    assert abs(da[DIAG_NAMES.index("Q_Q")] - db[DIAG_NAMES.index("Q_phi")] - db[DIAG_NAMES.index("Q_theta")]) < 1e-9


@pytest.mark.parametrize("over,prec", [(dict(g_gauge=0.0), 0), (dict(), PREC_FP32C), (dict(higgs_v=1.0), 0),
                                       (dict(g_gauge2=0.2), 0)])
def test_mf_refused(gpu, over, prec):
    """g_gauge = 0, FP32C, and with the Higgs or the second gauge (which the
    reference's validation rejects): SCP_EUNSUPPORTED at init."""
    st = seeds.mf_state(8, seed=96)
    p = Params(**{**st.params.__dict__, **over, "precision": prec})
    cols = st.cols()
    arr = (ctypes.c_void_p * 78)(*[c.ctypes.data for c in cols])
    cp = p.to_c()
    h = ctypes.c_void_p()
    assert native.lib().scp_gpu_init(ctypes.byref(cp), arr, ctypes.byref(h)) == -7


def test_mf_snapshots(gpu):
    """54 columns (C with the links, then L); f32 snapshots are the f64 values
    rounded; the asynchronous snapshot carries the same columns."""
    st = seeds.mf_state(12, seed=97, mf_lock_CQ=0, shift=1.0)
    p = st.params
    with Simulation(p, st.cols()) as sim:
        sim.step(9)
        s64 = sim.snapshot(DTYPE_F64)
        s32 = sim.snapshot(DTYPE_F32)
        bufs = [np.empty(p.N ** 3) for _ in range(54)]
        sim.snapshot_async(bufs, DTYPE_F64)
        sim.snapshot_wait()
        d = sim.snapshot_dict()
    assert len(s64) == len(s32) == 54 and list(d)[30] == "lphi_x"
    assert np.abs(s64[30]).max() > 0
    for c in range(54):
        assert np.array_equal(s32[c], s64[c].astype(np.float32)), c
        assert np.array_equal(bufs[c], s64[c]), c


@pytest.mark.parametrize("lock", [1, 0])
def test_mf_matches_reference_binary_48(gpu, reference, lock):
    """Three fabrics at 48^3 for 100 steps against the reference CPU binary."""
    st = seeds.mf_state(48, seed=78, shift=4.0, mf_lock_CQ=lock)
    p = st.params
    ref = oracle.run_reference(p, st.cols(), 100, diag_every=25)
    rows, got = run_rows(p, st.cols(), 100, 25)
    assert len(got) == 54
    for c in range(54):
        assert rel_l2(got[c], ref["cols"][c]) < TOL_FRAME, p.snap_names[c]
    check_diag(rows, ref["diag"], ref["diag_header"])


def test_mf_chunking_is_bitwise(gpu):
    """1 + 3 + 36 steps equal 40 steps in one call, bit for bit (the closing
    kick and sponge fused into the next step's first sweep keep the order of
    separate sweeps)."""
    st = seeds.mf_state(15, seed=80, shift=1.0, mf_lock_CQ=0, l_charge=0.05, bc_type=0, damp_width=2.5,
                        damp_rate=0.03)
    p = st.params
    with Simulation(p, st.cols()) as a, Simulation(p, st.cols()) as b:
        a.step(40)
        for k in (1, 3, 36):
            b.step(k)
        A, B = a.snapshot(), b.snapshot()
    assert all(np.array_equal(x, y) for x, y in zip(A, B))
