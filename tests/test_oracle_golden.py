"""Pins the C restatement (oracle/scp_oracle.c) against the reference's own
output: the fixtures in tests/golden/ hold final frames and diag rows of the
reference binary (sfa/sim/scp_sim.c built unmodified) on the same seeds
(tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import oracle
from scp_b200 import seeds

GOLD = os.path.join(os.path.dirname(__file__), "golden")
SMALL = ["ref_complex_n12", "ref_gauged_n12", "ref_gauged_n10_damped", "ref_complex_n13_damped"]


def load(name):
    return np.load(os.path.join(GOLD, name + ".npz"), allow_pickle=False)


def small_params(f):
    over = {}
    if int(f["bc_type"]) != 2:
        over = dict(bc_type=int(f["bc_type"]), damp_width=float(f["damp_width"]), damp_rate=float(f["damp_rate"]))
    return seeds.small_state(int(f["N"]), bool(int(f["gauged"])), **over)


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


@pytest.mark.parametrize("name", SMALL)
def test_oracle_matches_reference_frames(name):
    f = load(name)
    st = small_params(f)
    o = oracle.Oracle(st.params, st.cols())
    o.step(int(f["nsteps"]))
    got = o.cols()
    ref = f["final"]
    assert len(got) == ref.shape[0]
    for c in range(ref.shape[0]):
        assert rel_l2(got[c], ref[c]) < 1e-12, (name, str(f["names"][c]))


@pytest.mark.parametrize("name", SMALL)
def test_oracle_matches_reference_diag(name):
    f = load(name)
    st = small_params(f)
    o = oracle.Oracle(st.params, st.cols())
    hdr = [str(h) for h in f["diag_header"]]
    rows = f["diag"]
    de = int(f["diag_every"])
    for r in range(rows.shape[0]):
        if r > 0:
            o.step(de)
        d = o.diag()
        # columns after t in TSV order map onto oracle slots 0..; Q_p last
        for ci, h in enumerate(hdr[1:], start=1):
            slot = ci - 1
            if h in ("Q_p0", "Q_p1", "Q_p2"):
                slot = 28 + int(h[-1])
            elif h in ("gauss_max", "gauss_l2", "E_em", "Q_flux"):
                slot = {"gauss_max": 24, "gauss_l2": 25, "E_em": 26, "Q_flux": 27}[h]
            ref = rows[r, ci]
            scale = max(abs(ref), 1e-9)
            tol = 1e-5 if h in ("gauss_max", "gauss_l2", "Q_flux", "Q_phi", "Q_theta", "Q_total",
                                "Q_core", "Q_p0", "Q_p1", "Q_p2") else 2e-6
            if h in ("gauss_max", "gauss_l2", "Q_flux", "Q_phi", "Q_theta", "Q_total", "Q_p0", "Q_p1", "Q_p2",
                     "Q_core", "E_coupling", "thp1u", "thp1v", "thp2u", "thp2v"):
                # roundoff-level quantities: absolute agreement at the printed precision
                assert abs(d[slot] - ref) <= max(tol * scale, 1e-12), (name, r, h, d[slot], ref)
            else:
                assert abs(d[slot] - ref) <= tol * scale, (name, r, h, d[slot], ref)


def test_oracle_matches_reference_c0_64_1000():
    """64^3 ungauged workload, 1000 steps: the restatement stays within
    1e-10 relative of the reference on sampled sites and column norms."""
    f = load("ref_c0_64_1000")
    st = seeds.make_state("c0")
    o = oracle.Oracle(st.params, st.cols())
    o.step(int(f["nsteps"]))
    got = np.stack(o.cols())
    idx = f["sites"]
    for c in range(got.shape[0]):
        ref_s = f["sample"][c]
        assert np.linalg.norm(got[c, idx] - ref_s) <= 1e-10 * max(np.linalg.norm(ref_s), 1e-300) + 1e-300
        assert abs(np.linalg.norm(got[c]) - f["col_l2"][c]) <= 1e-10 * f["col_l2"][c] + 1e-300


def test_gauge_xform_kat_oracle():
    """Random lattice gauge transform leaves |acc|^2, E_acc and G unchanged
    (the reference's test_gauge_xform, sfa/sim/scp_sim.c:2461-2556)."""
    st = seeds.small_state(10, True)
    o = oracle.Oracle(st.params, st.cols())
    worst, rel = o.gauge_xform_test()
    assert worst <= 1e-12, rel


# ------------------------------------------------------------ gauged extensions

EXT = ["ref_higgs_gauge2_n12", "ref_higgs_gauge2_n11_damped", "ref_mf_lock_n12", "ref_mf_free_n11_damped"]
ROUNDOFF = ("gauss_max", "gauss_l2", "Q_flux", "Q_phi", "Q_theta", "Q_total", "Q_core", "Q_p0", "Q_p1", "Q_p2",
            "E_coupling", "Q_C", "Q_Q", "Q_L", "Q_em")
ORC_NAMES = ("E_phi_kin", "E_theta_kin", "E_grad", "E_mass", "E_pot", "E_tgrad", "E_tmass", "E_coupling",
             "E_total", "phi_max", "P_max", "P_int", "theta_rms", "Q_phi", "Q_theta", "Q_total", "s_max",
             "r_core", "omega_core", "Q_core", "thp1u", "thp1v", "thp2u", "thp2v", "gauss_max", "gauss_l2",
             "E_em", "Q_flux", "Q_p0", "Q_p1", "Q_p2", "Q_C", "Q_Q", "Q_L", "Q_em")


def ext_state(f):
    import json
    if "kw" in f.files:
        return seeds.mf_state(int(f["N"]), **json.loads(str(f["kw"])))
    return seeds.small_state(int(f["N"]), True, **json.loads(str(f["over"])))


def check_series(rows, want_rows, header):
    """Oracle diag vectors against the reference TSV rows, matched by name."""
    want = np.asarray(want_rows)
    have = np.array(rows)
    for ci, h in enumerate(header):
        if h == "t":
            continue
        ref, got = want[:, ci], have[:, ORC_NAMES.index(h)]
        scale = np.maximum(np.abs(ref), 1e-9)
        tol = np.maximum(1e-5 * scale, 1e-11) if h in ROUNDOFF else 2e-6 * scale
        assert np.all(np.abs(got - ref) <= tol), h


@pytest.mark.parametrize("name", EXT)
def test_oracle_matches_reference_extensions(name):
    """Higgs condensate + second gauge, and three fabrics (locked and free Q):
    the restatement against the reference's frames (36 / 54 columns) and every
    diag TSV column."""
    f = load(name)
    st = ext_state(f)
    o = oracle.Oracle(st.params, st.cols())
    rows = [o.diag()]
    every = int(f["diag_every"])
    for _ in range(int(f["nsteps"]) // every):
        o.step(every)
        rows.append(o.diag())
    got = o.cols()
    assert len(got) == f["final"].shape[0] == st.params.snap_ncols
    for c in range(len(got)):
        assert rel_l2(got[c], f["final"][c]) < 1e-12, (name, str(f["names"][c]))
    check_series(rows, f["diag"], [str(h) for h in f["diag_header"]])


@pytest.mark.skipif(not oracle.reference_available(), reason="reference binary not built (make -C oracle ref)")
@pytest.mark.parametrize("kind", ["higgs", "gauge2", "mf_lock", "mf_free"])
def test_oracle_matches_reference_binary_extensions(kind):
    """Each extension on its own at another size, seed and set of couplings,
    the restatement against the reference binary run here."""
    if kind == "higgs":
        st = seeds.small_state(14, True, seed=5, higgs_v=0.9, higgs_rvoid=2.0, higgs_lam=1.3, higgs_kap=2.5)
    elif kind == "gauge2":
        st = seeds.small_state(13, True, seed=6, g_gauge2=-0.25, gauge2_q0=0.5, gauge2_q1=2.0, gauge2_q2=-1.0)
    elif kind == "mf_lock":
        st = seeds.mf_state(13, seed=7, shift=1.0, q_C=0.4, q_Q=1.0, q_L=-2.0)
    else:
        st = seeds.mf_state(14, seed=8, shift=-1.5, mf_lock_CQ=0, l_charge=0.03, bc_type=0, damp_width=2.0,
                            damp_rate=0.04)
    p = st.params
    ref = oracle.run_reference(p, st.cols(), 30, diag_every=10)
    o = oracle.Oracle(p, st.cols())
    rows = [o.diag()]
    for _ in range(3):
        o.step(10)
        rows.append(o.diag())
    got = o.cols()
    assert len(got) == len(ref["cols"])
    for c in range(len(got)):
        assert rel_l2(got[c], ref["cols"][c]) < 1e-12, (kind, ref["names"][c])
    check_series(rows, ref["diag"], ref["diag_header"])


# ------------------------------------------------------------ real 6-field mode

@pytest.mark.parametrize("name", ["ref_real_n12", "ref_real_terms_n11_damped"])
def test_oracle_matches_reference_real_mode(name):
    """The real mode (compute_forces / compute_energy), plain and with every
    optional term under the sponge: frames and the 13 diag TSV columns."""
    import json
    f = load(name)
    st = seeds.real_state(int(f["N"]), **json.loads(str(f["over"])))
    o = oracle.Oracle(st.params, st.cols())
    rows = [o.diag()]
    every = int(f["diag_every"])
    for _ in range(int(f["nsteps"]) // every):
        o.step(every)
        rows.append(o.diag())
    got = o.cols()
    assert len(got) == 12 == f["final"].shape[0]
    for c in range(12):
        assert rel_l2(got[c], f["final"][c]) < 1e-12, (name, str(f["names"][c]))
    want = np.asarray(f["diag"])[:, 1:]
    have = np.array(rows)
    assert have.shape == want.shape
    assert np.all(np.abs(have - want) <= 1e-6 * np.abs(want) + 1e-12)


@pytest.mark.skipif(not oracle.reference_available(), reason="reference binary not built (make -C oracle ref)")
@pytest.mark.parametrize("terms", [dict(mode=1), dict(mode=3), dict(alpha_cs=0.3), dict(beta_h=0.5),
                                   dict(kappa_h=0.2)], ids=lambda t: "-".join(f"{k}{v}" for k, v in t.items()))
def test_oracle_real_terms_match_reference_binary(terms):
    st = seeds.real_state(13, seed=21, **terms)
    ref = oracle.run_reference(st.params, st.cols(), 30, diag_every=10)
    o = oracle.Oracle(st.params, st.cols())
    o.step(30)
    for c, (g, r) in enumerate(zip(o.cols(), ref["cols"])):
        assert rel_l2(g, r) < 1e-12, (terms, c)
