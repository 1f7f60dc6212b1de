import math

import numpy as np

from scp_b200 import Params, seeds


def test_splitmix64_known_answer():
    # canonical SplitMix64 outputs for seed 1234567
    assert [int(x) for x in seeds.splitmix64(1234567, 5)] == [
        6457827717110365317, 3203168211198807973, 9817491932198370423,
        4593380528125082431, 16408922859458223821]


def test_normals_deterministic_and_standard():
    a = seeds.normals(0, 3, 200001)
    b = seeds.normals(0, 3, 200001)
    assert np.array_equal(a, b)
    assert abs(a.mean()) < 0.01 and abs(a.std() - 1.0) < 0.01
    assert not np.array_equal(a[:100], seeds.normals(0, 4, 100))


def test_workload_grids():
    p = seeds.params_for("c1")
    assert p.N == 128 and p.dx == 0.5 and abs(p.dt - 0.1) < 1e-15 and p.gauged
    assert seeds.params_for("c0").ncols == 24 and p.ncols == 30


def test_c1_is_net_neutral_and_c2_neutralised():
    st = seeds.make_state("c1", seeds.params_for("c1", N=32, L=7.75))
    rho = seeds.charge_density(st)
    assert abs(rho.sum()) <= 1e-12 * np.abs(rho).sum()
    st2 = seeds.State(st.params)
    for k in st:
        st2[k] = st[k].copy()
    seeds.add_noise(st2, seeds.FIELD_COLS, 0.01, seed=1)
    seeds.neutralise(st2)
    rho2 = seeds.charge_density(st2)
    assert abs(rho2.sum()) <= 1e-12 * np.abs(rho2).sum()


def test_ball_is_phase_rotating():
    p = Params(N=16, L=3.75)
    st = seeds.State(p)
    seeds.add_balls(st, [seeds.Ball(omega=0.8)])
    # dPhi/dt = i omega Phi
    assert np.allclose(st["phi_vx"], -0.8 * st["phiim_x"])
    assert np.allclose(st["phiim_vy"], 0.8 * st["phi_y"])
    c = st.params.N // 2
    assert math.isclose(math.atan2(st["phiim_y"][c, c, c], st["phi_y"][c, c, c]), 2 * math.pi / 3, rel_tol=1e-12)


def test_gauged_extension_params():
    """Higgs / second-gauge keys: reference defaults, config text, snapshot width."""
    p = seeds.params_for("c1")
    assert (p.higgs_v, p.higgs_lam, p.higgs_kap, p.higgs_rvoid) == (0.0, 1.0, 2.0, 0.0)
    assert (p.g_gauge2, p.gauge2_q0, p.gauge2_q1, p.gauge2_q2) == (0.0, 1.0, 1.0, -2.0)
    assert p.snap_ncols == 30
    q = seeds.params_for("c1", g_gauge2=0.1, higgs_v=1.0)
    assert q.ncols == 30 and q.snap_ncols == 36
    assert "g_gauge2 = 0.1\n" in q.to_cfg() and "higgs_v = 1.0\n" in q.to_cfg()
    c = q.to_c()
    assert c.g_gauge2 == 0.1 and list(c.gauge2_q) == [1.0, 1.0, -2.0]
    assert seeds.params_for("c0", g_gauge2=0.1).snap_ncols == 24   # ignored without complex_gauge


def test_gauged_extension_fixtures():
    """The Higgs / second-gauge fixtures hold the reference's 36-column frame."""
    import json
    import os
    from scp_b200.params import COLUMN_NAMES
    gold = os.path.join(os.path.dirname(__file__), "golden")
    for name in ("ref_higgs_gauge2_n12", "ref_higgs_gauge2_n11_damped"):
        f = np.load(os.path.join(gold, name + ".npz"))
        over = json.loads(str(f["over"]))
        assert over["g_gauge2"] != 0 and over["higgs_v"] > 0
        assert list(f["names"]) == list(COLUMN_NAMES)
        assert f["final"].shape == (36, int(f["N"]) ** 3) and np.all(np.isfinite(f["final"]))
        assert np.abs(f["final"][30:33]).max() > 0          # th2 moved off its zero start
        assert len(f["diag"]) == int(f["nsteps"]) // int(f["diag_every"]) + 1


def test_three_fabric_params_and_fixtures():
    """n_fabrics = 3: 78 initial columns (C, Q, L), 54 snapshot columns (C, L),
    config keys; the committed fixtures hold the reference's 54-column frames."""
    import json
    import os
    st = seeds.mf_state(8, seed=3, mf_lock_CQ=0, q_L=-2.0)
    p = st.params
    assert p.ncols == 78 and p.snap_ncols == 54 and len(st.cols()) == 78
    assert p.input_names[30] == "qphi_x" and p.input_names[54] == "lphi_x" and p.snap_names[30] == "lphi_x"
    cfg = p.to_cfg()
    assert "n_fabrics = 3\n" in cfg and "mf_lock_CQ = 0\n" in cfg and "q_L = -2.0\n" in cfg
    c = p.to_c()
    assert c.n_fabrics == 3 and c.mf_lock_CQ == 0 and list(c.q_fab) == [0.0, 1.0, -2.0]
    from scp_b200.params import COLUMN_NAMES, L_COLUMN_NAMES, Q_COLUMN_NAMES
    for names in (COLUMN_NAMES[:24], Q_COLUMN_NAMES, L_COLUMN_NAMES):   # every fabric net-neutral
        v = [st[n] for n in names]   # complex order: phi theta phi_v theta_v, then the imaginary parts
        rho = sum(v[a] * v[18 + a] - v[12 + a] * v[6 + a] + v[3 + a] * v[21 + a] - v[15 + a] * v[9 + a]
                  for a in range(3))
        assert abs(rho.sum()) < 1e-12 * np.abs(rho).sum()
    gold = os.path.join(os.path.dirname(__file__), "golden")
    for name in ("ref_mf_lock_n12", "ref_mf_free_n11_damped"):
        f = np.load(os.path.join(gold, name + ".npz"))
        kw = json.loads(str(f["kw"]))
        q = seeds.mf_state(int(f["N"]), **kw).params
        assert list(f["names"]) == list(q.snap_names)
        assert f["final"].shape == (54, int(f["N"]) ** 3) and np.all(np.isfinite(f["final"]))
        assert np.abs(f["final"][30:54]).max() > 0               # fabric L evolved
        assert list(f["diag_header"][-7:-3]) == ["Q_C", "Q_Q", "Q_L", "Q_em"]


def test_real_mode_fixtures():
    """The real-mode fixtures hold the reference's 12-column frames and its
    real-mode diag TSV (energies and amplitudes only)."""
    import json
    import os
    gold = os.path.join(os.path.dirname(__file__), "golden")
    for name in ("ref_real_n12", "ref_real_terms_n11_damped"):
        f = np.load(os.path.join(gold, name + ".npz"))
        st = seeds.real_state(int(f["N"]), **json.loads(str(f["over"])))
        assert f["final"].shape == (12, int(f["N"]) ** 3) and np.all(np.isfinite(f["final"]))
        assert list(f["names"])[:3] == ["phi_x", "phi_y", "phi_z"] and len(f["diag_header"]) == 14
        assert st.params.real_fields == 1 and len(st.cols()) == 12
