"""Known-answer and failure-path tests of the CUDA stepper."""
import ctypes

import numpy as np
import pytest

from scp_b200 import Params, native, seeds
from scp_b200.api import Simulation

pytestmark = pytest.mark.gpu


def test_gauge_covariance(gpu):
    """A lattice gauge transform of the seed commutes with time stepping
    (the dynamic form of test_gauge_xform, sfa/sim/scp_sim.c:2461-2556):
    |Phi_a|^2, |Theta_a|^2, E and the Gauss residual agree after 20 steps."""
    st = seeds.small_state(16, True, seed=11)
    p = st.params
    rng = np.random.default_rng(5)
    alpha = rng.uniform(-10, 10, size=(p.N,) * 3)
    g = p.g_gauge
    ca, sa = np.cos(g * alpha), np.sin(g * alpha)
    tr = seeds.State(p)
    for k in st:
        tr[k] = st[k].copy()
    for pre_re, pre_im in (("phi_", "phiim_"), ("phi_v", "phiim_v"), ("theta_", "thetaim_"),
                           ("theta_v", "thetaim_v")):
        for ax in "xyz":
            u, v = st[pre_re + ax], st[pre_im + ax]
            tr[pre_re + ax] = ca * u + sa * v
            tr[pre_im + ax] = ca * v - sa * u
    for d, ax in enumerate("xyz"):
        t = st["th_" + ax] + g * (np.roll(alpha, -1, axis=d) - alpha)
        tr["th_" + ax] = t - 2 * np.pi * np.rint(t / (2 * np.pi))
    with Simulation(p, st.cols()) as a, Simulation(p, tr.cols()) as b:
        a.step(20)
        b.step(20)
        A, B = a.snapshot_dict(), b.snapshot_dict()
        da, db = a.diag(), b.diag()
    for ax in "xyz":
        ma = A["phi_" + ax] ** 2 + A["phiim_" + ax] ** 2
        mb = B["phi_" + ax] ** 2 + B["phiim_" + ax] ** 2
        assert np.max(np.abs(ma - mb)) <= 1e-11 * max(np.max(ma), 1.0)
        ta = A["theta_" + ax] ** 2 + A["thetaim_" + ax] ** 2
        tb = B["theta_" + ax] ** 2 + B["thetaim_" + ax] ** 2
        assert np.max(np.abs(ta - tb)) <= 1e-11 * max(np.max(ta), 1.0)
        assert np.max(np.abs(A["E_" + ax] - B["E_" + ax])) <= 1e-11 * max(np.max(np.abs(A["E_" + ax])), 1.0)
    for key in ("E_total", "Q_total", "gauss_max", "E_em"):
        assert abs(da[key] - db[key]) <= 1e-10 * max(abs(da[key]), 1.0), key


@pytest.mark.parametrize("prec", [0, 1])
def test_zero_coupling_runs_the_ungauged_stepper(gpu, prec):
    """complex_gauge=1 with g_gauge=0 is the reference's ungauged dispatch
    (scp_sim.c:1586, :2820): the 24 matter columns evolve bit for bit as in
    the ungauged run, th and E are carried unchanged, the energy is the
    ungauged one, and compute_gauss reports div E, 1/2 E^2 and Q_flux = 0."""
    st = seeds.small_state(16, True, seed=17, g_gauge=0.0, precision=prec)
    p = st.params
    pu = Params(**{**p.__dict__, "complex_gauge": 0})
    cols = st.cols()
    with Simulation(p, cols) as a, Simulation(pu, cols[:24]) as b:
        a.step(7)
        b.step(7)
        A, B = a.snapshot(), b.snapshot()
        da, db = a.diag(), b.diag()
    for c in range(24):
        assert np.array_equal(A[c], B[c]), c
    for c in range(24, 30):   # FP64 exactly; FP32C holds E in fp32 and th as an fp32 pair
        want = np.asarray(cols[c]).reshape(-1)
        if prec == 0:
            assert np.array_equal(A[c], want), c
        else:
            assert np.max(np.abs(A[c] - want)) <= 1e-7 * max(np.max(np.abs(want)), 1e-30), c
    # the same per-site terms; the ungauged FP64 handle sums them inside its
    # synchronous step launch, the g = 0 one in the separate pass, so the
    # totals agree to roundoff (the energy is the ungauged one: E_em, which the
    # gauged energy would add, is of order 1e-3 here)
    for key in ("E_total", "E_grad", "Q_total", "s_max", "r_core"):
        assert abs(da[key] - db[key]) <= 1e-12 * max(abs(db[key]), 1.0), key
    N, dx = p.N, p.dx
    E = [A[27 + d].reshape(N, N, N) for d in range(3)]
    div = sum(E[d] - np.roll(E[d], 1, axis=d) for d in range(3)) / dx
    assert abs(da["gauss_max"] - np.abs(div).max()) <= 1e-12 * max(np.abs(div).max(), 1.0)
    eem = 0.5 * sum((e ** 2).sum() for e in E) * dx ** 3
    assert abs(da["E_em"] - eem) <= 1e-12 * max(eem, 1.0)
    assert da["Q_flux"] == 0.0


def test_real_limit_keeps_imaginary_sector_zero(gpu):
    """v = tv = 0 with zero imaginary momenta stays exactly zero
    (the complex kernel's real limit, v66 reg_harness)."""
    p = Params(N=20, L=4.75)
    st = seeds.State(p)
    seeds.add_balls(st, [seeds.Ball(omega=0.0, phases=(0.0, np.pi, 0.0))])
    seeds.add_noise(st, ("theta_x", "theta_y", "phi_vz"), 1e-3, seed=2)
    for ax in "xyz":   # sin(pi) is not exactly zero: make the imaginary sector exactly zero
        for pre in ("phiim_", "thetaim_", "phiim_v", "thetaim_v"):
            st[pre + ax][:] = 0.0
    with Simulation(p, st.cols()) as sim:
        sim.step(50)
        s = sim.snapshot_dict()
    for ax in "xyz":
        for pre in ("phiim_", "thetaim_", "phiim_v", "thetaim_v"):
            assert not np.any(s[pre + ax]), pre + ax


def test_noether_charge_conserved(gpu):
    """eta = 0, periodic: Q_total stays flat to roundoff (v66 qcons)."""
    p = Params(N=24, L=5.75, eta=0.0)
    st = seeds.State(p)
    seeds.add_balls(st, [seeds.Ball(omega=0.8, sigma=1.5)])
    with Simulation(p, st.cols()) as sim:
        q0 = sim.diag()["Q_total"]
        for _ in range(5):
            sim.step(100)
        q1 = sim.diag()["Q_total"]
    assert abs(q1 - q0) <= 1e-11 * abs(q0)


def test_nonfinite_seed_is_reported(gpu):
    """A NaN planted in the seed (host-side fault injection) surfaces as
    SCP_ENONFINITE from sync and diag; the context stays usable."""
    st = seeds.small_state(12, False, seed=1)
    st["phi_x"][3, 4, 5] = np.nan
    with Simulation(st.params, st.cols()) as sim:
        sim.step(2)
        with pytest.raises(native.ScpError) as e:
            sim.sync()
        assert e.value.code == -6
    ok = seeds.small_state(12, False, seed=1)
    with Simulation(ok.params, ok.cols()) as sim:
        sim.step(2)
        sim.sync()


def test_charged_periodic_gauged_seed_refused(gpu):
    p = Params(N=16, L=3.75, complex_gauge=1, g_gauge=0.1)
    st = seeds.State(p)
    seeds.add_balls(st, [seeds.Ball(omega=0.8, sigma=1.0)])
    with pytest.raises(native.ScpError) as e:
        Simulation(p, st.cols())
    assert e.value.code == -4
    p2 = Params(N=16, L=3.75, complex_gauge=1, g_gauge=0.1, bc_type=0, damp_rate=0.0)
    with Simulation(p2, st.cols()) as sim:   # bc_type 0 keeps a frozen offset instead
        sim.step(3)
        assert sim.diag()["gauss_max"] < 1e-10


def test_bad_parameters(gpu):
    L = native.lib()
    h = ctypes.c_void_p()
    for bad in (dict(N=3), dict(bc_type=1), dict(complex_gauge=1, g_gauge=-0.1), dict(tile_variant=99)):
        p = Params(**bad)
        cols = [np.zeros(p.N ** 3) for _ in range(p.ncols)]
        arr = (ctypes.c_void_p * p.ncols)(*[c.ctypes.data for c in cols])
        rc = L.scp_gpu_init(ctypes.byref(p.to_c()), arr, ctypes.byref(h))
        assert rc in (-1, -7), bad
