"""Gauge covariance of the extension steppers (the dynamic form of the
reference's test_gauge_xform, sfa/sim/scp_sim.c:2461-2556): a lattice gauge
transform of the seed commutes with time stepping.  Size-independent checks
of the Higgs / second-gauge kernels and of the three-fabric kernels, whose
matter carries per-fabric charges."""
import numpy as np
import pytest

from scp_b200 import Params, seeds
from scp_b200.api import Simulation

pytestmark = pytest.mark.gpu

# complex 24-column order: (real, imaginary) column pairs of phi, theta, phi_v, theta_v
PAIRS = [(r + a, r + 12 + a) for r in (0, 3, 6, 9) for a in range(3)]


def rotate(cols24, phase):
    """Multiply every complex field of a fabric by exp(-i phase)."""
    out = [c.copy() for c in cols24]
    ca, sa = np.cos(phase), np.sin(phase)
    for re, im in PAIRS:
        u, v = cols24[re], cols24[im]
        out[re] = ca * u + sa * v
        out[im] = ca * v - sa * u
    return out


def shift_links(th3, g, alpha):
    out = []
    for d in range(3):
        t = th3[d] + g * (np.roll(alpha, -1, axis=d) - alpha)
        out.append(t - 2 * np.pi * np.rint(t / (2 * np.pi)))
    return out


def moduli(cols24):
    return [cols24[re] ** 2 + cols24[im] ** 2 for re, im in PAIRS]


def close(a, b, rtol):
    return np.max(np.abs(a - b)) <= rtol * max(np.max(np.abs(a)), 1.0)


def test_higgs_gauge2_covariance(gpu):
    """Higgs condensate and second gauge on: a gauge-1 transform of the seed
    leaves |Phi|, E, th2, E2 and the energies unchanged after 20 steps."""
    st = seeds.small_state(16, True, seed=31, higgs_v=1.0, higgs_rvoid=2.0, g_gauge2=0.2)
    p = st.params
    N = p.N
    alpha = np.random.default_rng(7).uniform(-10, 10, size=(N,) * 3)
    cols = [c.reshape(N, N, N) for c in st.cols()]
    tr = rotate(cols[:24], p.g_gauge * alpha) + shift_links(cols[24:27], p.g_gauge, alpha) + cols[27:30]
    with Simulation(p, [c.reshape(-1) for c in cols]) as a, Simulation(p, [c.reshape(-1) for c in tr]) as b:
        a.step(20)
        b.step(20)
        A, B = a.snapshot(), b.snapshot()
        da, db = a.diag(), b.diag()
    for ma, mb in zip(moduli(A[:24]), moduli(B[:24])):
        assert close(ma, mb, 1e-11)
    for c in list(range(27, 30)) + list(range(30, 36)):   # E, th2, E2
        assert close(A[c], B[c], 1e-11), c
    for key in ("E_total", "E_em", "Q_total", "gauss_max"):
        assert abs(da[key] - db[key]) <= 1e-10 * max(abs(da[key]), 1.0), key


@pytest.mark.parametrize("lock,q", [(1, (0.0, 1.0, -1.0)), (0, (2.0, 1.0, -1.0))])
def test_three_fabric_covariance(gpu, lock, q):
    """Three fabrics with integer charges: transforming fabric f by
    exp(-i q_f g alpha) and the shared links by g (alpha(x+d) - alpha(x))
    leaves every fabric's |Phi|, E and the energies unchanged after 20 steps
    (locked: C, and so Q, carries q_Q, the charge of its forces)."""
    st = seeds.mf_state(16, seed=41, shift=1.5, mf_lock_CQ=lock, q_C=q[0], q_Q=q[1], q_L=q[2])
    p = st.params
    N = p.N
    alpha = np.random.default_rng(9).uniform(-10, 10, size=(N,) * 3)
    cols = [c.reshape(N, N, N) for c in st.cols()]
    gC = (q[1] if lock else q[0]) * p.g_gauge
    tr = (rotate(cols[:24], gC * alpha) + shift_links(cols[24:27], p.g_gauge, alpha) + cols[27:30]
          + rotate(cols[30:54], q[1] * p.g_gauge * alpha) + rotate(cols[54:78], q[2] * p.g_gauge * alpha))
    with Simulation(p, [c.reshape(-1) for c in cols]) as a, Simulation(p, [c.reshape(-1) for c in tr]) as b:
        a.step(20)
        b.step(20)
        A, B = a.snapshot(), b.snapshot()
        da, db = a.diag(), b.diag()
    for ma, mb in zip(moduli(A[:24]) + moduli(A[30:54]), moduli(B[:24]) + moduli(B[30:54])):
        assert close(ma, mb, 1e-11)
    for c in range(27, 30):
        assert close(A[c], B[c], 1e-11), c
    for key in ("Q_C", "Q_Q", "Q_L", "Q_em", "gauss_max", "E_em"):
        assert abs(da[key] - db[key]) <= 1e-10 * max(abs(da[key]), 1.0), key


EXT_CASES = [("gext", 9), ("gext", 20), ("mf_lock", 9), ("mf_free", 20)]


@pytest.mark.parametrize("kind,N", EXT_CASES)
def test_extensions_match_oracle_in_chunks(gpu, kind, N):
    """The extension steppers against the C restatement (oracle/scp_oracle.c,
    itself pinned to the reference binary) after 1, 5 and 12 steps, grids the
    reference comparisons do not use."""
    import oracle
    if kind == "gext":
        st = seeds.small_state(N, True, seed=N, higgs_v=1.0, higgs_rvoid=1.5, g_gauge2=0.2, gauge2_q0=1.0,
                               gauge2_q1=-1.0, gauge2_q2=0.0)
    elif kind == "mf_lock":
        st = seeds.mf_state(N, seed=N, q_C=0.5)
    else:
        st = seeds.mf_state(N, seed=N, shift=1.0, mf_lock_CQ=0, l_charge=0.02, bc_type=0, damp_width=3.0,
                            damp_rate=0.05)
    p = st.params
    o = oracle.Oracle(p, st.cols())
    with Simulation(p, st.cols()) as sim:
        for chunk in (1, 4, 7):
            sim.step(chunk)
            o.step(chunk)
            got, want = sim.snapshot(), o.cols()
            assert len(got) == len(want) == p.snap_ncols
            for c in range(len(got)):
                a, b = got[c], want[c]
                nb = np.linalg.norm(b)
                err = np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)
                assert err < 1e-10, (chunk, c)
