"""Parity of the CUDA stepper (through the C ABI) with the CPU checker and
with the reference's own recorded output."""
import os

import numpy as np
import pytest

import oracle
from scp_b200 import Params, seeds
from scp_b200.api import DTYPE_F16, DTYPE_F32, DTYPE_F64, Simulation

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel_l2(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


def worst_rel(got, ref):
    return max(rel_l2(np.asarray(g).reshape(-1), np.asarray(r).reshape(-1)) for g, r in zip(got, ref))


@pytest.mark.parametrize("name", ["ref_complex_n12", "ref_gauged_n12", "ref_gauged_n10_damped",
                                  "ref_complex_n13_damped"])
def test_gpu_matches_reference_frames(gpu, name):
    f = np.load(os.path.join(GOLD, name + ".npz"))
    over = {}
    if int(f["bc_type"]) != 2:
        over = dict(bc_type=int(f["bc_type"]), damp_width=float(f["damp_width"]), damp_rate=float(f["damp_rate"]))
    st = seeds.small_state(int(f["N"]), bool(int(f["gauged"])), **over)
    with Simulation(st.params, st.cols()) as sim:
        sim.step(int(f["nsteps"]))
        got = sim.snapshot()
    assert worst_rel(got, f["final"]) < 1e-11


CASES = [(n, g, t) for n in (8, 13, 31, 33, 40) for g in (False, True) for t in (0, 2, 3, 4)]


@pytest.mark.parametrize("N,gauged,tile", CASES)
def test_gpu_matches_oracle_shapes(gpu, N, gauged, tile):
    st = seeds.small_state(N, gauged, seed=N, tile_variant=tile)
    o = oracle.Oracle(st.params, st.cols())
    with Simulation(st.params, st.cols()) as sim:
        for chunk in (1, 4, 7):
            sim.step(chunk)
            o.step(chunk)
            assert worst_rel(sim.snapshot(), o.cols()) < 1e-11, chunk


@pytest.mark.parametrize("gauged", [False, True])
@pytest.mark.parametrize("bc", [2, 0])
def test_gpu_diag_matches_oracle(gpu, gauged, bc):
    over = dict(bc_type=0, damp_width=3.0, damp_rate=0.02) if bc == 0 else {}
    st = seeds.small_state(24, gauged, seed=3, **over)
    o = oracle.Oracle(st.params, st.cols())
    with Simulation(st.params, st.cols()) as sim:
        for n in (0, 5, 10):
            if n:
                sim.step(5)
                o.step(5)
            g = sim.diag_vector()
            r = o.diag()
            for q in range(31):
                if not gauged and 24 <= q <= 27:
                    continue
                tol = 1e-9 * max(abs(r[q]), 1.0) if q in (7, 13, 14, 15, 19, 24, 25, 27, 28, 29, 30) \
                    else 1e-11 * max(abs(r[q]), 1e-300)
                assert abs(g[q] - r[q]) <= tol, (n, q, g[q], r[q])


def test_gpu_diag_deterministic(gpu):
    st = seeds.small_state(32, True, seed=5)
    with Simulation(st.params, st.cols()) as a:
        a.step(3)
        d1 = a.diag_vector()
        d2 = a.diag_vector()
    with Simulation(st.params, st.cols()) as b:
        b.step(3)
        d3 = b.diag_vector()
    assert np.array_equal(d1, d2) and np.array_equal(d1, d3)


def _f16_trunc(x):
    """The reference's f64_to_f16 (sfa/sim/scp_config.h:548-559) in numpy."""
    f = x.astype(np.float32).view(np.uint32)
    sign = ((f >> 16) & 0x8000).astype(np.uint16)
    e = ((f >> 23) & 0xFF).astype(np.int32) - 127 + 15
    mant = ((f >> 13) & 0x3FF).astype(np.uint16)
    out = (sign | (np.clip(e, 0, 31).astype(np.uint16) << 10) | mant).astype(np.uint16)
    out = np.where(e <= 0, sign, out)
    out = np.where(e >= 31, sign | 0x7C00, out)
    return out.astype(np.uint16)


def test_gpu_snapshot_dtypes(gpu):
    st = seeds.small_state(16, True, seed=9)
    with Simulation(st.params, st.cols()) as sim:
        sim.step(3)
        f64 = sim.snapshot(DTYPE_F64)
        f32 = sim.snapshot(DTYPE_F32)
        f16 = sim.snapshot(DTYPE_F16)
    for a, b, c in zip(f64, f32, f16):
        assert np.array_equal(a.astype(np.float32), b)
        assert np.array_equal(_f16_trunc(a), c)


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("dtype", [DTYPE_F64, DTYPE_F32, DTYPE_F16])
def test_snapshot_async_matches_sync_while_stepping(gpu, prec, dtype):
    """An asynchronous snapshot holds the state of the moment it was taken even
    though steps are enqueued before its copy lands, and equals the
    synchronous snapshot bit for bit."""
    st = seeds.small_state(20, True, seed=4, precision=prec)
    with Simulation(st.params, st.cols()) as sim:
        sim.step(5)
        want = sim.snapshot(dtype)
        bufs = [np.empty_like(w) for w in want]
        sim.snapshot_async(bufs, dtype)
        sim.step(5)
        sim.snapshot_wait()
        later = sim.snapshot(dtype)
    for c, (b, w) in enumerate(zip(bufs, want)):
        assert np.array_equal(b.view(np.uint8), w.view(np.uint8)), c
    assert not np.array_equal(later[0], want[0])


@pytest.mark.parametrize("N,nsteps,damped", [(16, 40, False), (33, 60, True), (64, 200, False)])
def test_real_mode_matches_reference_binary(gpu, reference, N, nsteps, damped):
    """The reference's real 6-field mode (complex_phi = 0, compute_forces with
    its default terms) run by the reference CPU binary and by this library on
    the same seed: final frame per column and every diag TSV column; odd N and
    the absorbing sponge included."""
    over = dict(bc_type=0, damp_width=3.0, damp_rate=0.02) if damped else {}
    st = seeds.real_state(N, seed=9, **over)
    p = st.params
    every = nsteps // 4
    ref = oracle.run_reference(p, st.cols(), nsteps, diag_every=every)
    rows = []
    with Simulation(p, st.cols()) as sim:
        rows.append(sim.diag_vector())
        for _ in range(4):
            sim.step(every)
            rows.append(sim.diag_vector())
        got = sim.snapshot()
    assert len(got) == 12 and len(ref["cols"]) == 12
    assert worst_rel(got, ref["cols"]) < 1e-11
    want = np.asarray(ref["diag"])[:, 1:]                 # drop t; %.6e columns in the reference's TSV
    have = np.array(rows)[:, :want.shape[1]]
    assert np.all(np.abs(have - want) <= 2e-6 * np.abs(want) + 1e-12)


REAL_TERMS = [dict(mode=1), dict(mode=3), dict(alpha_cs=0.3), dict(beta_h=0.5), dict(kappa_h=0.2),
              dict(mode=3, alpha_cs=0.2, beta_h=0.3, kappa_h=0.1, bc_type=0, damp_width=3.0, damp_rate=0.02)]


@pytest.mark.parametrize("terms", REAL_TERMS, ids=lambda t: "-".join(f"{k}{v}" for k, v in t.items()))
def test_real_mode_optional_terms_match_reference_binary(gpu, reference, terms):
    """The real mode's optional terms (mass modes 1 and 3, Cosserat strain,
    curl-squared hardening, chiral helicity; compute_forces, scp_sim.c:743-929)
    on the separate real-mode kernels, against the reference CPU binary: final
    frame per column and every diag TSV column."""
    st = seeds.real_state(17, seed=21, **terms)
    p = st.params
    ref = oracle.run_reference(p, st.cols(), 40, diag_every=10)
    rows = []
    with Simulation(p, st.cols()) as sim:
        rows.append(sim.diag_vector())
        for _ in range(4):
            sim.step(10)
            rows.append(sim.diag_vector())
        got = sim.snapshot()
    assert len(got) == 12 and len(ref["cols"]) == 12
    assert worst_rel(got, ref["cols"]) < 1e-11
    want = np.asarray(ref["diag"])[:, 1:]
    have = np.array(rows)[:, :want.shape[1]]
    assert np.all(np.abs(have - want) <= 2e-6 * np.abs(want) + 1e-12)


@pytest.mark.parametrize("name", ["ref_real_n12", "ref_real_terms_n11_damped"])
def test_real_mode_matches_golden(gpu, name):
    """The real 6-field mode, plain and with every optional term under the
    sponge, against frames and diag rows the reference binary recorded
    (tests/golden/make_golden.py)."""
    import json
    f = np.load(os.path.join(GOLD, name + ".npz"))
    st = seeds.real_state(int(f["N"]), **json.loads(str(f["over"])))
    p = st.params
    every = int(f["diag_every"])
    rows = []
    with Simulation(p, st.cols()) as sim:
        rows.append(sim.diag_vector())
        for _ in range(int(f["nsteps"]) // every):
            sim.step(every)
            rows.append(sim.diag_vector())
        got = sim.snapshot()
    assert len(got) == 12 == f["final"].shape[0]
    assert worst_rel(got, f["final"]) < 1e-11
    want = np.asarray(f["diag"])[:, 1:]
    have = np.array(rows)[:, :want.shape[1]]
    assert np.all(np.abs(have - want) <= 2e-6 * np.abs(want) + 1e-12)


def test_real_mode_fp32c_tracks_fp64(gpu):
    """FP32-compensated real mode against the FP64 real mode after 100 steps."""
    from scp_b200 import PREC_FP32C
    st = seeds.real_state(24, seed=12)
    p64 = st.params
    p32 = Params(**{**p64.__dict__, "precision": PREC_FP32C})
    with Simulation(p64, st.cols()) as a, Simulation(p32, st.cols()) as b:
        a.step(100)
        b.step(100)
        A, B = a.snapshot(), b.snapshot()
    assert len(A) == len(B) == 12
    worst = max(rel_l2(B[c], A[c]) for c in range(12) if np.linalg.norm(A[c]) > 1e-3 * np.sqrt(len(A[c])))
    assert worst < 1e-5, worst


def test_gpu_initial_state_roundtrip(gpu):
    st = seeds.small_state(12, False, seed=4)
    with Simulation(st.params, st.cols()) as sim:
        got = sim.snapshot()
    for g, r in zip(got, st.cols()):
        assert np.array_equal(g, r.reshape(-1))


def test_gpu_gauss_projection_matches_oracle(gpu):
    st = seeds.make_state("c1", seeds.params_for("c1", N=32, L=7.75))
    o = oracle.Oracle(st.params, st.cols())
    with Simulation(st.params, st.cols()) as sim:
        inf = sim.info()
        got = sim.snapshot()
        d = sim.diag()
    ref = o.cols()
    for c in range(27, 30):   # E after projection
        assert rel_l2(got[c], ref[c]) < 1e-10
    assert abs(inf.G_offset - o.g_offset) < 1e-12
    assert d["gauss_max"] < 1e-11


@pytest.mark.parametrize("N", [32, 48, 13])
def test_gpu_gauss_spectral_start_matches_oracle(gpu, N):
    """The start-up projection begins from the direct spectral solve of the
    periodic 7-point problem (radix-2 for N = 32, the direct transform for
    48 and 13) and finishes with the reference's CG stopping rule: E, the
    frozen offset and the Gauss residual agree with the CPU checker, whose CG
    starts from zero and takes many more iterations."""
    L = (N - 1) / 4.0
    st = seeds.make_state("c1", seeds.params_for("c1", N=N, L=L))
    o = oracle.Oracle(st.params, st.cols())
    with Simulation(st.params, st.cols()) as sim:
        inf = sim.info()
        got = sim.snapshot()
        d = sim.diag()
    ref = o.cols()
    for c in range(27, 30):
        assert rel_l2(got[c], ref[c]) < 1e-10, c
    assert abs(inf.G_offset - o.g_offset) < 1e-12
    assert d["gauss_max"] < 1e-11
    assert inf.cg_iterations <= max(60, o.cg_iterations // 4), (inf.cg_iterations, o.cg_iterations)


def test_gpu_c0_64_1000_parity(gpu):
    """Config-0 workload: 1000 FP64 steps within 1e-10 relative L2 per field of
    the CPU checker, energy series identical to the printed precision, and
    sampled sites within 1e-10 of the reference's own run."""
    st = seeds.make_state("c0")
    p = st.params
    o = oracle.Oracle(p, st.cols())
    e_gpu, e_orc = [], []
    with Simulation(p, st.cols()) as sim:
        for _ in range(100):
            sim.step(10)
            o.step(10)
            e_gpu.append(sim.diag()["E_total"])
            e_orc.append(o.diag()[8])
        got = sim.snapshot()
    ref = o.cols()
    for c in range(24):
        assert rel_l2(got[c], ref[c]) < 1e-10, c
    e_gpu, e_orc = np.array(e_gpu), np.array(e_orc)
    assert np.max(np.abs(e_gpu - e_orc) / np.abs(e_orc)) < 1e-11
    f = np.load(os.path.join(GOLD, "ref_c0_64_1000.npz"))
    idx = f["sites"]
    for c in range(24):
        assert rel_l2(got[c][idx], f["sample"][c]) < 1e-10


def test_gpu_gauged_64_1000_parity(gpu):
    """Gauged 64^3 (two opposite balls, g = 0.1): 1000 steps within 1e-10 per
    field; the Gauss residual stays at roundoff."""
    st = seeds.make_state("c1", seeds.params_for("c1", N=64, L=15.75))
    p = st.params
    o = oracle.Oracle(p, st.cols())
    with Simulation(p, st.cols()) as sim:
        gmax = []
        for _ in range(10):
            sim.step(100)
            o.step(100)
            gmax.append(sim.diag()["gauss_max"])
        got = sim.snapshot()
        d = sim.diag()
    ref = o.cols()
    for c in range(30):
        assert rel_l2(got[c], ref[c]) < 1e-10, c
    assert max(gmax) < 1e-10
    r = o.diag()
    assert abs(d["E_total"] - r[8]) < 1e-11 * abs(r[8])


FP32C_CASES = [(n, g, t) for n in (13, 31, 32, 40) for g in (False, True) for t in (0, 1, 3, 4)]


@pytest.mark.parametrize("N,gauged,tile", FP32C_CASES)
def test_fp32c_shapes_match_oracle(gpu, N, gauged, tile):
    """FP32-compensated mode on every tile shape, with the two-site packed
    kernel (even N) and the one-site kernel (odd N), against the FP64 checker
    after 1 and 7 steps."""
    from scp_b200 import PREC_FP32C
    st = seeds.small_state(N, gauged, seed=N, tile_variant=tile)
    o = oracle.Oracle(st.params, st.cols())
    p32 = Params(**{**st.params.__dict__, "precision": PREC_FP32C})
    with Simulation(p32, st.cols()) as sim:
        assert sim.info().sites_per_thread == (2 if N % 2 == 0 else 1)
        for chunk in (1, 6):
            sim.step(chunk)
            o.step(chunk)
            got, want = sim.snapshot(), o.cols()
            errs = [rel_l2(g, w) for g, w in zip(got, want) if np.linalg.norm(w) > 1e-3 * np.sqrt(len(w))]
            assert max(errs) < 1e-5, (chunk, max(errs))


@pytest.mark.parametrize("N", [48, 47])
@pytest.mark.parametrize("gauged", [False, True])
def test_fp32c_tracks_fp64(gpu, gauged, N):
    """FP32-compensated mode against FP64 on the same seed: field L2 error
    and relative energy drift stay small over 400 steps (even N runs the
    two-site packed kernel, odd N the one-site kernel)."""
    from scp_b200 import PREC_FP32C
    L = (N - 1) / 4.0
    if gauged:
        st = seeds.make_state("c1", seeds.params_for("c1", N=N, L=L))
    else:
        st = seeds.make_state("c0", seeds.params_for("c0", N=N, L=L))
    p64 = st.params
    p32 = Params(**{**p64.__dict__, "precision": PREC_FP32C})
    with Simulation(p64, st.cols()) as a, Simulation(p32, st.cols()) as b:
        e0a, e0b = a.diag()["E_total"], b.diag()["E_total"]
        a.step(400)
        b.step(400)
        da, db = a.diag(), b.diag()
        A, B = a.snapshot(), b.snapshot()
    assert abs(e0a - e0b) <= 1e-6 * abs(e0a)
    worst = max(rel_l2(B[c], A[c]) for c in range(len(A)) if np.linalg.norm(A[c]) > 1e-3 * np.sqrt(len(A[c])))
    assert worst < 1e-5, worst
    assert abs(db["E_total"] - da["E_total"]) <= 1e-6 * abs(da["E_total"])
    if gauged:
        assert db["gauss_max"] < 1e-5
