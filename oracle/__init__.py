"""TEST INFRASTRUCTURE ONLY -- the parity checker.

Two CPU implementations of the reference's complex / gauged stepper, used by
tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs only:

* ``Oracle``: ctypes face of liboracle.so, the C restatement in scp_oracle.c.
* ``run_reference``: the reference binary itself (oracle/_ref/scp_sim, built
  unmodified from kardianos/scp sfa/sim/scp_sim.c by oracle/Makefile), fed
  through an SFA seed file and read back from its output frame and diag TSV.

The product (scp_b200, libscpgpu.so) never imports this package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "scp_sim")
REF_GPU_BIN = os.path.join(HERE, "_ref", "scp_sim_cuda")   # the reference's CUDA stepper (sm_100a)
SFA_TOOL = os.path.join(HERE, "_ref", "sfa_tool")
NDIAG = 31


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int), ("L", ctypes.c_double), ("dx", ctypes.c_double), ("dt", ctypes.c_double),
        ("m2", ctypes.c_double), ("mtheta2", ctypes.c_double), ("eta", ctypes.c_double),
        ("mu", ctypes.c_double), ("kappa", ctypes.c_double), ("gauge", ctypes.c_int),
        ("g", ctypes.c_double), ("bc_type", ctypes.c_int), ("damp_width", ctypes.c_double),
        ("damp_rate", ctypes.c_double), ("qdiag_radius", ctypes.c_double),
        ("qdiag_probe1", ctypes.c_double), ("qdiag_probe2", ctypes.c_double),
        ("higgs_v", ctypes.c_double), ("higgs_lam", ctypes.c_double), ("higgs_kap", ctypes.c_double),
        ("higgs_rvoid", ctypes.c_double), ("g2", ctypes.c_double), ("q2", ctypes.c_double * 3),
        ("n_fabrics", ctypes.c_int), ("mf_lock", ctypes.c_int), ("q_fab", ctypes.c_double * 3),
        ("real_fields", ctypes.c_int), ("mode", ctypes.c_int), ("inv_alpha", ctypes.c_double),
        ("inv_beta", ctypes.c_double), ("kappa_gamma", ctypes.c_double), ("alpha_cs", ctypes.c_double),
        ("beta_h", ctypes.c_double), ("kappa_h", ctypes.c_double),
    ]


_lib = None


def build(ref: str | None = None) -> None:
    """Compile liboracle.so and, given the path of a kardianos/scp checkout
    (argument, else the SCP_REFERENCE environment variable), the reference
    binaries under _ref/.  Without a checkout only liboracle.so is built."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    ref = ref or os.environ.get("SCP_REFERENCE")
    if ref and os.path.isdir(os.path.join(ref, "sfa", "sim")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.POINTER(OrcParams), ctypes.POINTER(vp), ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_int)]
        L.orc_create.restype = vp
        L.orc_free.argtypes = [vp]
        L.orc_step.argtypes = [vp, ctypes.c_int]
        L.orc_get.argtypes = [vp, ctypes.POINTER(vp)]
        L.orc_diag.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.orc_g_offset.argtypes = [vp]
        L.orc_g_offset.restype = ctypes.c_double
        L.orc_cg_iterations.argtypes = [vp]
        L.orc_accelerations.argtypes = [vp, ctypes.POINTER(vp)]
        L.orc_gauge_xform_test.argtypes = [vp, ctypes.POINTER(ctypes.c_double)]
        L.orc_gauge_xform_test.restype = ctypes.c_double
        _lib = L
    return _lib


def _orc_params(p) -> OrcParams:
    o = OrcParams()
    o.N, o.L, o.dx, o.dt = p.N, p.L, p.dx, p.dt
    o.m2, o.mtheta2, o.eta, o.mu, o.kappa = p.m2, p.mtheta2, p.eta, p.mu, p.kappa
    o.gauge = 1 if p.gauged else 0
    o.g = p.g_gauge
    o.bc_type, o.damp_width, o.damp_rate = p.bc_type, p.damp_width, p.damp_rate
    o.qdiag_radius, o.qdiag_probe1, o.qdiag_probe2 = p.qdiag_radius, p.qdiag_probe1, p.qdiag_probe2
    o.higgs_v, o.higgs_lam = getattr(p, "higgs_v", 0.0), getattr(p, "higgs_lam", 1.0)
    o.higgs_kap, o.higgs_rvoid = getattr(p, "higgs_kap", 2.0), getattr(p, "higgs_rvoid", 0.0)
    o.g2 = getattr(p, "g_gauge2", 0.0)
    for a, k in enumerate(("gauge2_q0", "gauge2_q1", "gauge2_q2")):
        o.q2[a] = getattr(p, k, (1.0, 1.0, -2.0)[a])
    o.n_fabrics, o.mf_lock = getattr(p, "n_fabrics", 1), getattr(p, "mf_lock_CQ", 1)
    for a, k in enumerate(("q_C", "q_Q", "q_L")):
        o.q_fab[a] = getattr(p, k, (0.0, 1.0, -1.0)[a])
    o.real_fields, o.mode = getattr(p, "real_fields", 0), getattr(p, "mode", 0)
    for k, d in (("inv_alpha", 2.25), ("inv_beta", 5.0), ("kappa_gamma", 2.0), ("alpha_cs", 0.0),
                 ("beta_h", 0.0), ("kappa_h", 0.0)):
        setattr(o, k, getattr(p, k, d))
    return o


class Oracle:
    """C restatement of the reference stepper holding one state."""

    def __init__(self, params, cols: Sequence[np.ndarray], project: bool = True):
        self.params = params
        self.ncols = params.ncols
        src = [np.ascontiguousarray(c, dtype=np.float64).reshape(-1) for c in cols]
        arr = (ctypes.c_void_p * self.ncols)(*[c.ctypes.data for c in src])
        st = ctypes.c_int(0)
        h = lib().orc_create(ctypes.byref(_orc_params(params)), arr, 1 if project else 0, ctypes.byref(st))
        if not h:
            raise RuntimeError(f"orc_create failed with status {st.value}")
        self._h = ctypes.c_void_p(h)

    def step(self, n: int) -> None:
        lib().orc_step(self._h, int(n))

    def cols(self) -> list[np.ndarray]:
        """Current state in snapshot column order (th2 / E2 or fabric L
        appended when those extensions are on)."""
        n3 = self.params.N ** 3
        nc = getattr(self.params, "snap_ncols", self.ncols)
        out = [np.empty(n3) for _ in range(nc)]
        arr = (ctypes.c_void_p * nc)(*[c.ctypes.data for c in out])
        lib().orc_get(self._h, arr)
        return out

    def diag(self) -> np.ndarray:
        """The reference diag TSV columns after t (31), and Q_C, Q_Q, Q_L, Q_em
        with three fabrics."""
        buf = (ctypes.c_double * 40)()
        n = lib().orc_diag(self._h, buf)
        return np.array(buf[:n])

    def accelerations(self) -> list[np.ndarray]:
        n3 = self.params.N ** 3
        out = [np.empty(n3) for _ in range(15)]
        arr = (ctypes.c_void_p * 15)(*[c.ctypes.data for c in out])
        lib().orc_accelerations(self._h, arr)
        return out

    @property
    def g_offset(self) -> float:
        return lib().orc_g_offset(self._h)

    @property
    def cg_iterations(self) -> int:
        return lib().orc_cg_iterations(self._h)

    def gauge_xform_test(self) -> tuple[float, np.ndarray]:
        rel = (ctypes.c_double * 10)()
        worst = lib().orc_gauge_xform_test(self._h, rel)
        return worst, np.array(rel[:])

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().orc_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- reference binary

def reference_available() -> bool:
    return os.path.exists(REF_BIN) and os.path.exists(SFA_TOOL)


def write_seed(path: str, params, cols: Sequence[np.ndarray]) -> None:
    raw = path + ".raw"
    np.concatenate([np.ascontiguousarray(c, dtype=np.float64).reshape(-1) for c in cols]).tofile(raw)
    subprocess.run([SFA_TOOL, "write", path, str(params.N), repr(params.L), repr(params.dt),
                    str(len(cols)), raw], check=True, capture_output=True)
    os.remove(raw)


def read_frame(path: str, frame: int, n3: int) -> tuple[list[str], list[np.ndarray]]:
    raw = path + f".f{frame}.raw"
    res = subprocess.run([SFA_TOOL, "read", path, str(frame), raw], check=True, capture_output=True, text=True)
    names = [ln.split()[0] for ln in res.stdout.strip().splitlines()]
    data = np.fromfile(raw)
    os.remove(raw)
    return names, [data[i * n3:(i + 1) * n3] for i in range(len(names))]


def read_diag(path: str) -> tuple[list[str], np.ndarray]:
    """Header and rows of a diag TSV (a list of rows when their lengths
    differ, as in the reference CUDA build's file)."""
    with open(path) as f:
        header = f.readline().rstrip("\n").split("\t")
        rows = [[float(x) for x in ln.split("\t") if x.strip()] for ln in f if ln.strip()]
    if len({len(r) for r in rows}) > 1:
        return header, rows
    return header, np.array(rows)


def run_reference(params, cols: Sequence[np.ndarray], nsteps: int, diag_every: int | None = None,
                  threads: int | None = None, workdir: str | None = None, extra_cfg: dict | None = None,
                  read_final: bool = True, binary: str | None = None) -> dict:
    """Run the reference binary (CPU by default, or `binary`, e.g. REF_GPU_BIN)
    on the given initial columns for nsteps.

    Returns {'cols': final columns (SFA order) or None, 'names', 'diag_header',
    'diag' rows, 'wall_ms_per_step', 'stdout'}.
    """
    if not reference_available():
        raise RuntimeError("reference binary not built (oracle/_ref)")
    tmp = tempfile.mkdtemp(prefix="scpref_", dir=workdir)
    seed = os.path.join(tmp, "seed.sfa")
    fabric_seeds = {}
    if getattr(params, "n_fabrics", 1) == 3:
        # fabric C with the links, then the L (and, unlocked, Q) seeds the
        # reference loads by init_sfa_L / init_sfa_Q (24-column complex files)
        write_seed(seed, params, cols[:30])
        fabric_seeds["init_sfa_L"] = os.path.join(tmp, "seed_L.sfa")
        write_seed(fabric_seeds["init_sfa_L"], params, cols[54:78])
        if not params.mf_lock_CQ:
            fabric_seeds["init_sfa_Q"] = os.path.join(tmp, "seed_Q.sfa")
            write_seed(fabric_seeds["init_sfa_Q"], params, cols[30:54])
    else:
        write_seed(seed, params, cols)
    T = nsteps * params.dt
    de = diag_every if diag_every else nsteps
    kv = dict(init="sfa", init_sfa=seed, init_frame=0, T=repr(T), precision="f64",
              output=os.path.join(tmp, "out.sfa"), diag_file=os.path.join(tmp, "diag.tsv"),
              snap_dt=repr(T if read_final else 1e9 * params.dt), diag_dt=repr(de * params.dt), **fabric_seeds)
    if extra_cfg:
        kv.update(extra_cfg)
    cfg = os.path.join(tmp, "run.cfg")
    with open(cfg, "w") as f:
        f.write(params.to_cfg(**kv))
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads or os.cpu_count() or 1)
    res = subprocess.run([binary or REF_BIN, cfg], capture_output=True, text=True, env=env, cwd=tmp)
    if res.returncode != 0:
        raise RuntimeError(f"reference run failed ({res.returncode}): {res.stderr[-2000:]}")
    wall = None
    for ln in res.stdout.splitlines():
        if ln.startswith("Wall:") and "ms/step" in ln:
            wall = float(ln.split()[-1].replace("ms/step", ""))
    out = {"stdout": res.stdout, "wall_ms_per_step": wall, "dir": tmp}
    hdr, rows = read_diag(os.path.join(tmp, "diag.tsv"))
    out["diag_header"], out["diag"] = hdr, rows
    if read_final:
        names, fc = read_frame(os.path.join(tmp, "out.sfa"), -1, params.N ** 3)
        out["names"], out["cols"] = names, fc
    return out
