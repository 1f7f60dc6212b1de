"""Run parameters of the lattice stepper, mirroring the subset of the
reference ``Config`` (sfa/sim/scp_config.h:22-215) that the complex
(``complex_phi=1``) and gauged (``complex_gauge=1``) stepper reads.

Keys and defaults follow the reference: masses are given as ``m``/``m_theta``
and stored squared (scp_config.h:222-223), ``dx = 2L/(N-1)`` and
``dt = dt_factor*dx`` (sfa/sim/scp_sim.c:204-205).
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

PREC_FP64 = 0
PREC_FP32C = 1


class CParams(ctypes.Structure):
    """ctypes mirror of ``scp_gpu_params`` (include/scp_gpu.h)."""

    _fields_ = [
        ("N", ctypes.c_int32),
        ("L", ctypes.c_double),
        ("dx", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("m2", ctypes.c_double),
        ("mtheta2", ctypes.c_double),
        ("eta", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("kappa", ctypes.c_double),
        ("complex_gauge", ctypes.c_int32),
        ("g_gauge", ctypes.c_double),
        ("bc_type", ctypes.c_int32),
        ("damp_width", ctypes.c_double),
        ("damp_rate", ctypes.c_double),
        ("precision_mode", ctypes.c_int32),
        ("qdiag_radius", ctypes.c_double),
        ("qdiag_probe1", ctypes.c_double),
        ("qdiag_probe2", ctypes.c_double),
        ("gauss_project", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("tile_variant", ctypes.c_int32),
        ("real_fields", ctypes.c_int32),
        ("mode", ctypes.c_int32),
        ("inv_alpha", ctypes.c_double),
        ("inv_beta", ctypes.c_double),
        ("kappa_gamma", ctypes.c_double),
        ("alpha_cs", ctypes.c_double),
        ("beta_h", ctypes.c_double),
        ("kappa_h", ctypes.c_double),
        ("higgs_v", ctypes.c_double),
        ("higgs_lam", ctypes.c_double),
        ("higgs_kap", ctypes.c_double),
        ("higgs_rvoid", ctypes.c_double),
        ("g_gauge2", ctypes.c_double),
        ("gauge2_q", ctypes.c_double * 3),
        ("n_fabrics", ctypes.c_int32),
        ("mf_lock_CQ", ctypes.c_int32),
        ("q_fab", ctypes.c_double * 3),
    ]


@dataclasses.dataclass
class Params:
    """Grid, physics and mode settings of one simulation.

    Defaults are the reference defaults (scp_config.h:165-215) except the
    grid, which defaults to the 64^3, dx=0.5, dt=0.1 periodic case.
    """

    N: int = 64
    L: float = 15.75
    dt_factor: float = 0.2
    m: float = 1.5
    m_theta: float = 0.0
    eta: float = 0.5
    mu: float = -41.345
    kappa: float = 50.0
    complex_gauge: int = 0
    g_gauge: float = 0.05
    bc_type: int = 2
    damp_width: float = 3.0
    damp_rate: float = 0.01
    precision: int = PREC_FP64
    qdiag_radius: float = 8.0
    qdiag_probe1: float = 8.0
    qdiag_probe2: float = 16.0
    gauss_project: int = 1
    device: int = 0
    tile_variant: int = 0
    real_fields: int = 0      # 1: the reference's real 6-field mode (complex_phi = 0)
    # optional terms of the real mode (scp_config.h defaults)
    mode: int = 0
    inv_alpha: float = 2.25
    inv_beta: float = 5.0
    kappa_gamma: float = 2.0
    alpha_cs: float = 0.0
    beta_h: float = 0.0
    kappa_h: float = 0.0
    # extensions of the gauged stepper (scp_config.h defaults): Higgs condensate
    # (higgs_v > 0) and second compact U(1) gauge (g_gauge2 != 0)
    higgs_v: float = 0.0
    higgs_lam: float = 1.0
    higgs_kap: float = 2.0
    higgs_rvoid: float = 0.0
    g_gauge2: float = 0.0
    gauge2_q0: float = 1.0
    gauge2_q1: float = 1.0
    gauge2_q2: float = -2.0
    # three matter fabrics C, Q, L under the shared links (scp_config.h defaults)
    n_fabrics: int = 1
    mf_lock_CQ: int = 1
    q_C: float = 0.0
    q_Q: float = 1.0
    q_L: float = -1.0

    @property
    def dx(self) -> float:
        return 2.0 * self.L / (self.N - 1)

    @property
    def dt(self) -> float:
        return self.dt_factor * self.dx

    @property
    def m2(self) -> float:
        return self.m * self.m

    @property
    def mtheta2(self) -> float:
        return self.m_theta * self.m_theta

    @property
    def gauged(self) -> bool:
        return bool(self.complex_gauge) and self.g_gauge != 0.0

    @property
    def ncols(self) -> int:
        """Columns of an initial state (the second gauge starts at zero; three
        fabrics add Q and L, 24 each)."""
        if self.real_fields:
            return 12
        if self.n_fabrics == 3:
            return 78
        return 30 if self.complex_gauge else 24

    @property
    def input_names(self) -> tuple:
        if self.n_fabrics == 3:
            return COLUMN_NAMES[:30] + Q_COLUMN_NAMES + L_COLUMN_NAMES
        return COLUMN_NAMES[: self.ncols]

    @property
    def snap_names(self) -> tuple:
        if self.n_fabrics == 3:
            return COLUMN_NAMES[:30] + L_COLUMN_NAMES
        return COLUMN_NAMES[: self.snap_ncols]

    @property
    def gauge2(self) -> bool:
        return bool(self.complex_gauge) and self.g_gauge2 != 0.0

    @property
    def snap_ncols(self) -> int:
        """Columns of a snapshot: th2 and E2 follow when the second gauge is on;
        fabric L follows C with three fabrics."""
        if self.n_fabrics == 3:
            return 54
        return self.ncols + (6 if self.gauge2 else 0)

    def steps_for(self, T: float) -> int:
        """Step count of a run of length T, as the reference rounds it."""
        return int(math.floor(T / self.dt + 0.5))

    def to_c(self) -> CParams:
        c = CParams()
        c.N = self.N
        c.L = self.L
        c.dx = self.dx
        c.dt = self.dt
        c.m2 = self.m2
        c.mtheta2 = self.mtheta2
        c.eta = self.eta
        c.mu = self.mu
        c.kappa = self.kappa
        c.complex_gauge = 1 if self.complex_gauge else 0
        c.g_gauge = self.g_gauge
        c.bc_type = self.bc_type
        c.damp_width = self.damp_width
        c.damp_rate = self.damp_rate
        c.precision_mode = self.precision
        c.qdiag_radius = self.qdiag_radius
        c.qdiag_probe1 = self.qdiag_probe1
        c.qdiag_probe2 = self.qdiag_probe2
        c.gauss_project = self.gauss_project
        c.device = self.device
        c.tile_variant = self.tile_variant
        c.real_fields = 1 if self.real_fields else 0
        c.mode = self.mode
        c.inv_alpha = self.inv_alpha
        c.inv_beta = self.inv_beta
        c.kappa_gamma = self.kappa_gamma
        c.alpha_cs = self.alpha_cs
        c.beta_h = self.beta_h
        c.kappa_h = self.kappa_h
        c.higgs_v = self.higgs_v
        c.higgs_lam = self.higgs_lam
        c.higgs_kap = self.higgs_kap
        c.higgs_rvoid = self.higgs_rvoid
        c.g_gauge2 = self.g_gauge2
        c.gauge2_q[0] = self.gauge2_q0
        c.gauge2_q[1] = self.gauge2_q1
        c.gauge2_q[2] = self.gauge2_q2
        c.n_fabrics = self.n_fabrics
        c.mf_lock_CQ = self.mf_lock_CQ
        c.q_fab[0] = self.q_C
        c.q_fab[1] = self.q_Q
        c.q_fab[2] = self.q_L
        return c

    def to_cfg(self, **extra) -> str:
        """The same run as reference ``key = value`` config text."""
        kv = {
            "N": self.N, "L": repr(self.L), "dt_factor": repr(self.dt_factor),
            "m": repr(self.m), "m_theta": repr(self.m_theta), "eta": repr(self.eta),
            "mu": repr(self.mu), "kappa": repr(self.kappa), "complex_phi": 0 if self.real_fields else 1,
            "complex_gauge": int(self.complex_gauge), "g_gauge": repr(self.g_gauge),
            "bc_type": self.bc_type, "damp_width": repr(self.damp_width),
            "damp_rate": repr(self.damp_rate), "qdiag_radius": repr(self.qdiag_radius),
            "qdiag_probe1": repr(self.qdiag_probe1), "qdiag_probe2": repr(self.qdiag_probe2),
            "mode": self.mode, "inv_alpha": repr(self.inv_alpha), "inv_beta": repr(self.inv_beta),
            "kappa_gamma": repr(self.kappa_gamma), "alpha_cs": repr(self.alpha_cs), "beta_h": repr(self.beta_h),
            "kappa_h": repr(self.kappa_h),
            "higgs_v": repr(self.higgs_v), "higgs_lam": repr(self.higgs_lam), "higgs_kap": repr(self.higgs_kap),
            "higgs_rvoid": repr(self.higgs_rvoid), "g_gauge2": repr(self.g_gauge2),
            "gauge2_q0": repr(self.gauge2_q0), "gauge2_q1": repr(self.gauge2_q1), "gauge2_q2": repr(self.gauge2_q2),
            "n_fabrics": self.n_fabrics, "mf_lock_CQ": self.mf_lock_CQ,
            "q_C": repr(self.q_C), "q_Q": repr(self.q_Q), "q_L": repr(self.q_L),
        }
        kv.update(extra)
        return "".join(f"{k} = {v}\n" for k, v in kv.items())


# Column names of the SFA snapshot schema in registration order
# (sfa/sim/scp_sim.c:2862-2902; th2/E2 only with the second gauge).
COLUMN_NAMES = (
    "phi_x", "phi_y", "phi_z", "theta_x", "theta_y", "theta_z",
    "phi_vx", "phi_vy", "phi_vz", "theta_vx", "theta_vy", "theta_vz",
    "phiim_x", "phiim_y", "phiim_z", "thetaim_x", "thetaim_y", "thetaim_z",
    "phiim_vx", "phiim_vy", "phiim_vz", "thetaim_vx", "thetaim_vy", "thetaim_vz",
    "th_x", "th_y", "th_z", "E_x", "E_y", "E_z",
    "th2_x", "th2_y", "th2_z", "E2_x", "E2_y", "E2_z",
)

# Fabric L's snapshot columns (scp_sim.c:2907-2932), in the complex order
L_COLUMN_NAMES = (
    "lphi_x", "lphi_y", "lphi_z", "lth_x", "lth_y", "lth_z",
    "lphi_vx", "lphi_vy", "lphi_vz", "lth_vx", "lth_vy", "lth_vz",
    "lphiim_x", "lphiim_y", "lphiim_z", "lthim_x", "lthim_y", "lthim_z",
    "lphiim_vx", "lphiim_vy", "lphiim_vz", "lthim_vx", "lthim_vy", "lthim_vz",
)
# Fabric Q's initial columns (init only; the reference writes no Q columns)
Q_COLUMN_NAMES = tuple("q" + n[1:] for n in L_COLUMN_NAMES)

# Diagnostic slot names: the reference diag TSV columns after "t"
# (scp_sim.c:2993-3003), then centroid extras.
DIAG_NAMES = (
    "E_phi_kin", "E_theta_kin", "E_grad", "E_mass", "E_pot", "E_tgrad", "E_tmass",
    "E_coupling", "E_total", "phi_max", "P_max", "P_int", "theta_rms",
    "Q_phi", "Q_theta", "Q_total", "s_max", "r_core", "omega_core", "Q_core",
    "thp1u", "thp1v", "thp2u", "thp2v", "gauss_max", "gauss_l2", "E_em", "Q_flux",
    "Q_p0", "Q_p1", "Q_p2", "centroid_x", "centroid_y", "centroid_z",
    "Q_C", "Q_Q", "Q_L", "Q_em",
)
