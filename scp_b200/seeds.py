"""Seeded synthetic initial states for the stepper (host side, numpy).

The reference has no generator for these inputs (its Gaussian and Q-ball
seeds come from separate seed tools or profile files), so the state is built
here and handed to both the CUDA library and the CPU checker as plain FP64
columns in the SFA column order.

Random numbers: SplitMix64 streams turned into normals by Box-Muller.  The
n-th 64-bit output of the stream with seed ``s`` is ``mix(s + (n+1)*G)`` with
``G = 0x9E3779B97F4A7C15`` and the SplitMix64 finaliser ``mix``; array ``j``
of a noise draw uses stream seed ``mix(seed + (j+1)*0xD1B54A32D192ED03)``.
Output pairs ``(a, b)`` give ``u1 = ((a>>11)+1)*2^-53``, ``u2 = (b>>11)*2^-53``
and the normals ``r*cos(2*pi*u2)``, ``r*sin(2*pi*u2)``, ``r = sqrt(-2 ln u1)``,
in that order.  ``N(0, var)`` below is a normal of variance ``var``.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Iterable, Sequence

import numpy as np

from .params import Params

_G = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)
_K = 0xD1B54A32D192ED03
_MASK = (1 << 64) - 1


def _mix(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def _mix_int(z: int) -> int:
    z &= _MASK
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
    return z ^ (z >> 31)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """First n outputs of the SplitMix64 stream with the given seed."""
    idx = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        return _mix(np.uint64(seed & _MASK) + idx * _G)


def normals(seed: int, stream: int, n: int) -> np.ndarray:
    """n standard normals of array ``stream`` under ``seed``."""
    s = _mix_int(seed + (stream + 1) * _K)
    m = (n + 1) // 2
    raw = splitmix64(s, 2 * m)
    a, b = raw[0::2], raw[1::2]
    u1 = ((a >> np.uint64(11)).astype(np.float64) + 1.0) * 2.0 ** -53
    u2 = (b >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    r = np.sqrt(-2.0 * np.log(u1))
    out = np.empty(2 * m)
    out[0::2] = r * np.cos(2.0 * math.pi * u2)
    out[1::2] = r * np.sin(2.0 * math.pi * u2)
    return out[:n]


@dataclasses.dataclass
class Ball:
    """Gaussian Q-ball seed Phi_a = A exp(-r^2/2 sigma^2) exp(i(2 pi a/3 + phase)),
    dPhi_a/dt = i omega Phi_a, centred at (x0, y0, z0) in physical units."""

    x0: float = 0.0
    y0: float = 0.0
    z0: float = 0.0
    omega: float = 0.8
    A: float = 1.0
    sigma: float = 3.0
    phase: float = 0.0
    phases: Sequence[float] | None = None   # per-component phases; default 2 pi a/3


class State(dict):
    """Column name -> (N,N,N) float64 array; ``cols()`` gives SFA order."""

    def __init__(self, params: Params):
        super().__init__()
        self.params = params
        n = params.N
        for name in params.input_names:
            self[name] = np.zeros((n, n, n))

    def cols(self) -> list[np.ndarray]:
        return [np.ascontiguousarray(self[n]) for n in self.params.input_names]


def coords(p: Params) -> np.ndarray:
    """Physical coordinates -L + i*dx of the grid points along one axis."""
    return -p.L + np.arange(p.N) * p.dx


def add_balls(st: State, balls: Iterable[Ball]) -> None:
    p = st.params
    x = coords(p)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    for b in balls:
        env = b.A * np.exp(-((X - b.x0) ** 2 + (Y - b.y0) ** 2 + (Z - b.z0) ** 2) / (2.0 * b.sigma ** 2))
        for a, ax in enumerate("xyz"):
            ph = (b.phases[a] if b.phases is not None else 2.0 * math.pi * a / 3.0) + b.phase
            re, im = env * math.cos(ph), env * math.sin(ph)
            st["phi_" + ax] += re
            st["phiim_" + ax] += im
            # dPhi/dt = i omega Phi  ->  du/dt = -omega v, dv/dt = omega u
            st["phi_v" + ax] += -b.omega * im
            st["phiim_v" + ax] += b.omega * re


def add_noise(st: State, names: Sequence[str], var: float, seed: int) -> None:
    """Add N(0, var) to each named column, array j of the list using stream j."""
    n3 = st.params.N ** 3
    sd = math.sqrt(var)
    for j, name in enumerate(names):
        st[name] += sd * normals(seed, j, n3).reshape(st[name].shape)


def real_state(N: int, seed: int = 5, L: float | None = None, **over) -> State:
    """A test state of the real 6-field mode (complex_phi = 0): two Gaussian
    blobs with different amplitudes per component on phi (the triple product
    P = phi_x phi_y phi_z is non-zero in their cores), a breathing velocity
    phi_v = -0.3 phi, and N(0, 1e-3) noise on theta and on every velocity."""
    L = L if L is not None else (N - 1) / 2.0 * 0.9
    kw = dict(N=N, L=L, dt_factor=0.2, bc_type=2, complex_gauge=0, real_fields=1)
    kw.update(over)
    p = Params(**kw)
    st = State(p)
    x = coords(p)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    sig = max(1.0, p.L / 4)
    for cx, amps in ((-0.3 * p.L, (1.0, 0.9, 1.1)), (0.3 * p.L, (0.8, 1.2, 1.0))):
        env = np.exp(-((X - cx) ** 2 + Y ** 2 + Z ** 2) / (2 * sig * sig))
        for a, ax in enumerate("xyz"):
            st["phi_" + ax] += amps[a] * env
            st["phi_v" + ax] += -0.3 * amps[a] * env
    add_noise(st, ("theta_x", "theta_y", "theta_z"), 1e-3, seed=seed)
    add_noise(st, ("phi_vx", "phi_vy", "phi_vz", "theta_vx", "theta_vy", "theta_vz"), 1e-3, seed=seed + 1)
    return st


def charge_density(st: State) -> np.ndarray:
    """rho = sum_a u v' - v u' + tu tv' - tv tu' (sfa/sim/scp_sim.c:153-160)."""
    rho = np.zeros_like(st["phi_x"])
    for ax in "xyz":
        rho += st["phi_" + ax] * st["phiim_v" + ax] - st["phiim_" + ax] * st["phi_v" + ax]
        rho += st["theta_" + ax] * st["thetaim_v" + ax] - st["thetaim_" + ax] * st["theta_v" + ax]
    return rho


def neutralise(st: State) -> float:
    """Remove the net Noether charge with a uniform phase-rotation velocity of
    Phi: du/dt -= eps v, dv/dt += eps u adds eps*|Phi|^2 to rho everywhere;
    eps is chosen so the total vanishes.  Returns eps."""
    rho = charge_density(st)
    s2 = sum(st["phi_" + ax] ** 2 + st["phiim_" + ax] ** 2 for ax in "xyz")
    eps = -float(rho.sum()) / float(s2.sum())
    for ax in "xyz":
        u, v = st["phi_" + ax].copy(), st["phiim_" + ax].copy()
        st["phi_v" + ax] -= eps * v
        st["phiim_v" + ax] += eps * u
    return eps


THETA_COLS = ("theta_x", "theta_y", "theta_z", "thetaim_x", "thetaim_y", "thetaim_z")
FIELD_COLS = ("phi_x", "phi_y", "phi_z", "phiim_x", "phiim_y", "phiim_z") + THETA_COLS


# ---------------------------------------------------------------- workloads

def params_for(name: str, **over) -> Params:
    """Grid and mode of the named workload (dx = 0.5, dt = 0.1, reference couplings)."""
    n = {"c0": 64, "c1": 128, "c2": 256, "c4": 512}[name]
    kw = dict(N=n, L=(n - 1) / 4.0, dt_factor=0.2, bc_type=2)
    if name in ("c1", "c2", "c4"):
        kw.update(complex_gauge=1, g_gauge=0.1)
    if name == "c4":
        kw.update(bc_type=0, damp_rate=0.0)
    kw.update(over)
    return Params(**kw)


def make_state(name: str, params: Params | None = None) -> State:
    """Initial state of a named workload.

    c0  one ball at the origin, omega = 0.8; theta ~ N(0, 1e-3) (seed 0).
    c1  two balls at x = -5, +5 (20 sites apart) with omega = -0.8, +0.8
        (opposite charges), theta ~ N(0, 1e-3) (seed 0); links 0, E from the
        start-up Gauss projection.
    c2  c1 plus N(0, 0.01) on every u, v, tu, tv (seed 1), net charge removed
        by neutralise().
    c4  eight co-phase balls (omega = 0.8) on the vertices of a cube of side
        6 sites (3.0) about the centre; theta ~ N(0, 1e-3) (seed 3).  Net
        charged, so it runs with bc_type=0 and damp_rate=0 (no sponge, frozen
        Gauss offset).
    """
    p = params or params_for(name)
    st = State(p)
    if name == "c0":
        add_balls(st, [Ball(omega=0.8)])
        add_noise(st, THETA_COLS, 1e-3, seed=0)
    elif name in ("c1", "c2"):
        add_balls(st, [Ball(x0=-5.0, omega=-0.8), Ball(x0=5.0, omega=0.8)])
        add_noise(st, THETA_COLS, 1e-3, seed=0)
        if name == "c2":
            add_noise(st, FIELD_COLS, 0.01, seed=1)
            neutralise(st)
    elif name == "c4":
        h = 1.5
        balls = [Ball(x0=sx * h, y0=sy * h, z0=sz * h, omega=0.8)
                 for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)]
        add_balls(st, balls)
        add_noise(st, THETA_COLS, 1e-3, seed=3)
    else:
        raise ValueError(name)
    return st


def small_state(N: int, gauged: bool, seed: int = 7, L: float | None = None, **over) -> State:
    """A small generic test state: two opposite balls plus noise on every
    field (and on the links when gauged), net charge removed."""
    L = L if L is not None else (N - 1) / 2.0 * 0.9
    kw = dict(N=N, L=L, dt_factor=0.2, bc_type=2, complex_gauge=1 if gauged else 0,
              g_gauge=0.1 if gauged else 0.05)
    kw.update(over)
    p = Params(**kw)
    st = State(p)
    w = 0.3 * p.L
    add_balls(st, [Ball(x0=-w, omega=-0.8, sigma=max(1.0, p.L / 4)),
                   Ball(x0=w, y0=0.5 * p.dx, omega=0.8, sigma=max(1.0, p.L / 4))])
    add_noise(st, FIELD_COLS, 1e-3, seed=seed)
    add_noise(st, ("phi_vx", "phiim_vy", "theta_vz", "thetaim_vx"), 1e-3, seed=seed + 100)
    if gauged:
        add_noise(st, ("th_x", "th_y", "th_z"), 0.05, seed=seed + 200)
    neutralise(st)
    return st


def mf_state(N: int, seed: int = 7, L: float | None = None, shift: float = 0.0, l_charge: float = 0.0,
             **over) -> State:
    """A three-fabric test state (n_fabrics = 3): fabric C and the links are
    small_state(N, gauged) with `seed`; fabrics Q and L are two more complex
    small states (seeds seed+1, seed+2; L's balls moved by `shift` along y).
    Each fabric is net-neutral by itself, so every choice of charges is,
    unless `l_charge` != 0 adds l_charge |Phi_L|^2 to L's charge density (for
    runs with the sponge, which have no net-charge check)."""
    over = dict(over, n_fabrics=3)
    st = small_state(N, True, seed=seed, L=L, **over)
    p = st.params
    from .params import COLUMN_NAMES, L_COLUMN_NAMES, Q_COLUMN_NAMES
    for names, sd in ((Q_COLUMN_NAMES, seed + 1), (L_COLUMN_NAMES, seed + 2)):
        f = small_state(N, False, seed=sd, L=p.L)
        if names is L_COLUMN_NAMES and shift:
            for k in list(f):
                f[k] = np.roll(f[k], int(round(shift / p.dx)), axis=1)
        for dst, src in zip(names, COLUMN_NAMES[:24]):
            st[dst] = f[src].copy()
    if l_charge:
        for ax in "xyz":
            u, v = st["lphi_" + ax].copy(), st["lphiim_" + ax].copy()
            st["lphi_v" + ax] -= l_charge * v
            st["lphiim_v" + ax] += l_charge * u
    return st
