"""Regenerate the Q-conservation fixtures of tests/golden/ from the reference.

* profile_omega1.3900.txt: the radial Q-ball profile the reference's v66
  Q-conservation run reads (v66/cfg/qcons.cfg); the reference tree does not
  ship it, its own solver writes it (v66/radial_qball.c, built unmodified into
  oracle/_ref/radial_qball by `make -C oracle ref`).
* ref_qcons_v66.npz: the series the reference recorded for that run
  (v66/results/qcons_harness2.out: t, Q_total, Q_phi, Q_theta, s_max, E_total,
  r_core at every diag step of 1680 steps at 64^3, eta = 0, periodic).

Run in a checkout that has the reference tree:  python tests/golden/make_qcons.py
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.environ.get("SCP_REFERENCE", "")   # path of the kardianos/scp checkout (required)
SOLVER = os.path.join(ROOT, "oracle", "_ref", "radial_qball")
PROFILE = os.path.join(HERE, "profile_omega1.3900.txt")
SERIES = os.path.join(HERE, "ref_qcons_v66.npz")
COLUMNS = ("t", "Q_total", "Q_phi", "Q_theta", "s_max", "E_total", "r_core")


def write_profile(path: str) -> None:
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.run([SOLVER, "-omega", "1.39", "-profile", path, "-scan", os.path.join(tmp, "scan.tsv")],
                       check=True, capture_output=True, cwd=tmp)


def read_series(path: str) -> np.ndarray:
    rows = [[float(x) for x in ln.split()] for ln in open(path) if ln[:1].isdigit()]
    return np.array(rows)


if __name__ == "__main__":
    if not REF or not os.path.isdir(os.path.join(REF, "v66")):
        sys.exit("set SCP_REFERENCE to the path of the kardianos/scp checkout")
    if not os.path.exists(SOLVER):
        sys.exit("build the reference tools first: make -C oracle ref REF=$SCP_REFERENCE")
    write_profile(PROFILE)
    series = read_series(os.path.join(REF, "v66", "results", "qcons_harness2.out"))
    assert series.shape[1] == len(COLUMNS)
    np.savez_compressed(SERIES, columns=np.array(COLUMNS), series=series)
    print("wrote", PROFILE, "and", SERIES, series.shape)
