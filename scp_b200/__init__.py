"""scp_b200 -- B200 (sm_100a) lattice time-stepper for the complex / gauged
Cosserat Q-ball model of kardianos/scp ``sfa/sim``.

The compute path is libscpgpu.so (C ABI in include/scp_gpu.h, hand-written
CUDA in scp_b200/csrc/); this package holds the host-side mirror of the
reference's run parameters, seeded inputs and a ctypes face of the ABI.
"""
from .params import COLUMN_NAMES, DIAG_NAMES, PREC_FP32C, PREC_FP64, Params

__all__ = ["Params", "COLUMN_NAMES", "DIAG_NAMES", "PREC_FP64", "PREC_FP32C", "Simulation"]


def __getattr__(name):
    if name == "Simulation":
        from .api import Simulation
        return Simulation
    raise AttributeError(name)
