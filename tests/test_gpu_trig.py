"""The step kernel's own bounded-argument sine/cosine (Cody-Waite reduction +
Taylor series, scp_b200/csrc/trig.cuh) against CUDA's sin/cos on device."""
import ctypes

import numpy as np
import pytest

from scp_b200 import native

pytestmark = pytest.mark.gpu


def test_trig_matches_cuda(gpu):
    rng = np.random.default_rng(0)
    x = np.concatenate([
        rng.uniform(-np.pi, np.pi, 200000),            # link angles
        rng.uniform(-4 * np.pi, 4 * np.pi, 200000),    # plaquette angles
        np.array([0.0, -0.0, np.pi, -np.pi, np.pi / 2, np.pi / 4, 3 * np.pi / 4, 1e-300, 4 * np.pi]),
        np.nextafter(np.pi / 4, 0) * np.arange(-16, 17),
    ])
    err = np.zeros(4)
    native.check(native.lib().scp_gpu_check_trig(len(x), x.ctypes.data, err.ctypes.data), "check_trig")
    assert err[0] <= 4.5e-16 and err[1] <= 4.5e-16, err      # FP64: within ~2 ulp of 1
    assert err[2] <= 3.0e-7 and err[3] <= 3.0e-7, err        # FP32: within ~2-3 ulp of 1
