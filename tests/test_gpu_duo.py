"""The gauged FP64 step with two threads per site (one for the Phi fields,
one for the Theta fields and links, exchanging their curls and current terms
through shared memory) against the one-thread-per-site step: the same terms
in the same order, so the two agree to roundoff, on full and partial tiles,
with and without the sponge, across several calls."""
import os

import numpy as np
import pytest

from scp_b200 import seeds
from scp_b200.api import Simulation

pytestmark = pytest.mark.gpu


def _run(params, cols, staging, calls):
    old = os.environ.get("SCP_STAGING")
    os.environ["SCP_STAGING"] = staging
    try:
        with Simulation(params, cols) as sim:
            form = sim.info().tma_staging
            for n in calls:
                sim.step(n)
            out = sim.snapshot()
            d = sim.diag_vector()
    finally:
        if old is None:
            del os.environ["SCP_STAGING"]
        else:
            os.environ["SCP_STAGING"] = old
    return form, out, d


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / nb if nb > 0 else np.linalg.norm(a - b)


CASES = [(32, {}), (64, {}), (40, {}), (13, {}), (48, dict(bc_type=0, damp_width=5.0, damp_rate=0.05))]


@pytest.mark.parametrize("N,over", CASES)
def test_duo_matches_one_thread_step(gpu, N, over):
    st = seeds.small_state(N, True, seed=N + 7, **over)
    calls = (1, 5, 6)
    f_duo, a, da = _run(st.params, st.cols(), "duo", calls)
    f_cp, b, db = _run(st.params, st.cols(), "cp", calls)
    assert f_duo == 3 and f_cp == 0
    for c, (x, y) in enumerate(zip(a, b)):
        assert rel(x, y) <= 1e-13, c
    # diag slots that cancel to roundoff (Gauss residual, net charges) compare absolutely
    assert np.allclose(da, db, rtol=1e-10, atol=1e-9)


def test_duo_is_gauged_fp64_only(gpu):
    """Ungauged grids and other tile shapes keep the one-thread step."""
    st = seeds.small_state(32, False, seed=5)
    form, _, _ = _run(st.params, st.cols(), "duo", (2,))
    assert form == 0
    st = seeds.small_state(32, True, seed=5, tile_variant=2)
    form, _, _ = _run(st.params, st.cols(), "duo", (2,))
    assert form == 0
