"""Failure detection without a GPU fault: a halo-box load that never arrives
(injected by fvb_debug_drop_load: the copy is simply not issued) makes the
stage kernel's bounded mbarrier wait run out after one second of GPU time;
the kernel ends normally, the solver reports FVB_ERR_TIMEOUT and stops
stepping, and the GPU context stays usable for the next solver."""
from __future__ import annotations

import time

import numpy as np
import pytest

import fvstuff_b200 as F

pytestmark = pytest.mark.gpu

FVB_ERR_TIMEOUT = 7


@pytest.mark.parametrize("precision", ["f64", "f32c"])
def test_lost_halo_load_times_out_and_context_survives(precision):
    n = 96
    s = F.Solver(n, bc="periodic", precision=precision, x0=-5, y0=-5, length=10.0)
    s.init_case("vortex")
    s.step(2)
    assert s.sync().status == 0
    s.debug_drop_load()
    t0 = time.perf_counter()
    s.step(3)
    st = s.sync()
    waited = time.perf_counter() - t0
    assert st.status == FVB_ERR_TIMEOUT
    assert 0.9 < waited < 30.0
    # the solver stops stepping, as after a blow-up
    s.step(2)
    assert s.sync().steps == st.steps
    # the context is intact: a fresh solver runs and its result is finite
    s2 = F.Solver(n, bc="periodic", precision=precision, x0=-5, y0=-5, length=10.0)
    s2.init_case("vortex")
    s2.step(4)
    st2 = s2.sync()
    assert st2.status == 0 and st2.steps == 4
    assert np.isfinite(s2.get_state()).all()
