"""Failure detection without a GPU fault: the bounded wait that guards the
stage kernels' staged copies gives up when nothing completes its barrier,
reports it to the host, and leaves the context usable.

Tolerances: a wait that nothing completes gives up no earlier than its limit
and well before ten times it; a completed barrier is passed in under 5 ms.
"""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("limit_ms", [5.0, 40.0])
def test_wait_on_a_barrier_nothing_completes_gives_up(limit_ms):
    timed_out, elapsed = api.selftest_wait(False, limit_ms)
    assert timed_out
    assert limit_ms <= elapsed < 10 * limit_ms + 50.0, elapsed


def test_wait_on_a_completed_barrier_passes():
    timed_out, elapsed = api.selftest_wait(True, 1000.0)
    assert not timed_out
    assert elapsed < 5.0, elapsed


def test_context_usable_after_a_timed_out_wait():
    assert api.selftest_wait(False, 5.0)[0]
    geom = api.Geometry(3, 8, cases.EARTH_RADIUS)
    st, _ = cases.small(seed=2, nc=8, geom=geom)
    with api.Stepper(3, 8, st.dt, "RK4", radius=cases.EARTH_RADIUS) as s:
        s.set_geometry(geom)
        s.set_member(0, st.phi_s, st.u, st.v, st.phi)
        s.step(3)  # mcv_step -> mcv_sync: no stage error flag raised
        out = s.get_state(0)
    assert all(np.isfinite(out[k][:, geom.H:-geom.H, geom.H:-geom.H]).all() for k in ("u", "v", "phi"))
