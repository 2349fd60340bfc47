"""FP64 GPU path vs the CPU oracle on the benchmark configurations themselves.

Tolerance: relative L2 <= 1e-12 over the interior PVs of h = phi/g, u and v
(and the halo strips, relative to the field's interior norm) after the stated
step counts, as in test_parity_gpu.py:
  - the reference-method case, MCV3 Nc=32 RK4, seeded balanced tilted flow with
    degree 1-8 harmonics (RMS 10 m), for its full simulated day (557 steps);
  - one member of the 64-member MCV3 Nc=128 RK4 ensemble, the one whose jet
    axis is tilted nearest pi/2 (alpha = 1.546: the flow crosses the cube's
    corners), 30 steps;
  - the single large instance, MCV4 Nc=256 RK3_TVD with degree <= 32
    harmonics and the 2000 m mountain, 10 steps.
The oracle restates src/time_scheme_mod.F90:13-69 (RK4, RK3_TVD) with the
spatial operator and halo correction in the reference's evaluation order.
"""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases
from tests.helpers import oracle_for
from tests.test_parity_gpu import TOL, compare

pytestmark = pytest.mark.gpu


def run(st, geom, nsteps, precision="fp64"):
    o = oracle_for(st)
    o.step(nsteps)
    with api.Stepper(st.order, st.nc, st.dt, st.scheme, precision=precision, radius=cases.EARTH_RADIUS) as s:
        s.set_geometry(geom)
        s.set_member(0, st.phi_s, st.u, st.v, st.phi)
        s.step(nsteps)
        out = s.get_state(0)
    return compare(geom, o, out)


def test_reference_case_full_day():
    st, geom = cases.small(seed=1)
    assert st.order == 3 and st.nc == 32 and st.scheme == "RK4"
    assert abs(st.nsteps * st.dt - 86400.0) < 1e-6 and st.nsteps == 557
    errs = run(st, geom, st.nsteps)
    assert max(errs.values()) <= TOL, errs


def test_ensemble_member_across_the_corners():
    geom = api.Geometry(3, 128, cases.EARTH_RADIUS)
    st = cases.ensemble_member(geom, 1060)
    assert st.meta["alpha"] > 1.5
    errs = run(st, geom, 30)
    assert max(errs.values()) <= TOL, errs


def test_large_instance_ten_steps():
    st, geom = cases.large(seed=2)
    assert st.order == 4 and st.nc == 256 and st.scheme == "RK3_TVD"
    errs = run(st, geom, 10)
    assert max(errs.values()) <= TOL, errs
