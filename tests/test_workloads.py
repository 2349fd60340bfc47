"""The CPU reference arm's workloads (oracle/workloads.py: the oracle's mesh and
IC routines, no GPU library) are the product's workloads (mcv_sw_b200/cases.py
through the library's host init chain): same seeded draws, same dt, and the
same covariant state bit for bit."""
import numpy as np

from mcv_sw_b200 import cases
from oracle import workloads


def test_spec_draws_match():
    for seed, kw in [(1, dict(lmax=8, rms=10.0)), (2, dict(lmax=32, rms=20.0, mountain=True))]:
        a = cases.balanced_flow_spec(cases._Radius(cases.EARTH_RADIUS), np.random.default_rng(seed), 38.6, 0.05, **kw)
        b = workloads.draw_balanced_spec(np.random.default_rng(seed), 38.6, 0.05, **kw)
        assert a["gh0"] == b["gh0"] and np.array_equal(a["coef"], b["coef"])
        assert a["mountain"] == b["mountain"]


def test_small_workload_is_the_products():
    w, desc = workloads.build("small")
    st, geom = cases.small(seed=1)
    assert w.dt == st.dt and w.nsteps == st.nsteps
    assert np.array_equal(w.lon, geom.lonP) and np.array_equal(w.sqrtG, geom.sqrtG)
    for k in ("u", "v", "phi"):
        assert np.array_equal(w.o.state(k), getattr(st, k)), k
