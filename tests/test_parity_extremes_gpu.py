"""GPU step vs the CPU oracle at the extremes of the grid size: the smallest
grids (Nc = 2, 3: one ragged tile covers a whole panel, and the staged boxes
reach past every edge of the arrays) for every tile shape of both arithmetic
policies, and the full MCV4 Nc=256 grid of the headline configuration.

Tolerances: FP64 relative L2 <= 1e-12 of h = phi/g, u, v over the interior
PVs (the parity bar); split precision within 1e-6 normalized L2 of FP64 in h
and with mass conserved to 1e-9 after the same steps (FP32 rounding of the
increments on a few hundred points does not average out).
"""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases, diag
from tests.helpers import GRAVITY, oracle_for
from tests.test_parity_gpu import TOL, compare

pytestmark = pytest.mark.gpu


def seeded(order, nc, scheme, nsteps, seed, geom=None, **kw):
    geom = geom or api.Geometry(order, nc, cases.EARTH_RADIUS)
    zw, mw, phi, phis, _ = cases.balanced_flow(geom, np.random.default_rng(seed), **kw)
    return geom, cases.finish(geom, zw, mw, phi, phis, scheme, nsteps=nsteps)


@pytest.mark.parametrize("order,nc,scheme", [(3, 2, "RK4"), (4, 2, "RK3_TVD"), (3, 3, "RK3_TVD"), (4, 3, "RK4")])
def test_smallest_grids_every_shape(order, nc, scheme):
    nsteps = 10
    geom, st = seeded(order, nc, scheme, nsteps, 31, lmax=2, rms=10.0)
    o = oracle_for(st)
    o.step(nsteps)
    fp64_out = None
    for precision in ("fp64", "mixed"):
        with api.Stepper(order, nc, st.dt, scheme, precision=precision, radius=cases.EARTH_RADIUS) as s:
            s.set_geometry(geom)
            s.set_member(0, st.phi_s, st.u, st.v, st.phi)
            cands, _ = s.tuning()
            for i in range(len(cands)):
                s.select_tile(i)
                s.set_member(0, st.phi_s, st.u, st.v, st.phi)
                m0, _ = s.mass_energy(0)
                s.step(nsteps)
                m1, _ = s.mass_energy(0)
                out = s.get_state(0)
                if precision == "fp64":
                    errs = compare(geom, o, out)
                    assert max(errs.values()) <= TOL, (cands[i][0], errs)
                    fp64_out = out
                else:
                    err = diag.norms(geom, out["phi"] / GRAVITY, fp64_out["phi"] / GRAVITY)[1]
                    assert err < 1e-6, (cands[i][0], err)
                    assert abs(m1 - m0) / m0 < 1e-9, (cands[i][0], m1, m0)


def test_full_size_headline_grid():
    """MCV4 Nc=256 RK3_TVD (3,548,166 PVs per field), the benchmark's seeded
    state: one FP64 step against the oracle, split precision against FP64."""
    st, geom = cases.large(seed=2)
    o = oracle_for(st)
    o.step(1)
    outs = {}
    for precision in ("fp64", "mixed"):
        with api.Stepper(st.order, st.nc, st.dt, st.scheme, precision=precision, radius=cases.EARTH_RADIUS) as s:
            s.set_geometry(geom)
            s.set_member(0, st.phi_s, st.u, st.v, st.phi)
            s.step(1)
            outs[precision] = s.get_state(0)
    errs = compare(geom, o, outs["fp64"])
    assert max(errs.values()) <= TOL, errs
    err = diag.norms(geom, outs["mixed"]["phi"] / GRAVITY, outs["fp64"]["phi"] / GRAVITY)[1]
    assert err < 1e-6, err
