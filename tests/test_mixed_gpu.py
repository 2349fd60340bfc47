"""Split precision (FP32 tendencies on phi - phibar, FP64 state accumulation)
against the FP64 GPU path, which the parity tests tie to the oracle.

Error measure: normalized L2 of the height h = phi/g over cell averages
(calc_VIA, src/diag_mod.F90:69-93) weighted by the cell areas
(doc/orderCheck.m:70-75).  Mass drift (M - M0)/M0 with the compensated
device sums.
"""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases, diag
from tests.helpers import GRAVITY

pytestmark = pytest.mark.gpu

TILE_TOL = 1e-6  # FP32 rounding of other per-tile residuals, after 3 steps


def normalized_l2(geom, a, b):
    return diag.norms(geom, a, b)[1]


def run(geom, st, precision, nsteps):
    with api.Stepper(st.order, st.nc, st.dt, st.scheme, precision=precision, radius=cases.EARTH_RADIUS) as s:
        s.set_geometry(geom)
        s.set_member(0, st.phi_s, st.u, st.v, st.phi)
        m0, e0 = s.mass_energy(0)
        s.step(nsteps)
        m1, e1 = s.mass_energy(0)
        return s.get_state(0), (m1 - m0) / m0


@pytest.mark.parametrize("order,scheme", [(3, "RK4"), (4, "RK3_TVD"), (4, "RK4"), (3, "RK3_TVD")])
def test_mixed_tracks_fp64(order, scheme):
    geom = api.Geometry(order, 24, cases.EARTH_RADIUS)
    st = cases.finish(geom, *cases.balanced_flow(geom, np.random.default_rng(8), 38.6, 0.05, 8, 20.0,
                                                  mountain=True)[:4], scheme, seconds=6 * 3600.0)
    ref, _ = run(geom, st, "fp64", st.nsteps)
    out, drift = run(geom, st, "mixed", st.nsteps)
    err = normalized_l2(geom, out["phi"] / GRAVITY, ref["phi"] / GRAVITY)
    assert err < 1e-6, err
    assert abs(drift) < 1e-10, drift
    H, n = geom.H, geom.n
    du = np.abs(out["u"] - ref["u"])[:, H:H + n, H:H + n].max() / np.abs(ref["u"]).max()
    assert du < 1e-4, du


def test_mixed_one_day_error_bound():
    """MCV4 RK3 at Nc=64 over one simulated day stays within the 1e-5 bound."""
    geom = api.Geometry(4, 64, cases.EARTH_RADIUS)
    st = cases.finish(geom, *cases.balanced_flow(geom, np.random.default_rng(9), 38.6, 0.05, 16, 20.0,
                                                  mountain=True)[:4], "RK3_TVD", seconds=86400.0)
    ref, _ = run(geom, st, "fp64", st.nsteps)
    out, drift = run(geom, st, "mixed", st.nsteps)
    err = normalized_l2(geom, out["phi"] / GRAVITY, ref["phi"] / GRAVITY)
    assert err < 1e-5, err
    assert abs(drift) < 1e-9, drift


def test_mixed_tile_shapes_agree():
    """Each tile subtracts its own linear reference before rounding to FP32, so
    tile shapes agree to FP32 rounding of the residuals (not bit for bit), and a
    shape run twice gives identical bits."""
    geom = api.Geometry(4, 20, cases.EARTH_RADIUS)
    st = cases.finish(geom, *cases.balanced_flow(geom, np.random.default_rng(5))[:4], "RK3_TVD", nsteps=3)
    outs = []
    with api.Stepper(4, 20, st.dt, "RK3_TVD", precision="mixed", radius=cases.EARTH_RADIUS) as s:
        s.set_geometry(geom)
        s.set_member(0, st.phi_s, st.u, st.v, st.phi)
        cands, _ = s.tuning()
        for i in list(range(len(cands))) + [0]:
            s.select_tile(i)
            s.set_member(0, st.phi_s, st.u, st.v, st.phi)
            s.step(3)
            outs.append(s.get_state(0))
    for k in ("u", "v", "phi"):
        assert np.array_equal(outs[-1][k], outs[0][k]), k
    H, n = geom.H, geom.n
    for i in range(1, len(outs) - 1):
        for k in ("u", "v", "phi"):
            a, b = outs[i][k][:, H:H + n, H:H + n], outs[0][k][:, H:H + n, H:H + n]
            d = np.abs(a - b).max() / np.abs(b).max()
            assert d < TILE_TOL, (i, k, d)


@pytest.mark.parametrize("order,scheme", [(3, "RK3_TVD"), (4, "RK3_TVD"), (4, "RK4")])
def test_every_shape_members_and_active_set(order, scheme):
    """Each candidate shape (the persistent TMA form included) with three
    members of which two are active: every active member equals a one-member
    run of the same shape bit for bit (a member's arithmetic reads only its own
    data, whichever work items and CTAs carry it), and the inactive member keeps
    its state.  Nc = 20 leaves ragged tiles for every shape."""
    geom = api.Geometry(order, 20, cases.EARTH_RADIUS)
    states = [cases.finish(geom, *cases.balanced_flow(geom, np.random.default_rng(40 + m), mountain=bool(m % 2))[:4],
                           scheme, nsteps=2) for m in range(3)]
    dt = min(st.dt for st in states)
    with api.Stepper(order, 20, dt, scheme, members=3, precision="mixed", radius=cases.EARTH_RADIUS) as s, \
            api.Stepper(order, 20, dt, scheme, members=1, precision="mixed", radius=cases.EARTH_RADIUS) as one:
        s.set_geometry(geom)
        one.set_geometry(geom)
        for m, st in enumerate(states):
            s.set_member(m, st.phi_s, st.u, st.v, st.phi)
        cands, _ = s.tuning()  # runs the autotuner, which needs the members
        for i in range(len(cands)):
            s.select_tile(i)
            one.select_tile(i)
            for m, st in enumerate(states):
                s.set_member(m, st.phi_s, st.u, st.v, st.phi)
            s.set_active([2, 0])
            s.step(2)
            for m in (0, 2):
                st = states[m]
                one.set_member(0, st.phi_s, st.u, st.v, st.phi)
                one.step(2)
                a, b = s.get_state(m), one.get_state(0)
                for k in ("u", "v", "phi"):
                    assert np.array_equal(a[k], b[k]), (cands[i][0], m, k)
            idle = s.get_state(1)
            for k in ("u", "v", "phi"):
                assert np.array_equal(idle[k], getattr(states[1], k)), (cands[i][0], k)
            s.set_active([0, 1, 2])


@pytest.mark.parametrize("order,nc", [(4, 3), (4, 8), (3, 5)])
def test_geometry_of_another_radius_is_rejected(order, nc):
    """Split precision recomputes the metric from the handle's radius, so a
    geometry built for another radius is refused; the matching one (panel
    centre on a point or not) is accepted."""
    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
    with api.Stepper(order, nc, 60.0, "RK3_TVD", precision="mixed", radius=cases.EARTH_RADIUS) as s:
        s.set_geometry(geom)
    with api.Stepper(order, nc, 60.0, "RK3_TVD", precision="mixed", radius=0.99 * cases.EARTH_RADIUS) as s:
        with pytest.raises(api.MCVError):
            s.set_geometry(geom)
