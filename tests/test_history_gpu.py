"""Device history staging and error norms against the oracle.

mcv_get_history runs the reference's history-output sequence (MCV_SW.F90:62-67:
addFillValue, convert_wind_P2SP over the whole padded array, calc_VIA of u, v,
phi) on the device; the oracle's orc_history restates it on the host.  After
the same steps (the FP64 path is within 1e-12 of the oracle), every output is
compared with relative L2 <= 1e-12 (the wind rotation's A IG is evaluated on
the device from the same formulas; its math library differs by a few ulp).
FillValue corners must match exactly.  The norms of mcv_height_error_norms
are checked against the host restatement of orderCheck.m (diag.norms).
"""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases, diag
from tests.helpers import oracle_for, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-12
FILL = -9999999999999999.0


def corners(a, H):
    return np.concatenate([a[:, :H, :H].ravel(), a[:, :H, -H:].ravel(), a[:, -H:, :H].ravel(),
                           a[:, -H:, -H:].ravel()])


def strip_corners(a, H):
    b = a.copy()
    b[:, :H, :H] = b[:, :H, -H:] = b[:, -H:, :H] = b[:, -H:, -H:] = 0.0
    return b


@pytest.mark.parametrize("order,nc,scheme,precision", [(3, 12, "RK4", "fp64"), (4, 10, "RK3_TVD", "fp64"),
                                                       (4, 10, "RK3_TVD", "mixed")])
def test_history_matches_oracle(order, nc, scheme, precision):
    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
    st = cases.finish(geom, *cases.balanced_flow(geom, np.random.default_rng(7), mountain=True)[:4], scheme,
                      nsteps=5)
    o = oracle_for(st)
    o.step(5)
    ref = o.history()
    with api.Stepper(order, nc, st.dt, scheme, precision=precision, radius=cases.EARTH_RADIUS) as s:
        s.set_geometry(geom)
        s.set_member(0, st.phi_s, st.u, st.v, st.phi)
        s.step(5)
        out = s.get_history(0)
        part = s.get_history(0, fields=("zonal", "phiC"))
    tol = TOL if precision == "fp64" else 1e-6  # split precision: FP32 tendencies
    H = geom.H
    for k in ("u", "v", "phi", "zonal", "merid"):
        assert np.array_equal(corners(out[k], H), corners(ref[k], H)) or k in ("zonal", "merid"), k
        err = rel_l2(strip_corners(out[k], H), strip_corners(ref[k], H))
        assert err <= tol, (k, err)
    for k in ("zonal", "merid"):  # the rotated FillValue corners
        assert rel_l2(corners(out[k], H), corners(ref[k], H)) <= 1e-14, k
    for k in ("uC", "vC", "phiC"):
        assert out[k].shape == (6, nc + 2, nc + 2)
        assert not out[k][:, 0, :].any() and not out[k][:, :, 0].any()
        err = rel_l2(out[k], ref[k])
        assert err <= tol, (k, err)
    assert np.array_equal(part["zonal"], out["zonal"]) and np.array_equal(part["phiC"], out["phiC"])


def test_history_cell_values_are_calc_via_bit_for_bit():
    """With the state taken from the device, the device's cell values are the
    reference's calc_VIA of it exactly (same weights, same order, no FMA)."""
    geom = api.Geometry(4, 9, cases.EARTH_RADIUS)
    st = cases.finish(geom, *cases.balanced_flow(geom, np.random.default_rng(8))[:4], "RK4", nsteps=2)
    o = oracle_for(st)
    with api.Stepper(4, 9, st.dt, "RK4", radius=cases.EARTH_RADIUS) as s:
        s.set_geometry(geom)
        s.set_member(0, st.phi_s, st.u, st.v, st.phi)
        s.step(2)
        out = s.get_history(0)
    for k, c in (("u", "uC"), ("v", "vC"), ("phi", "phiC")):
        assert np.array_equal(out[c], o.calc_VIA(out[k])), c


def test_device_norms_match_host():
    geom = api.Geometry(3, 16, cases.EARTH_RADIUS)
    st = cases.finish(geom, *cases.balanced_flow(geom, np.random.default_rng(9), mountain=True)[:4], "RK3_TVD",
                      nsteps=40)
    with api.Stepper(3, 16, st.dt, "RK3_TVD", precision="mixed", radius=cases.EARTH_RADIUS) as a, \
            api.Stepper(3, 16, st.dt, "RK3_TVD", precision="fp64", radius=cases.EARTH_RADIUS) as b:
        for s in (a, b):
            s.set_geometry(geom)
            s.set_member(0, st.phi_s, st.u, st.v, st.phi)
            s.step(40)
        dev = a.height_error_norms(0, b, 0)
        host = diag.norms(geom, a.get_state(0)["phi"], b.get_state(0)["phi"])
        same = b.height_error_norms(0, b, 0)
    assert same == (0.0, 0.0, 0.0)
    assert all(x > 0 for x in dev)
    for d, h in zip(dev, host):
        assert abs(d - h) <= 1e-9 * h, (dev, host)
