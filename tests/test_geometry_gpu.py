"""Grid geometry computed on the device (mcv_set_geometry_equiangular) vs the
host builder (mcv_build_geometry), and FP64 steps on it vs the CPU oracle.

Tolerances: the metric planes agree with the host's to 1e-14 relative (the
device math library's tan/cos/atan2/pow differ by a few ulp); every ghost
point is located at the same coordinate to 1e-13 of the cell width (cell
indices differ only for points on a cell boundary); FP64
steps on the device geometry stay within the parity bar (relative L2 <= 1e-12)
of the oracle run on the host geometry.
"""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases
from tests.helpers import oracle_for
from tests.test_parity_gpu import TOL, compare

pytestmark = pytest.mark.gpu


def host_planes(geom):
    ig = geom.matrixIG.reshape(geom.shape + (4,))  # column-major 2x2: IG(1,1), IG(2,1), IG(1,2), IG(2,2)
    return {"sqrtG": geom.sqrtG, "ig11": ig[..., 0], "ig12": ig[..., 2], "ig22": ig[..., 3], "f": geom.f}


@pytest.mark.parametrize("order,nc,precision", [(3, 8, "fp64"), (4, 12, "mixed"), (4, 33, "fp64"), (3, 48, "mixed")])
def test_device_geometry_matches_host_builder(order, nc, precision):
    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
    with api.Stepper(order, nc, 60.0, "RK3_TVD", precision=precision, radius=cases.EARTH_RADIUS) as s:
        s.set_geometry_equiangular()
        dev = s.get_geometry()
    host = host_planes(geom)
    for k, ref in host.items():
        scale = np.abs(ref).max()
        err = np.abs(dev[k] - ref).max() / scale
        assert err <= 1e-14, (k, err)
    # every ghost point is located at the same panel-5 coordinate; a point on a
    # cell boundary (the panel corners map onto one) may be given as the end of
    # the lower cell or the start of the upper one -- the same point, whose
    # value either cell's polynomial interpolates -- depending on the last ulp
    # of tan/atan, so indices may differ there and only there
    pos_dev = (dev["ghost_iref"] - 1) * geom.dx + dev["ghost_coef"]
    pos_host = (geom.ghost_iref - 1) * geom.dx + geom.ghost_coef
    assert np.abs(pos_dev - pos_host).max() <= 1e-13 * geom.dx
    differ = dev["ghost_iref"] != geom.ghost_iref
    assert np.all(np.abs(dev["ghost_iref"] - geom.ghost_iref)[differ] == 1)
    at_tie = np.minimum(geom.ghost_coef, geom.dx - geom.ghost_coef) <= 1e-13 * geom.dx
    assert np.all(at_tie[differ])
    assert np.abs(dev["ghost_coef"] - geom.ghost_coef)[~differ].max() <= 1e-13 * geom.dx


def test_host_geometry_round_trip():
    """mcv_get_geometry returns what mcv_set_geometry installed, bit for bit."""
    geom = api.Geometry(4, 10, cases.EARTH_RADIUS)
    with api.Stepper(4, 10, 60.0, "RK4", radius=cases.EARTH_RADIUS) as s:
        s.set_geometry(geom)
        dev = s.get_geometry()
    for k, ref in host_planes(geom).items():
        assert np.array_equal(dev[k], ref), k
    assert np.array_equal(dev["ghost_iref"], geom.ghost_iref)
    assert np.array_equal(dev["ghost_coef"], geom.ghost_coef)


@pytest.mark.parametrize("order,nc,scheme,nsteps", [(3, 12, "RK4", 20), (4, 9, "RK3_TVD", 20)])
def test_steps_on_device_geometry_match_oracle(order, nc, scheme, nsteps):
    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
    zw, mw, phi, phis, _ = cases.balanced_flow(geom, np.random.default_rng(21), mountain=True)
    st = cases.finish(geom, zw, mw, phi, phis, scheme, nsteps=nsteps)
    o = oracle_for(st)
    o.step(nsteps)
    with api.Stepper(order, nc, st.dt, scheme, radius=cases.EARTH_RADIUS) as s:
        s.set_geometry_equiangular()
        s.set_member(0, st.phi_s, st.u, st.v, st.phi)
        s.step(nsteps)
        out = s.get_state(0)
    errs = compare(geom, o, out)
    assert max(errs.values()) <= TOL, errs


def test_split_precision_on_device_geometry():
    """Split precision reads the 1-D metric table; on the device-built table the
    run stays within split precision's own distance from FP64."""
    geom = api.Geometry(4, 12, cases.EARTH_RADIUS)
    st, _ = cases.small(seed=4, nc=12, order=4, scheme="RK3_TVD", geom=geom)
    outs = []
    for use_device in (False, True):
        with api.Stepper(4, 12, st.dt, "RK3_TVD", precision="mixed", radius=cases.EARTH_RADIUS) as s:
            if use_device:
                s.set_geometry_equiangular()
            else:
                s.set_geometry(geom)
            s.select_tile(0)
            s.set_member(0, st.phi_s, st.u, st.v, st.phi)
            s.step(20)
            outs.append(s.get_state(0))
    for k in ("u", "v", "phi"):
        a, b = outs[1][k], outs[0][k]
        H, n = geom.H, geom.n
        d = np.abs(a[:, H:H + n, H:H + n] - b[:, H:H + n, H:H + n]).max() / np.abs(b[:, H:H + n, H:H + n]).max()
        assert d < 1e-6, (k, d)
