"""Initial states generated on the device (mcv_set_member_balanced_flow) vs the
host init chain (cases.balanced_flow_from_spec + mcv_sphere_to_cov +
mcv_set_member) on the same seeded spec.

Tolerances: u, v, phi agree with the host chain's to 1e-13 of each field's
largest magnitude (device math library and summation order, a few ulp); mass
and energy to 1e-13 relative; FP64 steps from the device-built geometry and
state stay within the parity bar (relative L2 <= 1e-12) of the host-built run;
the generator is deterministic (bit-identical on repeated calls).
"""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases
from tests.helpers import interior, rel_l2

pytestmark = pytest.mark.gpu

CASES = [  # order, nc, precision, spec arguments
    (3, 8, "fp64", dict(lmax=8, rms=10.0, mountain=False)),
    (4, 12, "fp64", dict(lmax=16, rms=20.0, mountain=True, lmin=2)),
    (4, 10, "mixed", dict(lmax=8, rms=10.0, mountain=True)),
    (3, 16, "mixed", dict(lmax=0, mountain=True)),
    (4, 9, "fp64", dict(u0=25.0, alpha=1.1, lmax=32, rms=20.0, mountain=True)),
]


def host_state(geom, spec):
    zw, mw, phi, phis = cases.balanced_flow_from_spec(geom, spec)
    u, v = api.sphere_to_cov(geom, zw, mw)
    return phis, u, v, phi


@pytest.mark.parametrize("order,nc,precision,kw", CASES)
def test_device_state_matches_host_chain(order, nc, precision, kw):
    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
    spec = cases.balanced_flow_spec(geom, np.random.default_rng(7), **kw)
    phis, u, v, phi = host_state(geom, spec)
    with api.Stepper(order, nc, 60.0, "RK3_TVD", members=2, precision=precision, radius=cases.EARTH_RADIUS) as s:
        s.set_geometry(geom)
        s.set_member_balanced_flow(0, spec)
        s.set_member(1, phis, u, v, phi)
        dev, ref = s.get_state(0), s.get_state(1)
        if precision == "fp64":
            (m0, e0), (m1, e1) = s.mass_energy(0), s.mass_energy(1)
            assert abs(m0 - m1) <= 1e-13 * abs(m1) and abs(e0 - e1) <= 1e-13 * abs(e1)
    for k in ("u", "v", "phi"):
        d = np.abs(dev[k] - ref[k]).max() / np.abs(ref[k]).max()
        assert d <= 1e-13, (k, d)


def test_device_state_is_deterministic():
    geom = api.Geometry(4, 12, cases.EARTH_RADIUS)
    spec = cases.balanced_flow_spec(geom, np.random.default_rng(3), lmax=16, rms=15.0, mountain=True)
    with api.Stepper(4, 12, 60.0, "RK3_TVD", precision="mixed", radius=cases.EARTH_RADIUS) as s:
        s.set_geometry_equiangular()
        s.set_member_balanced_flow(0, spec)
        a = s.get_state(0)
        s.set_member_balanced_flow(0, spec)
        b = s.get_state(0)
    for k in ("u", "v", "phi"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("order,nc,scheme", [(3, 12, "RK4"), (4, 10, "RK3_TVD")])
def test_device_admission_steps_match_host_run(order, nc, scheme):
    """Geometry and state both built on the device, then stepped, vs the same
    run from the host-built geometry and state."""
    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
    spec = cases.balanced_flow_spec(geom, np.random.default_rng(11), lmax=8, rms=10.0, mountain=True)
    phis, u, v, phi = host_state(geom, spec)
    dt = cases.cfl_dt(geom, u, v, phi, 0.5)
    outs = []
    for device in (True, False):
        with api.Stepper(order, nc, dt, scheme, radius=cases.EARTH_RADIUS) as s:
            if device:
                s.set_geometry_equiangular()
                s.set_member_balanced_flow(0, spec)
            else:
                s.set_geometry(geom)
                s.set_member(0, phis, u, v, phi)
            s.step(20)
            outs.append(s.get_state(0))
    H, n = geom.H, geom.n
    for k in ("u", "v", "phi"):
        err = rel_l2(interior(outs[0][k], H, n), interior(outs[1][k], H, n))
        assert err <= 1e-12, (k, err)
