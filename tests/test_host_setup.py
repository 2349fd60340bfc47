"""The product's host-side init chain (mcv_build_geometry, initial-condition
helpers) against the oracle's restatement of initMesh / initGhost /
initTestCase: bit-identical, since the GPU step takes these arrays as input."""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases
from oracle.oracle import Oracle


@pytest.mark.parametrize("order,nc", [(3, 8), (4, 8), (3, 13), (4, 32), (3, 48)])
def test_geometry_bit_identical(order, nc):
    g = api.Geometry(order, nc, 6.371e6)
    o = Oracle(order, nc, 100.0, "RK4", 6.371e6)
    for name in ("lonP", "latP", "sqrtG", "f", "matrixG", "matrixIG", "matrixA", "matrixIA"):
        assert np.array_equal(getattr(g, name), o.mesh(name)), name
    assert np.array_equal(g.ghost_iref, o.mesh("ghost_iref"))
    assert np.array_equal(g.ghost_coef, o.mesh("ghost_coef"))


def test_grid_sizes():
    assert api.grid_sizes(3, 32) == (69, 65, 2)
    assert api.grid_sizes(4, 256) == (775, 769, 3)
    with pytest.raises(api.MCVError):
        api.grid_sizes(5, 32)


def test_sphere_to_cov_matches_init_test_case():
    g = api.Geometry(4, 8, 6.371e6)
    o = Oracle(4, 8, 100.0, "RK4", 6.371e6)
    zw, mw, phi, phis = api.williamson(g, 5)
    o.set_phi_s(phis)
    o.init_state(zw, mw, phi)
    u, v = api.sphere_to_cov(g, zw, mw)
    assert np.array_equal(u, o.state("u"))
    assert np.array_equal(v, o.state("v"))
    assert np.array_equal(phi * g.sqrtG, o.state("phiG"))


def test_williamson_case2_formula():
    g = api.Geometry(3, 8, 6371220.0)
    zw, mw, phi, phis = api.williamson(g, 2)
    R, Om = 6371220.0, 7.292e-5
    u0 = 2.0 * (2.0 * np.arcsin(1.0)) * R / (12.0 * 86400.0)
    s = np.sin(g.latP)
    assert np.array_equal(phi, 29400.0 - (R * Om * u0 + u0 * u0 / 2.0) * (s * s))
    assert np.array_equal(zw, u0 * np.cos(g.latP))
    assert not mw.any() and not phis.any()


def test_harmonics_orthonormal():
    """Each real harmonic has unit mean square over the unit sphere / (4 pi)."""
    g = api.Geometry(4, 24, 1.0)
    for l, m in ((1, 0), (3, 2), (5, -4), (8, 8)):
        c = np.zeros((8 + 1) ** 2)
        c[l * l + l + m] = 1.0
        h = np.zeros(g.shape)
        api.add_harmonics(g, h, c)
        w = g.pv_weights() * g.sqrtG
        ms = np.sum(w * h * h) / np.sum(w)
        assert abs(ms * 4 * np.pi - 1.0) < 1e-6, (l, m, ms)


def test_seeded_states_reproducible():
    a, g = cases.small(seed=7, nc=8)
    b, _ = cases.small(seed=7, nc=8, geom=g)
    for k in ("u", "v", "phi", "phi_s"):
        assert np.array_equal(getattr(a, k), getattr(b, k))
    base = api.tilted_zonal(g, cases.equator_gh0(38.6, g.radius), 38.6, 0.05)[2]
    h = (a.phi - base) / cases.GRAVITY
    assert abs(cases.area_mean(g, base) - cases.GH0) < 5.0
    assert abs(cases.area_rms(g, h) - 10.0) < 1e-9
    assert a.nsteps * a.dt == pytest.approx(86400.0)
