"""Host diagnostics against the oracle (no GPU): calc_VIA cell values with the
reference's weights (MCV4's /80 included) and mesh%areaCell, bit for bit."""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases, diag
from oracle.oracle import Oracle


@pytest.mark.parametrize("order,nc", [(3, 6), (4, 5)])
def test_cell_average_is_calc_via(order, nc):
    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
    o = Oracle(order, nc, 60.0, "RK4", cases.EARTH_RADIUS)
    f = np.random.default_rng(order).standard_normal(geom.shape)
    ref = o.calc_VIA(f)  # (6, nc+2, nc+2), halo cells 0
    assert np.array_equal(diag.cell_average(geom, f), ref[:, 1:-1, 1:-1])
    assert not ref[:, 0, :].any() and not ref[:, :, -1].any()


@pytest.mark.parametrize("order,nc", [(3, 6), (4, 16)])
def test_cell_areas_are_the_references(order, nc):
    o = Oracle(order, nc, 60.0, "RK4", cases.EARTH_RADIUS)
    assert np.array_equal(api.cell_areas(nc, cases.EARTH_RADIUS), o.mesh("areaCell"))


def test_norms_of_identical_fields_vanish():
    geom = api.Geometry(3, 6, cases.EARTH_RADIUS)
    f = 1.0 + np.random.default_rng(0).random(geom.shape)
    assert diag.norms(geom, f, f) == (0.0, 0.0, 0.0)
    l1, l2, linf = diag.norms(geom, 1.01 * f, f)
    assert abs(l1 - 0.01) < 1e-12 and abs(l2 - 0.01) < 1e-12 and abs(linf - 0.01) < 1e-12
