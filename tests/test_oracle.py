"""Known-answer tests that pin the CPU oracle (no GPU).

The reference ships no tests or golden vectors and cannot be compiled here (no
Fortran compiler), so the oracle is pinned by properties its algorithm must
have (src/spatial_operators_mod.F90:204-234, src/ghost_mod.f90:183-227,
src/mesh_mod.F90:227-276, doc/orderCheck.m:63-81):
  * one-sided derivatives exact for polynomials of degree <= DOF-1;
  * the MCV interior-point formulas exact for polynomials of degree <= DOF-1;
  * the ghost interpolation exact for polynomials of degree <= DOF-1;
  * the cell areas of the equiangular cube summing to 4 pi R^2;
  * Williamson case 2 steady: error small, converging at about the MCV order,
    mass conserved to round-off.
"""
import math

import numpy as np
import pytest

from oracle.oracle import Oracle


def poly(coefs, x):
    return sum(c * x ** k for k, c in enumerate(coefs))


def dpoly(coefs, x):
    return sum(k * c * x ** (k - 1) for k, c in enumerate(coefs) if k)


@pytest.mark.parametrize("order", [3, 4])
def test_polyfit_exact(order):
    o = Oracle(order, 8, 100.0, "RK4")
    dx = o.dx
    rng = np.random.default_rng(0)
    for deg in range(order):
        c = rng.standard_normal(deg + 1)
        x = np.linspace(0.0, dx, order)  # the DOF points of one cell
        pv = poly(c, x)
        assert abs(o.polyfit(pv, right=False) - dpoly(c, 0.0)) < 1e-9 * (1 + abs(dpoly(c, 0.0)))
        assert abs(o.polyfit(pv, right=True) - dpoly(c, dx)) < 1e-9 * (1 + abs(dpoly(c, dx)))


@pytest.mark.parametrize("order", [3, 4])
def test_calc_tendP_exact(order):
    """Derivatives at the centre cell's points equal the exact derivative for a
    polynomial (the interface Riemann average sees equal left/right states)."""
    o = Oracle(order, 8, 100.0, "RK4")
    dx = o.dx
    rng = np.random.default_rng(1)
    W = 3 * order - 2
    x = (np.arange(W) - (order - 1)) * dx / (order - 1)
    for deg in range(order):
        c = rng.standard_normal(deg + 1)
        f = poly(c, x)
        d = o.calc_tendP(f, f, 0.7, 1.3)
        xc = x[order - 1: 2 * order - 1]
        assert np.allclose(d, dpoly(c, xc), rtol=1e-9, atol=1e-9)


@pytest.mark.parametrize("order", [3, 4])
def test_ghost_interp_exact(order):
    o = Oracle(order, 8, 100.0, "RK4")
    X = o.mesh("ghost_X")  # ghost points' coordinate along the edge
    n, dx = o.n, o.dx
    xs = -np.pi / 4 + np.arange(n) * dx / (order - 1)
    rng = np.random.default_rng(2)
    for deg in range(order):
        c = rng.standard_normal(deg + 1)
        for h in range(1, o.H + 1):
            got = o.linear_interp(poly(c, xs), h)
            assert np.allclose(got, poly(c, X[h - 1]), rtol=1e-10, atol=1e-10)


def test_ghost_weights_in_cell():
    o = Oracle(4, 16, 100.0, "RK4")
    iref, coef = o.mesh("ghost_iref"), o.mesh("ghost_coef")
    assert iref.min() >= 1 and iref.max() <= 16
    assert coef.min() >= 0 and coef.max() <= o.dx * (1 + 1e-12)


@pytest.mark.parametrize("nc", [8, 20])
def test_cell_areas_cover_sphere(nc):
    R = 6371220.0
    o = Oracle(3, nc, 100.0, "RK4", R)
    area = o.mesh("areaCell")[:, 1:nc + 1, 1:nc + 1]
    assert abs(area.sum() / (4 * math.pi * R * R) - 1.0) < 1e-12


def tc2(o):
    R, Om = 6371220.0, 7.292e-5
    lat = o.mesh("latP")
    u0 = 2 * np.pi * R / (12 * 86400.0)
    phi = 29400.0 - (R * Om * u0 + u0 ** 2 / 2.0) * np.sin(lat) ** 2
    o.set_phi_s(np.zeros_like(phi))
    o.init_state(u0 * np.cos(lat), np.zeros_like(phi), phi)
    return phi


@pytest.mark.parametrize("order,expect", [(3, 2.5), (4, 3.5)])
def test_tc2_converges(order, expect):
    errs = []
    for nc in (8, 16):
        dt = 3600.0 / nc
        o = Oracle(order, nc, dt, "RK4")
        phi0 = tc2(o)
        m0 = o.total_mass()
        o.step(int(6 * 3600 / dt))
        H, n = o.H, o.n
        d = o.state("phi")[:, H:H + n, H:H + n] - phi0[:, H:H + n, H:H + n]
        errs.append(np.sqrt(np.sum(d * d) / np.sum(phi0[:, H:H + n, H:H + n] ** 2)))
        assert abs(o.total_mass() - m0) / m0 < 1e-13
    rate = math.log(errs[0] / errs[1], 2)
    assert errs[1] < 1e-4 and rate > expect, (errs, rate)


def test_rk3_and_rk4_agree_on_smooth_flow():
    errs = {}
    for scheme in ("RK3_TVD", "RK4"):
        o = Oracle(4, 8, 300.0, scheme)
        tc2(o)
        o.step(12)
        errs[scheme] = o.state("phi")
    d = errs["RK3_TVD"] - errs["RK4"]
    H, n = 3, 25
    assert np.abs(d[:, H:H + n, H:H + n]).max() < 1e-3 * 29400
