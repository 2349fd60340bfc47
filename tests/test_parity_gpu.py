"""GPU step vs the CPU oracle on identical seeded inputs, through the C ABI.

Tolerance: relative L2 <= 1e-12 over the interior PVs (ids:ide, jds:jde, all
panels) of h = phi/g, u and v after the stated step count.  The operation order
differs (FMA contraction, recomputed contravariant winds), so the match is not
bit-exact.  Halo strips are compared too (same tolerance, relative to the
field's interior norm).
"""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases
from tests.helpers import GRAVITY, halo_strips, interior, oracle_for, rel_l2

TOL = 1e-12
TILE_TOL = 1e-13

pytestmark = pytest.mark.gpu


def run_pair(order, nc, scheme, nsteps, seed=11, members=1, mountain=False):
    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
    rng = np.random.default_rng(seed)
    zw, mw, phi, phis, meta = cases.balanced_flow(geom, rng, 38.6, 0.05, 8, 10.0, mountain=mountain)
    st = cases.finish(geom, zw, mw, phi, phis, scheme, nsteps=nsteps)
    o = oracle_for(st)
    o.step(nsteps)
    with api.Stepper(order, nc, st.dt, scheme, members=members) as s:
        s.set_geometry(geom)
        for m in range(members):
            s.set_member(m, st.phi_s, st.u, st.v, st.phi)
        s.step(nsteps)
        outs = [s.get_state(m) for m in range(members)]
    return geom, o, outs


def compare(geom, o, out):
    H, n = geom.H, geom.n
    ref = {k: o.state(k) for k in ("u", "v", "phi", "phiG")}
    errs = {}
    errs["h"] = rel_l2(interior(out["phi"], H, n) / GRAVITY, interior(ref["phi"], H, n) / GRAVITY)
    errs["u"] = rel_l2(interior(out["u"], H, n), interior(ref["u"], H, n))
    errs["v"] = rel_l2(interior(out["v"], H, n), interior(ref["v"], H, n))
    for k in ("u", "v", "phi"):
        scale = np.sqrt(np.sum(interior(ref[k], H, n) ** 2))
        d = np.sqrt(np.sum((halo_strips(out[k], H, n) - halo_strips(ref[k], H, n)) ** 2))
        errs["halo_" + k] = float(d / scale)
    return errs


@pytest.mark.parametrize("order", [3, 4])
@pytest.mark.parametrize("scheme", ["RK3_TVD", "RK4"])
def test_one_step(order, scheme):
    geom, o, outs = run_pair(order, 8, scheme, 1)
    errs = compare(geom, o, outs[0])
    assert max(errs.values()) <= TOL, errs


@pytest.mark.parametrize("order,nc,scheme,nsteps", [
    (3, 8, "RK4", 30), (4, 8, "RK4", 30), (3, 8, "RK3_TVD", 30), (4, 8, "RK3_TVD", 30),
    (3, 32, "RK4", 40), (4, 16, "RK3_TVD", 40), (3, 13, "RK3_TVD", 20), (4, 11, "RK4", 20),
])
def test_multi_step(order, nc, scheme, nsteps):
    geom, o, outs = run_pair(order, nc, scheme, nsteps, mountain=True)
    errs = compare(geom, o, outs[0])
    assert max(errs.values()) <= TOL, errs


def test_members_independent():
    geom, o, outs = run_pair(4, 8, "RK3_TVD", 10, members=3)
    for out in outs:
        errs = compare(geom, o, out)
        assert max(errs.values()) <= TOL, errs
    for out in outs[1:]:
        for k in ("u", "v", "phi"):
            assert np.array_equal(out[k], outs[0][k])


def test_mass_energy_matches_oracle():
    geom = api.Geometry(3, 8, cases.EARTH_RADIUS)
    st, _ = cases.small(seed=3, nc=8, geom=geom)
    o = oracle_for(st)
    o.step(5)
    with api.Stepper(3, 8, st.dt, "RK4") as s:
        s.set_geometry(geom)
        s.set_member(0, st.phi_s, st.u, st.v, st.phi)
        s.step(5)
        mass, energy = s.mass_energy(0)
    assert abs(mass - o.total_mass()) <= 1e-12 * abs(o.total_mass())
    assert abs(energy - o.total_energy()) <= 1e-12 * abs(o.total_energy())


def test_tc2_steady_state_on_gpu():
    """Williamson case 2 stays steady to the scheme's accuracy (orderCheck.m norms)."""
    geom = api.Geometry(4, 16, 6371220.0)
    zw, mw, phi, phis = api.williamson(geom, 2)
    u, v = api.sphere_to_cov(geom, zw, mw)
    with api.Stepper(4, 16, 300.0, "RK4") as s:
        s.set_geometry(geom)
        s.set_member(0, phis, u, v, phi)
        m0, _ = s.mass_energy(0)
        s.step(72)
        out = s.get_state(0)
        m1, _ = s.mass_energy(0)
    H, n = geom.H, geom.n
    err = rel_l2(interior(out["phi"], H, n), interior(phi, H, n))
    assert err < 5e-6, err
    assert abs(m1 - m0) / m0 < 1e-13


@pytest.mark.parametrize("order", [3, 4])
def test_every_tile_shape_agrees(order):
    """The autotuner's candidates change the schedule; the arithmetic differs
    only in how the compiler contracts a*b+c into FMA, so shapes agree to
    TILE_TOL (and each candidate stays within TOL of the oracle through the
    other tests, which run the autotuner's choice)."""
    geom = api.Geometry(order, 20, cases.EARTH_RADIUS)
    st = cases.finish(geom, *cases.balanced_flow(geom, np.random.default_rng(5), mountain=True)[:4], "RK4",
                      nsteps=3)
    outs = []
    with api.Stepper(order, 20, st.dt, "RK4") as s:
        s.set_geometry(geom)
        s.set_member(0, st.phi_s, st.u, st.v, st.phi)
        cands, chosen = s.tuning()
        assert len(cands) >= 2 and 0 <= chosen < len(cands)
        for i in list(range(len(cands))) + [0]:
            s.select_tile(i)
            s.set_member(0, st.phi_s, st.u, st.v, st.phi)
            s.step(3)
            outs.append(s.get_state(0))
    for k in ("u", "v", "phi"):
        assert np.array_equal(outs[-1][k], outs[0][k]), k  # a shape is deterministic
    H, n = geom.H, geom.n
    for i in range(1, len(outs) - 1):
        for k in ("u", "v", "phi"):
            a, b = interior(outs[i][k], H, n), interior(outs[0][k], H, n)
            d = np.abs(a - b).max() / np.abs(b).max()
            assert d < TILE_TOL, (i, k, d)


@pytest.mark.parametrize("order,nc,members", [(4, 96, 1), (3, 64, 2)])
def test_every_persistent_shape_over_many_items(order, nc, members):
    """The TMA-staged persistent shapes walk several work items per CTA here
    (MCV4 Nc=96: 864 items; MCV3 Nc=64, two members: 1,536), so the staging
    buffer and its mbarrier phase cycle: every such FP64 shape stays within TOL
    of the oracle after 3 RK4 steps, for an identity active list and for a
    permuted one."""
    nsteps = 3
    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
    st = cases.finish(geom, *cases.balanced_flow(geom, np.random.default_rng(17), mountain=True)[:4], "RK4",
                      nsteps=nsteps)
    o = oracle_for(st)
    o.step(nsteps)
    with api.Stepper(order, nc, st.dt, "RK4", members=members) as s:
        s.set_geometry(geom)
        for m in range(members):
            s.set_member(m, st.phi_s, st.u, st.v, st.phi)
        cands, _ = s.tuning()  # runs the autotuner, which needs the members
        persistent = [i for i, (shape, _) in enumerate(cands) if shape[5] == 1]
        assert persistent
        for i in persistent:
            for active in ([*range(members)], [*range(members)][::-1]):
                s.select_tile(i)
                for m in range(members):
                    s.set_member(m, st.phi_s, st.u, st.v, st.phi)
                s.set_active(active)
                s.step(nsteps)
                for m in range(members):
                    errs = compare(geom, o, s.get_state(m))
                    assert max(errs.values()) <= TOL, (cands[i][0], active, m, errs)
            s.set_active([*range(members)])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_set_state_replaces_the_state(precision):
    """mcv_set_state (u, v, phi only) continues like mcv_set_member with the
    same phi_s: bit for bit in FP64; split precision keeps the first state's
    mean-depth reference, a constant offset of E that drops out of the
    derivatives (rounding-level difference)."""
    geom = api.Geometry(4, 8, cases.EARTH_RADIUS)
    a, _ = cases.small(seed=3, nc=8, order=4, geom=geom)
    b, _ = cases.small(seed=4, nc=8, order=4, geom=geom)
    outs = []
    for first in (a, b):
        with api.Stepper(4, 8, a.dt, "RK4", precision=precision, radius=cases.EARTH_RADIUS) as s:
            s.set_geometry(geom)
            s.select_tile(0)
            s.set_member(0, b.phi_s, first.u, first.v, first.phi)
            if first is a:
                s.set_state(0, b.u, b.v, b.phi)
            s.step(3)
            outs.append(s.get_state(0))
    H, n = geom.H, geom.n
    for k in ("u", "v", "phi"):
        if precision == "fp64":
            assert np.array_equal(outs[0][k], outs[1][k]), k
        else:
            assert rel_l2(interior(outs[0][k], H, n), interior(outs[1][k], H, n)) < 1e-12, k
