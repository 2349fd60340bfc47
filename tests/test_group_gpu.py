"""Several grids in one persistent launch (mcv_group_*): each grid of a group --
different Nc, dt and member counts, one order and arithmetic -- ends bit for bit
where the same handle stepped alone on the same stage-kernel candidate ends,
also with member subsets and with group steps interleaved with the handles'
own steps.  Reference: the per-grid time loop of src/MCV_SW.F90:57-60, run
once per grid."""
import numpy as np
import pytest

from mcv_sw_b200 import api, cases

pytestmark = pytest.mark.gpu

GRIDS = [(10, 1), (17, 2), (24, 3)]  # (nc, members)


def tma_candidate(stepper):
    cands, chosen = stepper.tuning()
    if cands[chosen][0][5] == 1:
        return chosen
    return max(i for i, (shape, _) in enumerate(cands) if shape[5] == 1)


def setup(order, precision, scheme):
    out = []
    for k, (nc, members) in enumerate(GRIDS):
        geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
        sts = [cases.finish(geom, *cases.balanced_flow(geom, np.random.default_rng(40 + 7 * k + m),
                                                        mountain=(m % 2 == 0))[:4], scheme, nsteps=1)
               for m in range(members)]
        out.append((geom, sts, min(st.dt for st in sts)))
    return out


def make(order, precision, scheme, grids, tile=None):
    steppers = []
    for geom, sts, dt in grids:
        s = api.Stepper(order, geom.nc, dt, scheme, members=len(sts), precision=precision,
                        radius=cases.EARTH_RADIUS)
        s.set_geometry(geom)
        for m, st in enumerate(sts):
            s.set_member(m, st.phi_s, st.u, st.v, st.phi)
        if tile is not None:
            s.select_tile(tile)
        steppers.append(s)
    return steppers


def states(steppers):
    return [[s.get_state(m) for m in range(s.members)] for s in steppers]


@pytest.mark.parametrize("order,precision,scheme", [(3, "fp64", "RK4"), (4, "fp64", "RK3_TVD"),
                                                    (3, "mixed", "RK4"), (4, "mixed", "RK3_TVD")])
def test_group_matches_each_handle_alone(order, precision, scheme):
    grids = setup(order, precision, scheme)
    probe = make(order, precision, scheme, grids[:1])[0]
    tile = tma_candidate(probe)
    probe.close()
    alone = make(order, precision, scheme, grids, tile)
    together = make(order, precision, scheme, grids, tile)
    # alone: 3 steps, member 0 of the last grid left out of 2 more, 2 more steps
    for s in alone:
        s.step(3)
    alone[2].set_active([1, 2])
    for s in alone:
        s.step(2)
    alone[2].set_active([0, 1, 2])
    alone[0].step(1)
    for s in alone:
        s.step(2)
    # the same schedule with group steps (and one step of grid 0 alone)
    with api.Group(together, tile=tile) as g:
        g.step(3)
        together[2].set_active([1, 2])
        g.step(2)
        together[2].set_active([0, 1, 2])
        together[0].step(1)
        g.step(2)
    a, b = states(alone), states(together)
    for k in range(len(GRIDS)):
        for m in range(GRIDS[k][1]):
            for f in ("u", "v", "phi"):
                assert np.array_equal(a[k][m][f], b[k][m][f]), (k, m, f)
    for s in alone + together:
        s.close()


def test_group_timing_and_errors():
    grids = setup(4, "mixed", "RK3_TVD")
    st = make(4, "mixed", "RK3_TVD", grids)
    tile = tma_candidate(st[0])
    with api.Group(st, tile=tile) as g:
        ms = g.time_steps(5)
        assert ms > 0
        assert g.query()
    with pytest.raises(api.MCVError):
        api.Group([st[0], st[0]])
    other = api.Stepper(3, 8, 60.0, "RK3_TVD", precision="mixed", radius=cases.EARTH_RADIUS)
    with pytest.raises(api.MCVError):
        api.Group([st[0], other])
    other.close()
    for s in st:
        s.close()
