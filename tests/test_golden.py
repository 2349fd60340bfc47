"""Committed golden fixtures (tests/golden/, made by make_golden.py from the
oracle): the oracle reproduces them bit-exactly (CPU), and the GPU step
reproduces the step fixtures within relative L2 1e-12 (GPU)."""
import glob
import os

import numpy as np
import pytest

from mcv_sw_b200 import api, cases
from oracle.oracle import Oracle
from tests.helpers import interior, rel_l2

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
STEP_FIXTURES = sorted(glob.glob(os.path.join(GOLD, "step_*.npz")))


def load(path):
    z = np.load(path, allow_pickle=False)
    return {k: z[k] for k in z.files}


def test_fixtures_present():
    assert len(STEP_FIXTURES) == 4 and os.path.exists(os.path.join(GOLD, "kernels.npz"))


@pytest.mark.parametrize("path", STEP_FIXTURES, ids=os.path.basename)
def test_oracle_reproduces_step_fixture(path):
    g = load(path)
    order, nc, scheme = int(g["order"]), int(g["nc"]), str(g["scheme"])
    o = Oracle(order, nc, float(g["dt"]), scheme, cases.EARTH_RADIUS)
    o.set_phi_s(g["phi_s"])
    o.init_state(g["zonal"], g["merid"], g["phi"])
    assert np.array_equal(o.state("u"), g["u"]) and np.array_equal(o.state("v"), g["v"])
    o.step(int(g["nsteps"]))
    for k in ("u", "v", "phi"):
        assert np.array_equal(o.state(k), g["out_" + k]), k


def test_oracle_reproduces_kernel_fixture():
    g = load(os.path.join(GOLD, "kernels.npz"))
    for order in (3, 4):
        o = Oracle(order, 8, 100.0, "RK4", cases.EARTH_RADIUS)
        f, q, lam = g[f"tendP_in_f_{order}"], g[f"tendP_in_q_{order}"], g[f"tendP_in_lam_{order}"]
        got = np.array([o.calc_tendP(f[k], q[k], lam[k, 0], lam[k, 1]) for k in range(len(f))])
        assert np.array_equal(got, g[f"tendP_out_{order}"])
        pv = g[f"polyfit_in_{order}"]
        got = np.array([[o.polyfit(p, False), o.polyfit(p, True)] for p in pv])
        assert np.array_equal(got, g[f"polyfit_out_{order}"])
        src = g[f"interp_in_{order}"]
        got = np.array([o.linear_interp(src[h - 1], h) for h in range(1, o.H + 1)])
        assert np.array_equal(got, g[f"interp_out_{order}"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", STEP_FIXTURES, ids=os.path.basename)
def test_gpu_reproduces_step_fixture(path):
    g = load(path)
    order, nc, scheme = int(g["order"]), int(g["nc"]), str(g["scheme"])
    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
    with api.Stepper(order, nc, float(g["dt"]), scheme) as s:
        s.set_geometry(geom)
        s.set_member(0, g["phi_s"], g["u"], g["v"], g["phi"])
        s.step(int(g["nsteps"]))
        out = s.get_state(0)
    H, n = geom.H, geom.n
    for k in ("u", "v", "phi"):
        err = rel_l2(interior(out[k], H, n), interior(g["out_" + k], H, n))
        assert err <= 1e-12, (k, err)
