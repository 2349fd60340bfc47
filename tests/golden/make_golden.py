"""Generates tests/golden/*.npz: small seeded fixtures of the oracle.

The reference (Fortran 90, no compiler in this image) ships no golden vectors,
so these fixtures are outputs of the CPU oracle (oracle/mcv_oracle.c), which is
itself pinned by the analytic known-answer tests in tests/test_oracle.py.  They
freeze the oracle's numbers (a CPU regression check, bit-exact) and give the
GPU tests fixed inputs and expected outputs.

Contents per fixture (Nc=4 grids, seeded balanced flow + harmonics + mountain):
  inputs : zonal, merid, phi, phi_s on all padded points (initTestCase inputs),
           u, v (covariant, as initTestCase projects them), dt
  outputs: u, v, phi after `nsteps` RK steps (full padded arrays)
Plus building-block vectors: polyfit / calc_tendP / linear_interp on seeded data.

Run: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mcv_sw_b200 import api, cases  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

CASES = [
    # name, order, nc, scheme, nsteps, seed
    ("mcv3_rk4", 3, 4, "RK4", 3, 101),
    ("mcv3_rk3", 3, 4, "RK3_TVD", 3, 102),
    ("mcv4_rk4", 4, 4, "RK4", 3, 103),
    ("mcv4_rk3", 4, 4, "RK3_TVD", 3, 104),
]


def make_step_fixture(name, order, nc, scheme, nsteps, seed):
    geom = api.Geometry(order, nc, cases.EARTH_RADIUS)
    zw, mw, phi, phis, _ = cases.balanced_flow(geom, np.random.default_rng(seed), 38.6, 0.3, 3, 50.0,
                                               mountain=True)
    st = cases.finish(geom, zw, mw, phi, phis, scheme, nsteps=nsteps)
    o = Oracle(order, nc, st.dt, scheme, cases.EARTH_RADIUS)
    o.set_phi_s(st.phi_s)
    o.init_state(st.zonal, st.merid, st.phi)
    o.step(nsteps)
    np.savez_compressed(os.path.join(HERE, f"step_{name}.npz"), order=order, nc=nc, scheme=scheme, nsteps=nsteps,
                        dt=st.dt, zonal=st.zonal, merid=st.merid, phi=st.phi, phi_s=st.phi_s, u=st.u, v=st.v,
                        out_u=o.state("u"), out_v=o.state("v"), out_phi=o.state("phi"))


def make_kernel_fixture():
    rng = np.random.default_rng(7)
    out = {}
    for order in (3, 4):
        o = Oracle(order, 8, 100.0, "RK4", cases.EARTH_RADIUS)
        W = 3 * order - 2
        f = rng.standard_normal((16, W))
        q = rng.standard_normal((16, W))
        lam = rng.uniform(0.1, 2.0, (16, 2))
        out[f"tendP_in_f_{order}"] = f
        out[f"tendP_in_q_{order}"] = q
        out[f"tendP_in_lam_{order}"] = lam
        out[f"tendP_out_{order}"] = np.array([o.calc_tendP(f[k], q[k], lam[k, 0], lam[k, 1]) for k in range(16)])
        pv = rng.standard_normal((16, order))
        out[f"polyfit_in_{order}"] = pv
        out[f"polyfit_out_{order}"] = np.array([[o.polyfit(p, False), o.polyfit(p, True)] for p in pv])
        src = rng.standard_normal((o.H, o.n))
        out[f"interp_in_{order}"] = src
        out[f"interp_out_{order}"] = np.array([o.linear_interp(src[h - 1], h) for h in range(1, o.H + 1)])
    np.savez_compressed(os.path.join(HERE, "kernels.npz"), **out)


if __name__ == "__main__":
    for c in CASES:
        make_step_fixture(*c)
    make_kernel_fixture()
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))
