"""Short fixed-configuration run for Nsight Compute captures.

`python -m mcv_sw_b200.profile_case --precision mixed --tile -1 --steps 2`
builds the single-large-instance workload (MCV4 Nc=256 RK3_TVD; ~0.5 GB of
device memory, every stage reading more than the 126 MB L2) and runs `steps` RK
steps.  --tile pins a stage-kernel tile shape (index into the autotuner's
candidate list; -1 lets the autotuner pick, which adds its timing launches).
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from mcv_sw_b200 import api, cases  # noqa: E402


def main():
    p = argparse.ArgumentParser()
    p.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    p.add_argument("--tile", type=int, default=-1)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--nc", type=int, default=256)
    p.add_argument("--order", type=int, default=4)
    p.add_argument("--scheme", default="RK3_TVD")
    a = p.parse_args()
    st, geom = cases.large(seed=2, nc=a.nc, order=a.order, scheme=a.scheme)
    with api.Stepper(st.order, st.nc, st.dt, st.scheme, precision=a.precision, radius=cases.EARTH_RADIUS) as s:
        s.set_geometry(geom)
        s.set_member(0, st.phi_s, st.u, st.v, st.phi)
        if a.tile >= 0:
            s.select_tile(a.tile)
        s.step(a.steps)
        cands, chosen = s.tuning()
        print("tile", cands[chosen][0], "of", [c for c, _ in cands])


if __name__ == "__main__":
    main()
