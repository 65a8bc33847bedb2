"""Stored state of the benchmarked 7-level refinement grid after one coarse
step, made by the CPU oracle (itself pinned to the reference's 3-level runs
and binary grid), for the benchmark's parity figure and its GPU test.

    python tests/golden/make_fmr_c3_fixture.py

The grid is baum_b200.workloads.FMR_SIZES (16.6 M points; about 15 GB of
host memory and ~12 minutes of the oracle on 8 cores).  The full state is
3.3 GB, so the fixture keeps, per level, every variable at 512 seeded points,
and per variable the sum, the sum of |u| and the largest |u| over all
points: tests/golden/fmr_c3_oracle.npz.
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from baum_b200 import workloads  # noqa: E402
from oracle import oracle  # noqa: E402

NSAMPLE = 512


def main():
    sizes = workloads.FMR_SIZES
    levels, params, dt = workloads.fmr_setup(sizes)
    t0 = time.time()
    u0 = [workloads.fmr_state_host(lev) for lev in levels]
    print("initial data %.1f s" % (time.time() - t0), flush=True)
    t0 = time.time()
    st = oracle.FmrState(levels, u0, 1, params, dt)
    del u0
    st.advance(1)
    print("oracle coarse step %.1f s" % (time.time() - t0), flush=True)
    out = {"sizes": np.array(sizes), "dx0": workloads.FMR_DX0, "coarse_steps": 1, "nsample": NSAMPLE}
    for l, lev in enumerate(levels):
        idx = workloads.sample_points(lev.npoints, NSAMPLE, 100 + l)
        u = st.u[l]
        out["idx_l%d" % l] = idx
        out["u_l%d" % l] = u[:, idx]
        out["sum_l%d" % l] = u.sum(axis=1)
        out["abssum_l%d" % l] = np.abs(u).sum(axis=1)
        out["max_l%d" % l] = np.abs(u).max(axis=1)
    np.savez_compressed(os.path.join(ROOT, "tests", "golden", "fmr_c3_oracle.npz"), **out)
    print("wrote fmr_c3_oracle.npz")


if __name__ == "__main__":
    main()
