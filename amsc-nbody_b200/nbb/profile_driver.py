"""Minimal driver for profiling: one simulation, `steps` graph-replayed
steps, per-stage times of one diagnostic force evaluation.

  python amsc-nbody_b200/nbb/profile_driver.py --n 1048576 --precision mixed --steps 2
  python amsc-nbody_b200/nbb/profile_driver.py --n 65536 --precision mixed --adjoint 32

Workload: the benchmark's Plummer sphere (theta 0.5, eps 0.01, dt 1e-3, G 1).
With --adjoint S the run is a rollout of S steps (checkpoints every 32) and
its backward pass for the loss sum(x_T) / n instead.
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import nbb  # noqa: E402
from nbb import ics  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=1 << 20)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--group-size", type=int, default=0, help="mixed walk group size (0 = tuned)")
    ap.add_argument("--adjoint", type=int, default=0, help="rollout steps for a backward pass (0: none)")
    args = ap.parse_args()
    prec = nbb.PRECISION_MIXED if args.precision == "mixed" else nbb.PRECISION_FP64
    p = ics.plummer(args.n, seed=0)
    sim = nbb.Simulation(p, nbb.SimulationConfig(1e-3, 0.5, 0.01, 1.0, precision=prec,
                                                 group_size=args.group_size))
    sim.initialize()
    if args.adjoint:
        import numpy as np

        sim.rollout(args.adjoint, 32)
        gm, gx, gv = sim.backward(np.full((3, args.n), 1.0 / args.n))
        print("backward done", float(gx[0, 0]))
        return
    sim.run(args.steps)
    stages, st = sim.profile()
    print({k: round(v, 4) for k, v in stages.items()}, "interactions", st.interactions,
          "mac_tests", st.mac_tests, "groups", st.n_groups, "nodes", st.n_octree_nodes)


if __name__ == "__main__":
    main()
