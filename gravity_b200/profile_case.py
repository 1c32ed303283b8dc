"""A named workload at a chosen size, stepped a few times: the command the
Nsight Compute captures in profiles/ run (a profiler replays each captured
kernel many times, so the captures use cases smaller than the benchmark's
but larger than the 126 MB L2).

  python -m gravity_b200.profile_case lattice --bodies 4000000 --grid 4096x1024
  python -m gravity_b200.profile_case plummer_walls
  python -m gravity_b200.profile_case adjoint --bodies 20000 --grid 512x256 --steps 8
  python -m gravity_b200.profile_case batch --sims 32

Order of the kernels launched: initializeAcceleration (one force build and
kick), then `--steps` steps (or, for `adjoint`, a checkpointed rollout of
`--steps` steps and its backward pass; for `batch`, batch steps).
"""

from __future__ import annotations

import argparse

import numpy as np

from . import _abi, scenarios
from .pipeline import GravityPipeline


def main(argv=None) -> None:
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", choices=["lattice", "plummer_walls", "uniform_torus", "adjoint", "batch"])
    ap.add_argument("--bodies", type=int, default=None)
    ap.add_argument("--grid", default=None, help="WxH")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--sims", type=int, default=32)
    ap.add_argument("--u32", action="store_true", help="lattice: uint32 deposit")
    args = ap.parse_args(argv)
    grid = tuple(int(v) for v in args.grid.split("x")) if args.grid else None

    if args.case == "batch":
        from .batch import GravityBatch

        scs = scenarios.batch(sims=args.sims)
        with GravityBatch([sc.config for sc in scs]) as b:
            for i, sc in enumerate(scs):
                b.upload(i, sc.bodies, sc.materials)
            b.initialize_acceleration()
            b.step(args.steps)
            b.synchronize()
        print("ok", sum(sc.n for sc in scs))
        return
    if args.case == "lattice":
        kw = {}
        if args.bodies:
            kw["n"] = args.bodies
        if grid:
            kw["grid"] = grid
        if args.u32:
            kw["deposit_mode"] = _abi.P3M_DEPOSIT_U32
        sc = scenarios.lattice_scale(**kw)
    elif args.case == "plummer_walls":
        sc = scenarios.plummer_walls(**({"n": args.bodies} if args.bodies else {}))
    elif args.case == "uniform_torus":
        sc = scenarios.uniform_torus(**({"n": args.bodies} if args.bodies else {}))
    else:
        kw = {}
        if args.bodies:
            kw["n_cluster"] = args.bodies - 1000
        if grid:
            kw["grid"] = grid
        sc = scenarios.adjoint_cluster(**kw)
    with GravityPipeline(sc.config) as p:
        p.upload(sc.bodies, sc.materials)
        if args.case == "adjoint":
            from .adjoint import Rollout

            r = Rollout(p, sc.n, args.steps, checkpoint_interval=max(1, args.steps // 2))
            r.forward()
            seed = np.zeros((sc.n, 4), np.float32)
            seed[-1000:, 0] = 1.0
            r.backward(seed)
        else:
            p.initialize_acceleration(sc.n)
            p.step(sc.n, args.steps)
        p.synchronize()
    print("ok", sc.n)


if __name__ == "__main__":
    main()
