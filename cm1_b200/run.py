"""Run a workload for a number of large steps on one GPU and print domain
diagnostics (the in-process counterpart of running cm1.exe through the
reference's cm1/run.py).

    python -m cm1_b200.run --workload supercell --steps 10 [--ni 128 --nj 128 --nk 80] [--graph]
"""
import argparse
import json
import sys

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="supercell")
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--ni", type=int)
    ap.add_argument("--nj", type=int)
    ap.add_argument("--nk", type=int)
    ap.add_argument("--graph", action="store_true")
    ap.add_argument("--seed", type=int, default=1234)
    args = ap.parse_args(argv)

    import torch
    from .cases import make_case
    from . import binding

    over = {k: getattr(args, k) for k in ("ni", "nj", "nk") if getattr(args, k)}
    case = make_case(args.workload, seed=args.seed, **over)
    ctx = binding.Context(case.cfg, case.grid)
    dev = binding.to_device(case.state)
    mass2 = cfl = None
    for _ in range(args.steps):
        mass2, cfl = ctx.step(dev, case.dt, case.mass1, use_graph=args.graph)
    torch.cuda.synchronize()
    lay = case.lay
    wmax, _, wloc = ctx.maxmin(dev["w3d"], 4)
    _, ppmin, ploc = ctx.maxmin(dev["pp3d"], 1)
    out = {"workload": args.workload, "grid": [lay.ni, lay.nj, lay.nk], "steps": args.steps,
           "max_w": wmax, "max_w_at": wloc[:3], "min_pp": ppmin, "min_pp_at": ploc[3:],
           "mass1": case.mass1, "mass2": mass2, "cflmax": cfl, "kernels": ctx.launches(),
           "theta_max": float(dev["th3d"][lay.interior(1)].max().item())}
    print(json.dumps(out))
    ctx.close()
    return 0 if np.isfinite(out["max_w"]) else 1


if __name__ == "__main__":
    sys.exit(main())
