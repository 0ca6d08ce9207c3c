"""Run a workload for a number of large steps on one GPU and print domain
diagnostics (the in-process counterpart of running cm1.exe through the
reference's cm1/run.py).

    python -m cm1_b200.run --workload supercell --steps 10 [--ni 128 --nj 128 --nk 80] [--graph]
                           [--time] [--profile] [--stats N] [--stats-file cm1out_stats.dat]
                           [--aux N] [--aux-dir DIR]

--time reports the device time per large step (CUDA events around the steps,
after one untimed step); --profile reports per-kernel device time per step,
the counterpart of the reference's timestats table.  --stats N runs the statistics package
(cm1g_statpack: every statistic this library builds) after the steps, N+1
times, and reports the device-resident time per call (CUDA events, the
first call untimed, rstat copied to the host each call) with the values;
--stats-file appends them as a record of the GrADS stats file.  --aux N
times, after the steps, N calls each of the other entry points of the path
with device-resident arrays (CUDA events, one untimed call first): the
2nd-order diffusion (kdiff2 = 75 m2/s), the records of the prognostic fields
(one gather and one copy to pinned host memory), a restart write and read
(files under --aux-dir), and for ptype=1 mp_driver.
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
    ap.add_argument("--time", action="store_true")
    ap.add_argument("--profile", action="store_true")
    ap.add_argument("--stats", type=int, default=0)
    ap.add_argument("--stats-file")
    ap.add_argument("--aux", type=int, default=0)
    ap.add_argument("--aux-dir", default=".")
    args = ap.parse_args(argv)

    import torch
    from .cases import make_case
    from . import binding

    over = {k: getattr(args, k) for k in ("ni", "nj", "nk") if getattr(args, k)}
    case = make_case(args.workload, seed=args.seed, **over)
    ctx = binding.Context(case.cfg, case.grid)
    dev = binding.to_device(case.state)
    mass2 = cfl = None
    timing = {}
    if args.time or args.profile:
        mass2, cfl = ctx.step(dev, case.dt, case.mass1, use_graph=args.graph)   # untimed
        steps = max(args.steps - 1, 1)
        if args.profile:
            ctx.profile(True)
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(steps):
            mass2, cfl = ctx.step(dev, case.dt, case.mass1, use_graph=args.graph)
        t1.record()
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1) / steps
        cells = case.lay.ni * case.lay.nj * case.lay.nk
        timing = {"ms_per_step": ms, "cell_updates_per_s": cells / (ms * 1e-3)}
        if args.profile:
            prof = ctx.profile_read()
            ctx.profile(False)
            timing["kernel_ms_per_step"] = {k: v[1] / steps for k, v in
                                            sorted(prof.items(), key=lambda kv: -kv[1][1])}
            timing["launches_per_step"] = {k: v[0] / steps for k, v in prof.items()}
    else:
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
    out.update(timing)
    if args.stats > 0:
        from .cases import stat_opts
        opts, keep = stat_opts(case)
        names = ctx.stat_setup(opts)
        fields = [dev[n] for n in ("ua", "va", "wa", "ppi", "tha", "prs", "rho")]
        extra = dict(qa=dev.get("qa") if case.cfg.imoist else None, pta=dev.get("pta") if case.cfg.iptra else None)
        if case.cfg.imoist:   # no moisture budgets are kept: their entries are zero
            extra.update(asq=np.zeros(case.cfg.numq), bsq=np.zeros(case.cfg.numq))
        mtime = case.dt * args.steps
        rstat = ctx.statpack(mtime, case.dt, *fields, **extra)   # untimed
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(args.stats):
            rstat = ctx.statpack(mtime, case.dt, *fields, **extra)
        t1.record()
        torch.cuda.synchronize()
        out["statpack_ms"] = t0.elapsed_time(t1) / args.stats
        out["stats"] = {n: float(v) for n, v in zip(names, rstat)}
        if args.stats_file:
            binding.stat_write(args.stats_file, 1, rstat)
    if args.aux > 0:
        out["aux"] = _time_aux(ctx, case, dev, args.aux, args.aux_dir)
    print(json.dumps(out))
    ctx.close()
    return 0 if np.isfinite(out["max_w"]) else 1


def _time_aux(ctx, case, dev, n, outdir):
    """Device time per call (ms) of the path's other entry points."""
    import os
    import time
    import torch
    lay, cfg = case.lay, case.cfg
    res = {}

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(reps):
            fn()
        t1.record()
        torch.cuda.synchronize()
        return t0.elapsed_time(t1) / reps

    ten = {k: torch.zeros_like(dev[k]) for k in ("uten1", "vten1", "wten1", "thten1", "qten", "ptten")}
    dz = cfg.dz
    zs = np.array([0.5, 1.5, 2.5]) * dz
    w = [float(np.prod([(0.0 - zs[m]) / (zs[l] - zs[m]) for m in range(3) if m != l])) for l in range(3)]
    qa = dev["qa"] if cfg.imoist else None
    pta = dev["pta"] if cfg.iptra else None
    res["diff2_ms"] = timed(lambda: ctx.diff2(75.0, 1, 1, 1, w, w, dev["u3d"], dev["v3d"], dev["w3d"], dev["rho"],
                                              dev["tha"], qa, pta, ten["uten1"], ten["vten1"], ten["wten1"],
                                              ten["thten1"], ten["qten"] if qa is not None else None,
                                              ten["ptten"] if pta is not None else None), n)
    names = ["rho", "prs", "ua", "va", "wa", "ppi", "tha", "ppx"]
    stag = [1, 1, 2, 3, 4, 1, 1, 1]
    fields = [dev[k] for k in names]
    k2 = [lay.nk, lay.nk, lay.nk, lay.nk, lay.nk + 1, lay.nk, lay.nk, lay.nk]
    nv = ctx.records_size(stag, [1] * len(stag), k2)
    host = torch.empty(nv, dtype=torch.float32).pin_memory()
    res["records_ms"] = timed(lambda: ctx.pack_records(fields, stag, [1] * len(stag), k2, out=host), n)
    res["records_bytes"] = nv * 4
    path = os.path.join(outdir, "cm1g_restart.bin")
    t0 = time.perf_counter()
    for _ in range(n):
        ctx.restart_write(path, dev, nstep=1, mtime=case.dt, dt=case.dt, dtlast=case.dt, mass1=case.mass1)
    res["restart_write_ms_wall"] = (time.perf_counter() - t0) * 1e3 / n
    res["restart_bytes"] = os.path.getsize(path)
    t0 = time.perf_counter()
    for _ in range(n):
        ctx.restart_read(path, dev)
    res["restart_read_ms_wall"] = (time.perf_counter() - t0) * 1e3 / n
    if cfg.ptype == 1:
        res["mp_driver_ms"] = timed(lambda: ctx.mp_driver(dev, case.dt), n)
    return res


if __name__ == "__main__":
    sys.exit(main())
