"""Benchmark of the CM1 dynamical-core large step on B200.

Metric: grid-cell updates per second per RK3 large step (cells x steps / s),
as an absolute number and as a fraction of the HBM roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload supercell]
    python bench.py --impl reference ...     # CPU restatement on the host cores

One "step" is one complete large step (solve2 + pdefq + solve3) of the
workload; the default workload is the 256x256x80 moist supercell-scale case
(WENO5 theta + 6 scalars, open-radiative boundaries, dt=3 s, nsound=8).
`value` is device-resident throughput (state already in HBM, CUDA-graph
replay); `e2e` runs the same step through the C-ABI with pinned host arrays,
so every step includes the host->device copy of the state and the copy back.
With N>1 ranks every GPU advances its own replica (ensemble-style weak
scaling, no collective on the data path); timing is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

# algorithmic bytes per cell per large step, per substep of the acoustic kernel
ACOUSTIC_FLOATS_PER_CELL = 23            # reads 15, writes 8 (u,v,w,pi',ppd + 3 averages)


def nloop_total(nsound):
    n1 = int(np.floor(nsound / 3.0 + 0.5))
    dt = 1.0
    if dt / (n1 * 3.0) > dt / nsound:
        n1 += 1
    return n1 + nsound // 2 + nsound


def algorithmic_bytes_per_cell(cfg):
    """B = 4 [3 (M + 3 + 4 N_adv + E) + 23 S + F] (floats per cell-step)."""
    moist = cfg.imoist == 1
    M = 16 if moist else 14
    nadv = 1 + (cfg.numq if moist else 0) + (cfg.npt if cfg.iptra else 0)
    E = 1 if (moist and cfg.eqtset == 2) else 0
    F = 5 if moist else 4
    S = nloop_total(cfg.nsound)
    return 4 * (3 * (M + 3 + 4 * nadv + E) + ACOUSTIC_FLOATS_PER_CELL * S + F)


def kernel_bytes_per_step(cfg):
    """Algorithmic bytes per cell per large step of the main kernels (each
    non-derivable input read once, each output written once, FP32), keyed by
    the names the library's per-kernel timing reports.

    k_scal_tile: the fused scalar pass, one launch per RK stage; a field it
    updates reads s, its RK base and its fixed tendency and writes the new
    value (16 B); each launch reads rru, rrv, rrw once (12 B) and, for moist
    theta (eqtset=2), thterm (4 B).  At stages 1-2 it updates theta, every q
    and every tracer; at stage 3 the fields without the positive-definite
    pass (theta, and tracers when pdtra=0).
    k_advs_tile: one field per launch (28 B, + 4 B thterm for moist theta).
    k_advs_tile_pdef1 + k_advs_pdef2: the final-stage positive-definite pass
    of one field, together the same 28 B (their six work arrays are scratch).
    k_sound_step: one acoustic small step, 23 floats (92 B) per cell.
    k_advu/k_advv/k_advw: read u, v, w and the fixed tendency, write the
    tendency (20 B each)."""
    moist = cfg.imoist == 1
    nq = cfg.numq if moist else 0
    npt = cfg.npt if cfg.iptra else 0
    nsc = 1 + nq + npt
    tht = 4 if (moist and cfg.eqtset == 2) else 0
    pdef3 = nq + (npt if cfg.pdtra == 1 else 0)
    fused_fields = 2 * nsc + (nsc - pdef3)
    S = nloop_total(cfg.nsound)
    return {"k_scal_tile": 16 * fused_fields + 3 * (12 + tht),
            "k_advs_tile": 3 * (28 * nsc + tht) - 28 * pdef3,
            "k_advs_tile_pdef1": 20 * pdef3, "k_advs_pdef2": 8 * pdef3,
            "k_sound_step": 4 * ACOUSTIC_FLOATS_PER_CELL * S,
            "k_advu": 3 * 20, "k_advv": 3 * 20, "k_advw": 3 * 20}


def kernel_roofline(name, prof, bpc, cells, hbm, peak_kind, traffic_per_launch=None):
    """Roofline entry of one kernel from the profiled pass (2 large steps):
    achieved = algorithmic bytes per launch / mean CUDA-event launch time."""
    n, ms = prof[name]
    launches_per_step = n / 2.0
    bytes_launch = bpc * cells / launches_per_step
    per_launch_ms = ms / n
    achieved = bytes_launch / (per_launch_ms * 1e-3) / 1e9
    tot = sum(v[1] for v in prof.values())
    return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": hbm, "peak_kind": peak_kind,
            "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic_per_launch,
            "algorithmic_bytes_per_launch": bytes_launch, "algorithmic_bytes_per_cell_step": bpc,
            "launches_per_step": launches_per_step, "avg_launch_ms": per_launch_ms,
            "share_of_step": ms / tot if tot else None}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) samples during the timed region:
    NVML reads every 20 ms on the benchmarked GPU (found by its UUID), or
    nvidia-smi every 200 ms where NVML is not importable.  Read-only."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.stop = gpu, [], threading.Event()
        self.nvml = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(gpu).uuid)
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            self.nvml = (pynvml, h)
        except Exception:
            self.nvml = None

    def _sample_nvml(self):
        nv, h = self.nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
        act = ["Active" if rs & b else "Not Active" for b in bits]
        self.rows.append([str(self.gpu), str(sm), str(mx), "", hex(rs)] + act)

    def _run(self):
        while not self.stop.is_set():
            if self.nvml is not None:
                try:
                    self._sample_nvml()
                except Exception:
                    self.nvml = None
                self.stop.wait(0.02)
                continue
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(timeout=10)

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) > 8:
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows),
                "source": "nvml" if self.nvml is not None else "nvidia-smi"}


def cpu_time_steps(case, nsteps):
    """Oracle (CPU restatement) timed on the host cores."""
    from oracle import oracle
    st = case.copy_state()
    oracle.step(case, st)          # warm caches and threads
    t0 = time.perf_counter()
    for _ in range(nsteps):
        st, _, _ = oracle.step(case, st)
    return time.perf_counter() - t0, oracle.threads()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from cm1_b200.cases import make_case
    case = make_case(args.workload)
    cells = case.cfg.ni * case.cfg.nj * case.cfg.nk
    for _ in range(max(0, min(args.warmup, 1))):
        cpu_time_steps(case, 0)
    steps = max(1, min(args.steps, args.ref_steps))
    sec, thr = cpu_time_steps(case, steps)
    v = cells * steps / sec
    line = {"impl": "reference", "metric": "cell-updates/s per RK3 large step", "value": v,
            "unit": "cell-updates/s", "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sec / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded, generated in-repo)",
            "config": workload_config(case, args),
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": thr, "kind": "port",
                             "sample": "%d full large steps of the %s workload, OpenMP on all host threads "
                                       "(CPU restatement of the Fortran: no Fortran compiler on this image)"
                                       % (steps, args.workload)},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def _shapes(tune, binding):
    """The launch shapes used (autotuner's choice, or the defaults)."""
    if tune is None:
        return {"autotuned": False}
    tab, stab = binding.tile_shapes(), binding.tile_shapes(scalar=True)
    forms = {0: "tile 32 columns x 8 warps", 1: "tile 32 columns x 4 warps", 2: "column sweep 32x4",
             3: "column sweep 32x2"}
    return {"autotuned": True, "scalar_tile_cells_xyz": stab[tune["adv_shape"]],
            "momentum_tile_xyz": tab[tune["mom_shape"]],
            "acoustic": forms.get(tune["sound_form"], tune["sound_form"]), "tuned_step_ms": tune["step_ms"]}


def workload_config(case, args):
    c = case.cfg
    return {"workload": args.workload, "grid": [c.ni, c.nj, c.nk], "dx_m": c.dx, "dz_m": c.dz, "dt_s": case.dt,
            "nsound": c.nsound, "advwenos": c.advwenos, "moist": bool(c.imoist), "passive_tracers": c.npt if c.iptra else 0,
            "lateral_bc": {1: "periodic", 2: "open-radiative"}[c.wbc], "l2": "inputs larger than L2 (no flush needed)",
            "parallelism": "replicas" if args.gpus > 1 else "single"}


def _tally(tunes):
    out = {}
    for t in tunes:
        k = (t["adv_shape"], t["mom_shape"], t["sound_form"])
        out[k] = out.get(k, 0) + 1
    return out


def other_workload(name, steps, warmup, hbm):
    """Device-resident throughput of another configuration (one GPU, the
    library's default launch shapes, CUDA-graph replay), measured after the
    main workload: the dry warm bubble (64x64x40) and the convective boundary
    layer (1024x1024x128, doubly periodic, WENO5 theta + 2 scalars)."""
    import torch
    from cm1_b200.cases import make_case
    from cm1_b200 import binding
    case = make_case(name)
    cfg = case.cfg
    cells = cfg.ni * cfg.nj * cfg.nk
    ctx = binding.Context(cfg, case.grid)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    dev = binding.to_device(case.state)
    del case.state
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            ctx.step(dev, case.dt, case.mass1, use_graph=True)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(steps):
        ctx.step(dev, case.dt, case.mass1, use_graph=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms_step = ev0.elapsed_time(ev1) / steps
    ctx.profile(True)
    with torch.cuda.stream(stream):
        ctx.step(dev, case.dt, case.mass1, use_graph=False)
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    ctx.close()
    del dev
    torch.cuda.empty_cache()
    B = algorithmic_bytes_per_cell(cfg)
    gbs = B * cells / (ms_step * 1e-3) / 1e9
    top = sorted(prof.items(), key=lambda kv: -kv[1][1])[:4]
    return {"workload": name, "grid": [cfg.ni, cfg.nj, cfg.nk], "steps": steps, "warmup": warmup,
            "ms_per_step": ms_step, "value": cells / (ms_step * 1e-3), "unit": "cell-updates/s",
            "launch_shapes": "library defaults",
            "step_roofline": {"algorithmic_bytes_per_cell": B, "achieved_gbs": gbs, "frac": gbs / hbm},
            "top_kernels_ms_per_step": {k: v[1] for k, v in top}}


def run_ensemble(args):
    """The uneven 64-member warm-bubble ensemble: one graph launch per large
    step for all members (cm1g_ensemble_step) against looping the members'
    own graph-replayed steps one after another.  Both legs are timed on the
    host around `steps` synchronised steps (each call returns after its
    results are read back)."""
    import torch
    from cm1_b200.cases import make_ensemble
    from cm1_b200 import binding
    members = make_ensemble(64)
    cells = sum(c.cfg.ni * c.cfg.nj * c.cfg.nk for c in members)
    ctxs = [binding.Context(c.cfg, c.grid) for c in members]
    dev = [binding.to_device(c.state) for c in members]
    # launch shapes per member grid from the autotuner (each member timed
    # alone; members of the same grid share the cached choice)
    tunes = []
    if not args.no_tune:
        for ctx, st, c in zip(ctxs, dev, members):
            tunes.append(ctx.autotune(st, c.dt, c.mass1, reps=3, cache=args.tune_cache))
    ens = binding.Ensemble(ctxs)
    dts, m1 = [c.dt for c in members], [c.mass1 for c in members]
    for _ in range(args.warmup):
        ens.step(dev, dts, m1, use_graph=True)
    torch.cuda.synchronize()
    with ClockSampler(0) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            ens.step(dev, dts, m1, use_graph=True)
        sec = time.perf_counter() - t0
    # looping the members: each its own captured step, one after another
    for ctx, st, c in zip(ctxs, dev, members):
        for _ in range(args.warmup):
            ctx.step(st, c.dt, c.mass1, use_graph=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for ctx, st, c in zip(ctxs, dev, members):
            ctx.step(st, c.dt, c.mass1, use_graph=True)
    sec_loop = time.perf_counter() - t0
    # and looping them with eager launches (no graphs): the plain per-member kernels
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for ctx, st, c in zip(ctxs, dev, members):
            ctx.step(st, c.dt, c.mass1, use_graph=False)
    sec_eager = time.perf_counter() - t0
    hbm, peak_kind = peaks()
    B = algorithmic_bytes_per_cell(members[0].cfg)
    value = cells * args.steps / sec
    loop_value = cells * args.steps / sec_loop
    line = {"metric": "cell-updates/s per RK3 large step", "value": value, "unit": "cell-updates/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded, generated in-repo)",
            "config": {"workload": "ensemble", "members": len(members), "total_cells": cells,
                       "grids": sorted({(c.cfg.ni, c.cfg.nj, c.cfg.nk) for c in members}),
                       "dt_s": members[0].dt, "nsound": members[0].cfg.nsound, "advwenos": 1,
                       "timing": "host clock around synchronised steps",
                       "tuned_members": len(tunes),
                       "tune_choices": {str(k): v for k, v in _tally(tunes).items()},
                       "l2": "all members together exceed L2 (no flush needed)"},
            "step_roofline": {"algorithmic_bytes_per_cell": B, "achieved_gbs": B * value / 1e9,
                              "frac": B * value / 1e9 / hbm, "peak": hbm, "peak_kind": peak_kind},
            "looping_members": {"value": loop_value, "ms_per_step": 1e3 * sec_loop / args.steps},
            "speedup_vs_looping": value / loop_value,
            "looping_members_eager": {"value": cells * args.steps / sec_eager, "ms_per_step": 1e3 * sec_eager / args.steps},
            "speedup_vs_looping_eager": sec_eager / sec,
            "gpu_launches": ens.kernels_per_step() * args.steps, "clocks": clk.summary()}
    print(json.dumps(line))
    ens.close()
    for c in ctxs:
        c.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="supercell")
    ap.add_argument("--impl", default="cm1g")
    ap.add_argument("--ref-steps", type=int, default=3)
    ap.add_argument("--cpu-steps", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="default launch shapes instead of the autotuner's")
    ap.add_argument("--no-other", action="store_true",
                    help="skip the dry-bubble and CBL throughput lines measured after the main workload")
    ap.add_argument("--tune-cache", default=None,
                    help="text file of autotuner results per grid (read if present, appended otherwise)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "ensemble":
        return run_ensemble(args)

    import torch
    from cm1_b200.cases import make_case
    from cm1_b200 import binding

    from cm1_b200.replicas import rank_env, replica_seed, max_over_ranks, job_value
    world, rank, local = rank_env()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    case = make_case(args.workload, seed=replica_seed(rank))
    cfg = case.cfg
    cells = cfg.ni * cfg.nj * cfg.nk
    ctx = binding.Context(cfg, case.grid)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    dev = binding.to_device(case.state)
    torch.cuda.synchronize()
    # ---- launch shapes for this grid (timed on a copy of the state, untimed here)
    tune = None if args.no_tune else ctx.autotune(dev, case.dt, case.mass1, reps=3, cache=args.tune_cache)

    # ---- device-resident throughput (graph replay)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            ctx.step(dev, case.dt, case.mass1, use_graph=True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    n0 = ctx.launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            ctx.step(dev, case.dt, case.mass1, use_graph=True)
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.launches() - n0
    ms = max_over_ranks(ms, dist, device="cuda")
    if dist:
        dist.barrier()
    ms_step = ms / args.steps
    value = job_value(world, cells, args.steps, ms)

    # ---- per-kernel device times (profiled pass, eager launches)
    ctx.profile(True)
    with torch.cuda.stream(stream):
        for _ in range(2):
            ctx.step(dev, case.dt, case.mass1, use_graph=False)
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    hbm, peak_kind = peaks()
    B = algorithmic_bytes_per_cell(cfg)
    step_gbs = B * cells / (ms_step * 1e-3) / 1e9
    # roofline of the dominant kernel (largest device time per step), and of
    # the acoustic kernel; DRAM traffic per launch from the ncu capture
    # summarised in profiles/roofline_traffic.json, when there is one
    traffic = {}
    tf = os.path.join(ROOT, "profiles", "roofline_traffic.json")
    if os.path.exists(tf):
        try:
            traffic = json.load(open(tf))
        except Exception:
            traffic = {}
    kb = kernel_bytes_per_step(cfg)
    ranked = sorted(prof, key=lambda k: -prof[k][1])
    top = ranked[0] if ranked else None
    roof = None
    if top in kb:
        roof = kernel_roofline(top, prof, kb[top], cells, hbm, peak_kind,
                               traffic.get("%s_bytes_per_launch_%s" % (top, args.workload)))
    elif top is not None:
        roof = {"kernel": top, "note": "no algorithmic byte count for this kernel"}
    roof_snd = None
    if "k_sound_step" in prof and top != "k_sound_step":
        roof_snd = kernel_roofline("k_sound_step", prof, kb["k_sound_step"], cells, hbm, peak_kind,
                                   traffic.get("k_sound_step_bytes_per_launch_%s" % args.workload))

    # ---- end-to-end through the C-ABI with pinned host arrays
    host = {k: torch.from_numpy(v.copy()).pin_memory() for k, v in case.state.items()}
    h2d = sum(v.numel() * 4 for v in host.values())
    d2h = sum(v.numel() * 4 for k, v in host.items() if k not in ("uten1", "vten1", "wten1", "ppten", "thten1",
                                                                    "qten", "ptten"))
    e2e_steps = max(2, min(args.steps, 5))
    with torch.cuda.stream(stream):
        ctx.step(host, case.dt, case.mass1)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        ctx.step(host, case.dt, case.mass1)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    ms_e2e = max_over_ranks(ms_e2e, dist, device="cuda")
    e2e_value = job_value(world, cells, e2e_steps, ms_e2e)

    # ---- CPU baseline (rank 0, N=1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sec, thr = cpu_time_steps(case, args.cpu_steps)
        cpu = {"value": cells * args.cpu_steps / sec, "unit": "cell-updates/s", "cores": thr, "kind": "port",
               "sample": "%d full large steps of the %s workload on the host (CPU restatement, OpenMP)"
                         % (args.cpu_steps, args.workload)}

    # ---- the other configurations' throughput (rank 0, N=1 only)
    others = None
    if rank == 0 and world == 1 and not args.no_other and args.workload == "supercell":
        ctx.close()
        del dev, host
        torch.cuda.empty_cache()
        others = [other_workload("dry_bubble", 50, 3, hbm), other_workload("cbl", 5, 3, hbm)]

    if rank == 0:
        line = {"metric": "cell-updates/s per RK3 large step", "value": value, "unit": "cell-updates/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded, generated in-repo)",
                "config": dict(workload_config(case, args), launch_shapes=_shapes(tune, binding)),
                "roofline": roof, "roofline_acoustic": roof_snd,
                "step_roofline": {"algorithmic_bytes_per_cell": B, "achieved_gbs": step_gbs, "frac": step_gbs / hbm,
                                  "roofline_cell_updates_per_s": hbm * 1e9 / B},
                "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "steps": e2e_steps},
                "gpu_launches": launches, "clocks": clk.summary(),
                "kernel_ms_per_step": {k: v[1] / 2 for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])},
                "other_workloads": others}
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
