"""Parity of the CUDA large step (through the C-ABI) with the CPU oracle.

Parity gate: after one large step every prognostic field
agrees with the oracle to max|err| <= 1e-5 of the field's range; after many
steps the domain extrema and the mass/theta budgets agree to 1e-3 relative.
The kernels keep the reference's binary32 operation order (built with
--fmad=false), so the observed errors are far below these bounds.
"""
import numpy as np
import pytest

from cm1_b200.cases import make_case

pytestmark = pytest.mark.gpu

TOL_RANGE = 1e-5        # max|err| / range(field), one large step
TOL_BUDGET = 1e-3       # relative, extrema and budgets after many steps

FIELDS = [("u3d", 2), ("v3d", 3), ("w3d", 4), ("pp3d", 1), ("th3d", 1), ("rho", 1), ("prs", 1),
          ("ua", 2), ("va", 3), ("wa", 4), ("ppi", 1), ("tha", 1), ("ppx", 1)]


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def interior(case, a, stag):
    return a[case.lay.interior(stag)]


def field_errors(case, got, ref):
    errs = {}
    for f, stag in FIELDS:
        g, r = interior(case, got[f], stag), interior(case, ref[f], stag)
        rng = float(r.max() - r.min()) or 1.0
        errs[f] = float(np.abs(g.astype(np.float64) - r).max()) / rng
    for f in ("q3d", "qa", "pt3d", "pta"):
        for n in range(ref[f].shape[0]):
            g, r = interior(case, got[f][n], 1), interior(case, ref[f][n], 1)
            rng = float(r.max() - r.min()) or 1.0
            errs["%s[%d]" % (f, n)] = float(np.abs(g.astype(np.float64) - r).max()) / rng
    return errs


CASES = [
    ("dry_bubble", {}),
    ("supercell", dict(ni=40, nj=36, nk=40)),
    ("supercell", dict(ni=40, nj=36, nk=40, advwenos=2)),
    ("cbl", dict(ni=48, nj=40, nk=40)),
    # 6th-order horizontal diffusion (idiff=1, difforder=6), with and without the mdiff limiter
    ("dry_bubble", dict(diff6=0.04)),
    ("supercell", dict(ni=40, nj=36, nk=40, diff6=0.04, mdiff=1)),
    # open-boundary phase speeds of Klemp-Wilhelmson form: from ua once per
    # large step (irbc=1) and from u3d at every small step (irbc=2)
    ("supercell", dict(ni=40, nj=36, nk=40, irbc=1)),
    ("supercell", dict(ni=40, nj=36, nk=40, irbc=2)),
    # open-boundary outflow restricted to the inflow at every acoustic step (roflux=1)
    ("supercell", dict(ni=40, nj=36, nk=40, roflux=1)),
    ("supercell", dict(ni=40, nj=36, nk=40, irbc=2, roflux=1)),
    # more levels than the acoustic tile form holds (column sweep with its
    # LU factors in global memory; column-averaged radiative phase speeds)
    ("cbl", dict(ni=24, nj=20, nk=160)),
    ("supercell", dict(ni=24, nj=20, nk=150)),
]


@pytest.mark.parametrize("name,over", CASES)
def test_one_large_step(name, over, cm1g, oracle_lib):
    torch = _torch()
    case = make_case(name, **over)
    ref, m2_ref, cfl_ref = oracle_lib.step(case)
    ctx = cm1g.Context(case.cfg, case.grid)
    dev = cm1g.to_device(case.state)
    m2, cfl = ctx.step(dev, case.dt, case.mass1)
    torch.cuda.synchronize()
    got = cm1g.to_host(dev)
    errs = field_errors(case, got, ref)
    worst = max(errs.values())
    print("%s %s worst max|err|/range = %.3e" % (name, over, worst))
    for f, e in errs.items():
        assert e <= TOL_RANGE, (f, e)
    assert abs(m2 - m2_ref) <= 1e-7 * abs(m2_ref)   # powf/summation-order rounding
    assert abs(cfl - cfl_ref) <= 1e-6 * max(cfl_ref, 1e-6)
    assert ctx.launches() > 0


@pytest.mark.parametrize("name,over", CASES)
def test_error_against_fp64_build(name, over, cm1g, oracle_lib):
    """The error of one large step against the FP64 (-r8) build of the
    oracle (oracle/make_r8.py), from the same inputs: the CUDA path's FP32
    result must be as close to it as the FP32 restatement's is (within 2x
    per field, or 1e-6 of the range)."""
    torch = _torch()
    case = make_case(name, **over)
    ref32, _, _ = oracle_lib.step(case)
    ref64 = oracle_lib.step_r8(case)
    ctx = cm1g.Context(case.cfg, case.grid)
    dev = cm1g.to_device(case.state)
    ctx.step(dev, case.dt, case.mass1)
    torch.cuda.synchronize()
    got = cm1g.to_host(dev)
    e_gpu, e_ref = field_errors(case, got, ref64), field_errors(case, ref32, ref64)
    worst = max(e_gpu, key=e_gpu.get)
    print("%s %s vs FP64: GPU worst %s %.3e, FP32 oracle %.3e" % (name, over, worst, e_gpu[worst], e_ref[worst]))
    for f in e_gpu:
        assert e_gpu[f] <= 2.0 * e_ref[f] + 1e-6, (f, e_gpu[f], e_ref[f])


@pytest.mark.parametrize("name,over", [CASES[1], CASES[3]])
def test_one_large_step_column_sweep_sound(name, over, cm1g, oracle_lib, monkeypatch):
    """The same step with the column-sweep acoustic kernel (the form large grids use)."""
    monkeypatch.setenv("CM1G_SOUND_FORM", "col")
    test_one_large_step(name, over, cm1g, oracle_lib)


@pytest.mark.parametrize("name,over", [("dry_bubble", {}), ("supercell", dict(ni=40, nj=36, nk=40, bc=1))])
def test_many_steps_budgets(name, over, cm1g, oracle_lib):
    """Domain max w, min pi', max theta', and the mass and theta budgets
    after 100 large steps (the dry bubble at c0 sizes; a reduced moist
    supercell with tracers, periodic), against the oracle; the distance of
    both from the FP64 build after the same 100 steps is printed.  The open
    radiative boundaries are left out of this test: with them the restated
    scheme itself separates a 1e-7 perturbation of theta into 1e-3 of pi''s
    range within 20 steps (inflow/outflow switches at the boundary), so a
    1e-3 bar after 100 steps holds for no pair of builds."""
    torch = _torch()
    case = make_case(name, **over)
    ref = case.copy_state()
    ctx = cm1g.Context(case.cfg, case.grid)
    dev = cm1g.to_device(case.state)
    nsteps = 100
    for n in range(nsteps):
        ref, m2r, _ = oracle_lib.step(case, ref)
        m2, _ = ctx.step(dev, case.dt, case.mass1, use_graph=(n > 0))
    torch.cuda.synchronize()
    got = cm1g.to_host(dev)
    lay = case.lay
    for f, stag, red in [("w3d", 4, np.max), ("pp3d", 1, np.min), ("th3d", 1, np.max)]:
        a, b = red(interior(case, got[f], stag)), red(interior(case, ref[f], stag))
        assert abs(a - b) <= TOL_BUDGET * abs(b), (f, a, b)
    mg = interior(case, got["rho"], 1).astype(np.float64).sum()
    mr = interior(case, ref["rho"], 1).astype(np.float64).sum()
    assert abs(mg - mr) <= TOL_BUDGET * abs(mr) * 1e-3
    th_g = (interior(case, got["rho"], 1).astype(np.float64) * interior(case, got["th3d"], 1)).sum()
    th_r = (interior(case, ref["rho"], 1).astype(np.float64) * interior(case, ref["th3d"], 1)).sum()
    assert abs(th_g - th_r) <= TOL_BUDGET * abs(th_r)
    assert abs(m2 - m2r) <= 1e-7 * abs(m2r)
    r64 = oracle_lib.step_r8(case, nsteps=nsteps)
    for f, stag, red in [("w3d", 4, np.max), ("pp3d", 1, np.min)]:
        a, b, c = red(interior(case, got[f], stag)), red(interior(case, ref[f], stag)), red(interior(case, r64[f], stag))
        print("%s %d steps %s: CUDA %.6e, FP32 oracle %.6e, FP64 %.6e" % (name, nsteps, f, a, b, c))
    del lay


def test_graph_replay_matches_eager(cm1g):
    torch = _torch()
    case = make_case("supercell", ni=32, nj=32, nk=40)
    ctx = cm1g.Context(case.cfg, case.grid)
    a = cm1g.to_device(case.state)
    b = cm1g.to_device(case.state)
    for _ in range(3):
        ctx.step(a, case.dt, case.mass1, use_graph=False)
        ctx.step(b, case.dt, case.mass1, use_graph=True)
    torch.cuda.synchronize()
    for k in a:
        assert torch.equal(a[k], b[k]), k


def test_host_pointer_path_matches_device(cm1g):
    torch = _torch()
    case = make_case("cbl", ni=32, nj=32, nk=40)
    ctx = cm1g.Context(case.cfg, case.grid)
    host = case.copy_state()
    dev = cm1g.to_device(case.state)
    m2h, cflh = ctx.step(host, case.dt, case.mass1)
    m2d, cfld = ctx.step(dev, case.dt, case.mass1)
    got = cm1g.to_host(dev)
    for k in host:
        assert np.array_equal(host[k], got[k]), k
    assert m2h == m2d and cflh == cfld


def test_nonfinite_state_is_reported(cm1g):
    torch = _torch()
    case = make_case("dry_bubble", ni=16, nj=16, nk=20)
    ctx = cm1g.Context(case.cfg, case.grid)
    dev = cm1g.to_device(case.state)
    lay = case.lay
    dev["u3d"][lay.kx(5), lay.jx(5), lay.ix(5)] = float("nan")
    with pytest.raises(cm1g.CM1GError) as ei:
        ctx.step(dev, case.dt, case.mass1)
    assert ei.value.code == -4
    # the context stays usable after the error
    dev2 = cm1g.to_device(case.state)
    ctx.step(dev2, case.dt, case.mass1)
    torch.cuda.synchronize()


def test_unsupported_option_is_an_error(cm1g):
    _torch()
    case = make_case("dry_bubble", ni=16, nj=16, nk=20)
    case.cfg.psolver = 2
    with pytest.raises(cm1g.CM1GError) as ei:
        cm1g.Context(case.cfg, case.grid)
    assert ei.value.code == -5
