"""Kessler warm-rain microphysics (ptype=1) through the C-ABI against the
oracle's restatement of kessler.F and mp_driver's Kessler branch.

The point arithmetic keeps the Fortran's order, but the scheme calls pow and
exp (fall speeds, accretion, evaporation, the saturation adjustment).  The
library evaluates them in binary64 and rounds once; the oracle, like the
reference built with gfortran, calls glibc's binary32 powf/expf, which are
not correctly rounded in every case (errors up to 0.82 ulp), so a few points
differ by one unit in the last place of a power.  The scheme then forms
pi' = (p/p00)^(rd/cp) - pi0 and theta' = T/pi - th0, where one ulp of pi
(~1e-7) or of theta (3e-5 K) is 5e-5 and 2e-5 of the perturbations' range.
The bars for mp_driver alone: theta' and pi' within 2 ulps of the full
theta and pi, every other field within 1e-5 of its range; FP64 budgets to
1e-5 relative.  For a whole large step the dynamical core's own last-place
differences (binary32 powers in p/rho, summation order of the mass fix) enter
the saturation adjustment, which turns one ulp of T (3e-5 K) into
dqvs/dT * 3e-5 K ~ 3e-8 kg/kg of cloud water: 3e-5 of qc's range here.  The
step's bars are therefore 1e-4 of range for qv, qc, qr and 4 ulps for theta'
and pi'; after several steps the extrema agree to 1e-3 relative of range.
"""
import numpy as np
import pytest

from cm1_b200.cases import make_case

pytestmark = pytest.mark.gpu

TOL_RANGE = 1e-5
MP_FIELDS = ["th3d", "pp3d", "prs", "rho"]


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _rel(case, g, r, stag=1):
    I = case.lay.interior(stag)
    gg, rr = g[I].astype(np.float64), r[I].astype(np.float64)
    rng = float(rr.max() - rr.min()) or 1.0
    return float(np.abs(gg - rr).max()) / rng


def _rel2(case, g, r):
    lay = case.lay
    sl = (slice(lay.jx(1), lay.jx(lay.nj) + 1), slice(lay.ix(1), lay.ix(lay.ni) + 1))
    gg, rr = g[sl].astype(np.float64), r[sl].astype(np.float64)
    rng = float(rr.max() - rr.min()) or 1.0
    return float(np.abs(gg - rr).max()) / rng


def _ulps(case, got, ref, base):
    """max |got - ref| in units of the last place of base + ref (the full
    theta or pi of which the perturbation is the difference)."""
    I = case.lay.interior(1)
    tot = (base[I] + ref[I]).astype(np.float32)
    return float((np.abs(got[I].astype(np.float64) - ref[I]) / np.spacing(np.abs(tot))).max())


TOL_Q_STEP = 1e-4       # water species after a whole step (see the module docstring)


def _check_fields(case, got, ref, tol=TOL_RANGE, tol_q=TOL_RANGE, ulps=2.0):
    errs = {}
    u_th = _ulps(case, got["th3d"], ref["th3d"], case.grid["th0"])
    u_pp = _ulps(case, got["pp3d"], ref["pp3d"], case.grid["pi0"])
    print("theta' %.2f ulp of theta, pi' %.2f ulp of pi" % (u_th, u_pp))
    assert u_th <= ulps and u_pp <= ulps, (u_th, u_pp)
    for f in MP_FIELDS:
        if f in ("th3d", "pp3d"):
            continue
        errs[f] = _rel(case, got[f], ref[f])
    for n in range(3):
        e = _rel(case, got["q3d"][n], ref["q3d"][n])
        print("q3d[%d] %.3e of range" % (n, e))
        assert e <= tol_q, (n, e)
    errs["rain"] = _rel2(case, got["rain"], ref["rain"])
    errs["prate"] = _rel2(case, got["prate"], ref["prate"])
    print("worst %.3e %s" % (max(errs.values()), max(errs, key=errs.get)))
    for f, e in errs.items():
        assert e <= tol, (f, e)


@pytest.mark.parametrize("eqtset", [2, 1])
def test_mp_driver_matches_oracle(eqtset, cm1g, oracle_lib):
    """mp_driver alone on a state one dynamical step in (cloud, rain and
    subsaturated air all present)."""
    _torch()
    case = make_case("kessler", ni=40, nj=36, nk=40, eqtset=eqtset)
    st, _, _ = oracle_lib.step(case)
    ref = {k: v.copy() for k, v in st.items()}
    qb_ref, asq_ref = oracle_lib.mp_driver(case, ref)
    I = case.lay.interior(1)
    assert ref["q3d"][1][I].max() > 0 and ref["q3d"][2][I].max() > 0 and ref["prate"].max() > 0
    ctx = cm1g.Context(case.cfg, case.grid)
    dev = cm1g.to_device(st)
    ctx.mp_driver(dev, case.dt)
    got = cm1g.to_host(dev)
    _check_fields(case, got, ref)
    qb, asq = ctx.mp_budget(reset=True)
    for a, b in zip(qb + asq, qb_ref + asq_ref):
        assert a == pytest.approx(b, rel=1e-5, abs=1e-6 * max(abs(x) for x in qb_ref)), (qb, qb_ref)
    assert all(b == 0.0 for b in ctx.mp_budget()[0])        # reset
    # host arrays (drop-in mode) give the same result
    hst = {k: v.copy() for k, v in st.items()}
    ctx.mp_driver(hst, case.dt)
    for f in MP_FIELDS + ["q3d", "rain", "prate"]:
        assert np.array_equal(hst[f], got[f]), f
    ctx.close()


@pytest.mark.parametrize("over", [dict(ni=40, nj=36, nk=40), dict(ni=33, nj=29, nk=40, bc=1)])
def test_one_large_step_with_kessler(over, cm1g, oracle_lib):
    torch = _torch()
    case = make_case("kessler", **over)
    ref, m2_ref, cfl_ref = oracle_lib.step(case)
    ctx = cm1g.Context(case.cfg, case.grid)
    dev = cm1g.to_device(case.state)
    m2, cfl = ctx.step(dev, case.dt, case.mass1)
    torch.cuda.synchronize()
    got = cm1g.to_host(dev)
    _check_fields(case, got, ref, tol_q=TOL_Q_STEP, ulps=4.0)
    for f, stag in (("u3d", 2), ("v3d", 3), ("w3d", 4), ("ua", 2), ("wa", 4)):
        assert _rel(case, got[f], ref[f], stag) <= TOL_RANGE, f
    for n in range(3):
        assert _rel(case, got["qa"][n], ref["qa"][n]) <= TOL_Q_STEP
    assert _ulps(case, got["tha"], ref["tha"], case.grid["th0"]) <= 4.0
    assert _ulps(case, got["ppi"], ref["ppi"], case.grid["pi0"]) <= 4.0
    assert abs(m2 - m2_ref) <= 1e-7 * abs(m2_ref)
    ctx.close()


def test_graph_replay_matches_eager(cm1g):
    torch = _torch()
    case = make_case("kessler", ni=40, nj=36, nk=40)
    ctx = cm1g.Context(case.cfg, case.grid)
    a, b = cm1g.to_device(case.state), cm1g.to_device(case.state)
    for _ in range(3):
        ctx.step(a, case.dt, case.mass1, use_graph=False)
        ctx.step(b, case.dt, case.mass1, use_graph=True)
    torch.cuda.synchronize()
    for k in a:
        assert torch.equal(a[k], b[k]), k
    ctx.close()


def test_several_steps_extrema(cm1g, oracle_lib):
    """Five steps: the extrema of the moist fields and the accumulated
    surface rain agree to 1e-3 of their range."""
    torch = _torch()
    case = make_case("kessler", ni=40, nj=36, nk=40)
    st = case.copy_state()
    ctx = cm1g.Context(case.cfg, case.grid)
    dev = cm1g.to_device(case.state)
    for _ in range(5):
        oracle_lib.step(case, st)
        ctx.step(dev, case.dt, case.mass1, use_graph=True)
    torch.cuda.synchronize()
    got = cm1g.to_host(dev)
    I = case.lay.interior(1)
    for name, g, r in [("qc", got["q3d"][1][I], st["q3d"][1][I]), ("qr", got["q3d"][2][I], st["q3d"][2][I]),
                       ("th", got["th3d"][I], st["th3d"][I]), ("w", got["w3d"][case.lay.interior(4)],
                                                               st["w3d"][case.lay.interior(4)]),
                       ("rain", got["rain"], st["rain"])]:
        rng = float(r.max() - r.min()) or 1.0
        assert abs(float(g.max()) - float(r.max())) <= 1e-3 * rng, name
        assert abs(float(g.min()) - float(r.min())) <= 1e-3 * rng, name
    assert float(got["rain"].max()) > 0.0
    ctx.close()


def test_config_checks(cm1g):
    _torch()
    case = make_case("kessler", ni=16, nj=16, nk=20)
    case.cfg.efall = 1
    with pytest.raises(cm1g.CM1GError):
        cm1g.Context(case.cfg, case.grid)
    case.cfg.efall = 0
    case.cfg.numq = 2
    with pytest.raises(cm1g.CM1GError):
        cm1g.Context(case.cfg, case.grid)


def test_autotune_leaves_the_kessler_state_unchanged(cm1g):
    """The autotuner times steps on a copy of the state: the caller's arrays,
    the accumulated rain included, are left as they were."""
    torch = _torch()
    case = make_case("kessler", ni=40, nj=36, nk=40)
    ctx = cm1g.Context(case.cfg, case.grid)
    dev = cm1g.to_device(case.state)
    dev["rain"] += 0.5
    before = {k: v.clone() for k, v in dev.items()}
    ctx.autotune(dev, case.dt, case.mass1, reps=1)
    torch.cuda.synchronize()
    for k in dev:
        assert torch.equal(dev[k], before[k]), k
    ctx.close()


def test_hundred_steps_periodic(cm1g, oracle_lib):
    """100 large steps with Kessler on a periodic domain: the extrema of qv,
    qc, qr, theta', w and the accumulated rain stay within 1e-3 of their
    range of the oracle's (measured: 1.6e-4 at most)."""
    torch = _torch()
    case = make_case("kessler", ni=40, nj=36, nk=40, bc=1)
    st = case.copy_state()
    ctx = cm1g.Context(case.cfg, case.grid)
    dev = cm1g.to_device(case.state)
    for _ in range(100):
        oracle_lib.step(case, st)
        ctx.step(dev, case.dt, case.mass1, use_graph=True)
    torch.cuda.synchronize()
    got = cm1g.to_host(dev)
    I, W = case.lay.interior(1), case.lay.interior(4)
    for name, g, r in [("qv", got["q3d"][0][I], st["q3d"][0][I]), ("qc", got["q3d"][1][I], st["q3d"][1][I]),
                       ("qr", got["q3d"][2][I], st["q3d"][2][I]), ("th", got["th3d"][I], st["th3d"][I]),
                       ("w", got["w3d"][W], st["w3d"][W]), ("rain", got["rain"], st["rain"])]:
        rng = float(r.max() - r.min()) or 1.0
        assert abs(float(g.max()) - float(r.max())) <= 1e-3 * rng, name
        assert abs(float(g.min()) - float(r.min())) <= 1e-3 * rng, name
    ctx.close()
