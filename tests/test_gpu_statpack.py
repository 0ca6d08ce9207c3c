"""cm1g_statpack (the statistics package on the device) through the C-ABI
against the statpack restatement of the oracle, on the same states.

Extrema of fields and of binary32 expressions evaluated in the reference's
order are compared bit for bit.  FP64 budgets may differ in the last bits of
their binary64 sums (a tree reduction per level instead of a serial loop), so
they are compared to 1e-6 relative.  Entries that call the math library
(pow for the pressure perturbation and theta-e, exp for the relative
humidity) are compared to 1e-5 relative; the pressure perturbation, a
difference of two values near 1e5 Pa, to 0.02 Pa (two units in the last
place of 1e5)."""
import numpy as np
import pytest

from cm1_b200.cases import make_case, stat_opts

pytestmark = pytest.mark.gpu

SUMS = {"tmass", "tmois", "massqv", "massqc", "massqr", "ek", "ei", "ep", "le", "et", "tmu", "tmv", "tmw", "tmfu",
        "tmfd"}
MATHLIB = {"rhmax", "rhmin", "themax", "themin", "sthemax", "sthemin"}
PP = {"ppmax", "ppmin"}


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _compare(names, got, ref):
    assert len(got) == len(ref) == len(names)
    for n, a, b in zip(names, got, ref):
        if n in SUMS:
            assert a == pytest.approx(b, rel=1e-6, abs=1e-30), n
        elif n in MATHLIB:
            assert a == pytest.approx(b, rel=1e-5), n
        elif n in PP:
            assert abs(float(a) - float(b)) <= 0.02, n
        else:
            assert a == b or (np.isnan(a) and np.isnan(b)), (n, a, b)


def _args(case, st):
    f = [st[n] for n in ("ua", "va", "wa", "ppi", "tha", "prs", "rho")]
    kw = {}
    if case.cfg.imoist:
        kw["qa"] = st["qa"]
    if case.cfg.iptra:
        kw["pta"] = st["pta"]
    return f, kw


@pytest.mark.parametrize("name,over,steps", [
    ("dry_bubble", dict(ni=40, nj=36, nk=20), 3),
    ("dry_bubble", dict(ni=16, nj=12, nk=10), 0),                  # at rest: every w ties
    ("supercell", dict(ni=48, nj=40, nk=44), 3),                    # moist, 5 tracers, open bcs, top 11 km
    ("supercell", dict(ni=33, nj=17, nk=44, bc=1), 2),              # periodic
    ("supercell", dict(ni=64, nj=64, nk=44), 1),                    # s-levels 1 chunk, u/v-levels 2
    ("dry_bubble", dict(ni=150, nj=61, nk=12), 2),                  # several chunks per level
])
def test_statpack_matches_oracle(name, over, steps, cm1g, oracle_lib):
    torch = _torch()
    case = make_case(name, **over)
    st = case.copy_state()
    for _ in range(steps):
        oracle_lib.step(case, st)
    o, keep = stat_opts(case)
    rng = np.random.default_rng(3)
    prate = rng.uniform(0, 1e-3, (case.lay.NJ, case.lay.NI)).astype(np.float32) if case.cfg.imoist else None
    nq = case.cfg.numq if case.cfg.imoist else 0
    asq, bsq = np.arange(1, nq + 1) * 1.5e3, -np.arange(1, nq + 1) * 2.5e2
    ref = oracle_lib.statpack(case, o, st, mtime=steps * case.dt, prate=prate, asq=asq, bsq=bsq)
    ctx = cm1g.Context(case.cfg, case.grid)
    names = ctx.stat_setup(o)
    dev = cm1g.to_device(st)
    f, kw = _args(case, dev)
    if prate is not None:
        kw["prate"] = torch.from_numpy(prate).cuda()
    got = ctx.statpack(steps * case.dt, case.dt, *f, asq=asq if nq else None, bsq=bsq if nq else None, **kw)
    _compare(names, got, ref)
    # host arrays (drop-in mode) give the same numbers
    fh, kwh = _args(case, st)
    if prate is not None:
        kwh["prate"] = prate
    got_h = ctx.statpack(steps * case.dt, case.dt, *fh, asq=asq if nq else None, bsq=bsq if nq else None, **kwh)
    assert np.array_equal(got, got_h)
    if steps == 0:
        v = dict(zip(names, got))
        assert v["wmax"] == v["wmin"] == v["zwmax"] == v["zwmin"] == 0.0
    ctx.close()


def test_statpack_switches_and_errors(cm1g, oracle_lib):
    _torch()
    case = make_case("supercell", ni=24, nj=20, nk=44)
    st = case.copy_state()
    oracle_lib.step(case, st)
    ctx = cm1g.Context(case.cfg, case.grid)
    # a subset of switches gives the subset of entries, in order
    o, keep = stat_opts(case, off=("stat_u", "stat_rh", "stat_vort", "stat_tenerg", "stat_wlevs", "stat_qsrc"))
    names = ctx.stat_setup(o)
    assert "umax" not in names and "rhmax" not in names and "vort1km" not in names and "ek" not in names
    ref = oracle_lib.statpack(case, o, st, mtime=3.0)
    dev = cm1g.to_device(st)
    f, kw = _args(case, dev)
    _compare(names, ctx.statpack(3.0, case.dt, *f, **kw), ref)
    # statistics that are not built are refused
    for sw in ("stat_km", "stat_rmw", "stat_rhi"):
        o2, keep2 = stat_opts(case)
        setattr(o2, sw, 1)
        with pytest.raises(cm1g.CM1GError):
            ctx.stat_setup(o2)
    # a field the statistics need must be given
    o3, keep3 = stat_opts(case)
    ctx.stat_setup(o3)
    with pytest.raises(cm1g.CM1GError):
        ctx.statpack(0.0, case.dt, f[0], f[1], None, *f[3:], asq=np.zeros(1), bsq=np.zeros(1), **kw)
    ctx.close()


def test_statpack_with_kessler_liquid(cm1g, oracle_lib):
    """Statistics of a Kessler state (qv, qc, qr): cloud top and base from qc,
    the total moisture and the masses of the liquid species, and the energy
    budget's liquid terms, against the oracle."""
    torch = _torch()
    case = make_case("kessler", ni=40, nj=36, nk=44)
    st = case.copy_state()
    for _ in range(2):
        oracle_lib.step(case, st)
    o, keep = stat_opts(case, qnames=("qv", "qc", "qr"), nql=(2, 3), cloud=(1,), budnames=("tcond", "tevac"))
    I = case.lay.interior(1)
    assert st["q3d"][1][I].max() > 1e-5
    qb = np.array([1.5e6, 2.5e5])
    asq, bsq = np.array([1.0, 2.0, 3.0]), np.array([-1.0, -2.0, -3.0])
    ref = oracle_lib.statpack(case, o, st, mtime=6.0, prate=st["prate"], qbudget=qb, asq=asq, bsq=bsq)
    ctx = cm1g.Context(case.cfg, case.grid)
    names = ctx.stat_setup(o)
    for n in ("maxqc", "minqr", "qctop", "qcbot", "tmois", "massqv", "massqc", "massqr", "le", "tcond", "asqr"):
        assert n in names, n
    dev = cm1g.to_device(st)
    f, kw = _args(case, dev)
    kw["prate"] = dev["prate"]
    got = ctx.statpack(6.0, case.dt, *f, qbudget=qb, asq=asq, bsq=bsq, **kw)
    _compare(names, got, ref)
    v = dict(zip(names, got))
    assert v["qctop"] > v["qcbot"] > 0.0 and v["le"] != 0.0 and v["pratemax"] > 0.0
    ctx.close()
