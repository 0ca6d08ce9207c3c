"""Smagorinsky LES tendencies (sgsmodel=2) through the C-ABI against the
oracle's restatement of calcnm, calcdef, turbsmag, gettau and turbu/v/w/s.

Both sides add and multiply in binary32 in the Fortran's order; they differ
only in the two transcendental calls: calcnm's log (N^2) and tconfig=1's cube
root, which the library evaluates in binary64 and rounds once while the
oracle calls the C library's binary32 logf/powf (not correctly rounded in
every case).  A last-place change of N^2 moves kmh/kmv by about one part in
1e7, so the bar is 1e-5 of each tendency increment's range (and of kmh/kmv's
range); measured on a turbulent periodic state: 1e-7 of range at most."""
import ctypes as C

import numpy as np
import pytest

from cm1_b200.cases import make_case

pytestmark = pytest.mark.gpu
P = C.POINTER(C.c_float)
TOL = 1e-5


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _fp(a):
    return a.ctypes.data_as(P) if a is not None and a.size else C.cast(None, P)


def _cg(case):
    dz = case.cfg.dz
    zs = np.array([0.5, 1.5, 2.5]) * dz
    w = [float(np.float32(np.prod([(0.0 - zs[m]) / (zs[l] - zs[m]) for m in range(3) if m != l]))) for l in range(3)]
    return w, w


def _wrap(lay, a):
    """Periodic halos in x and y for any staggering (u(ni+1) = u(1))."""
    xi = [lay.ix((m - lay.ix(0) - 1) % lay.ni + 1) for m in range(a.shape[-1])]
    yj = [lay.jx((m - lay.jx(0) - 1) % lay.nj + 1) for m in range(a.shape[-2])]
    a[...] = a[..., :, xi][..., yj, :]


def les_state(case, seed=5, amp=1.0):
    """The case's state with seeded velocity and theta turbulence (periodic
    halos), so that every deformation term is active."""
    lay = case.lay
    st = case.copy_state()
    rng = np.random.default_rng(seed)
    for name, stag in (("ua", 2), ("va", 3), ("wa", 4), ("tha", 1)):
        a = st[name]
        I = lay.interior(stag)
        a[I] += rng.normal(0.0, amp * (0.3 if name == "tha" else 1.0), a[I].shape).astype(np.float32)
        if stag == 4:
            a[lay.kx(1)] = 0.0
            a[lay.kx(lay.nk + 1)] = 0.0
        _wrap(lay, a)
    for n in range(st["pta"].shape[0]):
        _wrap(lay, st["pta"][n])
    return st


def _run_oracle(oracle_lib, case, st, ten, csm, tconfig, bcturbs, bbc, tbc):
    cgs, cgt = _cg(case)
    ref = {k: v.copy() for k, v in ten.items()}
    lay = case.lay
    kmh = np.zeros(lay.shape(4), np.float32)
    kmv = np.zeros(lay.shape(4), np.float32)
    g = case.grid_struct()
    rc = oracle_lib.lib().oracle_turbsmag(
        C.byref(case.cfg), C.byref(g), csm, tconfig, bcturbs, bbc, tbc, _fp(np.array(cgs, np.float32)),
        _fp(np.array(cgt, np.float32)), _fp(st["ua"]), _fp(st["va"]), _fp(st["wa"]), _fp(st["rho"]), _fp(st["tha"]),
        _fp(st["pta"]), _fp(ref["uten1"]), _fp(ref["vten1"]), _fp(ref["wten1"]), _fp(ref["thten1"]),
        _fp(ref["ptten"]), _fp(kmh), _fp(kmv))
    assert rc == 0
    return ref, kmh, kmv


def _rel(got, exp, base):
    inc = (exp - base).astype(np.float64)
    rng = float(inc.max() - inc.min()) or 1.0
    return float(np.abs(got.astype(np.float64) - exp).max()) / rng


@pytest.mark.parametrize("tconfig,bcturbs,bbc,tbc", [(2, 1, 1, 1), (1, 2, 2, 2), (2, 2, 1, 2), (1, 1, 2, 1)])
def test_turbsmag_matches_oracle(tconfig, bcturbs, bbc, tbc, cm1g, oracle_lib):
    torch = _torch()
    case = make_case("cbl", ni=40, nj=36, nk=30)
    st = les_state(case)
    rng = np.random.default_rng(3)
    ten = {n: rng.normal(0, 1e-3, st[n].shape).astype(np.float32) for n in ("uten1", "vten1", "wten1", "thten1")}
    ten["ptten"] = rng.normal(0, 1e-6, st["pta"].shape).astype(np.float32)
    csm = 0.18
    ref, kmh_ref, kmv_ref = _run_oracle(oracle_lib, case, st, ten, csm, tconfig, bcturbs, bbc, tbc)
    cgs, cgt = _cg(case)
    ctx = cm1g.Context(case.cfg, case.grid)
    d = cm1g.to_device(dict(st, **ten))
    lay = case.lay
    kmh = torch.zeros(lay.shape(4), dtype=torch.float32, device="cuda")
    kmv = torch.zeros_like(kmh)
    ctx.turbsmag(csm, tconfig, bcturbs, bbc, tbc, cgs, cgt, d["ua"], d["va"], d["wa"], d["rho"], d["tha"], d["pta"],
                 d["uten1"], d["vten1"], d["wten1"], d["thten1"], d["ptten"], kmh, kmv)
    torch.cuda.synchronize()
    worst = {}
    for n, stag in (("uten1", 2), ("vten1", 3), ("wten1", 4), ("thten1", 1)):
        I = lay.interior(stag)
        got, exp = d[n].cpu().numpy()[I], ref[n][I]
        assert np.abs(exp - ten[n][I]).max() > 0, n          # the turbulence acted
        worst[n] = _rel(got, exp, ten[n][I])
    I = lay.interior(1)
    for q in range(ref["ptten"].shape[0]):
        worst["pt%d" % q] = _rel(d["ptten"].cpu().numpy()[q][I], ref["ptten"][q][I], ten["ptten"][q][I])
    ring = (slice(None), slice(lay.jx(0), lay.jx(lay.nj + 1) + 1), slice(lay.ix(0), lay.ix(lay.ni + 1) + 1))
    for name, got, exp in (("kmh", kmh, kmh_ref), ("kmv", kmv, kmv_ref)):
        e = exp[ring].astype(np.float64)
        assert e.max() > 0
        worst[name] = float(np.abs(got.cpu().numpy()[ring] - e).max()) / float(e.max() - e.min())
    print({k: "%.2e" % v for k, v in worst.items()})
    for k, v in worst.items():
        assert v <= TOL, (k, v)
    # host arrays (drop-in mode) give the same tendencies as device arrays
    h = {k: v.copy() for k, v in ten.items()}
    ctx.turbsmag(csm, tconfig, bcturbs, bbc, tbc, cgs, cgt, st["ua"], st["va"], st["wa"], st["rho"], st["tha"],
                 st["pta"], h["uten1"], h["vten1"], h["wten1"], h["thten1"], h["ptten"])
    for n in ("uten1", "vten1", "wten1", "thten1", "ptten"):
        assert np.array_equal(h[n], d[n].cpu().numpy()), n
    ctx.close()


def test_turbsmag_scalar_flux_form_conserves(cm1g):
    """Periodic laterals and zero flux at the bottom and top (bcturbs=1):
    the scalar tendencies are a flux divergence, so sum(rho * dtheta) over
    the domain vanishes to rounding, at a larger size."""
    torch = _torch()
    case = make_case("cbl", ni=192, nj=160, nk=64)
    st = les_state(case, seed=9)
    lay = case.lay
    cgs, cgt = _cg(case)
    ctx = cm1g.Context(case.cfg, case.grid)
    d = cm1g.to_device(st)
    z = {n: torch.zeros_like(d[n]) for n in ("ua", "va", "wa", "tha", "pta")}
    ctx.turbsmag(0.18, 2, 1, 1, 1, cgs, cgt, d["ua"], d["va"], d["wa"], d["rho"], d["tha"], d["pta"], z["ua"], z["va"],
                 z["wa"], z["tha"], z["pta"])
    torch.cuda.synchronize()
    I = lay.interior(1)
    rho = st["rho"][I].astype(np.float64)
    for name, ten in (("theta", z["tha"].cpu().numpy()[I]), ("pt0", z["pta"].cpu().numpy()[0][I])):
        f = rho * ten.astype(np.float64)
        assert np.abs(f).sum() > 0
        assert abs(f.sum()) <= 1e-5 * np.abs(f).sum(), name
    ctx.close()


def test_turbsmag_refuses_what_is_not_built(cm1g):
    _torch()
    cgs = cgt = [1.0, 0.0, 0.0]
    case = make_case("supercell", ni=24, nj=20, nk=16)          # open boundaries, moist
    st = case.copy_state()
    ctx = cm1g.Context(case.cfg, case.grid)
    with pytest.raises(cm1g.CM1GError):
        ctx.turbsmag(0.18, 2, 1, 1, 1, cgs, cgt, st["ua"], st["va"], st["wa"], st["rho"], st["tha"], None,
                     st["ua"] * 0, st["va"] * 0, st["wa"] * 0)
    ctx.close()
    case = make_case("cbl", ni=24, nj=20, nk=16)
    st = case.copy_state()
    ctx = cm1g.Context(case.cfg, case.grid)
    with pytest.raises(cm1g.CM1GError):       # bbc=3 needs the surface layer
        ctx.turbsmag(0.18, 2, 1, 3, 1, cgs, cgt, st["ua"], st["va"], st["wa"], st["rho"], st["tha"], None,
                     st["ua"] * 0, st["va"] * 0, st["wa"] * 0)
    ctx.close()
