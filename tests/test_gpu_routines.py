"""Per-routine parity through the C-ABI entry points that replace the
reference's subroutines (bc.F bcs/bcp/bcu/bcv/bcw, adv.F advs/advu/advv/advw,
sound.F sound, misclibs.F pdefq/calcmass, maxmin.F maxmin)."""
import ctypes as C

import numpy as np
import pytest

from cm1_b200.cases import make_case

pytestmark = pytest.mark.gpu
f32 = np.float32


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def relerr(a, b):
    rng = float(b.max() - b.min()) or 1.0
    return float(np.abs(a.astype(np.float64) - b).max()) / rng


@pytest.mark.parametrize("bc", [1, 2, 3])
@pytest.mark.parametrize("which,stag", [("s", 1), ("p", 1), ("u", 2), ("v", 3), ("w", 4)])
def test_bc_fills_bitwise(bc, which, stag, cm1g, oracle_lib):
    _torch()
    case = make_case("dry_bubble", ni=20, nj=18, nk=12, bc=bc)
    rng = np.random.default_rng(7)
    a = rng.normal(size=case.lay.shape(stag)).astype(f32)
    ref = a.copy()
    code = {"s": 1, "p": 2, "u": 3, "v": 4, "w": 5}[which]
    assert oracle_lib.lib().oracle_bc(C.byref(case.cfg), code, _fp(ref), 1) == 0
    ctx = cm1g.Context(case.cfg, case.grid)
    d = cm1g.to_device({"a": a})["a"]
    ctx.bc(which, d, 1)
    got = d.cpu().numpy()
    assert np.array_equal(got, ref)


def _adv_inputs(case, rng, positive):
    lay = case.lay
    rru = rng.normal(0, 8, lay.shape(2)).astype(f32)
    rrv = rng.normal(0, 8, lay.shape(3)).astype(f32)
    rrw = rng.normal(0, 2, lay.shape(4)).astype(f32)
    rrw[lay.kx(1)] = 0.0
    rrw[lay.kx(case.lay.nk + 1)] = 0.0
    divx = rng.normal(0, 1e-3, lay.shape(1)).astype(f32)
    if positive:
        s = np.clip(rng.normal(0, 1e-3, lay.shape(1)), 0, None).astype(f32)
    else:
        x = np.linspace(0, 6 * np.pi, lay.NI)
        s = (np.sin(x)[None, None, :] * np.cos(np.linspace(0, 3, lay.NJ))[None, :, None]
             * np.linspace(1, 2, lay.NK)[:, None, None] + rng.normal(0, 0.05, lay.shape(1))).astype(f32)
    s0 = (s + rng.normal(0, 1e-4, s.shape)).astype(f32)
    if positive:
        s0 = np.clip(s0, 0, None).astype(f32)
    sten = rng.normal(0, 1e-4, lay.shape(1)).astype(f32)
    return rru, rrv, rrw, divx, s0, s, sten


@pytest.mark.parametrize("bc", [1, 2])
@pytest.mark.parametrize("weno,pdef,pdefweno", [(0, 0, 0), (1, 0, 0), (1, 0, 1), (1, 1, 0), (1, 1, 1), (0, 1, 1)])
def test_advs(bc, weno, pdef, pdefweno, cm1g, oracle_lib):
    _torch()
    case = make_case("dry_bubble", ni=24, nj=20, nk=16, bc=bc, advwenos=1 if weno else 0)
    rng = np.random.default_rng(11)
    rru, rrv, rrw, divx, s0, s, sten = _adv_inputs(case, rng, positive=bool(pdef or pdefweno))
    weps = float(np.float32(1e-2) * np.float32(1e-18))
    ref = sten.copy()
    g = case.grid_struct()
    rc = oracle_lib.lib().oracle_advs(C.byref(case.cfg), C.byref(g), 3, 1, _fp(rru), _fp(rrv), _fp(rrw), _fp(divx),
                                      _fp(s0), _fp(s), _fp(ref), pdef, pdefweno, case.dt, weps)
    assert rc == 0
    ctx = cm1g.Context(case.cfg, case.grid)
    d = cm1g.to_device(dict(rru=rru, rrv=rrv, rrw=rrw, divx=divx, s0=s0, s=s, sten=sten))
    ctx.advs(3, 1, d["divx"], d["rru"], d["rrv"], d["rrw"], d["s0"], d["s"], d["sten"], pdef, pdefweno, case.dt, weps)
    got = d["sten"].cpu().numpy()
    sl = case.lay.interior(1)
    e = relerr(got[sl], ref[sl])
    assert e <= 1e-6, e


@pytest.mark.parametrize("bc", [1, 2])
def test_advuvw(bc, cm1g, oracle_lib):
    _torch()
    case = make_case("supercell", ni=24, nj=20, nk=20, bc=bc)
    lay = case.lay
    rng = np.random.default_rng(3)
    u = (case.state["u3d"] + rng.normal(0, 1, lay.shape(2))).astype(f32)
    v = (case.state["v3d"] + rng.normal(0, 1, lay.shape(3))).astype(f32)
    w = rng.normal(0, 1, lay.shape(4)).astype(f32)
    w[lay.kx(1)] = 0
    w[lay.kx(lay.nk + 1)] = 0
    ut, vt, wt = (rng.normal(0, 1e-3, lay.shape(s)).astype(f32) for s in (2, 3, 4))
    rut, rvt, rwt = ut.copy(), vt.copy(), wt.copy()
    g = case.grid_struct()
    assert oracle_lib.lib().oracle_advuvw(C.byref(case.cfg), C.byref(g), _fp(u), _fp(v), _fp(w),
                                          _fp(rut), _fp(rvt), _fp(rwt)) == 0
    ctx = cm1g.Context(case.cfg, case.grid)
    d = cm1g.to_device(dict(u=u, v=v, w=w, ut=ut, vt=vt, wt=wt))
    ctx.advuvw(1, d["u"], d["v"], d["w"], d["ut"], d["vt"], d["wt"])
    i1 = 2 if bc != 1 else 1
    su = (slice(lay.kx(1), lay.kx(lay.nk) + 1), slice(lay.jx(1), lay.jx(lay.nj) + 1),
          slice(lay.ix(i1), lay.ix(lay.ni + (0 if bc != 1 else 1)) + 1))
    assert relerr(d["ut"].cpu().numpy()[su], rut[su]) <= 1e-6
    sv = (slice(lay.kx(1), lay.kx(lay.nk) + 1), slice(lay.jx(i1), lay.jx(lay.nj + (0 if bc != 1 else 1)) + 1),
          slice(lay.ix(1), lay.ix(lay.ni) + 1))
    assert relerr(d["vt"].cpu().numpy()[sv], rvt[sv]) <= 1e-6
    sw = (slice(lay.kx(2), lay.kx(lay.nk) + 1), slice(lay.jx(1), lay.jx(lay.nj) + 1), slice(lay.ix(1), lay.ix(lay.ni) + 1))
    assert relerr(d["wt"].cpu().numpy()[sw], rwt[sw]) <= 1e-6
    # the per-routine entries (advu, advv, advw) give the combined call's tendencies bit for bit
    e = cm1g.to_device(dict(u=u, v=v, w=w, ut=ut, vt=vt, wt=wt))
    ctx.advu(1, e["u"], e["ut"], e["v"], e["w"])
    ctx.advv(1, e["v"], e["vt"], e["u"], e["w"])
    ctx.advw(1, e["w"], e["wt"], e["u"], e["v"])
    for n in ("ut", "vt", "wt"):
        assert np.array_equal(e[n].cpu().numpy(), d[n].cpu().numpy()), n


@pytest.mark.parametrize("form", ["tile", "col"])
@pytest.mark.parametrize("bc,irbc,roflux", [(1, 4, 0), (2, 4, 0), (2, 2, 0), (2, 4, 1), (2, 2, 1)])
@pytest.mark.parametrize("nrk", [1, 2, 3])
def test_sound_stage(bc, irbc, roflux, nrk, form, cm1g, oracle_lib, monkeypatch):
    """Both forms of the acoustic kernel (3-phase tile, column sweep); with
    irbc=2 the routine forms the phase speeds at every small step and returns
    the last ones in radbcw/e/s/n; with roflux=1 the open boundaries' outflow
    is restricted to the inflow at every small step."""
    _torch()
    monkeypatch.setenv("CM1G_SOUND_FORM", form)
    case = make_case("supercell", ni=24, nj=20, nk=24, bc=bc, irbc=irbc, roflux=roflux)
    lay, st, gr = case.lay, case.state, case.grid
    rng = np.random.default_rng(5 + nrk)
    A = {}
    A["ua"] = (st["ua"] + rng.normal(0, 0.5, lay.shape(2))).astype(f32)
    A["va"] = (st["va"] + rng.normal(0, 0.5, lay.shape(3))).astype(f32)
    A["wa"] = rng.normal(0, 0.2, lay.shape(4)).astype(f32)
    A["wa"][lay.kx(1)] = 0
    A["wa"][lay.kx(lay.nk + 1)] = 0
    A["u3d"] = (A["ua"] + rng.normal(0, 0.1, lay.shape(2))).astype(f32)
    A["v3d"] = (A["va"] + rng.normal(0, 0.1, lay.shape(3))).astype(f32)
    A["w3d"] = A["wa"].copy()
    A["uten"] = rng.normal(0, 1e-3, lay.shape(2)).astype(f32)
    A["vten"] = rng.normal(0, 1e-3, lay.shape(3)).astype(f32)
    A["wten"] = rng.normal(0, 1e-2, lay.shape(4)).astype(f32)
    A["ppi"] = rng.normal(0, 1e-4, lay.shape(1)).astype(f32)
    A["pp3d"] = A["ppi"].copy()
    A["ppx"] = rng.normal(0, 1e-5, lay.shape(1)).astype(f32)
    A["piadv"] = (gr["pi0"] + A["ppi"]).astype(f32)
    A["ppten"] = rng.normal(0, 1e-7, lay.shape(1)).astype(f32)
    A["thv"] = (gr["th0"] + rng.normal(0, 0.5, lay.shape(1))).astype(f32)
    A["ppterm"] = (gr["pi0"] * np.float32(0.4)).astype(f32)
    for n, s in (("rru", 2), ("rrv", 3), ("rrw", 4)):
        A[n] = np.zeros(lay.shape(s), f32)
    for n in ("radbcw", "radbce"):
        A[n] = rng.uniform(-30, 0, (lay.NK, lay.NJ)).astype(f32) * (1 if n == "radbcw" else -1)
    for n in ("radbcs", "radbcn"):
        A[n] = rng.uniform(-30, 0, (lay.NK, lay.NI)).astype(f32) * (1 if n == "radbcs" else -1)
    names = ["ua", "u3d", "uten", "va", "v3d", "vten", "wa", "w3d", "wten", "ppi", "pp3d", "piadv", "ppten",
             "ppx", "thv", "ppterm", "rru", "rrv", "rrw", "radbcw", "radbce", "radbcs", "radbcn"]
    R = {k: v.copy() for k, v in A.items()}
    g = case.grid_struct()
    dttmp = case.dt / (4 - nrk)
    assert oracle_lib.lib().oracle_sound(C.byref(case.cfg), C.byref(g), nrk, case.dt, dttmp,
                                         *[_fp(R[n]) for n in names]) == 0
    ctx = cm1g.Context(case.cfg, case.grid)
    D = cm1g.to_device(A)
    ctx.sound(nrk, case.dt, dttmp, **D)
    G = cm1g.to_host(D)
    ni, nj, nk = lay.ni, lay.nj, lay.nk
    K = slice(lay.kx(1), lay.kx(nk) + 1)
    checks = [("u3d", (K, slice(lay.jx(1), lay.jx(nj) + 1), slice(lay.ix(1), lay.ix(ni + 1) + 1))),
              ("v3d", (K, slice(lay.jx(1), lay.jx(nj + 1) + 1), slice(lay.ix(1), lay.ix(ni) + 1))),
              ("w3d", (slice(lay.kx(2), lay.kx(nk) + 1),) + lay.interior(1)[1:]),
              ("pp3d", lay.interior(1)),
              ("rru", (K, slice(lay.jx(1), lay.jx(nj) + 1), slice(lay.ix(1), lay.ix(ni + 1) + 1))),
              ("rrv", (K, slice(lay.jx(1), lay.jx(nj + 1) + 1), slice(lay.ix(1), lay.ix(ni) + 1))),
              ("rrw", (K,) + lay.interior(1)[1:])]
    if nrk == 3:
        checks.append(("ppx", lay.interior(1)))
    if irbc == 2:
        checks += [(n, (K, slice(lay.jx(1), lay.jx(nj) + 1))) for n in ("radbcw", "radbce")]
        checks += [(n, (K, slice(lay.ix(1), lay.ix(ni) + 1))) for n in ("radbcs", "radbcn")]
    for n, sl in checks:
        e = relerr(G[n][sl], R[n][sl])
        assert e <= 1e-6, (n, e)


def test_pdefq_calcmass_maxmin(cm1g, oracle_lib):
    _torch()
    case = make_case("supercell", ni=24, nj=20, nk=16)
    lay = case.lay
    rng = np.random.default_rng(9)
    q = rng.normal(1e-3, 1e-3, lay.shape(1)).astype(f32)
    rho = case.state["rho"]
    ref = q.copy()
    g = case.grid_struct()
    asq_r = C.c_double(0.0)
    assert oracle_lib.lib().oracle_pdefq(C.byref(case.cfg), C.byref(g), 0.0, C.byref(asq_r), _fp(rho), _fp(ref)) == 0
    ctx = cm1g.Context(case.cfg, case.grid)
    d = cm1g.to_device(dict(q=q, rho=rho))
    asq = ctx.pdefq(0.0, d["rho"], d["q"])
    sl = lay.interior(1)
    assert relerr(d["q"].cpu().numpy()[sl], ref[sl]) <= 1e-6
    assert abs(asq - asq_r.value) <= 1e-6 * abs(asq_r.value) + 1e-30
    tm_r = C.c_double()
    assert oracle_lib.lib().oracle_calcmass(C.byref(case.cfg), C.byref(g), _fp(rho), C.byref(tm_r)) == 0
    assert abs(ctx.calcmass(d["rho"]) - tm_r.value) <= 1e-12 * tm_r.value
    for stag, a in ((1, q), (2, case.state["u3d"]), (4, rng.normal(size=lay.shape(4)).astype(f32))):
        mx, mn, loc = C.c_float(), C.c_float(), (C.c_int * 6)()
        oracle_lib.lib().oracle_maxmin(C.byref(case.cfg), _fp(a), stag, C.byref(mx), C.byref(mn), loc)
        gmx, gmn, gloc = ctx.maxmin(cm1g.to_device({"a": a})["a"], stag)
        assert (gmx, gmn) == (mx.value, mn.value)
        assert tuple(gloc) == tuple(loc)
