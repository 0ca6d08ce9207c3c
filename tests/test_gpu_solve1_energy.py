"""solve1's tendency initialisation (solve1.F:414-486) and calcener
(misclibs.F:3343-3454) through the C-ABI against the oracle."""
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
    return a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else C.cast(None, C.POINTER(C.c_float))


@pytest.mark.parametrize("irdamp", [0, 1, 2])
def test_tendency_init_bitwise(irdamp, cm1g, oracle_lib):
    _torch()
    case = make_case("supercell", ni=24, nj=20, nk=16)
    lay, st = case.lay, case.state
    rng = np.random.default_rng(31 + irdamp)
    tauh = rng.uniform(0, 1, lay.shape(1)).astype(f32)
    taus = rng.uniform(0, 1, lay.shape(1)).astype(f32)
    tauf = rng.uniform(0, 1, lay.shape(4)).astype(f32)
    uavg, vavg, thavg = (rng.normal(0, 3, lay.NK).astype(f32) for _ in range(3))
    ins = dict(ua=st["ua"], va=st["va"], wa=rng.normal(0, 1, lay.shape(4)).astype(f32), tha=st["tha"])
    outs = {n: rng.normal(0, 1, st[n].shape).astype(f32) for n in ("uten1", "vten1", "wten1", "thten1", "qten", "ptten")}
    ref = {k: v.copy() for k, v in outs.items()}
    g = case.grid_struct()
    assert oracle_lib.lib().oracle_tendency_init(
        C.byref(case.cfg), C.byref(g), irdamp, 1.0 / 300.0, _fp(tauh), _fp(taus), _fp(tauf), _fp(uavg), _fp(vavg),
        _fp(thavg), _fp(ins["ua"]), _fp(ins["va"]), _fp(ins["wa"]), _fp(ins["tha"]), *[_fp(ref[n]) for n in
        ("uten1", "vten1", "wten1", "thten1", "qten", "ptten")]) == 0
    ctx = cm1g.Context(case.cfg, case.grid)
    d = cm1g.to_device(dict(outs, tauh=tauh, taus=taus, tauf=tauf, uavg=uavg, vavg=vavg, thavg=thavg, **ins))
    ctx.tendency_init(irdamp, 1.0 / 300.0, d["uten1"], d["vten1"], d["wten1"], d["thten1"], d["qten"], d["ptten"],
                      d["tauh"], d["taus"], d["tauf"], d["uavg"], d["vavg"], d["thavg"], d["ua"], d["va"], d["wa"],
                      d["tha"])
    for n in ref:
        assert np.array_equal(d[n].cpu().numpy(), ref[n]), n


@pytest.mark.parametrize("moist", [False, True])
def test_calcener_matches_oracle(moist, cm1g, oracle_lib):
    _torch()
    case = make_case("supercell" if moist else "dry_bubble", ni=40, nj=36, nk=24)
    lay, st = case.lay, case.state
    rng = np.random.default_rng(5)
    zh = np.ascontiguousarray(np.broadcast_to(
        ((np.arange(lay.NK) - 0.5) * case.cfg.dz).astype(f32)[:, None, None], lay.shape(1)), dtype=f32)
    wa = rng.normal(0, 2, lay.shape(4)).astype(f32)
    qv = st["q3d"][0] if moist else None
    ql = rng.uniform(0, 1e-3, lay.shape(1)).astype(f32) if moist else None
    vr = rng.uniform(0, 5, lay.shape(1)).astype(f32) if moist else None
    out = (C.c_double * 5)()
    g = case.grid_struct()
    assert oracle_lib.lib().oracle_calcener(C.byref(case.cfg), C.byref(g), _fp(zh), _fp(st["rho"]), _fp(st["ua"]),
                                            _fp(st["va"]), _fp(wa), _fp(st["ppi"]), _fp(st["tha"]), _fp(qv), _fp(ql),
                                            _fp(None), _fp(vr), out) == 0
    ctx = cm1g.Context(case.cfg, case.grid)
    arrs = dict(zh=zh, rho=st["rho"], ua=st["ua"], va=st["va"], wa=wa, ppi=st["ppi"], tha=st["tha"])
    if moist:
        arrs.update(qv=np.ascontiguousarray(qv), ql=ql, vr=vr)
    d = cm1g.to_device(arrs)
    got = ctx.calcener(d["zh"], d["rho"], d["ua"], d["va"], d["wa"], d["ppi"], d["tha"], d.get("qv"), d.get("ql"),
                       None, d.get("vr"))
    for a, b in zip(got, tuple(out)):
        assert abs(a - b) <= 1e-12 * abs(b) + 1e-300, (got, tuple(out))
    # host pointers through the same entry point give the same numbers
    got_h = ctx.calcener(zh, st["rho"], st["ua"], st["va"], wa, st["ppi"], st["tha"], qv if moist else None,
                         ql, None, vr)
    assert got_h == got
