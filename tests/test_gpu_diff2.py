"""2nd-order diffusion with a fixed viscosity (difforder=2; diff2def and
diff2u/v/w/s, the block of solve1.F:686-734) through the C-ABI against the
oracle's restatement of diff2.F.  The arithmetic is binary32 additions,
products and divisions in the Fortran's order on both sides, so the
tendencies must agree bit for bit: with free-slip and no-slip lower and upper
boundaries, periodic and open lateral boundaries and both kinds of lateral
walls."""
import ctypes as C

import numpy as np
import pytest

from cm1_b200.cases import make_case

pytestmark = pytest.mark.gpu
P = C.POINTER(C.c_float)


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _fp(a):
    return a.ctypes.data_as(P) if a is not None and a.size else C.cast(None, P)


def _cg(case):
    """Extrapolation weights of rf to the bottom and top w-levels for the
    uniform grid (Lagrange weights from the three nearest s-levels)."""
    dz = case.cfg.dz
    zs = np.array([0.5, 1.5, 2.5]) * dz
    w = [float(np.float32(np.prod([(0.0 - zs[m]) / (zs[l] - zs[m]) for m in range(3) if m != l]))) for l in range(3)]
    return w, w


@pytest.mark.parametrize("name,over,bbc,tbc,idiff", [
    ("supercell", dict(ni=40, nj=36, nk=30), 1, 1, 1),                  # open lateral boundaries
    ("supercell", dict(ni=33, nj=29, nk=30, bc=1), 2, 2, 1),            # periodic, no-slip bottom and top
    ("dry_bubble", dict(ni=30, nj=26, nk=20, bc=3), 1, 2, 1),           # free-slip walls
    ("dry_bubble", dict(ni=30, nj=26, nk=20, bc=4), 2, 1, 2),           # no-slip walls, momentum only
])
def test_diff2_matches_oracle(name, over, bbc, tbc, idiff, cm1g, oracle_lib):
    torch = _torch()
    case = make_case(name, **over)
    st = case.copy_state()
    for _ in range(2):
        oracle_lib.step(case, st)
    rng = np.random.default_rng(11)
    ten = {n: rng.normal(0, 1e-3, st[n].shape).astype(np.float32) for n in ("uten1", "vten1", "wten1", "thten1")}
    ten["qten"] = rng.normal(0, 1e-6, st["qa"].shape).astype(np.float32)
    ten["ptten"] = rng.normal(0, 1e-6, st["pta"].shape).astype(np.float32)
    ref = {k: v.copy() for k, v in ten.items()}
    cgs, cgt = _cg(case)
    cgs_a, cgt_a = np.array(cgs, np.float32), np.array(cgt, np.float32)
    kd = 75.0
    g = case.grid_struct()
    rc = oracle_lib.lib().oracle_diff2(C.byref(case.cfg), C.byref(g), kd, idiff, bbc, tbc, _fp(cgs_a), _fp(cgt_a),
                                       _fp(st["u3d"]), _fp(st["v3d"]), _fp(st["w3d"]), _fp(st["rho"]), _fp(st["tha"]),
                                       _fp(st["qa"]), _fp(st["pta"]), _fp(ref["uten1"]), _fp(ref["vten1"]),
                                       _fp(ref["wten1"]), _fp(ref["thten1"]), _fp(ref["qten"]), _fp(ref["ptten"]))
    assert rc == 0
    ctx = cm1g.Context(case.cfg, case.grid)
    d = cm1g.to_device(dict(st, **ten))
    qa = d["qa"] if case.cfg.imoist else None
    pta = d["pta"] if case.cfg.iptra else None
    ctx.diff2(kd, idiff, bbc, tbc, cgs, cgt, d["u3d"], d["v3d"], d["w3d"], d["rho"], d["tha"], qa, pta,
              d["uten1"], d["vten1"], d["wten1"], d["thten1"], d["qten"] if qa is not None else None,
              d["ptten"] if pta is not None else None)
    torch.cuda.synchronize()
    lay = case.lay
    for n, stag in (("uten1", 2), ("vten1", 3), ("wten1", 4), ("thten1", 1)):
        I = lay.interior(stag)
        got, exp = d[n].cpu().numpy()[I], ref[n][I]
        assert not np.array_equal(exp, ten[n][I]) or (n == "thten1" and idiff != 1), n   # the diffusion acted
        assert np.array_equal(got, exp), (n, float(np.abs(got - exp).max()))
    for n in ("qten", "ptten"):
        for q in range(ref[n].shape[0]):
            I = lay.interior(1)
            assert np.array_equal(d[n].cpu().numpy()[q][I], ref[n][q][I]), (n, q)
    # host arrays give the same tendencies
    h = {k: v.copy() for k, v in ten.items()}
    ctx.diff2(kd, idiff, bbc, tbc, cgs, cgt, st["u3d"], st["v3d"], st["w3d"], st["rho"], st["tha"],
              st["qa"] if qa is not None else None, st["pta"] if pta is not None else None, h["uten1"], h["vten1"],
              h["wten1"], h["thten1"], h["qten"] if qa is not None else None, h["ptten"] if pta is not None else None)
    for n in ("uten1", "vten1", "wten1", "thten1"):
        assert np.array_equal(h[n], d[n].cpu().numpy()), n
    ctx.close()


def test_diff2_damps_a_wave(cm1g):
    """Known answer: a resting atmosphere with a 2-dx theta wave; the scalar
    tendency opposes the wave (diffusion), and a uniform field gets none."""
    torch = _torch()
    case = make_case("dry_bubble", ni=24, nj=20, nk=12, bc=1)
    st = case.copy_state()
    lay = case.lay
    th = np.zeros(lay.shape(1), np.float32)
    ii = np.arange(lay.NI)
    th[:] = np.where(ii % 2 == 0, 0.5, -0.5)[None, None, :].astype(np.float32)
    ten = np.zeros_like(th)
    z = {n: np.zeros_like(st[n]) for n in ("uten1", "vten1", "wten1")}
    ctx = cm1g.Context(case.cfg, case.grid)
    ctx.diff2(10.0, 1, 1, 1, *_cg(case), st["ua"] * 0, st["va"] * 0, st["wa"] * 0, st["rho"], th, None, None,
              z["uten1"], z["vten1"], z["wten1"], ten, None, None)
    I = lay.interior(1)
    assert np.all(ten[I] * th[I] < 0)
    assert np.all(z["uten1"] == 0) and np.all(z["wten1"] == 0)
    ctx.close()
