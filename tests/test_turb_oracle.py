"""Known answers of the oracle's Smagorinsky restatement (calcdef,
turbsmag, gettau, turbu, turbs), from the closure's own formulas: a linear
shear u = a z over a neutral, uniform-density column has defv = a^2, so with
tconfig=2 kmv = (csm dz)^2 |a| and kmh = (csm sqrt(dx dy))^2 sqrt(dmin); the
stress t13 is then the same on every level and the u tendency vanishes; a
uniform theta gets no scalar tendency."""
import ctypes as C

import numpy as np

from cm1_b200.cases import make_case

P = C.POINTER(C.c_float)
f32 = np.float32


def _fp(a):
    return a.ctypes.data_as(P) if a is not None and a.size else C.cast(None, P)


def test_linear_shear_known_answer(oracle_lib):
    case = make_case("cbl", ni=12, nj=10, nk=16)
    lay, cfg = case.lay, case.cfg
    st = case.copy_state()
    a_shear = 0.01
    zh = (np.arange(lay.NK) - 0.5) * cfg.dz
    st["ua"][:] = (a_shear * zh)[:, None, None].astype(f32)
    st["va"][:] = 0.0
    st["wa"][:] = 0.0
    st["tha"][:] = 0.0
    st["rho"][:] = 1.0
    th0 = case.grid["th0"]
    th0_saved = th0.copy()
    th0[:] = 300.0                       # neutral: N^2 = 0
    ten = {n: np.zeros_like(st[n]) for n in ("ua", "va", "wa", "tha")}
    pt = np.zeros_like(st["pta"])
    kmh = np.zeros(lay.shape(4), f32)
    kmv = np.zeros(lay.shape(4), f32)
    g = case.grid_struct()
    one = np.array([1.0, 0.0, 0.0], f32)
    csm = 0.18
    rc = oracle_lib.lib().oracle_turbsmag(C.byref(cfg), C.byref(g), csm, 2, 1, 1, 1, _fp(one), _fp(one),
                                          _fp(st["ua"]), _fp(st["va"]), _fp(st["wa"]), _fp(st["rho"]),
                                          _fp(st["tha"]), _fp(st["pta"]), _fp(ten["ua"]), _fp(ten["va"]),
                                          _fp(ten["wa"]), _fp(ten["tha"]), _fp(pt), _fp(kmh), _fp(kmv))
    th0[:] = th0_saved
    assert rc == 0
    I = lay.interior(1)
    K = (slice(lay.kx(2), lay.kx(lay.nk) + 1),) + I[1:]
    kv = (csm * cfg.dz) ** 2 * a_shear
    assert np.allclose(kmv[K], kv, rtol=2e-6)
    kh = (csm * np.sqrt(cfg.dx * cfg.dy)) ** 2 * np.sqrt(1e-10)
    assert np.allclose(kmh[K], kh, rtol=2e-6)
    assert np.all(kmv[lay.kx(1)] == 0) and np.all(kmv[lay.kx(lay.nk + 1)] == 0)
    U = lay.interior(2)
    assert np.abs(ten["ua"][U]).max() <= 1e-5 * a_shear * kv / cfg.dz   # rounding of u = a z
    assert np.all(ten["tha"][I] == 0.0)
    assert np.all(ten["va"][lay.interior(3)] == 0.0)
