"""Known-answer tests that pin the CPU oracle.

The reference ships no golden vectors for this path and cannot be compiled
here (no Fortran compiler), so the oracle is pinned by properties that follow
from the reference's formulas (adv_routines.F:5971-6355, adv.F:650-659,
sound.F, pdef.F, bc.F) and by committed regression fixtures.
"""
import ctypes as C
from fractions import Fraction as Fr

import numpy as np
import pytest

from cm1_b200.cases import make_case

f32 = np.float32


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def cell_avgs(m, start, n):
    return [float((Fr(k) ** (m + 1) - Fr(k - 1) ** (m + 1)) / (m + 1)) for k in range(start, start + n)]


def test_flx5_reproduces_quartics(oracle_lib):
    L = oracle_lib.lib()
    # cell averages over [0,1]..[4,5] -> value at the face x=3 (adv_routines.F:6006-6024)
    for m in range(5):
        s = cell_avgs(m, 1, 5)
        got = L.oracle_flx5(*s)
        assert abs(got - 3.0 ** m) <= 4e-6 * max(1.0, 3.0 ** m), (m, got)
    s = cell_avgs(5, 1, 5)
    assert abs(L.oracle_flx5(*s) - 243.0) > 1.0   # not exact for degree 5


def test_flx3_reproduces_quadratics(oracle_lib):
    L = oracle_lib.lib()
    for m in range(3):
        s = cell_avgs(m, 1, 3)   # face between cells 2 and 3: x = 2
        assert abs(L.oracle_flx3(*s) - 2.0 ** m) <= 4e-6 * max(1.0, 2.0 ** m)


def test_weno5_linear_weights_on_smooth_data(oracle_lib):
    L = oracle_lib.lib()
    # smooth data: the nonlinear weights tend to (0.1, 0.6, 0.3) and WENO5
    # tends to the 5th-order upwind value flx5 (adv_routines.F:6182-6191)
    for h in (0.1, 0.05, 0.025):
        s = [float(np.sin(1.0 + h * k)) for k in range(5)]
        d = abs(L.oracle_weno5(*s, 1e-17) - L.oracle_flx5(*s))
        assert d < 50 * h ** 3, (h, d)
    c = 2.5
    assert L.oracle_weno5(c, c, c, c, c, 1e-17) == pytest.approx(c, rel=1e-7)


def test_weno5_no_new_extrema_at_a_step(oracle_lib):
    L = oracle_lib.lib()
    for s in ([0, 0, 0, 1, 1], [1, 1, 1, 0, 0], [0, 0, 1, 1, 1], [0, 1, 1, 1, 1]):
        v = L.oracle_weno5(*[float(x) for x in s], 1e-17)
        assert -0.02 <= v <= 1.02, (s, v)


def test_upstrpd_keeps_positivity(oracle_lib):
    L = oracle_lib.lib()
    rng = np.random.default_rng(0)
    for _ in range(2000):
        s = rng.uniform(0, 1, 3) * (rng.uniform(size=3) > 0.3)
        assert L.oracle_upstrpd(float(s[0]), float(s[1]), float(s[2]), 1e-18) >= 0.0


def _no_perturbation_case(**over):
    return make_case("dry_bubble", ni=24, nj=20, nk=20, bubble=None, noise=None, **over)


def test_resting_atmosphere_stays_at_rest(oracle_lib):
    case = _no_perturbation_case()
    case.cfg.apmasscon = 0   # mass1 of the generator differs from the model's rho by rounding
    st, m2, cfl = oracle_lib.step(case)
    for f in ("u3d", "v3d", "w3d", "th3d", "pp3d", "ua", "wa"):
        assert np.abs(st[f]).max() == 0.0, f
    assert cfl == 0.0


def test_diffusion_keeps_rest_and_damps_noise(oracle_lib):
    """6th-order diffusion (adv.F:342-406 and the advu/v/w forms): a resting
    atmosphere stays at rest with it on; on a noisy field it only removes
    variance; the mdiff limiter changes the result."""
    case = _no_perturbation_case(diff6=0.04)
    case.cfg.apmasscon = 0
    st, _, _ = oracle_lib.step(case)
    for f in ("u3d", "v3d", "w3d", "th3d", "pp3d"):
        assert np.abs(st[f]).max() == 0.0, f
    runs = {}
    for label, over in (("plain", {}), ("diff", dict(diff6=0.04)), ("mdiff", dict(diff6=0.04, mdiff=1))):
        c = make_case("dry_bubble", ni=24, nj=20, nk=20, noise=dict(amp=0.5, zmax=None), **over)
        runs[label] = (c, oracle_lib.step(c)[0])
    c, plain = runs["plain"]
    lay = c.lay
    th = {k: v[1]["th3d"][lay.interior(1)] for k, v in runs.items()}
    # the 2-dx content of theta' (second differences in x) is damped
    d2 = {k: float(np.abs(v[:, :, 2:] - 2 * v[:, :, 1:-1] + v[:, :, :-2]).mean()) for k, v in th.items()}
    assert d2["diff"] < d2["plain"] and d2["mdiff"] < d2["plain"]
    assert not np.array_equal(th["diff"], th["mdiff"])
    for f, stag in (("u3d", 2), ("v3d", 3), ("w3d", 4)):
        assert not np.array_equal(runs["diff"][1][f][lay.interior(stag)], plain[f][lay.interior(stag)]), f


def test_fp64_build_agrees_with_fp32(oracle_lib):
    """The FP64 (-r8) build of the restatement (oracle/make_r8.py) runs the
    same step from the same inputs; one step apart the two agree to the
    binary32 rounding of the fields (well inside 1e-3 of each range)."""
    for name, over in (("dry_bubble", {}), ("supercell", dict(ni=24, nj=20, nk=24))):
        case = make_case(name, **over)
        r32, _, _ = oracle_lib.step(case)
        r64 = oracle_lib.step_r8(case)
        lay = case.lay
        for f, stag in (("u3d", 2), ("v3d", 3), ("w3d", 4), ("th3d", 1), ("pp3d", 1), ("rho", 1)):
            a, b = r32[f][lay.interior(stag)].astype(np.float64), r64[f][lay.interior(stag)]
            assert b.dtype == np.float64
            rng = float(b.max() - b.min()) or 1.0
            err = float(np.abs(a - b).max()) / rng
            assert 0.0 < err <= 1e-3, (name, f, err)


def test_constant_tracer_in_uniform_flow(oracle_lib):
    # flux-form advection of a constant by a non-divergent flow: the s*divx
    # term cancels the flux divergence (adv.F:650-659)
    case = make_case("cbl", ni=24, nj=20, nk=20, npt=1)
    lay = case.lay
    case.state["pta"][...] = 1.0e-3
    case.state["pt3d"][...] = 1.0e-3
    for k in ("tha", "th3d"):
        case.state[k][...] = 0.0
    st, _, _ = oracle_lib.step(case)
    pt = st["pt3d"][0][lay.interior(1)]
    assert np.abs(pt - 1.0e-3).max() <= 1e-3 * 1e-6


def test_periodic_translation_is_exact(oracle_lib):
    # the same arithmetic runs at every point of a periodic domain, so a
    # shifted start gives the shifted result bit for bit (mass fix off: its
    # domain sum depends on summation order)
    case = make_case("supercell", ni=24, nj=20, nk=20, bc=1)
    case.cfg.apmasscon = 0
    lay = case.lay
    shift, i0, ni = 5, lay.ix(1), lay.ni
    stag_of = {"ua": 2, "u3d": 2, "uten1": 2, "va": 3, "v3d": 3, "vten1": 3, "wa": 4, "w3d": 4, "wten1": 4}
    bc_code = {1: 1, 2: 3, 3: 4, 4: 5}

    def roll(arr, stag):
        """shift the physical points by `shift` cells in x, then refill the
        periodic halos with the oracle's own bc routine"""
        out = arr.copy()
        out[..., i0:i0 + ni] = np.roll(arr[..., i0:i0 + ni], shift, axis=-1)
        if stag == 2:
            out[..., i0 + ni] = out[..., i0]
        code = bc_code[stag]
        for k in range(out.shape[0] if out.ndim == 4 else 1):
            x = out[k] if out.ndim == 4 else out
            x = np.ascontiguousarray(x)
            oracle_lib.lib().oracle_bc(C.byref(case.cfg), code, _fp(x), 0)
            if out.ndim == 4:
                out[k] = x
            else:
                out = x
        return out

    a = case.copy_state()
    b = {k: (roll(v, stag_of.get(k, 1)) if v.ndim >= 3 and v.shape[-1] in (lay.NI, lay.NI + 1) and v.size else v)
         for k, v in a.items()}
    sa, _, _ = oracle_lib.step(case, a)
    sb, _, _ = oracle_lib.step(case, b)
    for f in ("u3d", "v3d", "w3d", "th3d", "pp3d", "q3d", "pt3d"):
        stag = stag_of.get(f, 1)
        x, y = roll(sa[f], stag), sb[f]
        sl = lay.interior(stag)
        if x.ndim == 4:
            sl = (slice(None),) + sl
        assert np.array_equal(x[sl], y[sl]), f


def test_mass_fix_restores_initial_mass(oracle_lib):
    case = make_case("dry_bubble", ni=24, nj=20, nk=20)
    st, m2, _ = oracle_lib.step(case)
    tot = st["rho"][case.lay.interior(1)].astype(np.float64).sum()
    assert abs(tot - case.mass1) <= 1e-6 * case.mass1


def test_tracer_mass_conserved_and_positive(oracle_lib):
    # flux form + periodic boundaries + pdef/pdefq are conservative
    case = make_case("cbl", ni=24, nj=20, nk=20, npt=2)
    lay = case.lay
    sl = lay.interior(1)
    before = [(case.state["rho"][sl].astype(np.float64) * case.state["pt3d"][n][sl]).sum() for n in range(2)]
    st, _, _ = oracle_lib.step(case)
    for n in range(2):
        after = (st["rho"][sl].astype(np.float64) * st["pt3d"][n][sl]).sum()
        assert abs(after - before[n]) <= 1e-4 * before[n]
        assert st["pt3d"][n][sl].min() >= 0.0


@pytest.mark.parametrize("bc", [1, 2])
def test_bcs_semantics(bc, oracle_lib):
    case = make_case("dry_bubble", ni=12, nj=10, nk=6, bc=bc)
    lay = case.lay
    a = np.random.default_rng(1).normal(size=lay.shape(1)).astype(f32)
    assert oracle_lib.lib().oracle_bc(C.byref(case.cfg), 1, _fp(a), 0) == 0
    k = lay.kx(3)
    ni, nj = lay.ni, lay.nj
    for j in range(1, nj + 1):
        if bc == 1:
            assert a[k, lay.jx(j), lay.ix(0)] == a[k, lay.jx(j), lay.ix(ni)]
            assert a[k, lay.jx(j), lay.ix(ni + 3)] == a[k, lay.jx(j), lay.ix(3)]
        else:
            assert a[k, lay.jx(j), lay.ix(-2)] == a[k, lay.jx(j), lay.ix(1)]
            assert a[k, lay.jx(j), lay.ix(ni + 2)] == a[k, lay.jx(j), lay.ix(ni)]
    if bc == 1:  # corners are periodic images once the rows are copied
        assert a[k, lay.jx(0), lay.ix(0)] == a[k, lay.jx(nj), lay.ix(ni)]


def test_golden_fixture_regression(oracle_lib):
    """The oracle reproduces the committed fixture of a small moist,
    open-boundary step bit for bit (tests/golden/make_golden.py)."""
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "supercell_12x10x8_step1.npz")
    fx = np.load(path)
    case = make_case("supercell", ni=12, nj=10, nk=8, seed=42)
    st, m2, cfl = oracle_lib.step(case)
    for k in fx.files:
        if k in ("mass2", "cflmax"):
            continue
        assert np.array_equal(st[k], fx[k]), k
    assert m2 == float(fx["mass2"]) and cfl == float(fx["cflmax"])


def _dtsmall(L, psolver, dx, dy, dz, dt, adapt=0, nx=64, ny=64):
    fdt, ddt, ns = C.c_float(dt), C.c_double(dt), C.c_int()
    rc = L.oracle_dtsmall(psolver, nx, ny, dx, dy, dz, adapt, C.byref(fdt), C.byref(ddt), C.byref(ns))
    return rc, ns.value, fdt.value, ddt.value


def test_dtsmall_known_answers(oracle_lib):
    """misclibs.F:817-915 for the three workloads' grids: dtsm = 0.6 min(dx,dy)/360."""
    L = oracle_lib.lib()
    assert _dtsmall(L, 3, 1000.0, 1000.0, 250.0, 6.0)[:2] == (0, 4)     # 64x64x40 bubble: 6/1.667 -> 4
    assert _dtsmall(L, 3, 500.0, 500.0, 250.0, 3.0)[:2] == (0, 4)       # supercell: 3/0.833 -> 4
    assert _dtsmall(L, 3, 50.0, 50.0, 20.0, 0.5)[:2] == (0, 6)          # CBL: 0.5/0.0833 -> 6
    assert _dtsmall(L, 3, 500.0, 500.0, 250.0, 3.4)[:2] == (0, 6)       # 4.08 -> 4, 3.4/4 > dtsm -> 6
    assert _dtsmall(L, 3, 500.0, 500.0, 250.0, 0.5)[:2] == (0, 4)       # at least 4
    assert _dtsmall(L, 1, 500.0, 500.0, 250.0, 3.0)[:2] == (0, 1)
    assert _dtsmall(L, 3, 50.0, 50.0, 20.0, 20.0)[0] == -2              # 240 > 192 small steps: stop
    rc, ns, fdt, ddt = _dtsmall(L, 3, 50.0, 50.0, 20.0, 20.0, adapt=1)  # adapt_dt: cap and shorten dt
    assert rc == 0 and ns == 192 and abs(ddt - 192 * (0.6 * 50 / 360)) < 1e-4 and fdt == np.float32(ddt)


def test_dtsmall_library_matches_oracle(oracle_lib, cm1g):
    """The C-ABI's dtsmall (host code, no GPU) against the oracle over a sweep."""
    L = oracle_lib.lib()
    for dx in (50.0, 125.0, 500.0, 1000.0, 2000.0):
        for dt in (0.5, 1.0, 3.0, 6.0, 10.0, 12.5):
            for psolver in (2, 3):
                rc, ns, _, _ = _dtsmall(L, psolver, dx, dx, 0.5 * dx, dt)
                if rc == 0:
                    assert cm1g.dtsmall(psolver, 64, 64, dx, dx, 0.5 * dx, dt)[0] == ns, (dx, dt, psolver)
                else:
                    with pytest.raises(cm1g.CM1GError):
                        cm1g.dtsmall(psolver, 64, 64, dx, dx, 0.5 * dx, dt)


def test_klemp_wilhelmson_phase_speeds(oracle_lib):
    """irbc=1 (radbcew/radbcns, bc.F:1948-2046): after a large step the
    stored phase speeds are the ones formed from the step's starting ua/va,
    u - cstar where negative at the west and south boundaries, u + cstar
    where positive at the east and north ones, else 0 (binary32)."""
    case = make_case("supercell", ni=20, nj=18, nk=12, irbc=1)
    lay, cstar = case.lay, np.float32(case.cfg.cstar)
    ua, va = case.state["ua"].copy(), case.state["va"].copy()
    st, _, _ = oracle_lib.step(case)
    K = slice(lay.kx(1), lay.kx(lay.nk) + 1)
    J = slice(lay.jx(1), lay.jx(lay.nj) + 1)
    I = slice(lay.ix(1), lay.ix(lay.ni) + 1)
    w = ua[K, J, lay.ix(1)] - cstar
    e = ua[K, J, lay.ix(lay.ni + 1)] + cstar
    s = va[K, lay.jx(1), I] - cstar
    n = va[K, lay.jx(lay.nj + 1), I] + cstar
    assert np.array_equal(st["radbcw"][K, J], np.where(w < 0, w, 0).astype(np.float32))
    assert np.array_equal(st["radbce"][K, J], np.where(e > 0, e, 0).astype(np.float32))
    assert np.array_equal(st["radbcs"][K, I], np.where(s < 0, s, 0).astype(np.float32))
    assert np.array_equal(st["radbcn"][K, I], np.where(n > 0, n, 0).astype(np.float32))
