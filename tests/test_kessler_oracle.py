"""Known-answer checks of the Kessler restatement (oracle/cm1_oracle.c,
mp_driver's Kessler branch), from the scheme's own equations: no cloud or
rain in subsaturated air leaves the state as it was; after the saturation
adjustment, cloudy air is at saturation; kessler and satadj only move water
between vapour, cloud and rain, so without rain at the surface the column's
water is conserved."""
import numpy as np

from cm1_b200.cases import make_case

f32 = np.float32


def _qvs(t, p, rd=287.04, rv=461.5):
    esl = 611.2 * np.exp(17.67 * (t - 273.15) / (t - 29.65))
    esl = np.minimum(esl, p * 0.5)
    return (rd / rv) * esl / (p - esl)


def test_dry_subsaturated_state_is_unchanged(oracle_lib):
    case = make_case("kessler", ni=16, nj=14, nk=30)
    st = case.copy_state()
    st["q3d"][1][:] = 0.0
    st["q3d"][2][:] = 0.0
    st["q3d"][0] *= f32(0.5)          # well below saturation everywhere
    ref = {k: v.copy() for k, v in st.items()}
    qb, asq = oracle_lib.mp_driver(case, st)
    for k in ("th3d", "pp3d", "prs", "rho", "q3d"):
        assert np.array_equal(st[k], ref[k]), k
    assert all(b == 0.0 for b in qb)
    assert float(st["prate"].max()) == 0.0


def test_cloudy_air_is_saturated(oracle_lib):
    case = make_case("kessler", ni=20, nj=18, nk=30)
    st = case.copy_state()
    oracle_lib.mp_driver(case, st)
    I = case.lay.interior(1)
    k = np.arange(case.lay.NK)[:, None, None]
    th0 = case.grid["th0"]
    pi0 = case.grid["pi0"]
    t = ((th0 + st["th3d"]) * (pi0 + st["pp3d"]))[I].astype(np.float64)
    qv, qc = st["q3d"][0][I].astype(np.float64), st["q3d"][1][I]
    qs = _qvs(t, st["prs"][I].astype(np.float64))
    cloudy = qc > 1.0e-6
    assert cloudy.sum() > 50
    assert np.abs(qv[cloudy] / qs[cloudy] - 1.0).max() < 2e-3


def test_column_water_without_fallout(oracle_lib):
    """Rain only above 3 km falls nowhere near the surface in one step, and
    the conversions conserve water: sum(rho*(qv+qc+qr)) is unchanged up to
    the pdefq clips (asq)."""
    case = make_case("kessler", ni=20, nj=18, nk=30)
    st = case.copy_state()
    z = (np.arange(case.lay.NK) - 0.5) * case.cfg.dz
    st["q3d"][2][z < 3000.0] = 0.0
    I = case.lay.interior(1)
    dv = case.cfg.dx * case.cfg.dy * case.cfg.dz

    def water(s):
        return float((s["rho"][I].astype(np.float64) * s["q3d"][:, I[0], I[1], I[2]].astype(np.float64).sum(0)).sum()
                     * dv)
    w0 = water(st)
    qb, asq = oracle_lib.mp_driver(case, st)
    assert qb[5] == 0.0 and float(st["prate"].max()) == 0.0     # nothing reached the ground
    assert abs(water(st) - w0 - sum(asq)) <= 1e-6 * w0
