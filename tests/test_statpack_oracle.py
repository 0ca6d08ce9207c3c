"""The statistics package on the CPU: the statpack restatement
(oracle/stat_oracle.c) checked against plain numpy reductions and the
calcmass/calcener restatements, and the GrADS stats record writer of the
library (host code, no device needed)."""
import numpy as np
import pytest

from cm1_b200.cases import make_case, stat_opts

f32 = np.float32


def _state(oracle_lib, name="supercell", steps=2, **over):
    case = make_case(name, **over)
    st = case.copy_state()
    for _ in range(steps):
        oracle_lib.step(case, st)
    return case, st


def _names(case, o):
    """Names in statpack's order for the switches of `o` (setup_stat_vars,
    statpack.F:666-1458), restated here for the CPU test."""
    cfg, nk = case.cfg, case.cfg.nk
    moist = cfg.imoist == 1
    out = ["mtime", "wmax", "wmin", "zwmax", "zwmin"]
    if nk * cfg.dz >= 10000.0:
        for s in ("500", "1000", "2500", "5000", "10k"):
            out += ["wmax" + s, "wmin" + s]
    out += ["umax", "umin", "sumax", "sumin", "vmax", "vmin", "svmax", "svmin", "ppimax", "ppimin", "ppmax", "ppmin",
            "thpmax", "thpmin", "sthpmax", "sthpmin"]
    if moist:
        out += ["maxqv", "minqv", "pratemax", "pratemin"]
    out += ["divmax", "divmin"]
    if moist:
        out += ["rhmax", "rhmin"]
    for n in range(cfg.npt if cfg.iptra else 0):
        out += ["maxpt%d" % (n + 1), "minpt%d" % (n + 1)]
    if moist:
        out += ["themax", "themin", "sthemax", "sthemin", "qctop", "qcbot"]
    out += ["sprsmax", "sprsmin", "psfcmax", "psfcmin", "wspmax", "wspmin", "zwspmax", "zwspmin", "swspmax",
            "swspmin", "cflmax", "vortsfc", "vort1km", "vort2km", "vort3km", "vort4km", "vort5km", "tmass"]
    if moist:
        out += ["tmois", "massqv"]
    out += ["ek", "ei", "ep", "le", "et", "tmu", "tmv", "tmw", "tmfu", "tmfd"]
    if moist:
        out += ["asqv", "bsqv"]
    return out


def test_oracle_statpack_against_numpy(oracle_lib):
    case, st = _state(oracle_lib, ni=20, nj=18, nk=44)
    lay = case.lay
    o, keep = stat_opts(case)
    r = oracle_lib.statpack(case, o, st, mtime=6.0)
    names = _names(case, o)
    assert len(r) == len(names)
    v = dict(zip(names, r))
    inner_w = (slice(1, lay.nk + 2),) + lay.interior(1)[1:]
    w = st["wa"][inner_w]
    assert v["wmax"] == w.max() and v["wmin"] == w.min()
    kmax = int(np.argmax(w.reshape(w.shape[0], -1).max(axis=1)))   # first level holding the max
    assert v["zwmax"] == f32(kmax * case.cfg.dz)
    u = st["ua"][lay.interior(2)]
    assert v["umax"] == u.max() and v["umin"] == u.min() and v["sumax"] == u[0].max()
    t = st["tha"][lay.interior(1)]
    assert v["thpmax"] == t.max() and v["sthpmin"] == t[0].min()
    for n in range(case.cfg.npt):
        p = st["pta"][n][lay.interior(1)]
        assert v["maxpt%d" % (n + 1)] == p.max() and v["minpt%d" % (n + 1)] == p.min()
    assert v["mtime"] == 6.0
    assert v["pratemax"] == 0.0 and v["qcbot"] == 0.0 and v["qctop"] == 0.0
    # tmass: the calcmass restatement
    import ctypes as C
    tm = C.c_double()
    g = case.grid_struct()
    rho = st["rho"]
    assert oracle_lib.lib().oracle_calcmass(C.byref(case.cfg), C.byref(g), rho.ctypes.data_as(C.POINTER(C.c_float)),
                                            C.byref(tm)) == 0
    assert v["tmass"] == f32(tm.value)
    # et is the sum of its parts
    assert v["et"] == pytest.approx(float(v["ek"]) + float(v["ei"]) + float(v["ep"]) + float(v["le"]), rel=1e-6)
    # cfl against a numpy restatement of calccfl (binary32 throughout)
    dt = f32(case.dt)
    dtdx = f32(f32(0.5) * dt) * f32(1.0 / case.cfg.dx)
    dtdz = f32(f32(0.5) * dt) * f32(f32(1.0) / f32(case.cfg.dz))
    ua, va, wa = st["ua"], st["va"], st["wa"]
    kk, jj, ii = lay.interior(1)
    cu = (ua[kk, jj, 3:3 + lay.ni] + ua[kk, jj, 4:4 + lay.ni]) * dtdx
    cv = (va[kk, 3:3 + lay.nj, ii] + va[kk, 4:4 + lay.nj, ii]) * dtdx
    cw = (wa[1:lay.nk + 1, jj, ii] + wa[2:lay.nk + 2, jj, ii]) * dtdz
    assert v["cflmax"] == np.sqrt((cu * cu + cv * cv) + cw * cw).max()


def test_oracle_statpack_ties_at_rest(oracle_lib):
    """A resting initial state: every w is 0, so the first level holds the
    extrema (maxmin.F's strict comparisons), zwmax = zwmin = zf(1) = 0."""
    case = make_case("dry_bubble", ni=16, nj=12, nk=10)
    o, keep = stat_opts(case)
    r = oracle_lib.statpack(case, o, case.copy_state())
    assert r[1] == 0.0 and r[2] == 0.0 and r[3] == 0.0 and r[4] == 0.0


def test_stat_write_records(tmp_path, cm1g):
    path = tmp_path / "cm1out_stats.dat"
    a = np.arange(7, dtype=f32)
    b = -np.arange(7, dtype=f32) - 0.5
    cm1g.stat_write(path, 1, a)
    cm1g.stat_write(path, 3, b)
    cm1g.stat_write(path, 2, a * 2)
    data = np.fromfile(path, dtype=f32).reshape(3, 7)
    assert np.array_equal(data[0], a) and np.array_equal(data[1], a * 2) and np.array_equal(data[2], b)
    with pytest.raises(cm1g.CM1GError):
        cm1g.stat_write(path, 0, a)
