"""Seeded synthetic inputs for the large-step workloads.

The reference hard-codes its bubble, noise amplitude and soundings
(init3d.F:450-487, 1446-1470; base.F:363-450, 842-908) and draws its noise
from a compiler-specific RNG, so the inputs are generated here and handed
identically to the CUDA library and to the CPU oracle.

Arrays use the reference's Fortran layout.  A numpy array of shape
(NK, NJ, NI) in C order is the Fortran array (ib:ie, jb:je, kb:ke).

Workloads (sizes can be overridden for small parity cases):
  dry_bubble   64x64x40, dx=1 km, dz=250 m, constant-N sounding, +2 K
               cos^2 bubble, periodic, 5th order, dt=6 s, nsound=6
  supercell    256x256x80, dx=500 m, dz=250 m, Weisman-Klemp sounding,
               curved hodograph, WENO5 theta/qv/5 tracers, open-radiative,
               dt=3 s, nsound=8
  cbl          1024x1024x128, dx=50 m, dz=20 m, mixed layer + inversion,
               WENO5 theta + 2 tracers, periodic, dt=0.5 s, nsound=6
"""
from dataclasses import dataclass, field
import ctypes as C
import math

import numpy as np

from .abi import Config, Grid, State, StatOpts, STAT_SWITCHES, GRID_FIELDS, STATE_FIELDS, fptr, CM1G_MAXQ

G = 9.81
RD = 287.04
RV = 461.5
CP = 1005.7
P00 = 1.0e5


def cm1_constants(testcase=0):
    """binary32 constants as constants.F:set_constants computes them."""
    f = np.float32
    rd, cp = f(287.04), f(1005.7)
    c = dict(g=f(9.81), rd=rd, cp=cp, rv=f(461.5))
    c["cv"] = f(cp - rd)
    c["rddcv"] = f(rd / c["cv"])
    c["cpdrd"] = f(cp / rd)
    c["reps"] = f(c["rv"] / rd)
    return c


class Layout:
    """Index helper for the Fortran-layout arrays of one grid."""

    def __init__(self, ni, nj, nk, ngxy=3):
        self.ni, self.nj, self.nk, self.ngxy = ni, nj, nk, ngxy
        self.ib, self.ie = 1 - ngxy, ni + ngxy
        self.jb, self.je = 1 - ngxy, nj + ngxy
        self.kb, self.ke = 0, nk + 1
        self.NI, self.NJ, self.NK = ni + 2 * ngxy, nj + 2 * ngxy, nk + 2

    def shape(self, stag=1):
        NI, NJ, NK = self.NI, self.NJ, self.NK
        return {1: (NK, NJ, NI), 2: (NK, NJ, NI + 1), 3: (NK, NJ + 1, NI), 4: (NK + 1, NJ, NI)}[stag]

    def zeros(self, stag=1, n=None):
        s = self.shape(stag)
        return np.zeros(((n,) + s) if n else s, np.float32)

    def ix(self, i):
        return i - self.ib

    def jx(self, j):
        return j - self.jb

    def kx(self, k):
        return k - self.kb

    def interior(self, stag=1):
        """Slice of the physical points (k, j, i) of an array."""
        ni, nj, nk = self.ni, self.nj, self.nk
        i1 = ni + (1 if stag == 2 else 0)
        j1 = nj + (1 if stag == 3 else 0)
        k1 = nk + (1 if stag == 4 else 0)
        return (slice(self.kx(1), self.kx(k1) + 1), slice(self.jx(1), self.jx(j1) + 1),
                slice(self.ix(1), self.ix(i1) + 1))


def _hydrostatic_pi(zh, theta_v_fn, psfc=P00):
    """Exner function at heights zh from dpi/dz = -g/(cp*theta_v)."""
    ztop = float(max(zh.max(), 0.0)) + 10.0
    zf = np.linspace(0.0, ztop, int(ztop / 2.0) + 2)
    integrand = G / (CP * theta_v_fn(zf))
    cum = np.concatenate([[0.0], np.cumsum(0.5 * (integrand[1:] + integrand[:-1]) * np.diff(zf))])
    pis = (psfc / P00) ** (RD / CP)
    return pis - np.interp(zh, zf, cum)


def _sounding(kind, z, **kw):
    """theta(z), qv(z) for the analytic soundings (float64)."""
    if kind == "constant_n":
        th_s, bv = kw.get("th_sfc", 300.0), kw.get("bv", 0.01)
        return th_s * np.exp(bv * bv * z / G), np.zeros_like(z)
    if kind == "cbl":
        zi, lapse = kw.get("zi", 1000.0), kw.get("lapse", 0.005)
        th = 300.0 + np.where(z > zi, lapse * (z - zi), 0.0)
        return th, np.zeros_like(z)
    if kind == "weisman_klemp":
        # Weisman and Klemp (1982, MWR) analytic sounding, as base.F isnd=5
        # describes it: theta0=300 K, tropopause 12 km at 343 K and 213 K,
        # RH 1-0.75(z/ztr)^1.25, qv capped at qv_pbl in the boundary layer.
        th0, thtr, ztr, ttr = 300.0, 343.0, 12000.0, 213.0
        qv_pbl = kw.get("qv_pbl", 0.014)
        ratio = np.clip(z / ztr, 0.0, None)
        th = np.where(z <= ztr, th0 + (thtr - th0) * ratio ** 1.25,
                      thtr * np.exp(G * (z - ztr) / (CP * ttr)))
        rh = np.where(z <= ztr, 1.0 - 0.75 * ratio ** 1.25, 0.25)
        qv = np.zeros_like(z)
        for _ in range(8):  # theta_v -> pi -> T,p -> qv fixed point
            qv_c = qv.copy()
            thv_fn = lambda zz: np.interp(zz, z, th * (1.0 + qv_c * RV / RD) / (1.0 + qv_c))
            pi = _hydrostatic_pi(z, thv_fn)
            t = th * pi
            p = P00 * pi ** (CP / RD)
            es = 611.2 * np.exp(17.67 * (t - 273.15) / (t - 29.65))
            qvs = (RD / RV) * es / np.maximum(p - es, 1.0)
            qv = np.minimum(qv_pbl, rh * qvs)
        return th, qv
    raise ValueError(kind)


def _hodograph(kind, z, **kw):
    if kind == "rest":
        return np.zeros_like(z), np.zeros_like(z)
    if kind == "uniform":
        return np.full_like(z, kw.get("u", 0.0)), np.full_like(z, kw.get("v", 0.0))
    if kind == "shear":
        # u grows linearly from 0 to `du` over the lowest `depth` metres, constant above
        du, depth = kw.get("du", 10.0), kw.get("depth", 6000.0)
        return du * np.clip(z / depth, 0.0, 1.0), np.zeros_like(z)
    if kind == "curved":
        # quarter circle of radius 10 m/s below 2 km, straight to U at 6 km,
        # constant above; shifted so the storm is roughly stationary.
        us, ztop = kw.get("U", 20.0), 6000.0
        zc, r = 2000.0, 10.0
        u = np.where(z < zc, r - r * np.cos(0.5 * np.pi * z / zc),
                     np.where(z < ztop, r + (us - r) * (z - zc) / (ztop - zc), us))
        v = np.where(z < zc, r * np.sin(0.5 * np.pi * z / zc), r)
        return u - 0.5 * us, v - 0.5 * r
    raise ValueError(kind)


@dataclass
class Case:
    name: str
    lay: Layout
    cfg: Config
    grid: dict
    state: dict
    dt: float
    mass1: float
    nsteps: int
    _keep: list = field(default_factory=list)

    def grid_struct(self):
        g = Grid()
        for n in GRID_FIELDS:
            setattr(g, n, fptr(self.grid[n].ctypes.data))
        return g

    def state_struct(self, arrays=None):
        """cm1g_state_t over host numpy arrays (default: this case's state)."""
        arrays = self.state if arrays is None else arrays
        s = State()
        for n in STATE_FIELDS:
            a = arrays.get(n)
            setattr(s, n, fptr(a.ctypes.data) if a is not None and a.size else C.cast(None, C.POINTER(C.c_float)))
        return s

    def copy_state(self):
        return {k: v.copy() for k, v in self.state.items()}


def _fill_lateral(lay, a, wbc, stag=1):
    """Fill the 3-wide lateral halos of a field for its initial state
    (periodic wrap or zero-gradient copy), over every level."""
    ng, ni, nj = lay.ngxy, lay.ni, lay.nj
    ie = ni + (1 if stag == 2 else 0)
    je = nj + (1 if stag == 3 else 0)
    i0, j0 = lay.ix(1), lay.jx(1)
    if wbc == 1:
        per_i = ni
        for h in range(1, ng + 1):
            a[..., :, i0 - h] = a[..., :, i0 - h + per_i]
        for h in range(1, ng + (2 if stag == 2 else 1)):
            a[..., :, lay.ix(ie) + h] = a[..., :, lay.ix(ie) + h - per_i]
        for h in range(1, ng + 1):
            a[..., j0 - h, :] = a[..., j0 - h + nj, :]
        for h in range(1, ng + (2 if stag == 3 else 1)):
            a[..., lay.jx(je) + h, :] = a[..., lay.jx(je) + h - nj, :]
    else:
        for h in range(1, ng + 1):
            a[..., :, i0 - h] = a[..., :, i0]
        for h in range(1, ng + (2 if stag == 2 else 1)):
            a[..., :, lay.ix(ie) + h] = a[..., :, lay.ix(ie)]
        for h in range(1, ng + 1):
            a[..., j0 - h, :] = a[..., j0, :]
        for h in range(1, ng + (2 if stag == 3 else 1)):
            a[..., lay.jx(je) + h, :] = a[..., lay.jx(je), :]


WORKLOADS = {
    "dry_bubble": dict(ni=64, nj=64, nk=40, dx=1000.0, dz=250.0, dt=6.0, nsound=6, nsteps=10,
                       sounding="constant_n", wind="rest", bc=1, moist=False, npt=0,
                       advwenos=0, bubble=dict(amp=2.0, xr=4000.0, zr=1400.0, zc=1400.0),
                       noise=dict(amp=0.01, zmax=None)),
    "supercell": dict(ni=256, nj=256, nk=80, dx=500.0, dz=250.0, dt=3.0, nsound=8, nsteps=60,
                      sounding="weisman_klemp", wind="curved", bc=2, moist=True, npt=5,
                      advwenos=1, bubble=dict(amp=3.0, xr=10000.0, zr=1400.0, zc=1400.0),
                      noise=dict(amp=0.1, zmax=None)),
    # the supercell with Kessler warm-rain microphysics (ptype=1: qv, qc, qr)
    # and seeded cloud and rain in the bubble, so that every process of the
    # scheme (condensation, autoconversion, accretion, evaporation, fallout)
    # acts from the first step
    "kessler": dict(ni=256, nj=256, nk=80, dx=500.0, dz=250.0, dt=3.0, nsound=8, nsteps=60,
                    sounding="weisman_klemp", wind="curved", bc=2, moist=True, npt=0, ptype=1,
                    advwenos=1, bubble=dict(amp=3.0, xr=10000.0, zr=1400.0, zc=1400.0),
                    noise=dict(amp=0.1, zmax=None)),
    "cbl": dict(ni=1024, nj=1024, nk=128, dx=50.0, dz=20.0, dt=0.5, nsound=6, nsteps=200,
                sounding="cbl", wind=("uniform", dict(u=5.0, v=0.0)), bc=1, moist=False, npt=2,
                advwenos=1, bubble=None, noise=dict(amp=0.1, zmax=400.0)),
}


def make_case(name, seed=1234, **over):
    """Build a seeded workload.  `over` may override ni, nj, nk, dx, dz, dt,
    nsound, advwenos, npt, bc, moist, ptype (for small parity cases), eqtset,
    irbc (the open boundaries' phase speeds: 1, 2 or 4), roflux (1: outflow
    restricted to the inflow), and add diff6 (kdiff6 of the 6th-order
    diffusion) and mdiff."""
    w = dict(WORKLOADS[name])
    w.update(over)
    ni, nj, nk = int(w["ni"]), int(w["nj"]), int(w["nk"])
    dx, dz = float(w["dx"]), float(w["dz"])
    lay = Layout(ni, nj, nk, 3)
    rng = np.random.default_rng(seed)
    moist, npt, bc = bool(w["moist"]), int(w["npt"]), int(w["bc"])

    cfg = Config()
    cfg.ni, cfg.nj, cfg.nk, cfg.ngxy = ni, nj, nk, 3
    cfg.dx, cfg.dy, cfg.dz = dx, dx, dz
    cfg.wbc = cfg.ebc = cfg.sbc = cfg.nbc = bc
    cfg.hadvordrs = cfg.vadvordrs = cfg.hadvordrv = cfg.vadvordrv = 5
    cfg.advwenos, cfg.advwenov, cfg.weno_order = int(w["advwenos"]), 0, 5
    cfg.nsound, cfg.alph, cfg.kdiv = int(w["nsound"]), 0.60, 0.10
    ptype = int(w.get("ptype", 0)) if moist else 0
    cfg.imoist, cfg.eqtset = (1 if moist else 0), int(w.get("eqtset", 2))
    cfg.numq, cfg.nqv = ((3 if ptype == 1 else 1), 1) if moist else (0, 1)
    # microphysics (cm1.F:311-319, param.F:3169-3175)
    cfg.ptype, cfg.efall = ptype, 0
    cfg.nql1, cfg.nql2 = (2, 3) if ptype == 1 else (0, 0)
    cfg.tsmall, cfg.qsmall = 1.0e-4, 1.0e-14
    cfg.iptra, cfg.npt, cfg.pdtra = (1 if npt > 0 else 0), npt, 1
    cfg.apmasscon = 1
    cfg.irbc, cfg.cstar, cfg.roflux = int(w.get("irbc", 4)), 30.0, int(w.get("roflux", 0))
    cfg.smeps = 1.0e-30
    cfg.testcase, cfg.psolver, cfg.terrain_flag, cfg.axisymm, cfg.icor = 0, 3, 0, 0, 0
    for q in range(CM1G_MAXQ):
        cfg.qmag[q] = 1.0e-2
    # 6th-order horizontal diffusion inside advection (idiff=1, difforder=6):
    # off unless `diff6` gives kdiff6 (the mdiff limiter with `mdiff`)
    kd = w.get("diff6")
    cfg.idiff, cfg.difforder = (1, 6) if kd is not None else (0, 6)
    cfg.kdiff6 = float(kd) if kd is not None else 0.0
    cfg.mdiff = int(w.get("mdiff", 0))

    # ---- grid metrics (uniform grid: param.F:7077-7081, 7459-7463, 7793-7802)
    f32 = np.float32
    gr = {}
    for n in ("uh", "ruh"):
        gr[n] = np.ones(lay.NI, f32)
    for n in ("uf", "ruf"):
        gr[n] = np.ones(lay.NI + 1, f32)
    for n in ("vh", "rvh"):
        gr[n] = np.ones(lay.NJ, f32)
    for n in ("vf", "rvf"):
        gr[n] = np.ones(lay.NJ + 1, f32)
    for n in ("mh", "rmh"):
        gr[n] = np.ones(lay.shape(1), f32)
    for n in ("mf", "rmf"):
        gr[n] = np.ones(lay.shape(4), f32)
    gr["c1"] = np.full(lay.shape(1), 0.5, f32)   # param.F:8603-8624, uniform dz
    gr["c2"] = np.full(lay.shape(1), 0.5, f32)

    # ---- base state on half levels k=0..nk+1 (zh(0) = -dz/2)
    kk = np.arange(lay.kb, lay.ke + 1)
    zh = (kk - 0.5) * dz
    snd_kind = w["sounding"]
    th, qv = _sounding(snd_kind, np.clip(zh, 0.0, None))
    thv_fn = lambda zz: np.interp(zz, np.clip(zh, 0, None), th * (1.0 + qv * RV / RD) / (1.0 + qv))
    pi = _hydrostatic_pi(zh, thv_fn)
    # extrapbcs (bc.F:1185-1203): 2nd-order extrapolation to zh(0), zh(nk+1)
    cgs = np.array([1.875, -1.25, 0.375])
    for arr in (th, qv, pi):
        arr[0] = cgs @ arr[1:4]
        arr[-1] = cgs @ arr[-2:-5:-1]
    prs = P00 * pi ** (CP / RD)
    rho = prs / (RD * th * pi * (1.0 + np.maximum(qv, 0.0) * RV / RD))
    rf = np.empty_like(rho)
    rf[2:nk + 1] = 0.5 * rho[1:nk] + 0.5 * rho[2:nk + 1]          # base.F:2168-2174
    rf[1] = cgs @ rho[1:4]
    rf[0] = rf[1]
    rf[nk + 1] = cgs @ rho[nk:nk - 3:-1]

    def col(prof, stag=1):
        a = np.empty(lay.shape(stag), f32)
        p = np.asarray(prof, np.float64)
        nkk = a.shape[0]
        pp = np.concatenate([p, p[-1:]])[:nkk] if nkk > len(p) else p[:nkk]
        a[...] = pp.astype(f32)[:, None, None]
        return a

    gr["th0"] = col(th)
    gr["pi0"] = col(pi)
    gr["prs0"] = col(prs)
    gr["rho0"] = col(rho)
    gr["qv0"] = col(qv)
    gr["qc0"] = col(np.zeros_like(th))
    gr["qi0"] = col(np.zeros_like(th))
    gr["rr0"] = (np.float32(1.0) / gr["rho0"]).astype(f32)
    gr["rf0"] = col(rf)
    gr["rrf0"] = (np.float32(1.0) / gr["rf0"]).astype(f32)
    gr["rth0"] = (np.float32(1.0) / gr["th0"]).astype(f32)

    wind = w["wind"]
    wkind, wkw = (wind, {}) if isinstance(wind, str) else wind
    if wkind == "curved":
        wkw = dict(U=20.0)
    u_prof, v_prof = _hodograph(wkind, np.clip(zh, 0, None), **wkw)
    gr["u0"] = col(u_prof, 2)
    gr["v0"] = col(v_prof, 3)

    # dtu0/dtv0 (param.F:9182-9218)
    ibw = ibe = ibs = ibn = (bc != 1)
    dtu0 = np.zeros((lay.NJ, lay.NI), f32)
    dtv0 = np.zeros((lay.NJ, lay.NI), f32)
    dtu0[lay.jx(1):lay.jx(nj) + 1, lay.ix(1):lay.ix(ni + 1) + 1] = 1.0
    if ibw:
        dtu0[lay.jx(1):lay.jx(nj) + 1, lay.ix(1)] = 0.0
    if ibe:
        dtu0[lay.jx(1):lay.jx(nj) + 1, lay.ix(ni + 1)] = 0.0
    dtv0[lay.jx(1):lay.jx(nj + 1) + 1, lay.ix(1):lay.ix(ni) + 1] = 1.0
    if ibs:
        dtv0[lay.jx(1), lay.ix(1):lay.ix(ni) + 1] = 0.0
    if ibn:
        dtv0[lay.jx(nj + 1), lay.ix(1):lay.ix(ni) + 1] = 0.0
    gr["dtu0"], gr["dtv0"] = dtu0, dtv0
    for k in gr:
        gr[k] = np.ascontiguousarray(gr[k], dtype=f32)

    # ---- initial state
    st = {}
    xs = (np.arange(lay.ib, lay.ie + 1) - 0.5) * dx
    ys = (np.arange(lay.jb, lay.je + 1) - 0.5) * dx
    th_p = lay.zeros(1)
    kin = slice(lay.kx(1), lay.kx(nk) + 1)
    Z = zh[1:nk + 1][:, None, None]
    X = xs[None, None, :]
    Y = ys[None, :, None]
    b = w.get("bubble")
    if b:
        xc, yc = 0.5 * ni * dx, 0.5 * nj * dx
        beta = np.sqrt(((X - xc) / b["xr"]) ** 2 + ((Y - yc) / b["xr"]) ** 2 + ((Z - b["zc"]) / b["zr"]) ** 2)
        th_p[kin] += np.where(beta < 1.0, b["amp"] * np.cos(0.5 * np.pi * beta) ** 2, 0.0)
    nz = w.get("noise")
    if nz:
        noise = rng.uniform(-nz["amp"], nz["amp"], size=(nk, lay.NJ, lay.NI))
        if nz.get("zmax"):
            noise *= (Z < nz["zmax"])
        th_p[kin] += noise
    _fill_lateral(lay, th_p, bc)
    th_p[lay.kx(nk + 1)] = th_p[lay.kx(nk)]      # init3d.F:1847
    st["tha"], st["th3d"] = th_p.copy(), th_p.copy()

    u = gr["u0"].copy()
    v = gr["v0"].copy()
    st["ua"], st["u3d"] = u.copy(), u.copy()
    st["va"], st["v3d"] = v.copy(), v.copy()
    st["wa"], st["w3d"] = lay.zeros(4), lay.zeros(4)
    for n in ("ppi", "pp3d", "ppx", "ppten", "thten1"):
        st[n] = lay.zeros(1)
    st["uten1"], st["vten1"], st["wten1"] = lay.zeros(2), lay.zeros(3), lay.zeros(4)

    if moist:
        q = np.zeros((cfg.numq,) + lay.shape(1), f32)
        q[0] = gr["qv0"]
        if ptype == 1 and b:
            # seeded cloud in the bubble, rain in a wider shell around it, and
            # a 3 % supersaturation of the bubble's core
            qc = np.where(beta < 1.0, 1.5e-3 * np.cos(0.5 * np.pi * beta) ** 2, 0.0)
            qr = np.where(beta < 1.6, 2.0e-3 * np.cos(0.5 * np.pi * beta / 1.6) ** 2, 0.0)
            q[1][kin] = qc
            q[2][kin] = qr
            q[0][kin] *= np.where(beta < 0.5, 1.03, 1.0)
            for n in range(3):
                _fill_lateral(lay, q[n], bc)
        st["qa"], st["q3d"], st["qten"] = q.copy(), q.copy(), np.zeros_like(q)
    else:
        st["qa"] = st["q3d"] = st["qten"] = np.zeros((0,) + lay.shape(1), f32)
    if npt > 0:
        pt = np.zeros((npt,) + lay.shape(1), f32)
        for n in range(npt):
            fld = np.zeros((nk, lay.NJ, lay.NI))
            for _ in range(4):
                cx, cy = rng.uniform(0, ni * dx), rng.uniform(0, nj * dx)
                cz = rng.uniform(0.1, 0.5) * nk * dz
                rx, rz = rng.uniform(0.1, 0.25) * ni * dx, rng.uniform(0.1, 0.3) * nk * dz
                amp = np.exp(rng.normal(math.log(1e-3), 0.75))
                fld += amp * np.exp(-(((X - cx) / rx) ** 2 + ((Y - cy) / rx) ** 2 + ((Z - cz) / rz) ** 2))
            fld -= 0.05 * fld.max()           # leaves zero-valued regions
            pt[n][kin] = np.clip(fld, 0.0, None)
            _fill_lateral(lay, pt[n], bc)
        st["pta"], st["pt3d"], st["ptten"] = pt.copy(), pt.copy(), np.zeros_like(pt)
    else:
        st["pta"] = st["pt3d"] = st["ptten"] = np.zeros((0,) + lay.shape(1), f32)

    # rho/prs of the initial state, in the model's binary32 form
    c = cm1_constants()
    pi_t = gr["pi0"] + st["pp3d"]
    prs_t = (np.float32(P00) * np.power(pi_t, c["cpdrd"])).astype(f32)
    if moist:
        qvp = np.maximum(st["q3d"][0], 0.0)
        rho_t = prs_t / ((gr["th0"] + st["th3d"]) * pi_t * (c["rd"] + qvp * c["rv"]))
    else:
        rho_t = prs_t / (c["rd"] * (gr["th0"] + st["th3d"]) * pi_t)
    st["rho"], st["prs"] = rho_t.astype(f32), prs_t
    st["radbcw"] = np.zeros((lay.NK, lay.NJ), f32)
    st["radbce"] = np.zeros((lay.NK, lay.NJ), f32)
    st["radbcs"] = np.zeros((lay.NK, lay.NI), f32)
    st["radbcn"] = np.zeros((lay.NK, lay.NI), f32)
    if ptype == 1:
        st["rain"] = np.zeros((lay.NJ, lay.NI), f32)
        st["prate"] = np.zeros((lay.NJ, lay.NI), f32)
    for k in st:
        st[k] = np.ascontiguousarray(st[k], dtype=f32)

    # mass1: initial dry-air mass as calcmass sums it (misclibs.F:3134-3191)
    inner = lay.interior(1)
    rr = st["rho"][inner].astype(np.float64)
    mass1 = float(rr.sum(dtype=np.float64))
    return Case(name=name, lay=lay, cfg=cfg, grid=gr, state=st, dt=float(w["dt"]),
                mass1=mass1, nsteps=int(w["nsteps"]))


# statistics this library does not build (turbulence, ice, axisymmetric runs)
_STAT_OFF = ("stat_rmw", "stat_tke", "stat_km", "stat_kh", "stat_rhi")


def stat_opts(case, off=(), qnames=("qv",), nql=(0, 0), cloud=(), budnames=()):
    """cm1g_stat_opts_t for a case: every statistic this library builds is on
    except those in `off`; level heights of the uniform grid, the surface
    extrapolation weights from zh(1..3) to z = 0 (Lagrange, as param.F's
    delta gives them), model top nk*dz.  Returns (opts, arrays to keep alive)."""
    cfg = case.cfg
    nk, dz = cfg.nk, cfg.dz
    o = StatOpts()
    for n in STAT_SWITCHES:
        setattr(o, n, 0 if (n in _STAT_OFF or n in off) else 1)
    o.adapt_dt, o.bbc, o.ptype, o.iice = 0, 1, 0, 0
    o.nql1, o.nql2 = nql
    for q in cloud:
        o.cloudvar[q] = 1
    zh = ((np.arange(nk + 2) - 0.5) * dz).astype(np.float32)
    zf = ((np.arange(nk + 3) - 1.0) * dz).astype(np.float32)
    z = zh[1:4].astype(np.float64)
    w = [np.prod([(0.0 - z[m]) / (z[l] - z[m]) for m in range(3) if m != l]) for l in range(3)]
    o.cgs1, o.cgs2, o.cgs3 = (float(np.float32(x)) for x in w)
    o.maxz = float(np.float32(nk * dz))
    o.zh, o.zf = fptr(zh.ctypes.data), fptr(zf.ctypes.data)
    for q, nm in enumerate(qnames[:CM1G_MAXQ]):
        o.qname[q].value = nm.encode()
    bud = b"".join(b.encode().ljust(6)[:6] for b in budnames)
    o.nbudget = len(budnames)
    o.budname = bud if budnames else None
    return o, [zh, zf, bud]


ENSEMBLE_SIZES = tuple(range(48, 193, 16))   # nx, ny in {48 .. 192}


def make_ensemble(n=64, seed=2024, sizes=ENSEMBLE_SIZES, levels=(40, 60, 80)):
    """Uneven ensemble of warm-bubble members (dx = dy = 1 km, dz = 250 m, WENO5
    scalars, periodic, dt = 6 s, nsound = 6): per member nx, ny drawn from
    `sizes`, nz from `levels`, a bubble of 1-3 K and 3-6 km horizontal radius,
    and a uniform background wind in +-10 m/s, all from `seed`."""
    rng = np.random.default_rng(seed)
    members = []
    for m in range(n):
        ni, nj = int(rng.choice(sizes)), int(rng.choice(sizes))
        nk = int(rng.choice(levels))
        amp, xr = float(rng.uniform(1.0, 3.0)), float(rng.uniform(3000.0, 6000.0))
        u, v = (float(x) for x in rng.uniform(-10.0, 10.0, 2))
        members.append(make_case("dry_bubble", seed=seed + 1 + m, ni=ni, nj=nj, nk=nk, advwenos=1,
                                 bubble=dict(amp=amp, xr=xr, zr=1400.0, zc=1400.0),
                                 wind=("uniform", dict(u=u, v=v))))
    return members
