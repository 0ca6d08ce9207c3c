"""ctypes/PyTorch binding of libcm1g.so.

Python drivers (the role cm1/run.py plays for the reference) and training
code use this module; it calls the C-ABI declared in include/cm1g.h.  There
is no CPU fallback: if the library or a CUDA device is missing the calls
raise.
"""
import ctypes as C
import os

import numpy as np

from .abi import Config, Grid, Restart, State, StatOpts, Tune, WriteoutOpts, WRITEOUT_SWITCHES, STATE_FIELDS, fptr, CM1G_OK

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcm1g.so")
_lib = None

_P = C.POINTER(C.c_float)


class CM1GError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("cm1g error %d: %s" % (code, msg))
        self.code = code


def lib():
    """Load libcm1g.so (raises if it has not been built).  CM1G_LIB names
    another build of the same library (e.g. one compiled with different
    tile parameters) to load instead."""
    global _lib
    if _lib is not None:
        return _lib
    path = os.environ.get("CM1G_LIB", LIB_PATH)
    if not os.path.exists(path):
        raise RuntimeError("%s not built: run `python -m cm1_b200.build` (no CPU fallback exists)" % path)
    L = C.CDLL(path)
    ctxp = C.c_void_p
    cfgp, grp, stp = C.POINTER(Config), C.POINTER(Grid), C.POINTER(State)
    L.cm1g_last_error.restype = C.c_char_p
    L.cm1g_version.argtypes = [C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    L.cm1g_init.argtypes = [cfgp, grp, C.POINTER(ctxp)]
    L.cm1g_finalize.argtypes = [ctxp]
    L.cm1g_set_stream.argtypes = [ctxp, C.c_void_p]
    L.cm1g_launch_count.argtypes = [ctxp, C.POINTER(C.c_int64)]
    L.cm1g_solve2.argtypes = [ctxp, C.c_int32, C.c_float, C.c_double, C.c_double, C.POINTER(C.c_double),
                              C.POINTER(C.c_float), stp]
    L.cm1g_step.argtypes = L.cm1g_solve2.argtypes + [C.c_int32]
    L.cm1g_solve3.argtypes = [ctxp, stp]
    L.cm1g_mp_driver.argtypes = [ctxp, C.c_float, stp]
    L.cm1g_diff2.argtypes = [ctxp, C.c_float, C.c_int32, C.c_int32, C.c_int32, _P, _P] + [_P] * 13
    L.cm1g_turbsmag.argtypes = [ctxp, C.c_float] + [C.c_int32] * 4 + [_P, _P] + [_P] * 15
    i32p = C.POINTER(C.c_int32)
    L.cm1g_records_size.argtypes = [ctxp, C.c_int32, i32p, i32p, i32p, C.POINTER(C.c_int64)]
    L.cm1g_pack_records.argtypes = [ctxp, C.c_int32, C.POINTER(_P), i32p, i32p, i32p, _P]
    L.cm1g_unpack_records.argtypes = [ctxp, C.c_int32, C.POINTER(_P), i32p, i32p, i32p, _P]
    L.cm1g_restart_write.argtypes = [ctxp, C.c_char_p, C.POINTER(Restart), stp]
    L.cm1g_writeout.argtypes = [ctxp, C.c_char_p, C.c_int32, C.c_double, C.POINTER(WriteoutOpts), stp]
    L.cm1g_restart_read.argtypes = [ctxp, C.c_char_p, C.POINTER(Restart), stp]
    L.cm1g_mp_budget.argtypes = [ctxp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32]
    L.cm1g_pdefq.argtypes = [ctxp, C.c_float, C.POINTER(C.c_double), _P, _P]
    for n in ("cm1g_bcs", "cm1g_bcp", "cm1g_bcu", "cm1g_bcv"):
        getattr(L, n).argtypes = [ctxp, _P]
    L.cm1g_bcw.argtypes = [ctxp, _P, C.c_int32]
    L.cm1g_advs.argtypes = [ctxp, C.c_int32, C.c_int32, _P, _P, _P, _P, _P, _P, _P, C.c_int32, C.c_int32,
                            C.c_float, C.c_double]
    L.cm1g_advuvw.argtypes = [ctxp, C.c_int32, _P, _P, _P, _P, _P, _P]
    for n in ("cm1g_advu", "cm1g_advv", "cm1g_advw"):
        getattr(L, n).argtypes = [ctxp, C.c_int32, _P, _P, _P, _P]
    L.cm1g_sound.argtypes = [ctxp, C.c_float] + [_P] * 23 + [C.c_int32, C.c_float]
    L.cm1g_calcmass.argtypes = [ctxp, _P, C.POINTER(C.c_double)]
    L.cm1g_maxmin.argtypes = [ctxp, _P, C.c_int32, _P, _P, C.POINTER(C.c_int32)]
    L.cm1g_profile.argtypes = [ctxp, C.c_int32]
    L.cm1g_profile_read.argtypes = [ctxp, C.c_int32, C.c_char_p, C.c_int32, C.POINTER(C.c_int64),
                                    C.POINTER(C.c_double)]
    L.cm1g_calcener.argtypes = [ctxp] + [_P] * 11 + [C.POINTER(C.c_double)]
    L.cm1g_stat_setup.argtypes = [ctxp, C.POINTER(StatOpts), C.POINTER(C.c_int32)]
    L.cm1g_stat_name.argtypes = [ctxp, C.c_int32, C.c_char_p, C.c_int32]
    L.cm1g_statpack.argtypes = ([ctxp, C.c_double, C.c_float] + [_P] * 10 +
                                [C.POINTER(C.c_double)] * 3 + [_P])
    L.cm1g_stat_write.argtypes = [C.c_char_p, C.c_int32, _P, C.c_int32]
    L.cm1g_dtsmall.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_float, C.c_int32,
                               C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int32)]
    L.cm1g_tendency_init.argtypes = [ctxp, C.c_int32, C.c_float] + [_P] * 16
    L.cm1g_ensemble_create.argtypes = [C.POINTER(ctxp), C.c_int32, C.POINTER(ctxp)]
    L.cm1g_ensemble_step.argtypes = [ctxp, stp, C.POINTER(C.c_float), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_float), C.c_int32]
    L.cm1g_ensemble_launch_count.argtypes = [ctxp, C.POINTER(C.c_int64)]
    L.cm1g_ensemble_destroy.argtypes = [ctxp]
    L.cm1g_mlp_param_count.restype = C.c_int32
    L.cm1g_mlp_param_count.argtypes = []
    L.cm1g_mlp_set_activation.argtypes = [C.c_int32]
    L.cm1g_mlp_get_activation.restype = C.c_int32
    L.cm1g_mlp_get_activation.argtypes = []
    L.cm1g_mlp_forward.argtypes = [_P, C.c_int32, _P, _P, _P, _P, _P, C.c_void_p]
    L.cm1g_mlp_backward.argtypes = [_P, C.c_int32, _P, _P, _P, _P, _P, C.c_void_p]
    L.cm1g_closure_loss.argtypes = [C.c_int32, _P, _P, _P, _P, _P, _P, _P, C.c_void_p, C.c_void_p]
    L.cm1g_adam.argtypes = [C.c_int32, _P, _P, _P, _P, C.c_int32, C.c_float, C.c_float, C.c_void_p]
    L.cm1g_face_features.argtypes = [C.c_int32] * 5 + [_P, _P, C.c_int32, _P, C.c_float, _P, _P, _P, _P,
                                                         C.c_void_p]
    L.cm1g_face_phi.argtypes = [C.c_int64, _P, _P, _P, _P, C.c_float, _P, C.c_void_p]
    L.cm1g_closure_faces.argtypes = [C.c_int32] * 5 + [_P, _P, C.c_int32, _P, C.c_float, _P, C.c_float, _P,
                                                       C.c_void_p]
    L.cm1g_closure_bounds.argtypes = [ctxp, C.c_float]
    L.cm1g_closure_set.argtypes = [ctxp, _P, C.c_int32]
    L.cm1g_capture_fluxes.argtypes = [ctxp, _P, _P, _P, _P]
    L.cm1g_pdefq_noalloc.argtypes = [cfgp, C.c_float, C.POINTER(C.c_double), _P, _P, _P, _P, _P, C.c_void_p]
    tunep = C.POINTER(Tune)
    L.cm1g_tile_shape.argtypes = [C.c_int32, C.POINTER(C.c_int32)]
    L.cm1g_scal_tile_shape.argtypes = [C.c_int32, C.POINTER(C.c_int32)]
    L.cm1g_set_tune.argtypes = [ctxp, tunep]
    L.cm1g_get_tune.argtypes = [ctxp, tunep]
    L.cm1g_autotune.argtypes = [ctxp, C.c_float, C.c_double, stp, C.c_int32, C.c_char_p, tunep]
    _lib = L
    return L


def check(rc):
    if rc != CM1G_OK:
        raise CM1GError(rc, lib().cm1g_last_error().decode())
    return rc


def ptr(a):
    """float* of a numpy array or a torch tensor (host or CUDA)."""
    if a is None:
        return C.cast(None, _P)
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(_P)
    return fptr(a.data_ptr())


def stat_write(path, nrec, rstat):
    """cm1g_stat_write: rstat as record nrec (1-based) of a GrADS stats file."""
    a = np.ascontiguousarray(rstat, np.float32)
    check(lib().cm1g_stat_write(str(path).encode(), int(nrec), a.ctypes.data_as(_P), a.size))


class Context:
    """A cm1g context for one grid (cm1g_init / cm1g_finalize)."""

    def __init__(self, cfg, grid_arrays):
        L = lib()
        self._grid_arrays = grid_arrays
        g = Grid()
        for n, a in grid_arrays.items():
            setattr(g, n, ptr(a))
        self.cfg = cfg
        h = C.c_void_p()
        check(L.cm1g_init(C.byref(cfg), C.byref(g), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().cm1g_finalize(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_handle):
        check(lib().cm1g_set_stream(self.h, C.c_void_p(int(stream_handle))))

    def launches(self):
        n = C.c_int64()
        check(lib().cm1g_launch_count(self.h, C.byref(n)))
        return n.value

    @staticmethod
    def state_struct(arrays):
        s = State()
        for n in STATE_FIELDS:
            a = arrays.get(n)
            empty = a is None or (a.numel() == 0 if hasattr(a, "numel") else a.size == 0)
            setattr(s, n, C.cast(None, _P) if empty else ptr(a))
        return s

    def step(self, state, dt, mass1, use_graph=False, solve2_only=False, nstep=0, mtime=0.0):
        """One large step on `state` (dict of torch CUDA tensors or numpy
        arrays).  Returns (mass2, cflmax)."""
        s = state if isinstance(state, State) else self.state_struct(state)
        m2, cfl = C.c_double(), C.c_float()
        L = lib()
        if solve2_only:
            check(L.cm1g_solve2(self.h, nstep, dt, mtime, mass1, C.byref(m2), C.byref(cfl), C.byref(s)))
        else:
            check(L.cm1g_step(self.h, nstep, dt, mtime, mass1, C.byref(m2), C.byref(cfl), C.byref(s),
                              1 if use_graph else 0))
        return m2.value, cfl.value

    @staticmethod
    def _rec_args(fields, stag, k1, k2):
        n = len(fields)
        a32 = lambda v: (C.c_int32 * n)(*v)
        return n, (_P * n)(*[ptr(f) for f in fields]), a32(stag), a32(k1), a32(k2)

    def records_size(self, stag, k1, k2):
        n = len(stag)
        out = C.c_int64()
        check(lib().cm1g_records_size(self.h, n, (C.c_int32 * n)(*stag), (C.c_int32 * n)(*k1), (C.c_int32 * n)(*k2),
                                      C.byref(out)))
        return out.value

    def pack_records(self, fields, stag, k1, k2, out=None):
        """cm1g_pack_records: the fields' records (level by level, i fastest) as
        one float32 array (numpy unless `out` is given)."""
        n, fp, s, a, b = self._rec_args(fields, stag, k1, k2)
        if out is None:
            out = np.zeros(self.records_size(stag, k1, k2), np.float32)
        check(lib().cm1g_pack_records(self.h, n, fp, s, a, b, ptr(out)))
        return out

    def unpack_records(self, fields, stag, k1, k2, buf):
        n, fp, s, a, b = self._rec_args(fields, stag, k1, k2)
        check(lib().cm1g_unpack_records(self.h, n, fp, s, a, b, ptr(buf)))

    def writeout(self, prefix, nwrite, state, mtime=0.0, switches=None, qnames=("qv", "qc", "qr")):
        """cm1g_writeout: GrADS files <prefix>_s/_u/_v/_w.dat (+ .ctl) at time
        nwrite; `switches` names the output_* switches that are on (all by default)."""
        o = WriteoutOpts()
        for n in WRITEOUT_SWITCHES:
            setattr(o, n, 1 if switches is None or n in switches else 0)
        for q, nm in enumerate(qnames[:8]):
            o.qname[q].value = nm.encode()
        s = state if isinstance(state, State) else self.state_struct(state)
        check(lib().cm1g_writeout(self.h, str(prefix).encode(), nwrite, mtime, C.byref(o), C.byref(s)))

    def restart_write(self, path, state, nstep=0, mtime=0.0, dt=0.0, dtlast=0.0, mass1=0.0):
        s = state if isinstance(state, State) else self.state_struct(state)
        h = Restart(nstep, mtime, dt, dtlast, mass1)
        check(lib().cm1g_restart_write(self.h, str(path).encode(), C.byref(h), C.byref(s)))

    def restart_read(self, path, state):
        """cm1g_restart_read into `state`; returns the header as a dict."""
        s = state if isinstance(state, State) else self.state_struct(state)
        h = Restart()
        check(lib().cm1g_restart_read(self.h, str(path).encode(), C.byref(h), C.byref(s)))
        return {n: getattr(h, n) for n, _ in Restart._fields_}

    def diff2(self, kdiff2, idiff, bbc, tbc, cgs, cgt, ua, va, wa, rho, tha=None, qa=None, pta=None,
              uten1=None, vten1=None, wten1=None, thten1=None, qten=None, ptten=None):
        """cm1g_diff2: 2nd-order diffusion tendencies added to uten1 ... ptten."""
        f3 = lambda v: (C.c_float * 3)(*[float(x) for x in v])
        check(lib().cm1g_diff2(self.h, kdiff2, idiff, bbc, tbc, f3(cgs), f3(cgt), ptr(ua), ptr(va), ptr(wa),
                               ptr(rho), ptr(tha), ptr(qa), ptr(pta), ptr(uten1), ptr(vten1), ptr(wten1),
                               ptr(thten1), ptr(qten), ptr(ptten)))

    def turbsmag(self, csm, tconfig, bcturbs, bbc, tbc, cgs, cgt, ua, va, wa, rho, tha, pta=None, uten1=None,
                 vten1=None, wten1=None, thten1=None, ptten=None, kmh=None, kmv=None):
        """cm1g_turbsmag: Smagorinsky LES tendencies added to uten1 ... ptten."""
        f3 = lambda v: (C.c_float * 3)(*[float(x) for x in v])
        check(lib().cm1g_turbsmag(self.h, csm, tconfig, bcturbs, bbc, tbc, f3(cgs), f3(cgt), ptr(ua), ptr(va),
                                  ptr(wa), ptr(rho), ptr(tha), None, ptr(pta), ptr(uten1), ptr(vten1), ptr(wten1),
                                  ptr(thten1), None, ptr(ptten), ptr(kmh), ptr(kmv)))

    def mp_driver(self, state, dt):
        """cm1g_mp_driver: the Kessler branch of mp_driver on `state` (ptype=1)."""
        s = state if isinstance(state, State) else self.state_struct(state)
        check(lib().cm1g_mp_driver(self.h, dt, C.byref(s)))

    def mp_budget(self, reset=False):
        """(qbudget(1..7), asq(1..3)) accumulated by the microphysics (FP64)."""
        qb, asq = (C.c_double * 7)(), (C.c_double * 3)()
        check(lib().cm1g_mp_budget(self.h, qb, asq, 1 if reset else 0))
        return list(qb), list(asq)

    def solve3(self, state):
        s = state if isinstance(state, State) else self.state_struct(state)
        check(lib().cm1g_solve3(self.h, C.byref(s)))

    def bc(self, which, a, flag=1):
        L = lib()
        f = {"s": L.cm1g_bcs, "p": L.cm1g_bcp, "u": L.cm1g_bcu, "v": L.cm1g_bcv}
        if which == "w":
            check(L.cm1g_bcw(self.h, ptr(a), flag))
        else:
            check(f[which](self.h, ptr(a)))

    def advs(self, nrk, wflag, divx, rru, rrv, rrw, s0, s, sten, pdef, pdefweno, dt, weps):
        """advs (adv.F:14-19): the kept arguments in the reference's order."""
        check(lib().cm1g_advs(self.h, nrk, wflag, ptr(divx), ptr(rru), ptr(rrv), ptr(rrw), ptr(s0), ptr(s),
                              ptr(sten), pdef, pdefweno, dt, weps))

    def advuvw(self, nrk, u, v, w, uten, vten, wten):
        check(lib().cm1g_advuvw(self.h, nrk, ptr(u), ptr(v), ptr(w), ptr(uten), ptr(vten), ptr(wten)))

    def advu(self, nrk, u3d, uten, v3d, w3d):
        check(lib().cm1g_advu(self.h, nrk, ptr(u3d), ptr(uten), ptr(v3d), ptr(w3d)))

    def advv(self, nrk, v3d, vten, u3d, w3d):
        check(lib().cm1g_advv(self.h, nrk, ptr(v3d), ptr(vten), ptr(u3d), ptr(w3d)))

    def advw(self, nrk, w3d, wten, u3d, v3d):
        check(lib().cm1g_advw(self.h, nrk, ptr(w3d), ptr(wten), ptr(u3d), ptr(v3d)))

    SOUND_ARRAYS = ["radbcw", "radbce", "radbcs", "radbcn", "rru", "ua", "u3d", "uten", "rrv", "va", "v3d", "vten",
                    "rrw", "wa", "w3d", "wten", "ppi", "pp3d", "piadv", "ppten", "ppx", "thv", "ppterm"]

    def sound(self, nrk, dt, dttmp, **a):
        """sound (sound.F:10-24): arrays by name, passed in the reference's order."""
        check(lib().cm1g_sound(self.h, dt, *[ptr(a[n]) for n in self.SOUND_ARRAYS], nrk, dttmp))

    def pdefq(self, rmax, rho, q):
        asq = C.c_double(0.0)
        check(lib().cm1g_pdefq(self.h, rmax, C.byref(asq), ptr(rho), ptr(q)))
        return asq.value

    def calcmass(self, rho):
        t = C.c_double()
        check(lib().cm1g_calcmass(self.h, ptr(rho), C.byref(t)))
        return t.value

    def maxmin(self, a, stag):
        mx, mn = C.c_float(), C.c_float()
        loc = (C.c_int32 * 6)()
        check(lib().cm1g_maxmin(self.h, ptr(a), stag, C.byref(mx), C.byref(mn), loc))
        return mx.value, mn.value, tuple(loc)

    def calcener(self, zh, rho, ua, va, wa, ppi, tha, qv=None, ql=None, qi=None, vr=None):
        """(ek, ei, ep, le, et) of calcener, FP64."""
        out = (C.c_double * 5)()
        check(lib().cm1g_calcener(self.h, ptr(zh), ptr(rho), ptr(ua), ptr(va), ptr(wa), ptr(ppi), ptr(tha),
                                  ptr(qv), ptr(ql), ptr(qi), ptr(vr), out))
        return tuple(out)

    def stat_setup(self, opts):
        """cm1g_stat_setup: builds the statistics list; returns the statistic names."""
        n = C.c_int32()
        check(lib().cm1g_stat_setup(self.h, C.byref(opts), C.byref(n)))
        buf = C.create_string_buffer(64)
        names = []
        for i in range(1, n.value + 1):
            check(lib().cm1g_stat_name(self.h, i, buf, 64))
            names.append(buf.value.decode())
        self._nstat = n.value
        return names

    def statpack(self, mtime, dt, ua, va, wa, ppi, tha, prs, rho, qa=None, pta=None, prate=None,
                 qbudget=None, asq=None, bsq=None):
        """cm1g_statpack: the statistics of the fields (host or device arrays) as a float32 array."""
        out = np.zeros(self._nstat, np.float32)

        def dp(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, np.float64)
            return a.ctypes.data_as(C.POINTER(C.c_double)), a
        qb, ab, bb = dp(qbudget), dp(asq), dp(bsq)
        check(lib().cm1g_statpack(self.h, float(mtime), float(dt), ptr(ua), ptr(va), ptr(wa), ptr(ppi), ptr(tha),
                                  ptr(prs), ptr(rho), ptr(qa), ptr(pta), ptr(prate),
                                  qb[0] if qb else None, ab[0] if ab else None, bb[0] if bb else None,
                                  out.ctypes.data_as(_P)))
        return out

    def tendency_init(self, irdamp, rdalpha, uten1, vten1, wten1, thten1, qten=None, ptten=None, tauh=None,
                      taus=None, tauf=None, uavg=None, vavg=None, thavg=None, ua=None, va=None, wa=None, tha=None):
        check(lib().cm1g_tendency_init(self.h, irdamp, rdalpha, ptr(tauh), ptr(taus), ptr(tauf), ptr(uavg), ptr(vavg),
                                       ptr(thavg), ptr(ua), ptr(va), ptr(wa), ptr(tha), ptr(uten1), ptr(vten1),
                                       ptr(wten1), ptr(thten1), ptr(qten), ptr(ptten)))

    def closure(self, params, enable=True, widen=None):
        """Learned closure of theta's horizontal faces on/off (params: FP32
        array); widen sets the bounds of the face values (cm1g_closure_bounds)."""
        check(lib().cm1g_closure_set(self.h, ptr(params), 1 if enable else 0))
        if widen is not None:
            check(lib().cm1g_closure_bounds(self.h, widen))

    def capture_fluxes(self, fx=None, fy=None, rx=None, ry=None):
        check(lib().cm1g_capture_fluxes(self.h, ptr(fx), ptr(fy), ptr(rx), ptr(ry)))

    def get_tune(self):
        """The context's launch shapes: dict of adv_shape, mom_shape, sound_form, step_ms."""
        t = Tune()
        check(lib().cm1g_get_tune(self.h, C.byref(t)))
        return {n: getattr(t, n) for n, _ in Tune._fields_}

    def set_tune(self, adv_shape=0, mom_shape=0, sound_form=-1, step_ms=0.0):
        t = Tune(adv_shape, mom_shape, sound_form, step_ms)
        check(lib().cm1g_set_tune(self.h, C.byref(t)))

    def autotune(self, state, dt, mass1, reps=3, cache=None):
        """Times the candidate launch shapes on a copy of `state` and keeps
        the fastest (cm1g_autotune); `cache` names a text file of results
        per grid shape.  Returns get_tune()."""
        s = state if isinstance(state, State) else self.state_struct(state)
        t = Tune()
        check(lib().cm1g_autotune(self.h, dt, mass1, C.byref(s), reps,
                                  None if cache is None else os.fsencode(cache), C.byref(t)))
        return {n: getattr(t, n) for n, _ in Tune._fields_}

    def profile(self, enable):
        check(lib().cm1g_profile(self.h, 1 if enable else 0))

    def profile_read(self):
        """{kernel: (launches, total_ms)} collected since profiling was enabled."""
        L = lib()
        out = {}
        buf = C.create_string_buffer(64)
        n, ms = C.c_int64(), C.c_double()
        i = 0
        while L.cm1g_profile_read(self.h, i, buf, 64, C.byref(n), C.byref(ms)) == CM1G_OK:
            out[buf.value.decode()] = (n.value, ms.value)
            i += 1
        return out


class Ensemble:
    """cm1g_ensemble_*: members advanced side by side, one graph per step.

    contexts: list of Context (one per member); states: list of dicts of
    CUDA tensors in the members' layouts."""

    def __init__(self, contexts):
        self.contexts = list(contexts)
        arr = (C.c_void_p * len(self.contexts))(*[c.h for c in self.contexts])
        h = C.c_void_p()
        check(lib().cm1g_ensemble_create(arr, len(self.contexts), C.byref(h)))
        self.h = h

    def step(self, states, dt, mass1, use_graph=True):
        n = len(self.contexts)
        self._structs = (State * n)(*[Context.state_struct(s) for s in states])
        dts = (C.c_float * n)(*dt)
        m1 = (C.c_double * n)(*mass1)
        m2, cfl = (C.c_double * n)(), (C.c_float * n)()
        check(lib().cm1g_ensemble_step(self.h, self._structs, dts, m1, m2, cfl, 1 if use_graph else 0))
        return list(m2), list(cfl)

    def kernels_per_step(self):
        n = C.c_int64()
        check(lib().cm1g_ensemble_launch_count(self.h, C.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "h", None):
            lib().cm1g_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def tile_shapes(scalar=False):
    """The tile-shape table of the momentum pass (x and y threads, levels),
    or with scalar=True that of the scalar passes (x and y cells, levels):
    list of (x, y, levels)."""
    f = lib().cm1g_scal_tile_shape if scalar else lib().cm1g_tile_shape
    out, i = [], 0
    a = (C.c_int32 * 3)()
    while f(i, a) == CM1G_OK:
        out.append(tuple(a))
        i += 1
    return out


def dtsmall(psolver, nx, ny, min_dx, min_dy, min_dz, dt, adapt_dt=0):
    """nsound (and dt, dbldt, changed only by adapt_dt) as dtsmall computes them."""
    fdt, ddt, ns = C.c_float(dt), C.c_double(dt), C.c_int32()
    check(lib().cm1g_dtsmall(psolver, nx, ny, min_dx, min_dy, min_dz, adapt_dt, C.byref(fdt), C.byref(ddt),
                             C.byref(ns)))
    return ns.value, fdt.value, ddt.value


def to_device(arrays, device="cuda"):
    import torch
    return {k: torch.from_numpy(np.ascontiguousarray(v)).to(device) for k, v in arrays.items()}


def to_host(arrays):
    return {k: v.detach().cpu().numpy() for k, v in arrays.items()}
