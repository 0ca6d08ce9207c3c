"""ctypes loader of the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arms may
import this module, as the checker or as the timed CPU restatement; the
product (libcm1g.so, cm1_b200) never does.  Parity unpinned: see the header
of cm1_oracle.c.
"""
import ctypes as C
import os
import subprocess

from cm1_b200.abi import Config, Grid, State, StatOpts

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-C", _HERE, "-s"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        P = C.POINTER(C.c_float)
        cfgp, grp, stp = C.POINTER(Config), C.POINTER(Grid), C.POINTER(State)
        L.oracle_solve2.argtypes = [cfgp, grp, stp, C.c_int, C.c_float, C.c_double, C.c_double,
                                    C.POINTER(C.c_double), C.POINTER(C.c_float)]
        L.oracle_step.argtypes = L.oracle_solve2.argtypes
        L.oracle_solve3.argtypes = [cfgp, grp, stp]
        L.oracle_pdefq.argtypes = [cfgp, grp, C.c_float, C.POINTER(C.c_double), P, P]
        L.oracle_bc.argtypes = [cfgp, C.c_int, P, C.c_int]
        L.oracle_advs.argtypes = [cfgp, grp, C.c_int, C.c_int, P, P, P, P, P, P, P, C.c_int, C.c_int,
                                  C.c_float, C.c_double]
        L.oracle_advuvw.argtypes = [cfgp, grp, P, P, P, P, P, P]
        L.oracle_sound.argtypes = [cfgp, grp, C.c_int, C.c_float, C.c_float] + [P] * 23
        L.oracle_calcmass.argtypes = [cfgp, grp, P, C.POINTER(C.c_double)]
        L.oracle_maxmin.argtypes = [cfgp, P, C.c_int, P, P, C.POINTER(C.c_int)]
        for n in ("oracle_flx5",):
            getattr(L, n).argtypes = [C.c_float] * 5
            getattr(L, n).restype = C.c_float
        L.oracle_flx3.argtypes = [C.c_float] * 3
        L.oracle_flx3.restype = C.c_float
        L.oracle_weno5.argtypes = [C.c_float] * 5 + [C.c_double]
        L.oracle_weno5.restype = C.c_float
        L.oracle_upstrpd.argtypes = [C.c_float] * 3 + [C.c_double]
        L.oracle_upstrpd.restype = C.c_float
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_dtsmall.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_int,
                                     C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.oracle_tendency_init.argtypes = [cfgp, grp, C.c_int, C.c_float] + [P] * 16
        L.oracle_calcener.argtypes = [cfgp, grp] + [P] * 11 + [C.POINTER(C.c_double)]
        L.oracle_threads.restype = C.c_int
        L.oracle_diff2.argtypes = [cfgp, grp, C.c_float, C.c_int, C.c_int, C.c_int, P, P] + [P] * 13
        L.oracle_turbsmag.argtypes = [cfgp, grp, C.c_float] + [C.c_int] * 4 + [P, P] + [P] * 13
        L.oracle_mp_driver.argtypes = [cfgp, grp, stp, C.c_float, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.oracle_statpack.argtypes = ([cfgp, grp, C.POINTER(StatOpts), C.c_double, C.c_float] + [P] * 10 +
                                      [C.POINTER(C.c_double)] * 3 + [P, C.POINTER(C.c_int)])
        _lib = L
    return _lib


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def step(case, state=None, solve2_only=False, mtime=0.0):
    """Advance `state` (dict of numpy arrays, default: a copy of the case's)
    by one large step in place; returns (state, mass2, cflmax)."""
    L = lib()
    st = case.copy_state() if state is None else state
    s = case.state_struct(st)
    g = case.grid_struct()
    m2, cfl = C.c_double(0.0), C.c_float(0.0)
    f = L.oracle_solve2 if solve2_only else L.oracle_step
    rc = f(C.byref(case.cfg), C.byref(g), C.byref(s), 1, case.dt, mtime, case.mass1, C.byref(m2), C.byref(cfl))
    if rc != 0:
        raise RuntimeError("oracle failed: %s" % L.oracle_last_error().decode())
    return st, m2.value, cfl.value


class pow_mode:
    """Context manager selecting how the oracle evaluates the binary32
    powers of the pressure/density relations and the Kessler scheme:
    "libm" (the C library's powf, as the reference build does; the default)
    or "binary64" (the power in binary64 rounded once, the CUDA path's
    choice)."""

    def __init__(self, mode):
        self.mode = {"libm": 0, "binary64": 1}[mode]

    def __enter__(self):
        L = lib()
        self.saved = L.oracle_get_pow_mode()
        L.oracle_set_pow_mode(self.mode)
        return self

    def __exit__(self, *a):
        lib().oracle_set_pow_mode(self.saved)


_LIB_R8 = os.path.join(_HERE, "_r8", "liboracle_r8.so")
_lib_r8 = None


def lib_r8():
    """The FP64 (-r8) build of the oracle (oracle/make_r8.py)."""
    global _lib_r8
    if _lib_r8 is None:
        if not os.path.exists(_LIB_R8):
            build()
        L = C.CDLL(_LIB_R8)
        cfgp, grp, stp = C.POINTER(Config), C.POINTER(Grid), C.POINTER(State)
        # every binary32 argument of the FP32 build is binary64 here
        L.oracle_step.argtypes = [cfgp, grp, stp, C.c_int, C.c_double, C.c_double, C.c_double,
                                  C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.oracle_last_error.restype = C.c_char_p
        _lib_r8 = L
    return _lib_r8


def step_r8(case, state=None, nsteps=1):
    """`nsteps` large steps of the FP64 build from the same (binary32) inputs
    promoted to float64; returns the float64 state dict."""
    import numpy as np
    from cm1_b200.abi import GRID_FIELDS, STATE_FIELDS
    L = lib_r8()
    src = case.state if state is None else state
    st = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in src.items()}
    grid = {k: np.ascontiguousarray(case.grid[k], dtype=np.float64) for k in GRID_FIELDS}
    P = C.POINTER(C.c_float)
    g = Grid()
    for n in GRID_FIELDS:
        setattr(g, n, C.cast(C.c_void_p(grid[n].ctypes.data), P))
    s = State()
    for n in STATE_FIELDS:
        a = st.get(n)
        setattr(s, n, C.cast(C.c_void_p(a.ctypes.data), P) if a is not None and a.size else C.cast(None, P))
    m2, cfl = C.c_double(0.0), C.c_double(0.0)
    for _ in range(nsteps):
        rc = L.oracle_step(C.byref(case.cfg), C.byref(g), C.byref(s), 1, case.dt, 0.0, case.mass1, C.byref(m2),
                           C.byref(cfl))
        if rc != 0:
            raise RuntimeError("FP64 oracle failed: %s" % L.oracle_last_error().decode())
    return st


def threads():
    return lib().oracle_threads()


def statpack(case, opts, st, mtime=0.0, prate=None, qbudget=None, asq=None, bsq=None, nmax=512):
    """The statistics of state dict `st` (numpy arrays) as the statpack
    restatement computes them; returns a float32 array."""
    import numpy as np
    L = lib()
    out = np.zeros(nmax, np.float32)
    n = C.c_int(0)

    def f(name):
        a = st.get(name)
        return _fp(a) if a is not None and a.size else None

    def d(a):
        if a is None:
            return None, None
        a = np.ascontiguousarray(a, np.float64)
        return a.ctypes.data_as(C.POINTER(C.c_double)), a
    qb, ab, bb = d(qbudget), d(asq), d(bsq)
    g = case.grid_struct()
    rc = L.oracle_statpack(C.byref(case.cfg), C.byref(g), C.byref(opts), mtime, case.dt, f("ua"), f("va"), f("wa"),
                           f("ppi"), f("tha"), f("prs"), f("rho"), f("qa"), f("pta"),
                           _fp(prate) if prate is not None else None, qb[0], ab[0], bb[0], _fp(out), C.byref(n))
    if rc != 0:
        raise RuntimeError("oracle statpack failed")
    return out[:n.value].copy()


def mp_driver(case, st, dt=None):
    """The Kessler branch of mp_driver on state dict `st` in place; returns
    (qbudget(1..7), asq(1..3)) of this call."""
    L = lib()
    s = case.state_struct(st)
    g = case.grid_struct()
    qb, asq = (C.c_double * 7)(), (C.c_double * 3)()
    rc = L.oracle_mp_driver(C.byref(case.cfg), C.byref(g), C.byref(s), case.dt if dt is None else dt, qb, asq)
    if rc != 0:
        raise RuntimeError("oracle mp_driver failed: %s" % L.oracle_last_error().decode())
    return list(qb), list(asq)
