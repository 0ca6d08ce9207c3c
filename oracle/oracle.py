"""ctypes loader of the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arms may
import this module, as the checker or as the timed CPU restatement; the
product (libcm1g.so, cm1_b200) never does.  Parity unpinned: see the header
of cm1_oracle.c.
"""
import ctypes as C
import os
import subprocess

from cm1_b200.abi import Config, Grid, State

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


def threads():
    return lib().oracle_threads()
