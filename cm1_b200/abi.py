"""ctypes mirror of include/cm1g.h (the library's C-ABI).

The structures below are byte-for-byte the C structs of cm1g.h, so the same
objects can be handed to libcm1g.so (the CUDA library) and, in the tests, to
the CPU oracle, which shares the struct definitions.
"""
import ctypes as C

CM1G_MAXQ = 8

CM1G_OK = 0
CM1G_ERR_ARG = -1
CM1G_ERR_CUDA = -2
CM1G_ERR_NOMEM = -3
CM1G_ERR_NONFINITE = -4
CM1G_ERR_UNSUPPORTED = -5
CM1G_ERR_STATE = -6

_P = C.POINTER(C.c_float)


class Config(C.Structure):
    """cm1g_config_t: globals of module `input` read by the large step."""
    _fields_ = [
        ("ni", C.c_int32), ("nj", C.c_int32), ("nk", C.c_int32), ("ngxy", C.c_int32),
        ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
        ("wbc", C.c_int32), ("ebc", C.c_int32), ("sbc", C.c_int32), ("nbc", C.c_int32),
        ("hadvordrs", C.c_int32), ("vadvordrs", C.c_int32),
        ("hadvordrv", C.c_int32), ("vadvordrv", C.c_int32),
        ("advwenos", C.c_int32), ("advwenov", C.c_int32), ("weno_order", C.c_int32),
        ("nsound", C.c_int32), ("alph", C.c_float), ("kdiv", C.c_float),
        ("imoist", C.c_int32), ("eqtset", C.c_int32), ("numq", C.c_int32), ("nqv", C.c_int32),
        ("iptra", C.c_int32), ("npt", C.c_int32), ("pdtra", C.c_int32),
        ("apmasscon", C.c_int32),
        ("irbc", C.c_int32), ("cstar", C.c_float), ("roflux", C.c_int32),
        ("smeps", C.c_float),
        ("testcase", C.c_int32), ("psolver", C.c_int32), ("terrain_flag", C.c_int32),
        ("axisymm", C.c_int32), ("icor", C.c_int32),
        ("qmag", C.c_float * CM1G_MAXQ),
        ("idiff", C.c_int32), ("difforder", C.c_int32), ("mdiff", C.c_int32), ("kdiff6", C.c_float),
        ("ptype", C.c_int32), ("nql1", C.c_int32), ("nql2", C.c_int32), ("efall", C.c_int32),
        ("tsmall", C.c_float), ("qsmall", C.c_float),
    ]


GRID_FIELDS = ["uh", "ruh", "uf", "ruf", "vh", "rvh", "vf", "rvf",
               "mh", "rmh", "c1", "c2", "mf", "rmf",
               "pi0", "rho0", "rr0", "rf0", "rrf0", "th0", "rth0",
               "qv0", "qc0", "qi0", "prs0", "u0", "v0", "dtu0", "dtv0"]


class Grid(C.Structure):
    """cm1g_grid_t: grid metrics and base state (host pointers)."""
    _fields_ = [(n, _P) for n in GRID_FIELDS]


STATE_FIELDS = ["ua", "u3d", "uten1", "va", "v3d", "vten1", "wa", "w3d", "wten1",
                "ppi", "pp3d", "ppx", "ppten", "tha", "th3d", "thten1", "rho", "prs",
                "qa", "q3d", "qten", "pta", "pt3d", "ptten",
                "radbcw", "radbce", "radbcs", "radbcn", "rain", "prate"]


class Tune(C.Structure):
    """cm1g_tune_t: launch shapes of the large step."""
    _fields_ = [("adv_shape", C.c_int32), ("mom_shape", C.c_int32), ("sound_form", C.c_int32),
                ("step_ms", C.c_float)]


STAT_SWITCHES = ["stat_w", "stat_wlevs", "stat_u", "stat_v", "stat_rmw", "stat_pipert", "stat_prspert",
                 "stat_thpert", "stat_q", "stat_tke", "stat_km", "stat_kh", "stat_div", "stat_rh", "stat_rhi",
                 "stat_the", "stat_cloud", "stat_sfcprs", "stat_wsp", "stat_cfl", "stat_vort", "stat_tmass",
                 "stat_tmois", "stat_qmass", "stat_tenerg", "stat_mo", "stat_tmf", "stat_pcn", "stat_qsrc"]


class StatOpts(C.Structure):
    """cm1g_stat_opts_t: switches and host values of the statistics package."""
    _fields_ = ([(n, C.c_int32) for n in STAT_SWITCHES] +
                [("adapt_dt", C.c_int32), ("bbc", C.c_int32), ("ptype", C.c_int32), ("iice", C.c_int32),
                 ("nql1", C.c_int32), ("nql2", C.c_int32), ("cloudvar", C.c_int32 * CM1G_MAXQ),
                 ("nbudget", C.c_int32), ("maxz", C.c_float), ("cgs1", C.c_float), ("cgs2", C.c_float),
                 ("cgs3", C.c_float), ("zh", _P), ("zf", _P), ("qname", (C.c_char * 4) * CM1G_MAXQ),
                 ("budname", C.c_char_p)])


WRITEOUT_SWITCHES = ["output_rain", "output_prate", "output_th", "output_thpert", "output_prs", "output_prspert",
                     "output_pi", "output_pipert", "output_rho", "output_rhopert", "output_qv", "output_qvpert",
                     "output_q", "output_u", "output_upert", "output_v", "output_vpert", "output_w"]


class WriteoutOpts(C.Structure):
    """cm1g_writeout_opts_t: writeout's output switches for the advanced fields."""
    _fields_ = [(n, C.c_int32) for n in WRITEOUT_SWITCHES] + [("qname", (C.c_char * 4) * CM1G_MAXQ)]


class Restart(C.Structure):
    """cm1g_restart_t: scalars of a restart file."""
    _fields_ = [("nstep", C.c_int32), ("mtime", C.c_double), ("dt", C.c_float), ("dtlast", C.c_float),
                ("mass1", C.c_double)]


class State(C.Structure):
    """cm1g_state_t: prognostic state and pre-RK tendencies."""
    _fields_ = [(n, _P) for n in STATE_FIELDS]


def fptr(addr):
    """A float* from an integer address (host numpy data or device pointer)."""
    return C.cast(C.c_void_p(int(addr)), _P)
