"""cm1g_pdefq_noalloc against cm1g_pdefq (the context-based entry point).

cm1g_pdefq_noalloc is the positive-definite column fix of pdefq
(misclibs.F:1037-1117) for host programs that may not allocate device memory:
it keeps its per-column budget in a fixed file-scope device array instead of
a context's scratch.  Two calls in a row on different grids check that the
shared array's leftover contents from the first call do not leak into the
second.  The file name makes pytest collect it last, so it also runs after
every other GPU test in the same process.
"""
import ctypes as C

import numpy as np
import pytest

from cm1_b200.cases import make_case

pytestmark = pytest.mark.gpu
f32 = np.float32


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def relerr(a, b):
    rng = float(b.max() - b.min()) or 1.0
    return float(np.abs(a.astype(np.float64) - b).max()) / rng


def _case(ni, nj, nk, seed):
    case = make_case("supercell", ni=ni, nj=nj, nk=nk)
    lay = case.lay
    # non-uniform metrics so that ruh, rvh and rmh all enter the budget
    case.grid["ruh"] = (1.0 + 0.05 * np.sin(np.arange(lay.NI))).astype(f32)
    case.grid["rvh"] = (1.0 + 0.03 * np.cos(np.arange(lay.NJ))).astype(f32)
    prof = (1.0 + 0.02 * np.arange(lay.NK)).astype(f32)
    case.grid["rmh"] = np.ascontiguousarray(np.broadcast_to(prof[:, None, None], lay.shape(1)), dtype=f32)
    rng = np.random.default_rng(seed)
    q = rng.normal(1e-3, 1e-3, lay.shape(1)).astype(f32)
    return case, q


def _noalloc(cm1g, torch, case, q, rmax):
    L = cm1g.lib()
    d = cm1g.to_device({"q": q, "rho": case.state["rho"], "ruh": case.grid["ruh"],
                        "rvh": case.grid["rvh"], "rmh": case.grid["rmh"]})
    torch.cuda.synchronize()
    asq = C.c_double(0.0)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    cm1g.check(L.cm1g_pdefq_noalloc(C.byref(case.cfg), rmax, C.byref(asq), cm1g.ptr(d["ruh"]),
                                    cm1g.ptr(d["rvh"]), cm1g.ptr(d["rmh"]), cm1g.ptr(d["rho"]),
                                    cm1g.ptr(d["q"]), stream))
    return d["q"].cpu().numpy(), asq.value


def _with_context(cm1g, case, q, rmax):
    ctx = cm1g.Context(case.cfg, case.grid)
    d = cm1g.to_device({"q": q, "rho": case.state["rho"]})
    asq = ctx.pdefq(rmax, d["rho"], d["q"])
    return d["q"].cpu().numpy(), asq


def test_pdefq_noalloc_matches_context_entry(cm1g):
    torch = _torch()
    # first call on the larger grid, second on a smaller one, then the larger again
    for ni, nj, nk, seed in ((40, 36, 20, 3), (24, 20, 16, 4), (40, 36, 20, 5)):
        case, q = _case(ni, nj, nk, seed)
        qa, asq_a = _noalloc(cm1g, torch, case, q, 0.0)
        qb, asq_b = _with_context(cm1g, case, q, 0.0)
        sl = case.lay.interior(1)
        assert relerr(qa[sl], qb[sl].astype(np.float64)) <= 1e-6
        assert asq_b != 0.0
        assert abs(asq_a - asq_b) <= 1e-6 * abs(asq_b) + 1e-30


def test_pdefq_noalloc_rejects_oversized_grid(cm1g):
    torch = _torch()
    case, q = _case(8, 8, 4, 6)
    L = cm1g.lib()
    d = cm1g.to_device({"q": q, "rho": case.state["rho"], "ruh": case.grid["ruh"],
                        "rvh": case.grid["rvh"], "rmh": case.grid["rmh"]})
    cfg = type(case.cfg).from_buffer_copy(case.cfg)
    cfg.ni, cfg.nj = 2048, 1024          # 2 Mi columns > 1 Mi
    asq = C.c_double(0.0)
    rc = L.cm1g_pdefq_noalloc(C.byref(cfg), 0.0, C.byref(asq), cm1g.ptr(d["ruh"]), cm1g.ptr(d["rvh"]),
                              cm1g.ptr(d["rmh"]), cm1g.ptr(d["rho"]), cm1g.ptr(d["q"]),
                              C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == -1
    assert "CM1G_PDEFQ_NOALLOC_MAX_COLUMNS" in L.cm1g_last_error().decode()
    assert asq.value == 0.0
