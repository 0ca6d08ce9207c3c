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


def _pdefq_columns(q, rho, ruh, rvh, rmh, ni, nj, nk, rmax, vol):
    """pdefq (misclibs.F:1037-1117) over every column at once with numpy:
    the binary32 products and binary64 sums of each column in k order.
    Returns the clipped field and the per-column budget change times vol."""
    g = 3
    sl = (slice(1, nk + 1), slice(g, g + nj), slice(g, g + ni))      # (k, j, i) of the C-order view
    qq = q[sl].copy()
    r, rm = rho[sl], rmh[sl]
    ru = ruh[g:g + ni][None, None, :].astype(f32)
    rv = rvh[g:g + nj][None, :, None].astype(f32)
    w = (r * qq * ru * rv * rm).astype(f32)                          # binary32, left to right
    t1 = np.zeros((nj, ni)); a1 = np.zeros((nj, ni)); t2 = np.zeros((nj, ni)); a2 = np.zeros((nj, ni))
    for k in range(nk):
        t1 = t1 + (r[k] * qq[k]).astype(np.float64)
        a1 = a1 + w[k].astype(np.float64)
        qq[k] = np.where(qq[k] < rmax, f32(0.0), qq[k])
        t2 = t2 + (r[k] * qq[k]).astype(np.float64)
    t3 = (t1 + 1.0e-20) / (t2 + 1.0e-20)
    t3 = np.where(t3 < 0.0, 1.0, t3)
    for k in range(nk):
        qq[k] = (t3 * qq[k].astype(np.float64)).astype(f32)
        a2 = a2 + (r[k] * qq[k] * ru[0] * rv[0] * rm[k]).astype(f32).astype(np.float64)
    out = q.copy()
    out[sl] = qq
    return out, float(((a2 - a1).sum(axis=1) * vol).sum()), float(np.abs(a2 - a1).sum() * vol)


def test_pdefq_noalloc_tall_thin_grid(cm1g):
    """A grid of 8 x 70000 columns: more rows than a launch grid's y extent
    (65535) holds, but within the column limit.  The call must clip every
    column and return the budget, not fail silently."""
    torch = _torch()
    base, _ = _case(8, 8, 6, 7)
    cfg = type(base.cfg).from_buffer_copy(base.cfg)
    ni, nj, nk = 8, 70000, 6
    cfg.ni, cfg.nj, cfg.nk = ni, nj, nk
    NI, NJ, NK = ni + 6, nj + 6, nk + 2
    rng = np.random.default_rng(11)
    q = rng.normal(1e-3, 1e-3, (NK, NJ, NI)).astype(f32)
    rho = (1.0 + 0.1 * rng.random((NK, NJ, NI))).astype(f32)
    rmh = (1.0 + 0.02 * rng.random((NK, NJ, NI))).astype(f32)
    ruh = (1.0 + 0.05 * np.sin(np.arange(NI))).astype(f32)
    rvh = (1.0 + 0.03 * np.cos(np.arange(NJ))).astype(f32)
    d = cm1g.to_device({"q": q, "rho": rho, "ruh": ruh, "rvh": rvh, "rmh": rmh})
    torch.cuda.synchronize()
    L = cm1g.lib()
    asq = C.c_double(0.0)
    cm1g.check(L.cm1g_pdefq_noalloc(C.byref(cfg), 0.0, C.byref(asq), cm1g.ptr(d["ruh"]), cm1g.ptr(d["rvh"]),
                                    cm1g.ptr(d["rmh"]), cm1g.ptr(d["rho"]), cm1g.ptr(d["q"]),
                                    C.c_void_p(torch.cuda.current_stream().cuda_stream)))
    got = d["q"].cpu().numpy()
    want, asq_want, scale = _pdefq_columns(q, rho, ruh, rvh, rmh, ni, nj, nk, f32(0.0),
                                    float(f32(cfg.dx) * f32(cfg.dy) * f32(cfg.dz)))
    assert np.array_equal(got, want)
    assert asq_want != 0.0
    assert abs(asq.value - asq_want) <= 1e-12 * scale


def test_pdefq_noalloc_allocates_no_device_memory(cm1g):
    """Free device memory is the same before and after calls (the first call
    loads the library's module and its fixed array, so it is made before the
    measurement)."""
    torch = _torch()
    case, q = _case(40, 36, 20, 8)
    L = cm1g.lib()
    d = cm1g.to_device({"q": q, "rho": case.state["rho"], "ruh": case.grid["ruh"],
                        "rvh": case.grid["rvh"], "rmh": case.grid["rmh"]})
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def call():
        asq = C.c_double(0.0)
        cm1g.check(L.cm1g_pdefq_noalloc(C.byref(case.cfg), 0.0, C.byref(asq), cm1g.ptr(d["ruh"]),
                                        cm1g.ptr(d["rvh"]), cm1g.ptr(d["rmh"]), cm1g.ptr(d["rho"]),
                                        cm1g.ptr(d["q"]), stream))
        return asq.value

    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
