"""Learned closure kernels (k_learned.cu) against the CPU reference of the MLP
(oracle/mlp_ref.py): tensor-core forward, backward gradients, loss, Adam,
face features, and the closure inside the large step."""
import ctypes as C

import numpy as np
import pytest

from cm1_b200.cases import make_case
from oracle import mlp_ref as R

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _p(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_float)) if t is not None else C.cast(None, C.POINTER(C.c_float))


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 0.3, (n, R.IN)).astype(np.float32)
    x[:, 6] = rng.uniform(0, 1, n)
    x[:, 7] = 0
    return x, rng


def _close(a, b, tol, gelu):
    """max|a-b| <= tol * scale.  With GELU the device's erff and the host's
    erf differ in the last place, and a BF16-rounded activation can then
    round the other way (one BF16 unit, 2^-8 relative): such entries are
    allowed in 0.1 % of the values, within 3e-2 of the scale."""
    err = np.abs(np.asarray(a, np.float64) - b)
    sc = max(1.0, float(np.abs(b).max()))
    if not gelu:
        return float(err.max()) <= tol * sc
    return float((err <= tol * sc).mean()) >= 0.999 and float(err.max()) <= 3e-2 * sc


@pytest.mark.parametrize("act", [0, 1])
def test_forward_and_backward_match_reference(act, cm1g):
    torch = _torch()
    L = cm1g.lib()
    assert L.cm1g_mlp_param_count() == R.P_TOTAL
    cm1g.check(L.cm1g_mlp_set_activation(act))
    try:
        _forward_and_backward(act == 1, cm1g, torch, L)
    finally:
        cm1g.check(L.cm1g_mlp_set_activation(0))
    assert L.cm1g_mlp_get_activation() == 0
    assert L.cm1g_mlp_set_activation(2) != 0


def _forward_and_backward(gelu, cm1g, torch, L):
    n = 1000                                          # not a multiple of 16: partial tiles
    x, rng = _data(n, 1)
    p = R.init_params(2)
    p[R.P_W3:R.P_B3] = rng.normal(0, 0.2, R.H * R.OUT).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    P, X = dev(p), dev(x)
    Y, Cc = torch.zeros(n, 8, device="cuda"), torch.zeros(n, 6, device="cuda")
    Z1, Z2 = torch.zeros(n, 64, device="cuda"), torch.zeros(n, 64, device="cuda")
    cm1g.check(L.cm1g_mlp_forward(_p(P), n, _p(X), _p(Y), _p(Cc), _p(Z1), _p(Z2), None))
    torch.cuda.synchronize()
    z1g, z2g = Z1.cpu().numpy().astype(np.float64), Z2.cpu().numpy().astype(np.float64)
    _, _, z1r, _ = R.forward(p, x, gelu=gelu)
    assert np.abs(z1g - z1r).max() <= 1e-5 * max(1.0, np.abs(z1r).max())
    # later layers from the GPU's pre-activations (same BF16 rounding points)
    yr, cr, _, z2r = R.forward(p, x, z1=z1g, gelu=gelu)
    assert _close(z2g, z2r, 1e-5, gelu)
    yr, cr, _, _ = R.forward(p, x, z1=z1g, z2=z2g, gelu=gelu)
    # ReLU is exact on both sides; what remains is the FP32 accumulation
    # order of the tensor-core products against the float64 reference
    assert _close(Y.cpu().numpy(), yr, 1e-5, gelu)
    assert _close(Cc.cpu().numpy(), cr, 1e-5, gelu)
    assert np.allclose(Cc.cpu().numpy().sum(1), 1.0, atol=1e-5)

    # loss and dy
    m = rng.normal(0, 1, n).astype(np.float32)
    d = rng.uniform(0.1, 2, n).astype(np.float32)
    tgt = (m + rng.normal(0, 0.1, n)).astype(np.float32)
    w = rng.uniform(0.5, 2, n).astype(np.float32)
    DY = torch.zeros(n, 8, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    Md, Dd, Td, Wd = dev(m), dev(d), dev(tgt), dev(w)          # keep the device copies alive
    cm1g.check(L.cm1g_closure_loss(n, _p(X), _p(Y), _p(Md), _p(Dd), _p(Td), _p(Wd), _p(DY),
                                   C.c_void_p(loss.data_ptr()), None))
    torch.cuda.synchronize()
    lr_, dyr = R.loss_and_dy(x, Y.cpu().numpy().astype(np.float64), m, d, tgt, w)
    assert abs(loss.item() - lr_) <= 1e-5 * abs(lr_)
    assert np.abs(DY.cpu().numpy() - dyr).max() <= 1e-4 * max(1e-6, np.abs(dyr).max())

    # backward
    G = torch.zeros(R.P_TOTAL, device="cuda")
    cm1g.check(L.cm1g_mlp_backward(_p(P), n, _p(X), _p(Z1), _p(Z2), _p(DY), _p(G), None))
    torch.cuda.synchronize()
    gr = R.backward(p, x, z1g, z2g, DY.cpu().numpy().astype(np.float64), gelu=gelu)
    gg = G.cpu().numpy()
    for a, b in ((R.P_W1, R.P_B1), (R.P_B1, R.P_W2), (R.P_W2, R.P_B2), (R.P_B2, R.P_W3), (R.P_W3, R.P_B3),
                 (R.P_B3, R.P_TOTAL)):
        scale = max(1e-12, np.abs(gr[a:b]).max())
        assert np.abs(gg[a:b] - gr[a:b]).max() <= 2e-3 * scale, (a, b)

    # Adam
    M1, M2 = torch.zeros(R.P_TOTAL, device="cuda"), torch.zeros(R.P_TOTAL, device="cuda")
    cm1g.check(L.cm1g_adam(R.P_TOTAL, _p(P), _p(G), _p(M1), _p(M2), 1, 1e-3, 0.5, None))
    torch.cuda.synchronize()
    pr, _, _ = R.adam(p.astype(np.float64), gg.astype(np.float64), 0.0, 0.0, 1, 1e-3, 0.5)
    assert np.abs(P.cpu().numpy() - pr).max() <= 1e-6


def test_face_features_match_numpy(cm1g):
    torch = _torch()
    L = cm1g.lib()
    case = make_case("dry_bubble", ni=20, nj=12, nk=10)
    lay, st, gr = case.lay, case.state, case.grid
    rng = np.random.default_rng(3)
    th = (st["th3d"] + rng.normal(0, 0.5, lay.shape(1))).astype(np.float32)
    u = rng.normal(0, 5, lay.shape(2)).astype(np.float32)
    th0 = gr["th0"][:, 3, 3].copy()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    nf = (lay.ni + 1) * lay.nj * lay.nk
    X, M, D, U = (torch.zeros(nf, 8, device="cuda"), torch.zeros(nf, device="cuda"), torch.zeros(nf, device="cuda"),
                  torch.zeros(nf, device="cuda"))
    TH, TH0, UU = dev(th), dev(th0), dev(u)                  # keep the device copies alive
    cm1g.check(L.cm1g_face_features(lay.ni, lay.nj, lay.nk, 3, 0, _p(TH), _p(TH0), 1, _p(UU), 0.3,
                                    _p(X), _p(M), _p(D), _p(U), None))
    torch.cuda.synchronize()
    X, M, D, U = X.cpu().numpy(), M.cpu().numpy(), D.cpu().numpy(), U.cpu().numpy()
    s = (th0[:, None, None] - np.float32(300.0)) + th       # (NK, NJ, NI), the advected value
    f = 0
    for k in range(1, lay.nk + 1):
        for j in range(1, lay.nj + 1):
            for i in range(1, lay.ni + 2):
                uu = u[lay.kx(k), lay.jx(j), lay.ix(i)]
                offs = range(-3, 3) if uu >= 0 else range(2, -4, -1)
                v = np.array([s[lay.kx(k), lay.jx(j), lay.ix(i + o)] for o in offs], np.float32)
                mean = v.sum(dtype=np.float32) / np.float32(6)
                sc = (v.max() - v.min()) + np.float32(1e-6)
                assert abs(M[f] - mean) <= 1e-6 * max(1.0, abs(mean)) and abs(D[f] - sc) <= 1e-6 * sc
                assert np.abs(X[f, :6] - (v - mean) / sc).max() <= 1e-5
                assert abs(X[f, 6] - abs(uu) * 0.3) <= 1e-6 * max(1.0, abs(uu)) and X[f, 7] == 0 and U[f] == uu
                f += 1


def test_fused_faces_equal_the_three_passes(cm1g):
    """cm1g_closure_faces (features, MLP and bounded face value in one
    kernel) gives the same phi as face_features -> mlp_forward -> face_phi,
    NaN (WENO5 fallback) at the same faces."""
    torch = _torch()
    L = cm1g.lib()
    case = make_case("dry_bubble", ni=37, nj=29, nk=11)
    lay, st, gr = case.lay, case.state, case.grid
    rng = np.random.default_rng(9)
    th = (st["th3d"] + rng.normal(0, 0.5, lay.shape(1))).astype(np.float32)
    p = R.init_params(4)
    p[R.P_W3:R.P_B3] = rng.normal(0, 0.05, R.H * R.OUT).astype(np.float32)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    TH, TH0, P = dev(th), dev(gr["th0"][:, 3, 3].copy()), dev(p)
    for dir_ in (0, 1):
        vel = rng.normal(0, 5, lay.shape(2 if dir_ == 0 else 3)).astype(np.float32)
        VEL = dev(vel)
        nf = (lay.ni + 1) * lay.nj * lay.nk if dir_ == 0 else lay.ni * (lay.nj + 1) * lay.nk
        X, M, D, U = (torch.zeros(nf, 8, device="cuda"), torch.zeros(nf, device="cuda"),
                      torch.zeros(nf, device="cuda"), torch.zeros(nf, device="cuda"))
        Y, Cc = torch.zeros(nf, 8, device="cuda"), torch.zeros(nf, 6, device="cuda")
        PHI3, PHI1 = torch.zeros(nf, device="cuda"), torch.full((nf,), 7.0, device="cuda")
        cm1g.check(L.cm1g_face_features(lay.ni, lay.nj, lay.nk, 3, dir_, _p(TH), _p(TH0), 1, _p(VEL), 0.2,
                                        _p(X), _p(M), _p(D), _p(U), None))
        cm1g.check(L.cm1g_mlp_forward(_p(P), nf, _p(X), _p(Y), _p(Cc), None, None, None))
        for widen in (0.0, 0.5):
            cm1g.check(L.cm1g_face_phi(nf, _p(X), _p(Cc), _p(M), _p(D), widen, _p(PHI3), None))
            cm1g.check(L.cm1g_closure_faces(lay.ni, lay.nj, lay.nk, 3, dir_, _p(TH), _p(TH0), 1, _p(VEL), 0.2,
                                            _p(P), widen, _p(PHI1), None))
            torch.cuda.synchronize()
            a, b = PHI3.cpu().numpy(), PHI1.cpu().numpy()
            assert np.array_equal(np.isnan(a), np.isnan(b))
            ok = ~np.isnan(a)
            if widen == 0.0:
                assert ok.mean() > 0.3 and (~ok).any()   # both outcomes occur
            assert np.array_equal(a[ok], b[ok])
            # the bound itself, from the features: within the widened range of stencil cells 2..5
            x, m, d = X.cpu().numpy(), M.cpu().numpy(), D.cpu().numpy()
            v = m[:, None].astype(np.float64) + d[:, None] * x[:, 1:5]
            lo = v.min(1) - (1e-6 + widen) * d
            hi = v.max(1) + (1e-6 + widen) * d
            assert np.all((a[ok] >= lo[ok] - 1e-5 * d[ok]) & (a[ok] <= hi[ok] + 1e-5 * d[ok]))


def test_closure_in_the_step(cm1g):
    """With the closure on, theta's horizontal faces come from the MLP where
    they stay inside the range of the four nearest stencil cells; the step stays
    finite and close to the plain step; turning it off restores the plain step
    bit for bit."""
    torch = _torch()
    case = make_case("dry_bubble", ni=40, nj=32, nk=24, advwenos=1)
    ctx = cm1g.Context(case.cfg, case.grid)
    plain = cm1g.to_device(case.state)
    learned = cm1g.to_device(case.state)
    again = cm1g.to_device(case.state)
    ctx.step(plain, case.dt, case.mass1)
    p = R.init_params(0)
    ctx.closure(torch.from_numpy(p).cuda())
    m2, cfl = ctx.step(learned, case.dt, case.mass1)
    assert np.isfinite(m2) and np.isfinite(cfl)
    ctx.closure(None, enable=False)
    ctx.step(again, case.dt, case.mass1)
    torch.cuda.synchronize()
    for k in plain:
        assert torch.equal(plain[k], again[k]), k
    th_p, th_l = plain["th3d"].cpu().numpy(), learned["th3d"].cpu().numpy()
    sl = case.lay.interior(1)
    rng_ = float(th_p[sl].max() - th_p[sl].min())
    diff = float(np.abs(th_l[sl] - th_p[sl]).max())
    assert 0.0 < diff <= 0.05 * rng_


@pytest.mark.parametrize("act", [0, 1])
def test_trained_network_beats_weno5_on_held_out_faces(act, cm1g, monkeypatch):
    """What training gains, at the face level: on quarter-size grids, fine
    runs of the plain method give the training faces (4 runs) and held-out
    faces (1 further run); the network trained by the library's kernels
    (forward, loss, backward, Adam; validation-selected epoch), with ReLU
    (act 0) or GELU (act 1) hidden units, reproduces the held-out target
    face values better than both the 5th-order upwind weights it starts
    from and WENO5, the plain method."""
    _torch()
    L = cm1g.lib()
    cm1g.check(L.cm1g_mlp_set_activation(act))
    try:
        _train_and_compare(monkeypatch)
    finally:
        cm1g.check(L.cm1g_mlp_set_activation(0))


def _train_and_compare(monkeypatch):
    from cm1_b200 import learned as Lm
    monkeypatch.setattr(Lm, "FINE", dict(ni=128, nj=128, nk=40, dx=250.0, dz=125.0, dt=1.5))
    monkeypatch.setattr(Lm, "COARSE", dict(ni=32, nj=32, nk=20, dx=1000.0, dz=250.0, dt=6.0))
    quiet = lambda s: None
    data, _ = Lm.generate(4, 8, 12, seed=11, log=quiet)
    held, _ = Lm.generate(1, 8, 12, seed=907, log=quiet)
    P, hist, _ = Lm.train(data, 20, batch=8192, val=held, log=quiet)
    fe = Lm.face_errors(P, held)
    print("held-out face errors: upwind5 %.3e, WENO5 %.3e, network %.3e" % (fe["upwind5"], fe["weno5"], fe["learned"]))
    assert fe["learned"] < 0.95 * fe["upwind5"]
    assert fe["learned"] < 0.95 * fe["weno5"]
    assert min(hist["validation"]) < Lm.baseline_loss(held)
