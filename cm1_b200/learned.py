"""Learned coarse-grid advection closure: data, training, evaluation.

Data.  Fine-grid runs of the plain method (WENO5, dry warm bubbles with
seeded 1-3 K amplitude and 0-20 m/s shear) record theta's face fluxes and
face mass fluxes at every final RK stage (cm1g_capture_fluxes).  Over one
coarse time step (4 fine steps) they are summed over each coarse face
(4 x 2 fine sub-faces of a 4x4x2 coarsening), and the face value the coarse
grid would need, phi* = sum(flux) / sum(mass flux), is the target for the
coarse face's stencil (theta coarsened conservatively at the start of the
coarse step) and Courant number.

Training.  The MLP's forward runs on tensor cores (cm1g_mlp_forward), the
loss w (phi - phi*)^2 with w = (mass flux)^2 normalised to mean 1
(cm1g_closure_loss), the backward (cm1g_mlp_backward) and Adam (cm1g_adam)
are the library's kernels; torch only holds the device buffers.

Evaluation.  From the coarsened initial state of held-out fine runs, coarse
runs with plain WENO5 and with the closure, and a plain run at twice the
coarse resolution, are compared with the coarsened fine run after the same
simulated time (L2 of theta'), together with each run's GPU time.

    python -m cm1_b200.learned [--runs 8] [--outputs 16] [--epochs 40] [--keep 1.0] [--minutes 30]
"""
import argparse
import ctypes as C
import json
import math
import os
import sys
import time

import numpy as np

FINE = dict(ni=512, nj=512, nk=80, dx=250.0, dz=125.0, dt=1.5)
COARSE = dict(ni=128, nj=128, nk=40, dx=1000.0, dz=250.0, dt=6.0)
MID = dict(ni=256, nj=256, nk=40, dx=500.0, dz=250.0, dt=3.0)      # plain method at 2x the coarse resolution
FX, FY, FZ = 4, 4, 2


N_PARAMS = 8 * 64 + 64 + 64 * 64 + 64 + 64 * 8 + 8


def init_params(seed=0):
    """Initial MLP parameters: small random hidden layers, a near-zero output
    layer, and output biases equal to the 5th-order upwind coefficients
    (2, -13, 47, 27, -3, 0)/60, so training starts from the plain 5th-order
    face value (layout of k_learned.cu: W1[8][64], b1, W2[64][64], b2, W3[64][8], b3)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    o = 0
    w1 = rng.normal(0, math.sqrt(2.0 / 7), (8, 64)).astype(np.float32)      # He initialisation
    w1[7] = 0
    p[o:o + 512] = w1.ravel(); o += 512 + 64
    p[o:o + 4096] = rng.normal(0, math.sqrt(2.0 / 64), 4096); o += 4096 + 64
    w3 = rng.normal(0, 0.01, (64, 8)).astype(np.float32)
    w3[:, 6:] = 0
    p[o:o + 512] = w3.ravel(); o += 512
    p[o:o + 6] = np.array([2, -13, 47, 27, -3, 0], np.float32) / 60.0
    return p


def _lib():
    from . import binding
    return binding


def _fp(t):
    return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_float)) if t is not None else C.cast(None, C.POINTER(C.c_float))


def member(grid, seed, amp, xr, shear):
    """A dry warm-bubble case on `grid` (dict of ni, nj, nk, dx, dz, dt)."""
    from .cases import make_case
    b = _lib()
    nsound = b.dtsmall(3, grid["ni"], grid["nj"], grid["dx"], grid["dx"], grid["dz"], grid["dt"])[0]
    return make_case("dry_bubble", seed=seed, ni=grid["ni"], nj=grid["nj"], nk=grid["nk"], dx=grid["dx"],
                     dz=grid["dz"], dt=grid["dt"], nsound=nsound, advwenos=1,
                     bubble=dict(amp=amp, xr=xr, zr=1400.0, zc=1400.0), wind=("shear", dict(du=shear)),
                     noise=dict(amp=0.01, zmax=None))


def draw(rng):
    return dict(amp=float(rng.uniform(1.0, 3.0)), xr=float(rng.uniform(3000.0, 6000.0)),
                shear=float(rng.uniform(0.0, 20.0)))


# ---------------------------------------------------------------- coarsening
def _interior(lay, a, stag):
    import torch
    ni, nj, nk = lay.ni, lay.nj, lay.nk
    if stag == 1:
        return a[lay.kx(1):lay.kx(nk) + 1, lay.jx(1):lay.jx(nj) + 1, lay.ix(1):lay.ix(ni) + 1]
    raise ValueError(stag)


def coarsen_s(lay, a, fac=(FX, FY, FZ)):
    """Cell average over fx x fy x fz fine cells (interior only)."""
    fx, fy, fz = fac
    v = _interior(lay, a, 1)
    nk, nj, ni = v.shape
    return v.reshape(nk // fz, fz, nj // fy, fy, ni // fx, fx).mean(dim=(1, 3, 5))


def coarsen_uface(lay, u, fac=(FX, FY, FZ)):
    """x-faces: the fine faces at i = fx(I-1)+1 averaged over their fy x fz fine sub-faces."""
    fx, fy, fz = fac
    ni, nj, nk = lay.ni, lay.nj, lay.nk
    v = u[lay.kx(1):lay.kx(nk) + 1, lay.jx(1):lay.jx(nj) + 1, lay.ix(1):lay.ix(ni + 1) + 1:fx]
    return v.reshape(nk // fz, fz, nj // fy, fy, -1).mean(dim=(1, 3))


def coarsen_vface(lay, v, fac=(FX, FY, FZ)):
    fx, fy, fz = fac
    ni, nj, nk = lay.ni, lay.nj, lay.nk
    w = v[lay.kx(1):lay.kx(nk) + 1, lay.jx(1):lay.jx(nj + 1) + 1:fy, lay.ix(1):lay.ix(ni) + 1]
    return w.reshape(nk // fz, fz, -1, ni // fx, fx).mean(dim=(1, 4))


def coarsen_wface(lay, w, fac=(FX, FY, FZ)):
    fx, fy, fz = fac
    ni, nj, nk = lay.ni, lay.nj, lay.nk
    v = w[lay.kx(1):lay.kx(nk + 1) + 1:fz, lay.jx(1):lay.jx(nj) + 1, lay.ix(1):lay.ix(ni) + 1]
    return v.reshape(v.shape[0], nj // fy, fy, ni // fx, fx).mean(dim=(2, 4))


def sum_uface(lay, a):
    ni, nj, nk = lay.ni, lay.nj, lay.nk
    v = a[lay.kx(1):lay.kx(nk) + 1, lay.jx(1):lay.jx(nj) + 1, lay.ix(1):lay.ix(ni + 1) + 1:FX]
    return v.reshape(nk // FZ, FZ, nj // FY, FY, -1).sum(dim=(1, 3))


def sum_vface(lay, a):
    ni, nj, nk = lay.ni, lay.nj, lay.nk
    v = a[lay.kx(1):lay.kx(nk) + 1, lay.jx(1):lay.jx(nj + 1) + 1:FY, lay.ix(1):lay.ix(ni) + 1]
    return v.reshape(nk // FZ, FZ, -1, ni // FX, FX).sum(dim=(1, 4))


def coarse_state(fcase, fdev, ccase, cctx, fac=(FX, FY, FZ)):
    """Device state of the coarse case from the fine one (conservative averages, halos filled)."""
    import torch
    b = _lib()
    fl, cl = fcase.lay, ccase.lay
    th0f = torch.from_numpy(fcase.grid["th0"]).cuda()
    th0c = torch.from_numpy(ccase.grid["th0"]).cuda()
    dev = b.to_device(ccase.state)
    full = coarsen_s(fl, th0f + fdev["th3d"], fac)
    ci = (slice(cl.kx(1), cl.kx(cl.nk) + 1), slice(cl.jx(1), cl.jx(cl.nj) + 1), slice(cl.ix(1), cl.ix(cl.ni) + 1))
    th = full - th0c[ci]
    for name in ("th3d", "tha"):
        dev[name][ci] = th
    for name in ("pp3d", "ppi"):
        dev[name][ci] = coarsen_s(fl, fdev["pp3d"], fac)
    dev["rho"][ci] = coarsen_s(fl, fdev["rho"], fac)
    dev["prs"][ci] = coarsen_s(fl, fdev["prs"], fac)
    cu = (slice(cl.kx(1), cl.kx(cl.nk) + 1), slice(cl.jx(1), cl.jx(cl.nj) + 1), slice(cl.ix(1), cl.ix(cl.ni + 1) + 1))
    cv = (slice(cl.kx(1), cl.kx(cl.nk) + 1), slice(cl.jx(1), cl.jx(cl.nj + 1) + 1), slice(cl.ix(1), cl.ix(cl.ni) + 1))
    cw = (slice(cl.kx(1), cl.kx(cl.nk + 1) + 1), slice(cl.jx(1), cl.jx(cl.nj) + 1), slice(cl.ix(1), cl.ix(cl.ni) + 1))
    for name in ("u3d", "ua"):
        dev[name][cu] = coarsen_uface(fl, fdev["u3d"], fac)
    for name in ("v3d", "va"):
        dev[name][cv] = coarsen_vface(fl, fdev["v3d"], fac)
    for name in ("w3d", "wa"):
        dev[name][cw] = coarsen_wface(fl, fdev["w3d"], fac)
    dev["ppx"].zero_()
    torch.cuda.synchronize()
    for name, which in (("th3d", "s"), ("tha", "s"), ("pp3d", "p"), ("ppi", "p"), ("rho", "p"), ("prs", "p"),
                        ("u3d", "u"), ("ua", "u"), ("v3d", "v"), ("va", "v"), ("w3d", "w"), ("wa", "w")):
        cctx.bc(which, dev[name])
    torch.cuda.synchronize()
    return dev


def coarse_mass(ccase, dev):
    """mass1 of a coarsened state as apmasscon counts it: the FP64 sum of
    rho*ruh*rvh*rmh over the physical cells without the cell volume
    (solve2.F:1617-1648; the grids here are uniform, so the metrics are 1)."""
    lay = ccase.lay
    ci = (slice(lay.kx(1), lay.kx(lay.nk) + 1), slice(lay.jx(1), lay.jx(lay.nj) + 1), slice(lay.ix(1), lay.ix(lay.ni) + 1))
    return float(dev["rho"][ci].double().sum().item())


# ---------------------------------------------------------------- data
def face_samples(ccase, cdev, fx_sum, fy_sum, rx_sum, ry_sum, dt_c, keep_quiet, keep_active=1.0):
    """Features and targets of the coarse x- and y-faces for one coarse step:
    a random `keep_active` of the faces whose stencil varies by more than
    1e-3 K, and `keep_quiet` of the others."""
    import torch
    b = _lib()
    L = b.lib()
    cl, cfg = ccase.lay, ccase.cfg
    th0 = torch.from_numpy(ccase.grid["th0"][:, 3, 3].copy()).cuda()
    out = []
    for dir_, vel, fsum, rsum in ((0, cdev["u3d"], fx_sum, rx_sum), (1, cdev["v3d"], fy_sum, ry_sum)):
        nfx, nfy = (cl.ni + 1, cl.nj) if dir_ == 0 else (cl.ni, cl.nj + 1)
        nf = nfx * nfy * cl.nk
        x = torch.zeros(nf, 8, device="cuda")
        m, d, u = (torch.zeros(nf, device="cuda") for _ in range(3))
        b.check(L.cm1g_face_features(cl.ni, cl.nj, cl.nk, 3, dir_, _fp(cdev["th3d"]), _fp(th0), 1, _fp(vel),
                                     dt_c / cfg.dx, _fp(x), _fp(m), _fp(d), _fp(u), None))
        phi = (fsum / torch.where(rsum.abs() > 0, rsum, torch.ones_like(rsum))).reshape(-1)
        wgt = (rsum * rsum).reshape(-1)
        ok = (rsum.abs().reshape(-1) > 1e-6) & torch.isfinite(phi)
        active = d > 1e-3
        draw_ = torch.rand(nf, device="cuda")
        sel = ok & torch.where(active, draw_ < keep_active, draw_ < keep_quiet)
        out.append((x[sel], m[sel], d[sel], phi[sel], wgt[sel]))
    return out


def generate(runs, outputs, spacing, seed=11, keep_active=1.0, log=print):
    """Training samples from `runs` fine-grid runs, `outputs` coarse steps each."""
    import torch
    b = _lib()
    rng = np.random.default_rng(seed)
    torch.manual_seed(seed)
    chunks = []
    t_gpu = 0.0
    for r in range(runs):
        prm = draw(rng)
        fcase = member(FINE, seed + 100 * r, **prm)
        ccase = member(COARSE, seed + 100 * r + 1, **prm)
        fctx, cctx = b.Context(fcase.cfg, fcase.grid), b.Context(ccase.cfg, ccase.grid)
        fdev = b.to_device(fcase.state)
        fl = fcase.lay
        cap = [torch.zeros(fl.shape(2), device="cuda"), torch.zeros(fl.shape(3), device="cuda"),
               torch.zeros(fl.shape(2), device="cuda"), torch.zeros(fl.shape(3), device="cuda")]
        t0 = time.perf_counter()
        for o in range(outputs):
            for _ in range(spacing - FX):
                fctx.step(fdev, fcase.dt, fcase.mass1, use_graph=True)
            cdev = coarse_state(fcase, fdev, ccase, cctx)
            fctx.capture_fluxes(*cap)
            sums = [torch.zeros(sum_uface(fl, cap[0]).shape, device="cuda"),
                    torch.zeros(sum_vface(fl, cap[1]).shape, device="cuda")] * 2
            sums = [s.clone() for s in sums]
            for _ in range(FX):
                fctx.step(fdev, fcase.dt, fcase.mass1, use_graph=True)
                sums[0] += sum_uface(fl, cap[0]); sums[1] += sum_vface(fl, cap[1])
                sums[2] += sum_uface(fl, cap[2]); sums[3] += sum_vface(fl, cap[3])
            fctx.capture_fluxes()
            chunks.extend(face_samples(ccase, cdev, sums[0], sums[1], sums[2], sums[3], ccase.dt, 0.05 * keep_active,
                                       keep_active))
        torch.cuda.synchronize()
        t_gpu += time.perf_counter() - t0
        log("run %d %s: %d samples so far" % (r, prm, sum(c[0].shape[0] for c in chunks)))
        fctx.close(); cctx.close()
    cat = [torch.cat([c[q] for c in chunks]) for q in range(5)]
    cat[4] = cat[4] / cat[4].mean()
    return cat, t_gpu


# ---------------------------------------------------------------- training
def _loss_of(P, data, chunk=1 << 22):
    """Mean weighted face loss of parameters P over a data set (library kernels)."""
    import torch
    b = _lib()
    L = b.lib()
    x, m, d, tgt, w = data
    n = x.shape[0]
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    y = torch.empty(min(n, chunk), 8, device="cuda")
    dy = torch.empty(min(n, chunk), 8, device="cuda")
    for s0 in range(0, n, chunk):
        k = min(chunk, n - s0)
        xs, ms, ds, ts, ws = (a[s0:s0 + k].contiguous() for a in (x, m, d, tgt, w))
        b.check(L.cm1g_mlp_forward(_fp(P), k, _fp(xs), _fp(y), None, None, None, None))
        b.check(L.cm1g_closure_loss(k, _fp(xs), _fp(y), _fp(ms), _fp(ds), _fp(ts), _fp(ws), _fp(dy),
                                    C.c_void_p(loss.data_ptr()), None))
    return float(loss.item()) / max(1, n)


def train(data, epochs, batch=65536, lr=2e-3, lr_end=5e-5, seed=5, val=None, log=print):
    """Adam over shuffled mini-batches, all on the library's kernels; the step
    size follows a cosine from lr to lr_end over the whole run.  With a
    validation set (samples of other runs), the parameters of the epoch with
    the lowest validation loss are returned."""
    import torch
    b = _lib()
    L = b.lib()
    x, m, d, tgt, w = data
    n = x.shape[0]
    batch = max(256, min(batch, n // 8 // 256 * 256))
    total = epochs * (n // batch)
    P = torch.from_numpy(init_params(seed)).cuda()
    M1, M2, G = torch.zeros_like(P), torch.zeros_like(P), torch.zeros_like(P)
    Y = torch.zeros(batch, 8, device="cuda")
    Z1, Z2 = torch.zeros(batch, 64, device="cuda"), torch.zeros(batch, 64, device="cuda")
    DY = torch.zeros(batch, 8, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    step, hist, vhist = 0, [], []
    best, best_P = None, None
    t0 = time.perf_counter()
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=gen)
        loss.zero_()
        for s0 in range(0, n - batch + 1, batch):
            idx = perm[s0:s0 + batch]
            xb, mb, db, tb, wb = (x[idx].contiguous(), m[idx].contiguous(), d[idx].contiguous(),
                                  tgt[idx].contiguous(), w[idx].contiguous())
            b.check(L.cm1g_mlp_forward(_fp(P), batch, _fp(xb), _fp(Y), None, _fp(Z1), _fp(Z2), None))
            b.check(L.cm1g_closure_loss(batch, _fp(xb), _fp(Y), _fp(mb), _fp(db), _fp(tb), _fp(wb), _fp(DY),
                                        C.c_void_p(loss.data_ptr()), None))
            G.zero_()
            b.check(L.cm1g_mlp_backward(_fp(P), batch, _fp(xb), _fp(Z1), _fp(Z2), _fp(DY), _fp(G), None))
            lr_t = lr_end + 0.5 * (lr - lr_end) * (1.0 + math.cos(math.pi * step / max(1, total)))
            step += 1
            b.check(L.cm1g_adam(P.numel(), _fp(P), _fp(G), _fp(M1), _fp(M2), step, lr_t, 1.0 / batch, None))
        torch.cuda.synchronize()
        nb = max(1, n // batch)
        hist.append(loss.item() / (nb * batch))
        if val is not None:
            vhist.append(_loss_of(P, val))
            if best is None or vhist[-1] < best:
                best, best_P = vhist[-1], P.clone()
        if ep % 5 == 0 or ep == epochs - 1:
            log("epoch %d loss %.4e%s" % (ep, hist[-1], " validation %.4e" % vhist[-1] if vhist else ""))
    torch.cuda.synchronize()
    t = time.perf_counter() - t0
    if best_P is not None:
        P = best_P
    return P, {"train": hist, "validation": vhist}, t


def baseline_loss(data):
    """Loss of the plain 5th-order coefficients (the initial point) for reference."""
    import torch
    x, m, d, tgt, w = data
    c = torch.tensor([2, -13, 47, 27, -3, 0], dtype=torch.float32, device="cuda") / 60.0
    phi = m + d * (x[:, :6] * c).sum(1)
    return float(((w * (phi - tgt) ** 2).sum() / x.shape[0]).item())


# ---------------------------------------------------------------- evaluation
def weno5_faces(v, weps=1e-17):
    """WENO5 face values with the Borges et al. (2008) weights (the plain
    method of the scalar pass), float64, from the upwind-ordered stencil
    values v[:, 0..4] (v[:, 2] and v[:, 3] are the cells beside the face)."""
    s1, s2, s3, s4, s5 = (v[:, q] for q in range(5))
    b1 = 13.0 / 12.0 * (s1 - 2 * s2 + s3) ** 2 + 0.25 * (s1 - 4 * s2 + 3 * s3) ** 2
    b2 = 13.0 / 12.0 * (s2 - 2 * s3 + s4) ** 2 + 0.25 * (s2 - s4) ** 2
    b3 = 13.0 / 12.0 * (s3 - 2 * s4 + s5) ** 2 + 0.25 * (3 * s3 - 4 * s4 + s5) ** 2
    q1 = (2 * s1 - 7 * s2 + 11 * s3) / 6.0
    q2 = (-s2 + 5 * s3 + 2 * s4) / 6.0
    q3 = (2 * s3 + 5 * s4 - s5) / 6.0
    tau = (b1 - b3).abs()
    a1 = 0.1 * (1 + (tau / (b1 + weps)) ** 2)
    a2 = 0.6 * (1 + (tau / (b2 + weps)) ** 2)
    a3 = 0.3 * (1 + (tau / (b3 + weps)) ** 2)
    return (a1 * q1 + a2 * q2 + a3 * q3) / (a1 + a2 + a3)


def face_errors(P, data, widens=(0.0, 1.0), chunk=1 << 22):
    """Weighted mean squared error of the coarse face values against the
    fine-run targets, for the 5th-order upwind weights, WENO5, the network,
    and the network with the WENO5 fallback outside the neighbour bounds (the
    form the large step uses)."""
    import torch
    b = _lib()
    L = b.lib()
    x, m, d, tgt, w = data
    n = x.shape[0]
    c = torch.empty(n, 6, device="cuda")
    y = torch.empty(min(n, chunk), 8, device="cuda")
    for s0 in range(0, n, chunk):
        k = min(chunk, n - s0)
        xs = x[s0:s0 + k].contiguous()
        cs = torch.empty(k, 6, device="cuda")
        b.check(L.cm1g_mlp_forward(_fp(P), k, _fp(xs), _fp(y), _fp(cs), None, None, None))
        c[s0:s0 + k] = cs
    torch.cuda.synchronize()
    xd, md, dd, td, wd = x[:, :6].double(), m.double(), d.double(), tgt.double(), w.double()
    v = md[:, None] + dd[:, None] * xd
    c5 = torch.tensor([2, -13, 47, 27, -3, 0], dtype=torch.float64, device="cuda") / 60.0
    phi5 = md + dd * (xd @ c5)
    phiw = weno5_faces(v)
    phil = md + dd * (c.double() * xd).sum(1)
    lo, hi = v[:, 1:5].min(1).values, v[:, 1:5].max(1).values
    err = lambda phi: float((wd * (phi - td) ** 2).sum().item() / n)
    out = {"samples": int(n), "upwind5": err(phi5), "weno5": err(phiw), "learned": err(phil)}
    for widen in widens:
        tol = (1e-6 + widen) * dd
        inside = lambda phi: (phi >= lo - tol) & (phi <= hi + tol)
        frac_out = lambda phi: float(1.0 - inside(phi).double().mean().item())
        out["widen_%g" % widen] = {"learned_with_fallback": err(torch.where(inside(phil), phil, phiw)),
                                   "fallback_fraction": frac_out(phil), "upwind5_outside": frac_out(phi5),
                                   "target_outside": frac_out(td)}
    return out


class _Run:
    """A run advanced in segments; its GPU time is the sum of CUDA-event
    times of the replayed step graphs.  The first step of the run captures
    the graph (host work) and is not timed; the run's time is scaled by
    steps / timed steps."""

    def __init__(self, ctx, dev, case, mass1):
        self.ctx, self.dev, self.case, self.mass1 = ctx, dev, case, mass1
        self.steps = self.timed = 0
        self.ms = 0.0
        self.failed = None          # the library's error if the run went unstable

    def advance(self, n):
        if n <= 0 or self.failed:
            return
        try:
            self._advance(n)
        except Exception as e:      # a non-finite velocity ends this run only
            self.failed = "step %d: %s" % (self.steps, e)

    def _advance(self, n):
        import torch
        if self.steps == 0:
            self.ctx.step(self.dev, self.case.dt, self.mass1, use_graph=True)
            self.steps += 1
            n -= 1
            torch.cuda.synchronize()
        if n <= 0:
            return
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n):
            self.ctx.step(self.dev, self.case.dt, self.mass1, use_graph=True)
        e1.record()
        torch.cuda.synchronize()
        self.ms += e0.elapsed_time(e1)
        self.steps += n
        self.timed += n

    def gpu_seconds(self):
        return self.ms / 1e3 * self.steps / max(1, self.timed)


def evaluate(P, tests, minutes, seed=77, horizons=(2, 10, 50), widens=(0.0, 1.0), log=print):
    """Held-out runs: L2 of theta' against the coarsened fine run after
    `horizons` coarse steps and after `minutes`, for the coarse grid without
    and with the closure and for the plain method at twice the coarse
    resolution, with each run's GPU time to that point."""
    import torch
    b = _lib()
    rng = np.random.default_rng(seed)
    res = []
    for t in range(tests):
        prm = draw(rng)
        fcase = member(FINE, seed + 100 * t, **prm)
        ccase = member(COARSE, seed + 100 * t + 1, **prm)
        mcase = member(MID, seed + 100 * t + 2, **prm)
        fctx, pctx, mctx = (b.Context(c.cfg, c.grid) for c in (fcase, ccase, mcase))
        lctx = {w: b.Context(ccase.cfg, ccase.grid) for w in widens}
        for w, c in lctx.items():
            c.closure(P, widen=w)
        fdev = b.to_device(fcase.state)
        # initial coarse/mid states from the fine initial state (same bubble, same shear)
        c_plain = coarse_state(fcase, fdev, ccase, pctx)
        c_learn = {w: {k: v.clone() for k, v in c_plain.items()} for w in widens}
        mdev = coarse_state(fcase, fdev, mcase, mctx, (2, 2, 2))
        m1c = coarse_mass(ccase, c_plain)
        runs = {"fine_plain_250m": _Run(fctx, fdev, fcase, fcase.mass1),
                "coarse_plain": _Run(pctx, c_plain, ccase, m1c),
                "plain_500m": _Run(mctx, mdev, mcase, coarse_mass(mcase, mdev))}
        ratio = {"fine_plain_250m": FX, "coarse_plain": 1, "plain_500m": 2}
        for w in widens:
            runs["coarse_learned_widen_%g" % w] = _Run(lctx[w], c_learn[w], ccase, m1c)
            ratio["coarse_learned_widen_%g" % w] = 1
        total = int(round(minutes * 60 / ccase.dt))
        cl, ml = ccase.lay, mcase.lay
        ci = (slice(cl.kx(1), cl.kx(cl.nk) + 1), slice(cl.jx(1), cl.jx(cl.nj) + 1), slice(cl.ix(1), cl.ix(cl.ni) + 1))
        done, rows = 0, []
        for hz in sorted(set([h for h in horizons if h < total] + [total])):
            for name, r in runs.items():
                r.advance((hz - done) * ratio[name])
            done = hz
            ref = coarse_state(fcase, fdev, ccase, pctx)["th3d"][ci]
            l2 = lambda a: float(torch.sqrt(((a - ref) ** 2).mean()).item())
            mth = mdev["th3d"][ml.kx(1):ml.kx(ml.nk) + 1, ml.jx(1):ml.jx(ml.nj) + 1, ml.ix(1):ml.ix(ml.ni) + 1]
            mth = mth.reshape(ml.nk, ml.nj // 2, 2, ml.ni // 2, 2).mean(dim=(2, 4))
            l2s = {"coarse_plain": l2(c_plain["th3d"][ci]), "plain_500m": l2(mth), "no_change": l2(torch.zeros_like(ref))}
            for w in widens:
                r = runs["coarse_learned_widen_%g" % w]
                l2s["coarse_learned_widen_%g" % w] = None if r.failed else l2(c_learn[w]["th3d"][ci])
            row = {"coarse_steps": hz, "seconds": hz * ccase.dt, "l2_theta": l2s,
                   "unstable": {k: r.failed for k, r in runs.items() if r.failed},
                   "gpu_seconds": {k: r.gpu_seconds() for k, r in runs.items()}}
            log(json.dumps(row))
            rows.append(row)
        res.append({"params": prm, "horizons": rows})
        for c in [fctx, pctx, mctx] + list(lctx.values()):
            c.close()
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--runs", type=int, default=8)
    ap.add_argument("--outputs", type=int, default=16)
    ap.add_argument("--spacing", type=int, default=40, help="fine steps between samples (>= 4)")
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--keep", type=float, default=1.0, help="fraction of the active faces kept per output")
    ap.add_argument("--val-runs", type=int, default=2, help="runs of the validation / held-out face set")
    ap.add_argument("--params", default=None, help="evaluate these parameters (.npy) instead of training")
    ap.add_argument("--widens", default="0,1", help="bound widenings of the face values to evaluate")
    ap.add_argument("--tests", type=int, default=2)
    ap.add_argument("--minutes", type=float, default=30.0)
    ap.add_argument("--out", default="closure_out")
    ap.add_argument("--small", action="store_true", help="quarter-size grids (a quick end-to-end check)")
    ap.add_argument("--act", choices=("relu", "gelu"), default="relu", help="hidden activation of the network")
    args = ap.parse_args(argv)
    import torch
    b = _lib()
    b.check(b.lib().cm1g_mlp_set_activation(1 if args.act == "gelu" else 0))
    if args.small:
        for grid in (FINE, COARSE, MID):
            grid["ni"] //= 4
            grid["nj"] //= 4
            grid["nk"] //= 2
    os.makedirs(args.out, exist_ok=True)
    logf = open(os.path.join(args.out, "log.txt"), "w")

    def log(s):
        print(s)
        logf.write(s + "\n")
        logf.flush()

    widens = tuple(float(w) for w in args.widens.split(","))
    # samples of other runs: validation for the choice of epoch, and the
    # held-out face errors reported below
    held, _ = generate(args.val_runs, args.outputs, args.spacing, seed=907, keep_active=args.keep, log=log)
    if args.params:
        # evaluate given parameters (no data generation, no training)
        P = torch.from_numpy(np.load(args.params).astype(np.float32)).cuda()
        t_gen = t_train = 0.0
        base, hist, n_samples, faces_train = None, {"train": [None], "validation": []}, 0, None
    else:
        data, t_gen = generate(args.runs, args.outputs, args.spacing, keep_active=args.keep, log=log)
        base = baseline_loss(data)
        P, hist, t_train = train(data, args.epochs, lr=args.lr, val=held, log=log)
        n_samples = int(data[0].shape[0])
        faces_train = face_errors(P, [a[: min(a.shape[0], 1 << 24)] for a in data], widens)
        del data
        torch.cuda.empty_cache()
    np.save(os.path.join(args.out, "params.npy"), P.cpu().numpy())
    faces = face_errors(P, held, widens)
    log(json.dumps({"held_out_face_errors": faces, "training_face_errors": faces_train}))
    del held
    torch.cuda.empty_cache()
    ev = evaluate(P, args.tests, args.minutes, widens=widens, log=log)
    rep = {"samples": n_samples, "data_gpu_seconds": t_gen, "train_gpu_seconds": t_train,
           "loss_5th_order_start": base, "loss_final": hist["train"][-1], "loss_history": hist,
           "held_out_face_errors": faces, "training_face_errors": faces_train,
           "grids": {"fine": FINE, "coarse": COARSE, "plain_2x": MID}, "runs": args.runs,
           "outputs_per_run": args.outputs, "epochs": args.epochs, "activation": args.act, "evaluation": ev}
    json.dump(rep, open(os.path.join(args.out, "report.json"), "w"), indent=1)
    log(json.dumps({k: v for k, v in rep.items() if k != "loss_history"}))
    return 0


if __name__ == "__main__":
    sys.exit(main())
