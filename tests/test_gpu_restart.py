"""Output records and restart files through the C-ABI.

Records: a field's physical points, one record per level, i fastest then j
(writeout's GrADS layout and restart_write's writer), checked against numpy
slicing of the same arrays, for s-, u-, v-, w- and 2-D arrays, from host and
device arrays, and unpacked back.

Restart: a run that writes a restart after three steps and goes on for two
more must equal, bit for bit, a run that reads that restart into other
arrays and takes the same two steps (dry, moist with tracers and open
boundaries, Kessler with rain).
"""
import numpy as np
import pytest

from cm1_b200.cases import make_case

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_records_layout_and_round_trip(cm1g):
    torch = _torch()
    case = make_case("supercell", ni=37, nj=21, nk=12)
    lay, st = case.lay, case.state
    rng = np.random.default_rng(7)
    arrs = {"th": rng.normal(size=lay.shape(1)).astype(np.float32), "u": rng.normal(size=lay.shape(2)).astype(np.float32),
            "v": rng.normal(size=lay.shape(3)).astype(np.float32), "w": rng.normal(size=lay.shape(4)).astype(np.float32),
            "sfc": rng.normal(size=(lay.NJ, lay.NI)).astype(np.float32)}
    names, stag, k1, k2 = ["th", "u", "v", "w", "sfc"], [1, 2, 3, 4, 1], [1, 1, 1, 1, 0], [12, 12, 12, 13, 0]
    ctx = cm1g.Context(case.cfg, case.grid)
    out = ctx.pack_records([arrs[n] for n in names], stag, k1, k2)
    expect = []
    for n, sg, a, b in zip(names, stag, k1, k2):
        if n == "sfc":
            I = lay.interior(1)
            expect.append(arrs[n][I[1], I[2]].ravel())
            continue
        I = lay.interior(sg)
        kk = slice(lay.kx(a), lay.kx(b) + 1)
        expect.append(arrs[n][(kk,) + I[1:]].ravel())
    expect = np.concatenate(expect)
    assert out.shape == expect.shape and np.array_equal(out, expect)
    # device arrays and a device buffer give the same records
    dev = {n: torch.from_numpy(a).cuda() for n, a in arrs.items()}
    dbuf = torch.zeros(out.size, dtype=torch.float32, device="cuda")
    ctx.pack_records([dev[n] for n in names], stag, k1, k2, out=dbuf)
    assert np.array_equal(dbuf.cpu().numpy(), out)
    # unpacking into zeroed arrays restores the physical points
    back = {n: np.zeros_like(a) for n, a in arrs.items()}
    ctx.unpack_records([back[n] for n in names], stag, k1, k2, out)
    assert np.array_equal(ctx.pack_records([back[n] for n in names], stag, k1, k2), out)
    ctx.close()


def _interior_equal(case, a, b):
    lay = case.lay
    for k, stag in (("ua", 2), ("va", 3), ("wa", 4), ("u3d", 2), ("v3d", 3), ("w3d", 4), ("ppi", 1), ("pp3d", 1),
                    ("tha", 1), ("th3d", 1), ("rho", 1), ("prs", 1), ("ppx", 1)):
        I = lay.interior(stag)
        assert np.array_equal(a[k][I], b[k][I]), k
    for k in ("qa", "q3d", "pta", "pt3d"):
        for n in range(a[k].shape[0]):
            assert np.array_equal(a[k][n][lay.interior(1)], b[k][n][lay.interior(1)]), (k, n)
    for k in ("radbcw", "radbce", "radbcs", "radbcn", "rain"):
        if k in a:
            assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("name,over", [("dry_bubble", dict(ni=40, nj=36, nk=20)),
                                       ("supercell", dict(ni=40, nj=36, nk=40)),
                                       ("kessler", dict(ni=40, nj=36, nk=40))])
def test_restart_resumes_bit_for_bit(name, over, tmp_path, cm1g):
    torch = _torch()
    case = make_case(name, **over)
    ctx = cm1g.Context(case.cfg, case.grid)
    a = cm1g.to_device(case.state)
    for _ in range(3):
        ctx.step(a, case.dt, case.mass1, use_graph=True)
    path = tmp_path / "rst.bin"
    ctx.restart_write(path, a, nstep=3, mtime=3 * case.dt, dt=case.dt, dtlast=case.dt, mass1=case.mass1)
    for _ in range(2):
        ctx.step(a, case.dt, case.mass1, use_graph=True)
    # other arrays: the initial state with a different seed, then the restart
    other = make_case(name, seed=99, **over)
    b = cm1g.to_device(other.state)
    hdr = ctx.restart_read(path, b)
    assert hdr["nstep"] == 3 and hdr["mtime"] == 3 * case.dt and hdr["mass1"] == case.mass1
    for _ in range(2):
        ctx.step(b, case.dt, hdr["mass1"], use_graph=True)
    torch.cuda.synchronize()
    _interior_equal(case, cm1g.to_host(a), cm1g.to_host(b))
    # host arrays read the same file to the same values
    h = other.copy_state()
    ctx.restart_read(path, h)
    d = cm1g.to_device(other.state)
    ctx.restart_read(path, d)
    hd = cm1g.to_host(d)
    for k in ("ua", "tha", "ppi", "rho", "qa", "pta", "radbcw"):
        assert np.array_equal(h[k][...], hd[k][...]), k
    ctx.close()


def test_restart_rejects_other_grid(tmp_path, cm1g):
    _torch()
    case = make_case("dry_bubble", ni=24, nj=20, nk=12)
    ctx = cm1g.Context(case.cfg, case.grid)
    path = tmp_path / "rst.bin"
    ctx.restart_write(path, case.state)
    other = make_case("dry_bubble", ni=24, nj=22, nk=12)
    ctx2 = cm1g.Context(other.cfg, other.grid)
    with pytest.raises(cm1g.CM1GError):
        ctx2.restart_read(path, other.copy_state())
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"not a restart file")
    with pytest.raises(cm1g.CM1GError):
        ctx.restart_read(bad, case.copy_state())
    ctx.close()
    ctx2.close()


def test_writeout_grads_files(tmp_path, cm1g):
    """writeout's GrADS files for a Kessler state: each variable's records
    (one per level, i fastest) equal writeout's formula applied to the state
    with numpy; two output times land as consecutive time blocks."""
    torch = _torch()
    case = make_case("kessler", ni=24, nj=20, nk=16)
    lay, gr = case.lay, case.grid
    ctx = cm1g.Context(case.cfg, case.grid)
    dev = cm1g.to_device(case.state)
    for _ in range(2):
        ctx.step(dev, case.dt, case.mass1, use_graph=True)
    prefix = tmp_path / "cm1out"
    ctx.writeout(prefix, 1, dev, mtime=2 * case.dt)
    h1 = cm1g.to_host(dev)
    ctx.step(dev, case.dt, case.mass1, use_graph=True)
    ctx.writeout(prefix, 2, dev, mtime=3 * case.dt)
    h2 = cm1g.to_host(dev)
    I, U, V, W = lay.interior(1), lay.interior(2), lay.interior(3), lay.interior(4)
    f32 = np.float32

    def s_vars(h):
        pi = np.power((h["prs"][I] * f32(1.0 / 1.0e5)).astype(np.float64),
                      float(np.float32(287.04) / np.float32(1005.7))).astype(f32)
        sfc = (slice(lay.jx(1), lay.jx(lay.nj) + 1), slice(lay.ix(1), lay.ix(lay.ni) + 1))
        return [h["rain"][sfc], h["prate"][sfc], gr["th0"][I] + h["tha"][I], h["tha"][I], h["prs"][I],
                h["prs"][I] - gr["prs0"][I], pi, pi - gr["pi0"][I], h["rho"][I], h["rho"][I] - gr["rho0"][I],
                h["qa"][0][I], h["qa"][0][I] - gr["qv0"][I], h["qa"][1][I], h["qa"][2][I]]

    per_s = sum(v.size for v in s_vars(h1))
    s = np.fromfile(str(prefix) + "_s.dat", dtype=f32)
    assert s.size == 2 * per_s
    for t, h in ((0, h1), (1, h2)):
        off = t * per_s
        for n, v in enumerate(s_vars(h)):
            got = s[off:off + v.size].reshape(v.shape)
            if n in (6, 7):    # pi and pipert: binary64 power rounded once on both sides
                assert np.abs(got - v).max() <= 2 * np.spacing(f32(1.0)), n
            else:
                assert np.array_equal(got, v), n
            off += v.size
    u = np.fromfile(str(prefix) + "_u.dat", dtype=f32).reshape(2, 2, -1)
    assert np.array_equal(u[1, 0], h2["ua"][U].ravel()) and np.array_equal(u[1, 1], (h2["ua"][U] - gr["u0"][U]).ravel())
    w = np.fromfile(str(prefix) + "_w.dat", dtype=f32).reshape(2, -1)
    assert np.array_equal(w[0], h1["wa"][W].ravel())
    ctl = open(str(prefix) + "_s.ctl").read()
    assert "vars 14" in ctl and "tdef 2" in ctl and "qc " in ctl
    ctx.close()
