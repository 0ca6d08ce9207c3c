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
