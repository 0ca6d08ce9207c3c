"""Launch shapes and the autotuner (cm1g_set_tune / cm1g_autotune).

The tile shapes of the scalar and momentum passes and the two tile forms
(or two column forms) of the acoustic kernel change only which thread
computes which cell, so every choice must give the default step bit for
bit.  The tile and column-sweep forms of the acoustic kernel order the
tridiagonal elimination differently and agree to rounding.  The autotuner
must leave the caller's state unchanged, pick valid shapes and reuse
cached results."""
import os

import numpy as np
import pytest

from cm1_b200.cases import make_case

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _one_step(cm1g, case, tune):
    ctx = cm1g.Context(case.cfg, case.grid)
    if tune is not None:
        ctx.set_tune(**tune)
    st = cm1g.to_device(case.state)
    ctx.step(st, case.dt, case.mass1, use_graph=True)
    ctx.step(st, case.dt, case.mass1, use_graph=True)
    out = {k: v.cpu().numpy() for k, v in st.items()}
    ctx.close()
    return out


CASES = {
    # odd sizes: partial tiles in x, y and in the level chunks
    "dry": dict(name="dry_bubble", ni=70, nj=45, nk=37),
    # moisture with the positive-definite two-pass scalar form and a tracer
    "moist": dict(name="supercell", ni=52, nj=40, nk=30, npt=1),
}


@pytest.mark.parametrize("which", sorted(CASES))
def test_every_launch_shape_gives_the_same_step(cm1g, which):
    _torch()
    kw = dict(CASES[which])
    case = make_case(kw.pop("name"), **kw)
    base = _one_step(cm1g, case, dict(adv_shape=0, mom_shape=0, sound_form=0))
    shapes = cm1g.tile_shapes()
    assert len(shapes) >= 2 and shapes[0] == (32, 8, 16)
    variants = [dict(adv_shape=a, mom_shape=0, sound_form=0) for a in range(1, len(shapes))]
    variants += [dict(adv_shape=0, mom_shape=m, sound_form=0) for m in range(1, len(shapes))]
    variants += [dict(adv_shape=len(shapes) - 1, mom_shape=len(shapes) - 1, sound_form=1)]
    for v in variants:
        got = _one_step(cm1g, case, v)
        for k in base:
            assert np.array_equal(got[k], base[k]), (v, k)
    # the two column-sweep forms agree with each other bit for bit, and
    # with the tile form to rounding
    col4 = _one_step(cm1g, case, dict(adv_shape=0, mom_shape=0, sound_form=2))
    col2 = _one_step(cm1g, case, dict(adv_shape=2, mom_shape=3, sound_form=3))
    for k in base:
        assert np.array_equal(col4[k], col2[k]), k
        if base[k].size == 0:
            continue
        b = base[k].astype(np.float64)
        rng = float(b.max() - b.min()) or 1.0
        assert np.abs(col4[k] - b).max() <= 1e-5 * rng, k


def test_set_tune_rejects_bad_shapes(cm1g):
    _torch()
    case = make_case("dry_bubble", ni=24, nj=20, nk=16)
    ctx = cm1g.Context(case.cfg, case.grid)
    n = len(cm1g.tile_shapes())
    for bad in (dict(adv_shape=n), dict(mom_shape=-1), dict(sound_form=4), dict(sound_form=-2)):
        with pytest.raises(cm1g.CM1GError):
            ctx.set_tune(**bad)
    assert ctx.get_tune()["sound_form"] == -1


def test_autotune_keeps_state_and_caches(cm1g, tmp_path):
    torch = _torch()
    case = make_case("dry_bubble", ni=96, nj=80, nk=40)
    ctx = cm1g.Context(case.cfg, case.grid)
    st = cm1g.to_device(case.state)
    before = {k: v.clone() for k, v in st.items()}
    cache = str(tmp_path / "tune.txt")
    t = ctx.autotune(st, case.dt, case.mass1, reps=2, cache=cache)
    torch.cuda.synchronize()
    for k in st:
        assert torch.equal(st[k], before[k]), k
    n = len(cm1g.tile_shapes())
    assert 0 <= t["adv_shape"] < n and 0 <= t["mom_shape"] < n and 0 <= t["sound_form"] < 4
    assert t["step_ms"] > 0
    assert ctx.get_tune() == t
    lines = open(cache).read().split("\n")
    assert any(l.split()[1:4] == [str(t["adv_shape"]), str(t["mom_shape"]), str(t["sound_form"])]
               for l in lines if l.strip())
    # a second context of the same grid takes the cached choice
    ctx2 = cm1g.Context(case.cfg, case.grid)
    assert ctx2.autotune(st, case.dt, case.mass1, reps=2, cache=cache) == t
    # the tuned step equals the default step
    a = cm1g.to_device(case.state)
    b = cm1g.to_device(case.state)
    ctx.step(a, case.dt, case.mass1, use_graph=True)
    ctx3 = cm1g.Context(case.cfg, case.grid)
    ctx3.set_tune(adv_shape=0, mom_shape=0, sound_form=t["sound_form"])
    ctx3.step(b, case.dt, case.mass1, use_graph=True)
    torch.cuda.synchronize()
    for k in a:
        assert torch.equal(a[k], b[k]), k
    for c in (ctx, ctx2, ctx3):
        c.close()
