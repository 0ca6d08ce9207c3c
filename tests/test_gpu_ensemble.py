"""Ensembles of uneven members (cm1g_ensemble_*): one ensemble step must leave
every member exactly where stepping it alone through cm1g_step leaves it
(same kernels, only run side by side), with and without the captured graph."""
import numpy as np
import pytest

from cm1_b200.cases import make_ensemble

pytestmark = pytest.mark.gpu


def _torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("use_graph", [False, True])
def test_ensemble_matches_members_alone(use_graph, cm1g):
    torch = _torch()
    members = make_ensemble(5, seed=7, sizes=(48, 64, 80), levels=(40, 60))
    ctxs = [cm1g.Context(c.cfg, c.grid) for c in members]
    alone = [cm1g.to_device(c.state) for c in members]
    together = [cm1g.to_device(c.state) for c in members]
    ens = cm1g.Ensemble(ctxs)
    dts = [c.dt for c in members]
    m1 = [c.mass1 for c in members]
    for _ in range(2):
        m2e, cfle = ens.step(together, dts, m1, use_graph=use_graph)
        m2a, cfla = [], []
        for ctx, st, c in zip(ctxs, alone, members):
            a, b = ctx.step(st, c.dt, c.mass1)
            m2a.append(a); cfla.append(b)
        torch.cuda.synchronize()
        assert m2e == m2a and cfle == cfla
        for a, b in zip(alone, together):
            for k in a:
                assert torch.equal(a[k], b[k]), k
    if use_graph:
        assert ens.kernels_per_step() > 40 * len(members)
    ens.close()


def test_ensemble_rejects_host_states(cm1g):
    _torch()
    members = make_ensemble(2, seed=3, sizes=(48,), levels=(40,))
    ctxs = [cm1g.Context(c.cfg, c.grid) for c in members]
    ens = cm1g.Ensemble(ctxs)
    with pytest.raises(cm1g.CM1GError) as ei:
        ens.step([c.state for c in members], [c.dt for c in members], [c.mass1 for c in members])
    assert ei.value.code == -1
    ens.close()
