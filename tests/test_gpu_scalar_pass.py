"""The fused scalar pass (k_scal_tile: every field of an RK stage in one
launch, rows staged by bulk copies) against one k_advs_tile launch per field.

Both evaluate every face and update with the same operations, so the large
step must agree bit for bit: on odd grid sizes (partial tiles and level
chunks), with and without WENO, on periodic and open boundaries, moist
with tracers (whose final stage takes the positive-definite per-field path),
for every tile shape, and with state arrays whose base address is not
16-byte aligned (the row copies take aligned supersets of the caller's
rows).  Each case is also checked against the oracle."""
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


def _context(cm1g, case, perfield, monkeypatch):
    if perfield:
        monkeypatch.setenv("CM1G_SCALAR_PASS", "perfield")
    else:
        monkeypatch.delenv("CM1G_SCALAR_PASS", raising=False)
    return cm1g.Context(case.cfg, case.grid)


def _misaligned(torch, arrays, shift):
    """Device copies whose data start `shift` floats past a 256-byte boundary."""
    out = {}
    for k, v in arrays.items():
        buf = torch.zeros(v.size + 64, dtype=torch.float32, device="cuda")
        t = buf[shift:shift + v.size].view(v.shape)
        t.copy_(torch.from_numpy(np.ascontiguousarray(v)))
        out[k] = t
    return out


def _steps(cm1g, torch, case, perfield, monkeypatch, nsteps=2, tune=None, shift=None):
    ctx = _context(cm1g, case, perfield, monkeypatch)
    if tune is not None:
        ctx.set_tune(**tune)
    st = cm1g.to_device(case.state) if shift is None else _misaligned(torch, case.state, shift)
    for _ in range(nsteps):
        ctx.step(st, case.dt, case.mass1, use_graph=True)
    torch.cuda.synchronize()
    out = {k: v.cpu().numpy() for k, v in st.items()}
    ctx.close()
    return out


CASES = {
    "dry_flx5": dict(name="dry_bubble", ni=70, nj=45, nk=37),
    "dry_weno": dict(name="dry_bubble", ni=70, nj=45, nk=37, advwenos=1),
    "dry_weno_final": dict(name="dry_bubble", ni=41, nj=33, nk=21, advwenos=2),
    "moist_open": dict(name="supercell", ni=52, nj=40, nk=30, npt=2),
    "moist_periodic": dict(name="supercell", ni=37, nj=29, nk=24, npt=1, bc=1),
    "cbl": dict(name="cbl", ni=48, nj=40, nk=40),
}


@pytest.mark.parametrize("which", sorted(CASES))
def test_fused_scalar_pass_equals_per_field_launches(cm1g, which, monkeypatch):
    torch = _torch()
    kw = dict(CASES[which])
    case = make_case(kw.pop("name"), **kw)
    ref = _steps(cm1g, torch, case, True, monkeypatch)
    got = _steps(cm1g, torch, case, False, monkeypatch)
    for k in ref:
        assert np.array_equal(got[k], ref[k], equal_nan=True), k


@pytest.mark.parametrize("shape", [1, 2, 3, 4])
def test_fused_scalar_pass_every_tile_shape(cm1g, shape, monkeypatch):
    torch = _torch()
    case = make_case("supercell", ni=45, nj=38, nk=27, npt=1)
    ref = _steps(cm1g, torch, case, True, monkeypatch, tune=dict(adv_shape=shape, mom_shape=0, sound_form=0))
    got = _steps(cm1g, torch, case, False, monkeypatch, tune=dict(adv_shape=shape, mom_shape=0, sound_form=0))
    for k in ref:
        assert np.array_equal(got[k], ref[k], equal_nan=True), k


@pytest.mark.parametrize("shift", [1, 2, 3])
def test_fused_scalar_pass_unaligned_arrays(cm1g, shift, monkeypatch):
    torch = _torch()
    case = make_case("supercell", ni=33, nj=27, nk=22, npt=2)
    ref = _steps(cm1g, torch, case, True, monkeypatch)
    got = _steps(cm1g, torch, case, False, monkeypatch, shift=shift)
    for k in ref:
        assert np.array_equal(got[k], ref[k], equal_nan=True), k


def test_fused_scalar_pass_matches_oracle(cm1g, oracle_lib, monkeypatch):
    """One large step of a moist open-boundary case against the oracle, at
    the 1e-5-of-range bar of the step parity tests."""
    from test_gpu_parity import field_errors, TOL_RANGE
    torch = _torch()
    case = make_case("supercell", ni=40, nj=36, nk=40)
    got = _steps(cm1g, torch, case, False, monkeypatch, nsteps=1)
    ref, _, _ = oracle_lib.step(case)
    errs = field_errors(case, got, ref)
    assert max(errs.values()) <= TOL_RANGE, errs
