"""CPU-side checks of the C-ABI: the library loads, exports every entry point
include/cm1g.h declares, and its structs match the ctypes mirror."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cm1g.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(cm1g_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(cm1g):
    lib = C.CDLL(cm1g.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_struct_layout_matches_ctypes(tmp_path):
    from cm1_b200.abi import Config, Grid, State
    prog = tmp_path / "sz.c"
    prog.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "%s"\n'
                    'int main(void){printf("%%zu %%zu %%zu %%zu %%zu\\n", sizeof(cm1g_config_t), '
                    'sizeof(cm1g_grid_t), sizeof(cm1g_state_t), offsetof(cm1g_config_t, qmag), '
                    'offsetof(cm1g_state_t, radbcn));return 0;}\n' % HEADER)
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-o", str(exe), str(prog)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    assert [int(x) for x in out] == [C.sizeof(Config), C.sizeof(Grid), C.sizeof(State),
                                     Config.qmag.offset, State.radbcn.offset]


def test_no_cpu_fallback_without_a_device(cm1g):
    """Without a CUDA device the library refuses to run instead of falling
    back to a CPU path."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from cm1_b200.cases import make_case
    case = make_case("dry_bubble", ni=8, nj=8, nk=8)
    with pytest.raises(cm1g.CM1GError) as ei:
        cm1g.Context(case.cfg, case.grid)
    assert ei.value.code == -2


def test_version(cm1g):
    a, b = C.c_int32(), C.c_int32()
    assert cm1g.lib().cm1g_version(C.byref(a), C.byref(b)) == 0
    assert (a.value, b.value) == (0, 1)


def test_oracle_header_and_threads(oracle_lib):
    assert oracle_lib.threads() >= 1
    assert "parity unpinned" in open(os.path.join(ROOT, "oracle", "cm1_oracle.c")).read().lower()
