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


# Argument lists of the reference routines the per-routine entry points
# replace, as declared (src/adv.F:14-19, 911-912, 1847-1848, 2778-2781;
# src/sound.F:10-24; src/misclibs.F:1037).
REFERENCE_ARGS = {
    "advs": "nrk,wflag,bflag,bsq,xh,rxh,arh1,arh2,uh,ruh,xf,vh,rvh,gz,rgz,mh,rmh,rho0,rr0,rf0,rrf0,advx,advy,"
            "advz,dumx,dumy,dumz,mass,subs,divx,rru,rrv,rrw,s0,s,sten,pdef,pdefweno,dt,weps,flag,sw31,sw32,se31,"
            "se32,ss31,ss32,sn31,sn32,rdsf,c1,c2,rho,ri,diffit,dobud,ibd,ied,jbd,jed,kbd,ked,ndiag,diag,sd_hadv,"
            "sd_vadv,sd_lsw,sd_hidiff,sd_vidiff,sd_hediff,wprof,dumk1,dumk2,hadvorder,vadvorder,kbdy,bndy,hflxw,"
            "hflxe,hflxs,hflxn,out3d",
    "advu": "nrk,arh1,arh2,uh,xf,rxf,arf1,arf2,uf,vh,gz,rgz,gzu,mh,rho0,rr0,rf0,rrf0,dumx,dumy,dumz,advx,advy,"
            "advz,subs,divx,rru,u3d,uten,rrv,rrw,rdsf,c1,c2,rho,dt,doubud,udiag,wprof,bndy,kbdy,hflxw,hflxe,hflxs,"
            "hflxn,vf,mf,v3d,w3d",
    "advv": "nrk,xh,rxh,arh1,arh2,uh,xf,vh,vf,gz,rgz,gzv,mh,rho0,rr0,rf0,rrf0,dumx,dumy,dumz,advx,advy,advz,subs,"
            "divx,rru,rrv,v3d,vten,rrw,rdsf,c1,c2,rho,dt,dovbud,vdiag,wprof,bndy,kbdy,hflxw,hflxe,hflxs,hflxn,uf,"
            "mf,u3d,w3d",
    "advw": "nrk,xh,rxh,arh1,arh2,uh,xf,vh,gz,rgz,mh,mf,rho0,rr0,rf0,rrf0,dumx,dumy,dumz,advx,advy,advz,subs,"
            "divx,rru,rrv,rrw,w3d,wten,rds,rdsf,c1,c2,rho,dt,dowbud,wdiag,hadvorder,vadvorder,advweno,bndy,kbdy,uf,"
            "vf,u3d,v3d,hflxw,hflxe,hflxs,hflxn,iamw",
    "sound": "dt,xh,arh1,arh2,uh,ruh,xf,uf,yh,vh,rvh,yf,vf,rds,sigma,rdsf,sigmaf,zh,mh,rmh,c1,c2,mf,zf,pi0,rho0,"
             "rr0,rf0,rrf0,th0,rth0,zs,gz,rgz,gzu,rgzu,gzv,rgzv,dzdx,dzdy,gx,gxu,gy,gyv,radbcw,radbce,radbcs,"
             "radbcn,dtu,dtu0,dtv,dtv0,dum1,dum2,dum3,dum4,mm,bk,ppd,fpk,qk,pk1,pk2,wtens,u0,rru,ua,u3d,uten,v0,"
             "rrv,va,v3d,vten,rrw,wa,w3d,wten,ppi,pp3d,piadv,ppten,ppx,thv,ppterm,nrk,dttmp,rtime,mtime,"
             "get_time_avg,bndy,kbdy,pw1,pw2,pe1,pe2,ps1,ps2,pn1,pn2,reqs_p",
    "pdefq": "rmax,asq,ruh,rvh,rmh,rho,q3d",
}
# C entry point -> the reference routine whose argument order it keeps
ENTRY_ROUTINE = {"cm1g_advs": "advs", "cm1g_advu": "advu", "cm1g_advv": "advv", "cm1g_advw": "advw",
                 "cm1g_sound": "sound", "cm1g_pdefq": "pdefq", "cm1g_pdefq_noalloc": "pdefq"}
# arguments of the C entries that carry no reference argument
NOT_REFERENCE = {"ctx", "cfg", "stream"}


def c_arguments(name):
    src = re.sub(r"/\*.*?\*/", " ", open(HEADER).read(), flags=re.S)
    m = re.search(r"\bint\s+%s\s*\(([^;]*?)\)\s*;" % name, src, flags=re.S)
    assert m, name
    out = []
    for a in m.group(1).split(","):
        out.append(re.findall(r"[A-Za-z_][A-Za-z0-9_]*", a.split("[")[0])[-1])
    return out


def fortran_arguments(name):
    src = open(os.path.join(ROOT, "cm1_b200", "fortran", "cm1g_iso.F90")).read().replace("&\n", " ")
    m = re.search(r"function\s+%s\s*\(([^)]*)\)" % name, src)
    assert m, name
    return [a.strip() for a in m.group(1).split(",")]


@pytest.mark.parametrize("entry", sorted(ENTRY_ROUTINE))
def test_entry_keeps_reference_argument_order(entry):
    """Every argument an entry point shares with its reference routine is a
    reference argument, and they come in the reference's order."""
    ref = REFERENCE_ARGS[ENTRY_ROUTINE[entry]].split(",")
    kept = [a for a in c_arguments(entry) if a not in NOT_REFERENCE]
    assert kept, entry
    missing = [a for a in kept if a not in ref]
    assert not missing, (entry, missing)
    pos = [ref.index(a) for a in kept]
    assert pos == sorted(pos), (entry, kept)


@pytest.mark.parametrize("entry", ["cm1g_advs", "cm1g_advu", "cm1g_advv", "cm1g_advw", "cm1g_sound",
                                   "cm1g_pdefq"])
def test_fortran_interface_matches_header(entry):
    """The ISO_C_BINDING interface lists the C arguments in the same order."""
    assert fortran_arguments(entry) == c_arguments(entry)


def test_oracle_header_and_threads(oracle_lib):
    assert oracle_lib.threads() >= 1
    assert "parity unpinned" in open(os.path.join(ROOT, "oracle", "cm1_oracle.c")).read().lower()


@pytest.mark.parametrize("field,value,code", [
    ("roflux", 2, -1),                 # roflux is 0 or 1
    ("irbc", 3, -5),                   # open boundaries with phase speeds 1, 2 or 4 only
    ("nk", 70000, -5),                 # levels index a launch grid's y or z extent
    ("ni", 20000, -5),                 # with nj = 20000: arrays of 2^31 points or more
])
def test_config_limits_are_refused_before_any_device_work(field, value, code, cm1g):
    """cm1g_init checks the configuration before it looks for a device, so
    these refusals hold on a host without a GPU too."""
    from cm1_b200.cases import make_case
    case = make_case("supercell", ni=16, nj=16, nk=12)
    setattr(case.cfg, field, value)
    if field == "ni":
        case.cfg.nj = 20000
    with pytest.raises(cm1g.CM1GError) as ei:
        cm1g.Context(case.cfg, case.grid)
    assert ei.value.code == code, (field, ei.value.code, str(ei.value))


def test_tile_shape_tables(cm1g):
    """The autotuner's two tables: the momentum tiles (threads of a block)
    and the scalar tiles (cells of a tile, one thread row more per block),
    indexed alike; both end with CM1G_ERR_ARG."""
    mom, scal = cm1g.tile_shapes(), cm1g.tile_shapes(scalar=True)
    assert len(mom) == len(scal) == 5
    assert mom[0] == (32, 8, 16) and scal[0] == (32, 7, 16)
    for m, s in zip(mom, scal):
        assert s[0] == m[0] and s[1] + 1 == m[1] and s[2] == m[2]


def test_c_program_links_and_calls_the_library(tmp_path, cm1g):
    """A C caller (the form a Fortran or C host binds) compiled against
    include/cm1g.h and linked with libcm1g.so: the host-side entry points
    answer, and a configuration the library refuses returns its error code
    and message through the C-ABI."""
    prog = tmp_path / "drv.c"
    prog.write_text(r'''
#include <stdio.h>
#include <string.h>
#include "%s"
int main(void) {
  int32_t ma = 0, mi = 0, sh[3] = {0, 0, 0}, ns = 0;
  float dts = 0.0f; double dd = 0.0;
  if (cm1g_version(&ma, &mi) != CM1G_OK) return 1;
  if (cm1g_scal_tile_shape(0, sh) != CM1G_OK || sh[0] != 32 || sh[1] != 7) return 2;
  if (cm1g_tile_shape(99, sh) != CM1G_ERR_ARG) return 3;
  dts = 3.0f;
  if (cm1g_dtsmall(3, 256, 256, 500.0f, 500.0f, 250.0f, 0, &dts, &dd, &ns) != CM1G_OK) return 4;
  cm1g_config_t cfg; memset(&cfg, 0, sizeof cfg);
  cfg.ni = 16; cfg.nj = 16; cfg.nk = 12; cfg.ngxy = 3; cfg.psolver = 2;   /* sound.F's solver is 3 */
  cm1g_grid_t gr; memset(&gr, 0, sizeof gr);
  cm1g_ctx_t *ctx = NULL;
  int rc = cm1g_init(&cfg, &gr, &ctx);
  printf("%%d.%%d %%d %%d %%s\n", ma, mi, ns, rc, cm1g_last_error());
  return rc == CM1G_ERR_UNSUPPORTED && ctx == NULL ? 0 : 5;
}
''' % HEADER)
    exe = tmp_path / "drv"
    libdir = os.path.dirname(cm1g.LIB_PATH)
    subprocess.run(["gcc", "-o", str(exe), str(prog), "-L" + libdir, "-lcm1g", "-Wl,-rpath," + libdir], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    ver, nsound, rc = r.stdout.split()[:3]
    assert int(nsound) >= 2 and int(rc) == -5 and "psolver=2" in r.stdout
