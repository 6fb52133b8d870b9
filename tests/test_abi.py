"""The C ABI library (no GPU needed): builds for sm_100a, loads, exports every
entry point include/diva.h declares, and its struct layouts match the ctypes
mirror.  No compute call is made here."""
import ctypes as C
import os
import re
import subprocess

import pytest

from imau_ice_b200 import _abi, build, diva

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"^\s*(?:int|int32_t|void|int64_t|const char\*)\s+(diva_\w+)\s*\(", src,
                                flags=re.M))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    path = build.build()
    return C.CDLL(path)


def test_library_exports_every_declared_entry_point(lib):
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_only_the_c_abi_is_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", build.LIB], capture_output=True, text=True, check=True).stdout
    syms = [l.split()[-1] for l in out.splitlines() if " T " in l]
    assert syms and all(s.startswith("diva_") for s in syms), [s for s in syms if not s.startswith("diva_")]


def test_struct_layout_matches_ctypes(tmp_path):
    prog = tmp_path / "layout.c"
    prog.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "diva.h"
#include "diva_cnn.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(diva_grid_t), sizeof(diva_config_t), sizeof(diva_report_t), sizeof(diva_fields_t));
  printf("%zu %zu %zu %zu\n", offsetof(diva_config_t, lin_rtol), offsetof(diva_config_t, precision),
         offsetof(diva_config_t, prescribed_tauc), offsetof(diva_report_t, elapsed_ms));
  printf("%d\n", (int)DIVA_NUM_FIELDS);
  printf("%zu %zu %zu\n", offsetof(diva_config_t, calving_threshold_thickness),
         offsetof(diva_config_t, continental_shelf_min_height), offsetof(diva_config_t, reserved));
  return 0;
}
''')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    a, b, n, tail = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")[:4]
    sizes = [int(x) for x in a.split()]
    offs = [int(x) for x in b.split()]
    assert sizes[:3] == [C.sizeof(_abi.Grid), C.sizeof(_abi.Config), C.sizeof(_abi.Report)]
    assert offs == [_abi.Config.lin_rtol.offset, _abi.Config.precision.offset, _abi.Config.prescribed_tauc.offset,
                    _abi.Report.elapsed_ms.offset]
    assert [int(x) for x in tail.split()] == [_abi.Config.calving_threshold_thickness.offset,
                                              _abi.Config.continental_shelf_min_height.offset,
                                              _abi.Config.reserved.offset]
    assert sizes[3] == int(n) * C.sizeof(C.c_void_p)


def test_field_table_and_defaults_host_only():
    b = diva.cuda_backend()
    fields = b.fields()
    names = [f[0] for f in fields]
    header = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "diva_fields.h")).read(), flags=re.S)
    assert names == re.findall(r"X\((?:\w+),\s*(\w+),", header)
    assert ("u_vav_cx", "CX", "f8") in fields and ("mask_ice_a", "A", "i4") in fields
    cfg = b.default_config()
    # configuration_module.f90:271-302 defaults
    assert cfg.choice_ice_dynamics == _abi.DYN["DIVA"] and cfg.n_flow == 3.0
    assert cfg.DIVA_visc_it_relax == 0.4 and cfg.DIVA_visc_eff_min == 1e3 and cfg.DIVA_vel_max == 5000.0
    assert cfg.DIVA_epsilon_sq_0 == 1e-15 and cfg.DIVA_beta_max == 1e20 and cfg.DIVA_visc_it_nit == 50
    o = __import__("oracle_backend").oracle_backend().default_config()
    for k, _ in _abi.Config._fields_:
        if k != "reserved" and k not in ("lin_maxit",):
            assert getattr(o, k) == getattr(cfg, k), k


def test_no_cpu_fallback_without_gpu():
    """Creating a context on a machine without a GPU fails loudly, it never falls back."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    g = diva.Grid(9, 9, 1e3)
    with pytest.raises(diva.DivaError) as e:
        diva.Context(g, {})
    assert e.value.status == _abi.CUDA_ERROR
