"""The boundary's struct layouts agree across C, ctypes and Fortran.

A C program compiled with gcc against include/ddcosmo_gpu.h prints sizeof and
offsetof of ddc_params, ddc_solve_info and ddc_run_info and the defaults that
ddc_default_params writes through the linked library; the test compares them
with the ctypes mirrors in ddpcm_b200/ddcosmo.py.  The Fortran module's
bind(c) types (ddpcm_b200/fortran/ddcosmo_gpu.f90) are read as text and their
field order and kinds compared with the same structs (no Fortran compiler is
available to compile them).  No GPU is needed.
"""
import ctypes
import json
import os
import re
import shutil
import subprocess

import pytest

from conftest import ROOT

STRUCTS = {
    "ddc_params": ["lmax", "ngrid", "iconv", "igrad", "eps", "eta", "iprint", "max_iter",
                   "ndiis", "precision", "guess", "device", "device_pointers", "stream",
                   "timing", "pair_solves"],
    "ddc_solve_info": ["iterations", "converged", "diis_restarts", "refinements", "final_norm",
                       "seconds", "norms"],
    "ddc_run_info": ["direct", "adjoint", "t_init", "t_mkrhs", "t_direct", "t_adjoint",
                     "t_forces", "t_efld", "nsph", "ncav", "nylm", "ngrid", "ntriples",
                     "npairs"],
}


def _c_program():
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "ddcosmo_gpu.h"',
             "int main(void) {", "  ddc_params p;", "  int rc = ddc_default_params(&p);",
             '  printf("{\\"rc\\": %d, ", rc);',
             '  printf("\\"defaults\\": [%d, %d, %d, %d, %.17g, %.17g, %d, %d, %d, %d, %d, %d, '
             '%d, %d, %d], ", p.lmax, p.ngrid, p.iconv, p.igrad, p.eps, p.eta, p.iprint, '
             'p.max_iter, p.ndiis, p.precision, p.guess, p.device, p.device_pointers, '
             'p.timing, p.pair_solves);']
    for s, fields in STRUCTS.items():
        lines.append(f'  printf("\\"{s}\\": {{\\"size\\": %zu", sizeof({s}));')
        for f in fields:
            lines.append(f'  printf(", \\"{f}\\": %zu", offsetof({s}, {f}));')
        lines.append('  printf("}, ");')
    lines += ['  printf("\\"end\\": 0}\\n");', "  return 0;", "}"]
    return "\n".join(lines) + "\n"


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    from ddpcm_b200.build import build
    lib = build()
    d = tmp_path_factory.mktemp("abi")
    src = d / "layout.c"
    src.write_text(_c_program())
    exe = d / "layout"
    libdir = os.path.dirname(lib)
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", libdir, "-lddcosmo_gpu",
                    "-Wl,-rpath," + libdir], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return json.loads(out)


def test_c_struct_layout_matches_ctypes(c_layout):
    from ddpcm_b200.ddcosmo import Params, RunInfo, SolveInfo
    assert c_layout["rc"] == 0
    for name, cls in (("ddc_params", Params), ("ddc_solve_info", SolveInfo),
                      ("ddc_run_info", RunInfo)):
        got = c_layout[name]
        assert [f for f, _ in cls._fields_] == STRUCTS[name]
        assert got["size"] == ctypes.sizeof(cls), name
        for f in STRUCTS[name]:
            assert got[f] == getattr(cls, f).offset, (name, f)


def test_defaults_seen_from_c_match_ctypes(c_layout):
    from ddpcm_b200.ddcosmo import Params, load_library
    p = Params()
    assert load_library().ddc_default_params(ctypes.byref(p)) == 0
    want = [p.lmax, p.ngrid, p.iconv, p.igrad, p.eps, p.eta, p.iprint, p.max_iter, p.ndiis,
            p.precision, p.guess, p.device, p.device_pointers, p.timing, p.pair_solves]
    assert c_layout["defaults"] == want


def _fortran_types():
    src = open(os.path.join(ROOT, "ddpcm_b200", "fortran", "ddcosmo_gpu.f90")).read()
    types = {}
    for m in re.finditer(r"type, bind\(c\) :: (\w+)\n(.*?)\n\s*end type", src, re.S):
        fields = []
        for line in m.group(2).splitlines():
            kind, names = line.split("::")
            for nm in names.split(","):
                nm = nm.strip()
                dim = re.match(r"(\w+)\((\d+)\)", nm)
                fields.append((dim.group(1) if dim else nm, kind.strip(),
                               int(dim.group(2)) if dim else 1))
        types[m.group(1)] = fields
    return types


def test_fortran_bind_c_types_match_the_c_structs():
    from ddpcm_b200.ddcosmo import Params, SolveInfo
    kinds = {ctypes.c_int: "integer(c_int)", ctypes.c_double: "real(c_double)",
             ctypes.c_void_p: "type(c_ptr)"}
    ft = _fortran_types()
    for name, cls in (("ddc_params", Params), ("ddc_solve_info", SolveInfo)):
        want = []
        for f, t in cls._fields_:
            n = getattr(t, "_length_", 1)
            base = getattr(t, "_type_", t) if n > 1 else t
            want.append((f, kinds[base], n))
        assert ft[name] == want, name
