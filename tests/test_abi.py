"""The C-ABI library loads, exports every symbol include/rcabf.h declares, and
the ctypes mirror of its structs has the C layout.  No GPU needed: nothing
here launches a kernel."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from simu_rca_ab_b200 import _lib as L
from simu_rca_ab_b200.build import HOST_CXX, INCLUDE, LIB

HEADER = INCLUDE / "rcabf.h"


def header_functions():
    txt = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(rcabf_[a-z0-9_]+)\s*\(", txt)))


def test_library_built_and_loads():
    assert LIB.exists(), "run `python -m simu_rca_ab_b200.build`"
    assert L.lib().rcabf_abi_version() == 1


def test_every_declared_symbol_is_exported_and_bound():
    names = header_functions()
    assert len(names) >= 12
    lib = C.CDLL(str(LIB))
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(L.declared_symbols()) == names


def test_status_strings_carry_reference_identifiers():
    s = L.lib().rcabf_status_string
    assert s(16).decode() == "bfVirtualSourceGeneric_RCA:tiltsNotSameLength"
    assert s(26).decode() == "bfVirtualSourceGeneric_RCA:startTimeInvalid"
    assert s(105).decode() == "rcabf:timeout"


def test_struct_layouts_match_header(tmp_path):
    src = tmp_path / "sz.c"
    fields_g = [f[0] for f in L.GeometryDesc._fields_]
    fields_b = [f[0] for f in L.BeamformArgs._fields_]
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "rcabf.h"', "int main(void){"]
    lines.append('printf("G %zu\\n", sizeof(rcabf_geometry_desc));')
    lines.append('printf("B %zu\\n", sizeof(rcabf_beamform_args));')
    for f in fields_g:
        lines.append(f'printf("g.{f} %zu\\n", offsetof(rcabf_geometry_desc, {f}));')
    for f in fields_b:
        lines.append(f'printf("b.{f} %zu\\n", offsetof(rcabf_beamform_args, {f}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "sz"
    gcc = HOST_CXX.replace("g++", "gcc")
    subprocess.run([gcc, "-I", str(INCLUDE), str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    assert int(out["G"]) == C.sizeof(L.GeometryDesc)
    assert int(out["B"]) == C.sizeof(L.BeamformArgs)
    for f in fields_g:
        assert int(out[f"g.{f}"]) == getattr(L.GeometryDesc, f).offset, f
    for f in fields_b:
        assert int(out[f"b.{f}"]) == getattr(L.BeamformArgs, f).offset, f


def test_null_arguments_are_rejected_without_a_device():
    lib = L.lib()
    assert lib.rcabf_create_geometry(None, None, None) == 100
    n = C.c_size_t()
    assert lib.rcabf_beamform_workspace_size(None, None, C.byref(n)) == 100
    assert lib.rcabf_destroy_geometry(None) == 108
