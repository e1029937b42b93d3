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
    assert L.lib().rcabf_abi_version() == 2


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
    structs = {"g": (L.GeometryDesc, "rcabf_geometry_desc"), "b": (L.BeamformArgs, "rcabf_beamform_args"),
               "c": (L.ServerConfig, "rcabf_server_config"), "s": (L.ServerStats, "rcabf_server_stats"),
               "t": (L.TuneResult, "rcabf_tune_result"), "u": (L.UlmBins, "rcabf_ulm_bins")}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "rcabf.h"', "int main(void){"]
    for tag, (py, cname) in structs.items():
        lines.append(f'printf("{tag} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{tag}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "sz"
    gcc = HOST_CXX.replace("g++", "gcc")
    subprocess.run([gcc, "-I", str(INCLUDE), str(src), "-o", str(exe)], check=True)
    out = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for tag, (py, cname) in structs.items():
        assert int(out[tag]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(out[f"{tag}.{f}"]) == getattr(py, f).offset, (cname, f)


def test_null_arguments_are_rejected_without_a_device():
    lib = L.lib()
    assert lib.rcabf_create_geometry(None, None, None) == 100
    n = C.c_size_t()
    assert lib.rcabf_beamform_workspace_size(None, None, C.byref(n)) == 100
    assert lib.rcabf_destroy_geometry(None) == 108


def test_server_argument_checks_need_no_device():
    lib = L.lib()
    cfg = L.ServerConfig()
    cfg.struct_size = C.sizeof(L.ServerConfig)
    cfg.hbm_budget_bytes = 1 << 20
    cfg.n_streams, cfg.max_queue, cfg.max_batch = 0, 4, 4      # no launch slot
    h = C.c_void_p()
    assert lib.rcabf_server_create(C.byref(cfg), C.byref(h)) == 100
    cfg.n_streams, cfg.max_batch = 2, 25                      # more jobs than one launch holds
    assert lib.rcabf_server_create(C.byref(cfg), C.byref(h)) == 100
    cfg.struct_size = 8
    assert lib.rcabf_server_create(C.byref(cfg), C.byref(h)) == 100
    t = C.c_uint64()
    st = C.c_int()
    assert lib.rcabf_server_submit(None, None, None, C.byref(t)) == 108
    assert lib.rcabf_server_poll(None, 1, C.byref(st)) == 108
    assert lib.rcabf_server_wait_for(None, 1, 0.0, C.byref(st)) == 108
    assert lib.rcabf_server_destroy(None) == 108


def test_host_pipeline_argument_checks_need_no_device():
    lib = L.lib()
    n = C.c_size_t()
    assert lib.rcabf_beamform_host_workspace_size(None, None, 0, C.byref(n)) == 108
    assert lib.rcabf_beamform_host(None, None, 0, None) == 108


def test_ulm_argument_checks_need_no_device():
    lib = L.lib()
    assert lib.rcabf_ulm_psf_corr(None, None, None, 1.0, 8, 8, 2, 3, 3, None) == 100
    assert lib.rcabf_ulm_ensemble(None, None, None, 5, 8, 8, 2, None) == 100
    n = C.c_uint64()
    assert lib.rcabf_ulm_detect(None, None, C.byref(n), None, None, 8, 8, 2, 3, 0, 0, None) == 100
    assert lib.rcabf_ulm_gauss_fit(None, None, None, 1, None, 8, 8, 2, 3, None, None) == 100
    b = L.UlmBins()
    b.struct_size = 8                                          # wrong size
    assert lib.rcabf_ulm_density(None, None, None, 0, None, C.byref(b), 0, None) == 100
    b.struct_size = C.sizeof(L.UlmBins)
    b.pos_rows = 5
    for k in range(3):
        b.n[k], b.step[k] = 4, 1.0
    assert lib.rcabf_ulm_density(C.c_void_p(1), None, None, 0, None, C.byref(b), 0, None) == 0   # nothing to bin
    b.step[1] = 0.0
    assert lib.rcabf_ulm_density(C.c_void_p(1), None, None, 0, None, C.byref(b), 0, None) == 101

