"""CPU tests of the C ABI boundary: the library loads and exports every declared symbol,
and argument checks fail with status codes before touching any device."""
import ctypes as C
import os
import re

import pytest

from mordred_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mordred_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(mb_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("mb_star_query", "mb_build_pht", "mb_q11_query", "mb_q21_probe", "mb_q41_probe",
                 "mb_join_build", "mb_join_probe", "mb_filter_probe_group_by_GPU2", "mb_build_GPU2"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_functions()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    unbound = [n for n in names if n not in L.SIGNATURES]
    assert not unbound, unbound


def test_library_is_the_in_tree_build():
    assert os.path.dirname(L.lib_path()) == os.path.join(ROOT, "mordred_b200")
    assert os.path.exists(L.lib_path())


def test_argument_errors_return_codes():
    lib = L.lib()
    assert lib.mb_star_query(None, None) == 1  # MB_ERR_ARG
    assert lib.mb_build_pht(None, 0, 0, 0, None, None, 10, None, 10, 0, None, None) == 1
    assert lib.mb_q11_query(None, None, None, None, 10, None, None, None) == 1
    assert lib.mb_join_build(None, None, 1, None, 1, None) == 1
    assert lib.mb_build_GPU2(None, None, None, 1, None, 0, None, None) == 1
    assert lib.mb_gen_fact_column_host(99, 1, 0, 10, 1, 1, 1, None, 1) == 1
    assert lib.mb_error_string(1).decode() == "invalid argument"
    assert lib.mb_version() >= 1


def test_struct_layouts_match_c_abi():
    # sizes computed from the C declarations on x86-64 (LP64)
    assert C.sizeof(L.MbFilter) == 24
    assert C.sizeof(L.MbProbe) == 48
    assert C.sizeof(L.MbFilterArgsGPU) == 40
    assert C.sizeof(L.MbProbeArgsGPU) == 96
    assert C.sizeof(L.MbGroupbyArgsGPU) == 88
    assert C.sizeof(L.MbBuildArgsGPU) == 32


def test_struct_sizes_agree_with_compiler(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include "mordred_b200.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(){printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(mb_filter), sizeof(mb_probe),'
                   'sizeof(mb_star_args), sizeof(mb_filterArgsGPU), sizeof(mb_probeArgsGPU),'
                   'sizeof(mb_groupbyArgsGPU), offsetof(mb_star_args, grid));return 0;}\n')
    exe = tmp_path / "sz"
    import subprocess
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert out == [C.sizeof(L.MbFilter), C.sizeof(L.MbProbe), C.sizeof(L.MbStarArgs), C.sizeof(L.MbFilterArgsGPU),
                   C.sizeof(L.MbProbeArgsGPU), C.sizeof(L.MbGroupbyArgsGPU), L.MbStarArgs.grid.offset]


def test_no_device_reports_error_not_crash():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert L.lib().mb_init(0) != 0
