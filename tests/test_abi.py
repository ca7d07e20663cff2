"""The C-ABI library loads and exports every entry point include/*.h declares;
struct layouts agree between C and the Python binding. No GPU needed."""

import ctypes
import glob
import os
import re
import subprocess

import pytest

from alpacc_b200 import native

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(REPO, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(alpacc_\w+)\s*\(", src, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("alpacc_gpu_load", "alpacc_gpu_free", "alpacc_gpu_parse", "alpacc_gpu_parse_device",
                 "alpacc_gpu_parse_batch", "alpacc_gpu_run_case", "alpacc_gpu_layout", "alpacc_result_free",
                 "alpacc_strerror"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = native.lib()
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing


def test_struct_layout_matches_c(tmp_path):
    src = tmp_path / "layout.c"
    fields = [f[0] for f in native.Tables._fields_]
    rfields = [f[0] for f in native.Result._fields_]
    body = ['#include <stdio.h>', '#include <stddef.h>', '#include "alpacc_b200.h"', "int main(void){",
            'printf("%zu\\n", sizeof(alpacc_tables));', 'printf("%zu\\n", sizeof(alpacc_result));']
    body += ['printf("%%zu\\n", offsetof(alpacc_tables, %s));' % f for f in fields]
    body += ['printf("%%zu\\n", offsetof(alpacc_result, %s));' % f for f in rfields]
    body.append("return 0;}")
    src.write_text("\n".join(body))
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)])
    vals = [int(x) for x in subprocess.check_output([str(exe)]).split()]
    assert vals[0] == ctypes.sizeof(native.Tables)
    assert vals[1] == ctypes.sizeof(native.Result)
    offs = vals[2:2 + len(fields)]
    assert offs == [getattr(native.Tables, f).offset for f in fields]
    roffs = vals[2 + len(fields):]
    assert roffs == [getattr(native.Result, f).offset for f in rfields]


def test_strerror_and_invalid_tables_without_gpu():
    lib = native.lib()
    assert lib.alpacc_strerror(native.REJECT) == b"input rejected"
    assert lib.alpacc_strerror(native.E_TIMEOUT) == b"device wait timed out"
    bad = native.Tables()
    bad.abi_version = 999
    err = ctypes.c_int(0)
    h = lib.alpacc_gpu_load(ctypes.byref(bad), 0, 0, ctypes.byref(err))
    assert not h and err.value == native.E_INVALID


def test_parts_validation_without_gpu():
    """Tables of a lexer-mode or parser-mode program are checked for the part
    they carry before any device work; an unknown parts value is refused."""
    lib = native.lib()
    err = ctypes.c_int(0)
    for parts in (native.PARTS["lexer"], native.PARTS["parser"], 7):
        t = native.Tables()
        t.abi_version = native.ABI_VERSION
        t.terminal_size, t.index_size, t.length_size = 1, 4, 4
        t.state_size, t.production_size, t.bracket_size = 2, 1, 1
        t.parts = parts  # no tables attached
        h = lib.alpacc_gpu_load(ctypes.byref(t), 0, 0, ctypes.byref(err))
        assert not h and err.value == native.E_INVALID
