"""ctypes access to the C restatement oracle (oracle/oracle.c).

TEST INFRASTRUCTURE ONLY. ``PortOracle(tables).run_case(data)`` returns the
response record the reference's run_case writes, computed by the sequential
restatement with the tables passed at run time.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
SRC = os.path.join(HERE, "oracle.c")
SO = os.path.join(HERE, "_port", "liboracle_port.so")


def build(force: bool = False) -> str:
    os.makedirs(os.path.dirname(SO), exist_ok=True)
    hdr = os.path.join(REPO, "include", "alpacc_b200.h")
    if force or not os.path.exists(SO) or os.path.getmtime(SO) < max(os.path.getmtime(SRC), os.path.getmtime(hdr)):
        subprocess.check_call(["gcc", "-O2", "-std=c99", "-shared", "-fPIC", SRC, "-o", SO])
    return SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(SO)
        L.oracle_run_case.restype = ctypes.c_int
        L.oracle_run_case.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_char_p,
                                      ctypes.POINTER(ctypes.POINTER(ctypes.c_uint8)), ctypes.POINTER(ctypes.c_size_t)]
        L.oracle_free.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


class PortOracle:
    def __init__(self, tables):
        from alpacc_b200.native import make_tables

        self.struct, self._keep = make_tables(tables)

    def run_case(self, data: bytes) -> bytes:
        out = ctypes.POINTER(ctypes.c_uint8)()
        n = ctypes.c_size_t()
        # the parser-mode program's input is counted in terminal ids
        count = len(data) // self.struct.terminal_size if self.struct.parts == 2 else len(data)
        lib().oracle_run_case(ctypes.addressof(self.struct), count, data, ctypes.byref(out), ctypes.byref(n))
        try:
            return ctypes.string_at(out, n.value)
        finally:
            lib().oracle_free(out)
