"""Build a grammar's wire-protocol program on the B200 path.

The program is what alpacc's C emitter would generate for the tables' mode
(combined, lexer-only or parser-only), except that ``run_case`` goes through
the C ABI: the grammar's constants
(emitted as the reference emitter writes them, ``grammar/emit_c.py``), the glue
that fills ``alpacc_tables`` from them (``csrc/wire_glue.h``) and the batch /
server / layout loop (``csrc/wire_main.c``), linked against
``_lib/libalpacc_b200.so``.
"""

from __future__ import annotations

import os
import subprocess

from .build import LIB, LIBDIR, REPO, build_lib
from .grammar import emit_c

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def source(tables) -> str:
    parts = [
        emit_c.constants(tables),
        '#include "wire_glue.h"',
        '#include "wire_main.c"',
    ]
    return "".join(p + "\n" for p in parts)


def build_program(tables, name: str, force: bool = False) -> str:
    build_lib()
    out = os.path.join(LIBDIR, "wire_%s" % name)
    src = os.path.join(LIBDIR, "wire_%s.c" % name)
    stamp = out + ".stamp"
    key = tables.digest()
    deps = [os.path.join(CSRC, "wire_main.c"), os.path.join(CSRC, "wire_glue.h"), LIB]
    if not force and os.path.exists(out) and os.path.exists(stamp) and open(stamp).read() == key and all(
            os.path.getmtime(d) <= os.path.getmtime(out) for d in deps):
        return out
    with open(src, "w") as f:
        f.write(source(tables))
    subprocess.check_call(["gcc", "-std=c99", "-O2", "-D_POSIX_C_SOURCE=200809L", "-I", CSRC, "-I",
                           os.path.join(REPO, "include"), src, "-o", out, "-L", LIBDIR, "-lalpacc_b200",
                           "-Wl,-rpath,$ORIGIN"])
    with open(stamp, "w") as f:
        f.write(key)
    os.remove(src)
    return out
