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
                           "-Wl,-rpath,$ORIGIN:" + LIBDIR])
    with open(stamp, "w") as f:
        f.write(key)
    os.remove(src)
    return out


def main(argv=None) -> int:
    """``python -m alpacc_b200.wire_program grammar.alp [--lexer|--parser]
    [--index32] [-o program]``: the counterpart of ``alpacc c grammar.alp``
    followed by ``cc`` (tests/testc.sh:89-95 of the reference), building the
    wire-protocol program of that mode on the B200 path."""
    import argparse
    import shutil

    from .grammar.cache import load_tables

    ap = argparse.ArgumentParser(prog="python -m alpacc_b200.wire_program")
    ap.add_argument("grammar")
    mode = ap.add_mutually_exclusive_group()
    mode.add_argument("--lexer", action="store_true", help="lexer-only program")
    mode.add_argument("--parser", action="store_true", help="parser-only program")
    ap.add_argument("--index32", action="store_true", help="32-bit index_t")
    ap.add_argument("-o", "--output", help="path of the program (default: the grammar's name)")
    a = ap.parse_args(argv)
    parts = "lexer" if a.lexer else "parser" if a.parser else "both"
    t = load_tables(a.grammar, index32=a.index32, parts=parts)
    name = "%s_%s%s" % (t.name, "i32" if a.index32 else "i64", "" if parts == "both" else "_" + parts)
    exe = build_program(t, name)
    out = a.output or os.path.splitext(os.path.basename(a.grammar))[0]
    shutil.copy2(exe, out)
    print(out)
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())
