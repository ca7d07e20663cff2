"""Build recipe for ``oracle/_ref``: the reference's own C backend, compiled here.

TEST INFRASTRUCTURE ONLY. This script assembles the program that alpacc's C
emitter would generate for a grammar (src/Alpacc/Generator/C/Generator.hs:161-201,
``Both`` mode) from

* the constant sections produced by ``alpacc_b200.grammar`` (the restated
  generator; see ``alpacc_b200/grammar/emit_c.py``), and
* the reference's runtime templates, read where they lie:
  ``backends/c/lexer.c``, ``backends/c/parser.c``, ``backends/c/cli.c``, and the
  ``run_case`` text of ``bothTestCase`` (C/Generator.hs:114-159), extracted from
  the Haskell string list at build time,

then compiles it with ``cc -std=c99 -O2`` (as tests/test-long-input.sh:72 does)
into ``oracle/_ref/<config>`` (the wire-protocol CLI) and, together with
``oracle/ref_harness.c``, into ``oracle/_ref/lib<config>.so`` for in-memory calls.

The lexer-mode and parser-mode programs (C/Generator.hs:161-186) are assembled
the same way from ``lexerTestCase`` / ``parserTestCase`` with only the lexer's
(``backends/c/lexer.c``) or only the parser's (``backends/c/parser.c``, no tree
constants) part, as ``<config>_lexer`` and ``<config>_parser``.
Nothing from the reference is written outside ``oracle/_ref/`` (git-ignored).

Usage: python oracle/build_ref.py [--reference DIR] [config ...]

The reference sources are read from ``--reference``, else from the
environment variable ALPACC_REFERENCE, else from /root/reference (where they
are mounted read-only in the build container); ``reference_dir()`` gives the
same answer to the tests, which skip when the sources are absent.
"""

from __future__ import annotations

import argparse
import ast
import hashlib
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
sys.path.insert(0, REPO)

# config name -> (grammar file, index32)
CONFIGS = {
    "arithmetic_i32": ("arithmetic.alp", True),
    "arithmetic_i64": ("arithmetic.alp", False),
    "json_i32": ("json.alp", True),
    "json_ext_i32": ("json_ext.alp", True),
    "json_ext_i64": ("json_ext.alp", False),
    "sexp_i64": ("sexp.alp", False),
    "sexp_i32": ("sexp.alp", True),
    "paper_grammar_i64": ("paper_grammar.alp", False),
    "list_i64": ("list.alp", False),
    "llp01_i64": ("llp01.alp", False),
}


def haskell_text_block(hs_source: str, name: str) -> str:
    """The ``Text.unlines [ "...", ... ]`` value bound to ``name``."""
    m = re.search(r"^%s\s*=\s*Text\.unlines\s*\n(.*?)^\s*\]" % re.escape(name), hs_source, re.S | re.M)
    if not m:
        raise RuntimeError("could not find %s" % name)
    lits = re.findall(r'"((?:[^"\\]|\\.)*)"', m.group(1))
    lines = [ast.literal_eval('"%s"' % s) for s in lits]
    return "".join(l + "\n" for l in lines)


# configurations whose lexer-mode and parser-mode programs are also built
MODE_CONFIGS = ("arithmetic_i64", "json_i32", "json_ext_i32", "sexp_i64", "paper_grammar_i64", "llp01_i64")
# lexer-mode programs built beside those: json_ext with 64-bit starts checks
# the chunked lexing of inputs beyond 2^31 bytes
EXTRA_LEXER_CONFIGS = ("json_ext_i64",)


def reference_dir():
    """Directory of the reference's sources (ALPACC_REFERENCE, else the build
    container's mount), or None when they are not present (the GPU box)."""
    d = os.environ.get("ALPACC_REFERENCE", "/root/reference")
    return d if d and os.path.isdir(d) else None


def assemble(reference: str, tables) -> str:
    from alpacc_b200.grammar import emit_c

    def rd(p):
        with open(os.path.join(reference, p), "r", encoding="utf-8") as f:
            return f.read()

    gen_hs = rd("src/Alpacc/Generator/C/Generator.hs")
    if tables.parts == "lexer":  # auxiliary, Lex case (C/Generator.hs:164-174)
        parts = [emit_c.program_prefix(tables), emit_c.lexer_constants(tables), rd("backends/c/lexer.c"),
                 haskell_text_block(gen_hs, "lexerTestCase"), rd("backends/c/cli.c")]
        return "".join(p + "\n" for p in parts)
    if tables.parts == "parser":  # auxiliary, Parse case (C/Generator.hs:176-186)
        parts = [emit_c.program_prefix(tables), emit_c.parser_constants(tables, with_tree=False),
                 rd("backends/c/parser.c"), haskell_text_block(gen_hs, "parserTestCase"), rd("backends/c/cli.c")]
        return "".join(p + "\n" for p in parts)
    both_case = haskell_text_block(gen_hs, "bothTestCase")
    parts = [
        emit_c.program_prefix(tables),
        emit_c.lexer_constants(tables),
        rd("backends/c/lexer.c"),
        emit_c.parser_constants(tables, with_tree=True),
        rd("backends/c/parser.c"),
        both_case,
        rd("backends/c/cli.c"),
    ]
    return "".join(p + "\n" for p in parts)


def build(config: str, reference: str, cc: str = "gcc", force: bool = False, parts: str = "both") -> str:
    from alpacc_b200.grammar.cache import load_tables

    gfile, index32 = CONFIGS[config]
    name = config if parts == "both" else "%s_%s" % (config, parts)
    tables = load_tables(os.path.join(REPO, "grammars", gfile), index32=index32, parts=parts)
    return compile_program(tables, name, OUT, reference, cc, force)


def build_tables(tables, name: str, reference: str, cc: str = "gcc") -> str:
    """The reference program for tables generated from any grammar text (the
    random grammars of the differential fuzz tests), under oracle/_ref/fuzz/."""
    return compile_program(tables, name, os.path.join(OUT, "fuzz"), reference, cc, False, opt="-O1")


def compile_program(tables, name: str, out: str, reference: str, cc: str = "gcc", force: bool = False,
                    opt: str = "-O2") -> str:
    os.makedirs(out, exist_ok=True)
    src = os.path.join(out, name + ".c")
    exe = os.path.join(out, name)
    so = os.path.join(out, "lib%s.so" % name)
    stamp = os.path.join(out, name + ".stamp")
    with open(os.path.join(HERE, "ref_harness.c"), "rb") as f:
        key = tables.digest() + ":" + hashlib.sha256(f.read()).hexdigest()[:12]
    if not force and os.path.exists(so) and os.path.exists(exe) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == key:
                return so
    text = assemble(reference, tables)
    with open(src, "w", encoding="utf-8") as f:
        f.write(text)
    subprocess.check_call([cc, "-std=c99", opt, "-o", exe, src])
    subprocess.check_call([cc, "-std=c99", opt, "-shared", "-fPIC", "-o", so,
                           "-DALPACC_GENERATED=\"%s\"" % src, os.path.join(HERE, "ref_harness.c")])
    with open(stamp, "w") as f:
        f.write(key)
    return so


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("configs", nargs="*")
    a = ap.parse_args(argv)
    a.reference = a.reference or reference_dir() or ""
    if not os.path.isdir(a.reference):
        print("reference sources not present; oracle/_ref not rebuilt")
        return 0
    for c in a.configs or list(CONFIGS):
        print("building", c, "->", build(c, a.reference, force=a.force))
        if c in MODE_CONFIGS:
            for parts in ("lexer", "parser"):
                print("building", c, parts, "->", build(c, a.reference, force=a.force, parts=parts))
        elif c in EXTRA_LEXER_CONFIGS:
            print("building", c, "lexer", "->", build(c, a.reference, force=a.force, parts="lexer"))
    return 0


if __name__ == "__main__":
    sys.exit(main())
