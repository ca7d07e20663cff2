"""Wire protocol (docs/wire-protocols.md): record and batch round trips."""

import json
import os

import numpy as np

from alpacc_b200 import wire
from tests import cases

HERE = os.path.dirname(os.path.abspath(__file__))


def test_record_round_trip_golden():
    records = json.load(open(os.path.join(HERE, "golden", "records.json")))
    for config, items in records.items():
        lay = wire.Layout.of(cases.tables(config))
        for it in items:
            rec = bytes.fromhex(it["record"])
            r, end = wire.decode_record(rec, lay)
            assert end == len(rec)
            assert wire.encode_record(r, lay) == rec


def test_batch_framing():
    payloads = [b"", b"1+2", b"x" * 300]
    buf = wire.encode_batch(payloads)
    assert int.from_bytes(buf[:8], "little") == 3
    assert int.from_bytes(buf[8:16], "little") == 8
    lay = wire.Layout(1, 1, 8, 8)
    recs = [wire.ParseResult(False), wire.ParseResult(True, np.array([1]), np.array([0]), np.array([3]),
                                                     np.array([2]), np.array([0]), np.array([0]))]
    out = (2).to_bytes(8, "little") + b"".join(wire.encode_record(r, lay) for r in recs)
    dec, end = wire.decode_batch(out, lay)
    assert end == len(out) and not dec[0].valid and dec[1].equal(recs[1])


def test_layout_text():
    lay = wire.Layout.of(cases.tables("json_ext_i32"))
    assert lay.text() == "terminal_t=1\nproduction_t=1\nindex_t=4\nlength_t=2\n"


def test_mode_records_round_trip_golden():
    """Lexer-mode and parser-mode records decode and re-encode to the
    reference's bytes."""
    recs = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "records_modes.json")))
    for name, items in recs.items():
        parts = "lexer" if name.endswith("_lexer") else "parser"
        config = name[: -len(parts) - 1]
        lay = wire.Layout.of(cases.tables(config, parts))
        for item in items:
            rec = bytes.fromhex(item["record"])
            if parts == "lexer":
                r, pos = wire.decode_lex_record(rec, lay)
                assert wire.encode_lex_record(r, lay) == rec
            else:
                r, pos = wire.decode_token_parse_record(rec, lay)
                assert wire.encode_token_parse_record(r, lay) == rec
            assert pos == len(rec)


def test_mode_layout_text_and_frames():
    lex = wire.Layout.of(cases.tables("json_i32", "lexer"))
    par = wire.Layout.of(cases.tables("json_i32", "parser"))
    assert lex.text() == "terminal_t=1\nindex_t=4\nlength_t=2\n"  # json.alp: 16-bit lengths
    assert par.text() == "terminal_t=1\nproduction_t=1\nindex_t=4\n"
    frame = wire.encode_mode_frame(b"\x01\x02\x03", par)
    assert frame[:16] == (11).to_bytes(8, "little") + (3).to_bytes(8, "little")


def test_wire_program_layout_matches_reference_without_gpu():
    """The wire-protocol programs of all three modes print the reference
    programs' --layout (from the types in scope; no device is touched)."""
    import subprocess

    from alpacc_b200.wire_program import build_program
    from oracle.ref import REF_DIR
    for config in ("arithmetic_i64", "json_i32", "sexp_i64"):
        for parts in ("both", "lexer", "parser"):
            name = cases.mode_name(config, parts)
            exe = build_program(cases.tables(config, parts), name)
            got = subprocess.run([exe, "--layout"], capture_output=True, check=True).stdout
            assert got.decode() == wire.Layout.of(cases.tables(config, parts)).text()
            ref = os.path.join(REF_DIR, name)
            if os.path.exists(ref):
                assert got == subprocess.run([ref, "--layout"], capture_output=True, check=True).stdout


def test_reference_cli_with_b200_run_case_builds(tmp_path):
    """The binding a maintainer adds to the Haskell generator's C output: the
    emitted constants and runtime templates, the glue of csrc/wire_glue.h, a
    run_case calling alpacc_gpu_run_case and the reference's own cli.c
    compile together in all three modes, and --layout (no device) prints the
    reference program's lines. Needs the reference sources."""
    import subprocess

    import pytest

    from alpacc_b200.build import LIBDIR, REPO
    from alpacc_b200.grammar import emit_c
    from oracle.ref import REF_DIR

    from oracle.build_ref import reference_dir
    ref = reference_dir()
    if ref is None:
        pytest.skip("reference sources not present")

    def rd(p):
        return open(os.path.join(ref, p)).read()

    glue = open(os.path.join(REPO, "alpacc_b200", "csrc", "wire_glue.h")).read()
    for parts in ("both", "lexer", "parser"):
        t = cases.tables("json_i32", parts)
        ib = "#define INPUT_BYTES(n) ((n) * sizeof(terminal_t))" if parts == "parser" else "#define INPUT_BYTES(n) (n)"
        run_case = "\n".join([ib, "static void run_case(uint64_t n, const uint8_t *in, FILE *out) {",
                              "  int rc = alpacc_gpu_run_case(gpu_grammar(), n, in, out);",
                              '  if (rc < 0) { fprintf(stderr, "%s\\n", alpacc_strerror(rc)); exit(1); }', "}"])
        secs = [emit_c.program_prefix(t)]
        if parts != "parser":
            secs += [emit_c.lexer_constants(t), rd("backends/c/lexer.c")]
        if parts != "lexer":
            secs += [emit_c.parser_constants(t, with_tree=parts == "both"), rd("backends/c/parser.c")]
        secs += [glue, run_case, rd("backends/c/cli.c")]
        src = tmp_path / ("b200_%s.c" % parts)
        src.write_text("\n".join(secs))
        exe = str(tmp_path / ("b200_%s" % parts))
        subprocess.check_call(["gcc", "-std=c99", "-O1", "-I", os.path.join(REPO, "include"), "-o", exe, str(src),
                               "-L", LIBDIR, "-lalpacc_b200", "-Wl,-rpath," + LIBDIR])
        got = subprocess.run([exe, "--layout"], capture_output=True, check=True).stdout
        want = os.path.join(REF_DIR, cases.mode_name("json_i32", parts))
        if os.path.exists(want):
            assert got == subprocess.run([want, "--layout"], capture_output=True, check=True).stdout
        else:
            assert got.decode() == wire.Layout.of(t).text()


def test_wire_program_frame_errors_without_gpu():
    """Malformed requests end the program with status 1 before any device
    work, as the reference's cli.c does: a truncated count, a truncated frame,
    and a frame whose length disagrees with n (for the parser-mode program
    with n counted in terminal ids)."""
    import struct
    import subprocess

    from alpacc_b200.wire_program import build_program
    for parts in ("both", "lexer", "parser"):
        t = cases.tables("sexp_i64", parts)
        exe = build_program(t, cases.mode_name("sexp_i64", parts))
        cases_bad = [b"\x01\x00", struct.pack("<Q", 1) + struct.pack("<QQ", 20, 12) + b"(a)",
                     struct.pack("<Q", 1) + struct.pack("<QQ", 8 + 4, 3) + b"\x00\x01\x02\x03"]
        for data in cases_bad:
            r = subprocess.run([exe], input=data, capture_output=True, timeout=60)
            assert r.returncode == 1, (parts, data, r.stderr)
        assert subprocess.run([exe, "--help"], capture_output=True, timeout=60).returncode == 0
