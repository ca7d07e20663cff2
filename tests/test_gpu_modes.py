"""Lexer-only and parser-only modes on the GPU against the reference's
lexer-mode and parser-mode programs (oracle/_ref/<config>_lexer, _parser),
byte for byte.

* ``alpacc_gpu_lex`` on lexer-mode tables: the record of the lexer-mode
  run_case (src/Alpacc/Generator/C/Generator.hs:87-102);
* ``alpacc_gpu_parse_tokens`` on parser-mode tables: the record of the
  parser-mode run_case (Generator.hs:65-79) for terminal-id inputs, including
  ids outside the grammar's terminal range;
* both entry points on combined tables agree with the combined result;
* the wire-protocol programs of both modes against the reference's programs.
"""

import json
import os
import subprocess

import numpy as np
import pytest

from alpacc_b200 import wire
from oracle.port import PortOracle
from oracle.ref import REF_DIR, RefOracle, available
from tests import cases

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
_PARSERS = {}


def parser(config, parts="both"):
    from alpacc_b200.native import Parser
    key = (config, parts)
    if key not in _PARSERS:
        _PARSERS[key] = Parser(cases.tables(config, parts))
    return _PARSERS[key]


def checker(config, parts):
    """The reference's own program when it was built here, else the oracle."""
    name = cases.mode_name(config, parts)
    if available(name):
        return RefOracle(name)
    return PortOracle(cases.tables(config, parts))


@pytest.mark.parametrize("config", cases.MODE_CONFIGS)
def test_lexer_mode_parity(gpu, config):
    ref = checker(config, "lexer")
    p = parser(config, "lexer")
    for data in cases.case_inputs(config):
        assert p.run_case(data) == ref.run_case(data), data[:60]


@pytest.mark.parametrize("config", cases.MODE_CONFIGS)
def test_parser_mode_parity(gpu, config):
    ref = checker(config, "parser")
    p = parser(config, "parser")
    ins = cases.token_inputs(config, sizes=(1, 64, 1000, 20000, 60000), seeds=(0, 1))
    valid = 0
    for data in ins:
        rec = p.run_case(data)
        assert rec == ref.run_case(data), data[:60]
        valid += rec[0]
    assert 0 < valid < len(ins)


def test_mode_golden_records(gpu):
    recs = json.load(open(os.path.join(HERE, "golden", "records_modes.json")))
    for name, items in recs.items():
        parts = "lexer" if name.endswith("_lexer") else "parser"
        p = parser(name[: -len(parts) - 1], parts)
        for it in items:
            data = bytes.fromhex(it["input"])
            assert p.run_case(data).hex() == it["record"], (name, data[:60])


@pytest.mark.parametrize("config", ["json_ext_i32", "sexp_i64"])
def test_combined_tables_modes_agree(gpu, config):
    """On a combined handle, lex() gives the combined result's tokens and
    parse_tokens() of those tokens the parser-mode productions."""
    p = parser(config)
    po = PortOracle(cases.tables(config, "parser"))
    lay = wire.Layout.of(cases.tables(config, "parser"))
    for data in cases.case_inputs(config, sizes=(64, 20000, 40000), seeds=(0,)):
        full = p.parse(data)
        lx = p.lex(data)
        if full.valid:
            assert lx.valid
            for a in ("token_ids", "token_starts", "token_lengths"):
                assert np.array_equal(getattr(lx, a), getattr(full, a))
        if not lx.valid:
            continue
        toks = np.asarray(lx.token_ids).astype(wire._dt(lay.terminal))
        got = wire.encode_token_parse_record(p.parse_tokens(toks), lay)
        assert got == po.run_case(toks.tobytes())


def test_large_modes_vs_oracle(gpu):
    """A multi-MiB document through both modes (many lexer tiles, ~10^6
    tokens through the pair stage and the bracket walk)."""
    config = "json_ext_i32"
    data = cases.generated(config, 6 << 20, 77)
    lex_rec = parser(config, "lexer").run_case(data)
    assert lex_rec == PortOracle(cases.tables(config, "lexer")).run_case(data)
    full = parser(config).parse(data)
    assert full.valid
    lay = wire.Layout.of(cases.tables(config, "parser"))
    toks = np.asarray(full.token_ids).astype(wire._dt(lay.terminal)).tobytes()
    assert parser(config, "parser").run_case(toks) == PortOracle(cases.tables(config, "parser")).run_case(toks)


def test_mode_handles_refuse_other_modes(gpu):
    from alpacc_b200.native import AlpaccError
    with pytest.raises(AlpaccError):
        parser("sexp_i64", "lexer").parse(b"(a)")
    with pytest.raises(AlpaccError):
        parser("sexp_i64", "lexer").parse_tokens(np.zeros(2, dtype=np.uint8))
    with pytest.raises(AlpaccError):
        parser("sexp_i64", "parser").lex(b"(a)")


@pytest.mark.parametrize("parts", ["lexer", "parser"])
@pytest.mark.parametrize("config", ["arithmetic_i64", "json_i32"])
def test_mode_wire_program_matches_reference(gpu, config, parts):
    from alpacc_b200.wire_program import build_program
    name = cases.mode_name(config, parts)
    ref = os.path.join(REF_DIR, name)
    if not os.path.exists(ref):
        pytest.skip("reference program not built")
    t = cases.tables(config, parts)
    prog = build_program(t, name)
    lay = wire.Layout.of(t)
    ins = (cases.case_inputs(config, sizes=(1, 64, 2000), seeds=(0,)) if parts == "lexer"
           else cases.token_inputs(config, sizes=(1, 64, 2000)))
    import struct
    data = struct.pack("<Q", len(ins)) + b"".join(wire.encode_mode_frame(d, lay) for d in ins)
    want = subprocess.run([ref], input=data, capture_output=True, check=True).stdout
    got = subprocess.run([prog], input=data, capture_output=True, check=True).stdout
    assert got == want
    twice = subprocess.run([prog, "--server"], input=data + data, capture_output=True, check=True).stdout
    assert twice == want + want
    assert (subprocess.run([prog, "--layout"], capture_output=True, check=True).stdout ==
            subprocess.run([ref, "--layout"], capture_output=True, check=True).stdout)
