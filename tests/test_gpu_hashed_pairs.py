"""The hashed form of the pair table on the GPU.

Grammars whose (q + k)-terminal key space exceeds 2^26 keys get the
reference's own open-addressing table on the device, probed as lookup_key
probes it (backends/c/parser.c:30-45): a random LLP(3, 3) grammar with
85.8M keys runs in all three modes against the C restatement oracle (itself
checked against the reference's programs for this grammar on the CPU in
tests/test_fuzz.py). ALPACC_PAIR_LOOKUP=hashed selects that form for any
grammar, so every grammar configuration's cases are also run through it and
compared byte for byte with the reference's C backend's records
(oracle/_ref) and the committed golden records.
"""

import json
import os

import pytest

from oracle.ref import RefOracle, available
from tests import cases

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "records.json")


@pytest.mark.parametrize("config", ["json_ext_i32", "arithmetic_i64", "sexp_i64", "json_i32", "paper_grammar_i64"])
def test_hashed_pair_table_parity(gpu, config, monkeypatch):
    from alpacc_b200.native import Parser
    monkeypatch.setenv("ALPACC_PAIR_LOOKUP", "hashed")
    p = Parser(cases.tables(config))
    try:
        assert p.info()["pair_hashed"] == 1
        golden = json.load(open(GOLDEN)).get(config, [])
        for it in golden:
            data = bytes.fromhex(it["input"])
            assert p.run_case(data).hex() == it["record"], data[:60]
        if available(config):
            ref = RefOracle(config)
            for data in cases.case_inputs(config)[:60]:
                assert p.run_case(data) == ref.run_case(data), data[:60]
    finally:
        p.close()


def test_hashed_pair_table_large_document(gpu, monkeypatch):
    from alpacc_b200 import workloads as W
    from alpacc_b200.native import Parser
    from oracle.port import PortOracle
    monkeypatch.setenv("ALPACC_PAIR_LOOKUP", "hashed")
    t = cases.tables("json_ext_i32")
    p = Parser(t)
    try:
        data = W.json_doc(6 << 20, 17)
        assert p.run_case(data) == PortOracle(t).run_case(data)
    finally:
        p.close()


def test_key_space_beyond_dense_table(gpu):
    from alpacc_b200.grammar.tables import generate_parts
    from alpacc_b200.native import Parser
    from oracle.port import PortOracle
    from tests.random_grammars import big_keyspace_grammar, token_sentences
    name, g, t = big_keyspace_grammar()
    ins = g.inputs(0, sentences=(8, 64, 2000), noise=(100, 15000))
    accepted = 0
    for parts, tables, inputs in (("both", t, ins),
                                  ("parser", generate_parts(g.text(), name, False, "parser"), token_sentences(g))):
        p = Parser(tables)
        po = PortOracle(tables)
        try:
            assert p.info()["pair_hashed"] == 1
            for d in inputs:
                rec = p.run_case(d)
                assert rec == po.run_case(d), (parts, d[:40])
                accepted += rec[0]
        finally:
            p.close()
    assert accepted > 0
