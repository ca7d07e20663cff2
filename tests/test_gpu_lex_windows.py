"""The lexer's window variants on the GPU.

Each chunk's start state is settled by walking the 16 bytes before it in the
window machine (the subset automaton of the lexer machine's live states);
grammars whose window machine exceeds its budget walk those bytes as explicit
state sets instead. ALPACC_LEX_WINDOW=sets selects the state-set walk for any
grammar, so every grammar configuration's cases run through both kernels and
are compared byte for byte with the reference's C backend's records
(oracle/_ref) and the committed golden records; inputs whose windows never
settle (a numeric array is valid inside and outside a JSON string) exercise
the per-candidate walks and the tile look-back in both.
"""

import json
import os

import numpy as np
import pytest

from oracle.ref import RefOracle, available
from tests import cases

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "records.json")


def _open_chunk_inputs():
    rng = np.random.default_rng(7)
    nums = b"[" + b", ".join(str(int(x)).encode() for x in rng.integers(0, 1000, 60000)) + b"]"
    return [nums, b'{"a": ' + nums + b', "b": "x y z"}', nums[:100000] + b"\x01" + nums[100000:],
            b'["' + b"ab cd " * 20000 + b'", 1]']


@pytest.mark.parametrize("variant", ["window", "sets"])
@pytest.mark.parametrize("config", ["json_ext_i32", "arithmetic_i64", "sexp_i64", "json_i32", "paper_grammar_i64"])
def test_lexer_window_variants(gpu, config, variant, monkeypatch):
    from alpacc_b200.native import Parser
    if variant == "sets":
        monkeypatch.setenv("ALPACC_LEX_WINDOW", "sets")
    p = Parser(cases.tables(config))
    try:
        info = p.info()
        assert info["lex_variant"] == (2 if variant == "sets" else 0), info
        assert variant == "sets" or info["window_sets"] > 0
        golden = json.load(open(GOLDEN)).get(config, [])
        for it in golden:
            data = bytes.fromhex(it["input"])
            assert p.run_case(data).hex() == it["record"], data[:60]
        if available(config):
            ref = RefOracle(config)
            extra = _open_chunk_inputs() if config.startswith("json") else []
            for data in cases.case_inputs(config)[:60] + extra:
                assert p.run_case(data) == ref.run_case(data), data[:60]
    finally:
        p.close()
