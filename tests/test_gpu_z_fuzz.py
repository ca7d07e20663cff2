"""Random-grammar differential fuzzing of the CUDA path: for grammars drawn like
``alpacc random`` (tests/random_grammars.py, the reference's (q, k) matrix), the device
path's records against the C restatement oracle (itself checked against the
reference's C programs on the same grammars in tests/test_fuzz.py) in the
combined, lexer-only and parser-only modes, and the batched form against the
single-input form."""

import pytest

from alpacc_b200.grammar.tables import generate_parts
from oracle.port import PortOracle
from tests import cases
from tests.random_grammars import fuzz_grammars

pytestmark = pytest.mark.gpu

COUNT = 24


@pytest.fixture(scope="module")
def grammars():
    return list(fuzz_grammars(COUNT))


def _check(t, inputs):
    from alpacc_b200.native import Parser
    p = Parser(t)
    po = PortOracle(t)
    valid = 0
    try:
        for d in inputs:
            rec = p.run_case(d)
            assert rec == po.run_case(d), (t.name, t.parts, d[:50])
            valid += rec[0]
    finally:
        p.close()
    return valid


def test_random_grammars_all_modes(gpu, grammars):
    accepted = {"both": 0, "lexer": 0, "parser": 0}
    for name, g, t in grammars:
        ins = g.inputs(0)
        accepted["both"] += _check(t, ins)
        accepted["lexer"] += _check(generate_parts(g.text(), name, False, "lexer"), ins)
        accepted["parser"] += _check(generate_parts(g.text(), name, False, "parser"),
                                     cases.token_inputs_for(t, ins))
    assert all(v > 0 for v in accepted.values()), accepted


def test_random_grammars_batch_equals_single(gpu, grammars):
    from alpacc_b200.native import Parser
    for name, g, t in grammars[:8]:
        ins = g.inputs(1)
        p = Parser(t)
        try:
            batch = p.parse_batch(ins)
            for d, r in zip(ins, batch):
                assert r.equal(p.parse(d)), (name, d[:50])
        finally:
            p.close()


@pytest.mark.parametrize("nkw", [8, 16, 24, 32])
def test_keyword_lexers(gpu, nkw):
    """C-like keyword lexers of 50, 86, 124 and 164 machine states (above 64:
    256-bit candidate sets; window machines of up to 347 sets), in all three
    modes against the oracle, on inputs up to several lexer tiles."""
    from alpacc_b200.native import Parser
    from tests.random_grammars import keyword_grammar, keyword_inputs
    text = keyword_grammar(nkw)
    name = "kw%d" % nkw
    t = generate_parts(text, name, False, "both")
    ins = keyword_inputs(nkw, seed=nkw)
    p = Parser(t)
    try:
        assert (p.info()["M"] > 64) == (nkw >= 16)
    finally:
        p.close()
    assert _check(t, ins) > 0
    assert _check(generate_parts(text, name, False, "lexer"), ins) > 0
    assert _check(generate_parts(text, name, False, "parser"), cases.token_inputs_for(t, ins)) > 0
