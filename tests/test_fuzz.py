"""Random-grammar differential fuzzing on the CPU: for grammars drawn like
``alpacc random`` (tests/random_grammars.py), the C restatement oracle
against the reference's own C programs built here from the same tables, in
the combined, lexer-only and parser-only modes (the reference's
tests/testc.sh does the same with its Haskell-generated expected outputs).
Needs the reference sources to build those programs; skipped without them."""

import pytest

from alpacc_b200.grammar.tables import generate_parts
from oracle.build_ref import reference_dir
from oracle.port import PortOracle
from oracle.ref import RefOracle
from tests import cases
from tests.random_grammars import fuzz_grammars

REFERENCE = reference_dir()
COUNT = 16


@pytest.fixture(scope="module")
def grammars():
    if REFERENCE is None:
        pytest.skip("reference sources not present")
    return list(fuzz_grammars(COUNT))


def _check(t, name, inputs):
    from oracle.build_ref import build_tables
    po = PortOracle(t)
    ro = RefOracle(name, build_tables(t, name, REFERENCE))
    valid = 0
    for d in inputs:
        rec = po.run_case(d)
        assert rec == ro.run_case(d), (name, d[:50])
        valid += rec[0]
    return valid


def test_random_grammars_all_modes(grammars):
    accepted = {"both": 0, "lexer": 0, "parser": 0}
    for name, g, t in grammars:
        ins = g.inputs(0)
        accepted["both"] += _check(t, name, ins)
        tl = generate_parts(g.text(), name, False, "lexer")
        accepted["lexer"] += _check(tl, name + "_lexer", ins)
        tp = generate_parts(g.text(), name, False, "parser")
        accepted["parser"] += _check(tp, name + "_parser", cases.token_inputs_for(t, ins))
    assert all(v > 0 for v in accepted.values()), accepted


def test_random_grammars_cover_qk():
    qks = {(g.q, g.k) for _, g, _ in fuzz_grammars(COUNT)}
    assert len(qks) >= 3, qks


@pytest.mark.parametrize("nkw", [8, 24])
def test_keyword_lexers_all_modes(nkw):
    """C-like keyword lexers (machines of 50 and 124 states), all three modes."""
    if REFERENCE is None:
        pytest.skip("reference sources not present")
    from tests.random_grammars import keyword_grammar, keyword_inputs
    text = keyword_grammar(nkw)
    ins = keyword_inputs(nkw)
    name = "kw%d" % nkw
    t = generate_parts(text, name, False, "both")
    assert 0 < _check(t, name, ins) < len(ins)
    _check(generate_parts(text, name, False, "lexer"), name + "_lexer", ins)
    _check(generate_parts(text, name, False, "parser"), name + "_parser", cases.token_inputs_for(t, ins))


def test_key_space_beyond_dense_table_vs_reference():
    """The oversized-key-space grammar (hashed pair table on the device): the
    oracle against the reference's programs built from its tables."""
    if REFERENCE is None:
        pytest.skip("reference sources not present")
    from tests.random_grammars import big_keyspace_grammar
    name, g, t = big_keyspace_grammar()
    from tests.random_grammars import token_sentences
    ins = g.inputs(0, sentences=(8, 64, 2000), noise=(100, 15000))
    _check(t, name, ins)  # lexed random strings: mostly rejected, every record compared
    assert _check(generate_parts(g.text(), name, False, "parser"), name + "_parser", token_sentences(g)) > 0
