"""The batched entry point (alpacc_gpu_parse_batch): many documents of uneven
length through one launch per stage. Every document's result must be
identical to parsing it alone, whatever its neighbours are - empty documents,
rejects (lexer and parser), multi-tile documents and deep nesting included."""

import numpy as np
import pytest

from alpacc_b200 import native, wire, workloads as W
from oracle.ref import RefOracle, available
from tests import cases

pytestmark = pytest.mark.gpu

_P = {}


def parser(config):
    if config not in _P:
        _P[config] = native.Parser(cases.tables(config), device=0)
    return _P[config]


def mixed_docs(config, seed):
    rng = np.random.default_rng(seed)
    docs = []
    for i, n in enumerate([2, 7, 60, 61, 500, 4000, 15360, 15361, 40000, 120000]):
        docs.append(cases.generated(config, n, seed * 100 + i))
    docs.append(b"")
    docs += [cases.mutate(d, rng) for d in docs[3:8]]  # rejects of every kind
    docs += list(cases.FIXED.get(cases.family(config), []))
    order = rng.permutation(len(docs))
    return [docs[i] for i in order]


@pytest.mark.parametrize("config", ["json_ext_i32", "arithmetic_i64", "sexp_i64", "paper_grammar_i64"])
def test_batch_equals_single(gpu, config):
    p = parser(config)
    lay = p.layout
    docs = mixed_docs(config, 7)
    got = p.parse_batch(docs)
    assert len(got) == len(docs)
    for d, r in zip(docs, got):
        assert wire.encode_record(r, lay) == p.run_case(d), d[:60]


@pytest.mark.parametrize("config", ["json_ext_i32", "sexp_i64"])
def test_batch_against_reference(gpu, config):
    if not available(config):
        pytest.skip("oracle/_ref/%s not built" % config)
    ref = RefOracle(config)
    p = parser(config)
    docs = [cases.generated(config, n, 500 + n) for n in (10, 300, 3000, 20000)]
    if config.startswith("sexp"):
        docs.append(W.sexp_doc(50000, 9, max_depth=2000))
    for d, r in zip(docs, p.parse_batch(docs)):
        assert wire.encode_record(r, p.layout) == ref.run_case(d)


def test_batch_many_small_documents(gpu):
    """The configured batch shape at reduced scale: log-normal lengths."""
    buf, offs = W.json_batch(count=300, median=2048, lo=200, hi=64 << 10, seed=4)
    docs = [buf[offs[i]:offs[i + 1]] for i in range(len(offs) - 1)]
    p = parser("json_ext_i32")
    got = p.parse_batch(docs)
    for d, r in zip(docs[::15], got[::15]):
        assert wire.encode_record(r, p.layout) == p.run_case(d)
    assert all(r.valid for r in got)


def test_batch_then_single_reuse(gpu):
    p = parser("json_ext_i32")
    a = cases.generated("json_ext_i32", 3 << 20, 3)
    b = [cases.generated("json_ext_i32", 1000, k) for k in range(5)]
    first = p.run_case(a)
    p.parse_batch(b)
    assert p.run_case(a) == first
    assert [wire.encode_record(r, p.layout) for r in p.parse_batch(b)] == [p.run_case(x) for x in b]


def test_batch_empty(gpu):
    assert parser("json_ext_i32").parse_batch([]) == []
