"""Limits and large inputs on the GPU, against the reference's own C backend.

* ``length_t`` overflow: json_ext's token lengths are 16-bit
  (``params { length=16 }``), and the reference's ``lex_string`` rejects the
  input when a kept token's length does not fit (backends/c/lexer.c:68-72).
  A 70 000-byte and a 65 536-byte string token are rejected, a 65 535-byte one
  is accepted, a 70 000-byte whitespace run (an ignored token: never length
  checked) is accepted - through the single-input parse, the batched parse,
  and the lexer-only program. Each token spans several lexer tiles.
* The s-expression configuration at scale: 256 MiB with nesting depths drawn
  from 1..10 000 and 64-bit indices, balanced (accepted; the whole record
  compared by SHA-256 with the reference's) and with 5% of the forms carrying
  an extra ``)`` (the single byte 0, as the reference writes).
"""

import pytest

from oracle.port import PortOracle
from oracle.ref import RefOracle, available
from tests import cases

pytestmark = pytest.mark.gpu


def _docs():
    """(input, accepted?) pairs around the 16-bit length limit."""
    out = []
    for body, ok in ((70000 - 2, False), (65536 - 2, False), (65535 - 2, True)):
        out.append((b'{"a": [1, "' + b"x" * body + b'", 2]}', ok))
    out.append((b"[1," + b" " * 70000 + b"2]", True))
    return out


def _check_both(config, got_of, parts="both"):
    name = cases.mode_name(config, parts)
    po = PortOracle(cases.tables(config, parts))
    ref = RefOracle(name) if available(name) else None
    for data, ok in _docs():
        got = got_of(data)
        assert got[0] == (1 if ok else 0), (len(data), ok)
        assert got == po.run_case(data)
        if ref is not None:
            assert got == ref.run_case(data)


def test_length_overflow_single_parse(gpu):
    from alpacc_b200.native import Parser
    p = Parser(cases.tables("json_ext_i32"))
    try:
        _check_both("json_ext_i32", p.run_case)
    finally:
        p.close()


def test_length_overflow_lexer_mode(gpu):
    from alpacc_b200.native import Parser
    p = Parser(cases.tables("json_ext_i32", "lexer"))
    try:
        _check_both("json_ext_i32", p.run_case, "lexer")
    finally:
        p.close()


def test_length_overflow_batch(gpu):
    """The batched form: documents over the limit reject alone, their
    neighbours in the batch are unaffected."""
    from alpacc_b200 import wire
    from alpacc_b200.native import Parser
    p = Parser(cases.tables("json_ext_i32"))
    po = PortOracle(cases.tables("json_ext_i32"))
    try:
        small = cases.generated("json_ext_i32", 30000, 3)
        docs = [small]
        for data, _ in _docs():
            docs += [data, small]
        outs = p.parse_batch(docs)
        for d, r in zip(docs, outs):
            assert wire.encode_record(r, p.layout) == po.run_case(d), len(d)
        assert [r.valid for r in outs[1::2]] == [ok for _, ok in _docs()]
    finally:
        p.close()


def _sexp_parity(data):
    import numpy as np

    from alpacc_b200.native import Parser
    t = cases.tables("sexp_i64")
    p = Parser(t, max_input=len(data))
    a = np.frombuffer(data, dtype=np.uint8)
    try:
        rc, got, size = p.record_digest_raw(a.ctypes.data, len(data))
    finally:
        p.close()
    if available("sexp_i64"):
        want, want_size = RefOracle("sexp_i64").record_digest(a)
        assert (got, size) == (want, want_size)
    return rc


def test_sexp_256mib_deep_balanced(gpu):
    from alpacc_b200 import workloads as W
    data = W.sexp_doc(256 << 20, 4, max_depth=10000)
    assert _sexp_parity(data) == 0


def test_sexp_256mib_deep_unbalanced(gpu):
    from alpacc_b200 import workloads as W
    data = W.sexp_doc(256 << 20, 4, unbalanced_frac=0.05, max_depth=10000)
    assert _sexp_parity(data) == 1
