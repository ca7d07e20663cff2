"""Chunked lexing (``alpacc_gpu_lex_stream``) on the GPU.

* Small windows on ordinary inputs: the lexemes equal one ``alpacc_gpu_lex``
  call (itself checked against the reference's lexer-mode program) for every
  window size, including windows shorter than a token (the window is widened)
  and inputs that are rejected.
* An input beyond 2^31 bytes (json_ext, 64-bit index_t): the whole lexeme
  stream equals the lexer-mode record of the reference's own C program
  (oracle/_ref, SHA-256 of the lexemes in record order, streamed on both
  sides); two different windowings give the same lexeme sequence
  (order-sensitive checksums); the spans are ordered and inside the input;
  and the lexemes near the start and near the end equal single calls on the
  input cut at a token boundary.
"""

import numpy as np
import pytest

from tests import cases

pytestmark = pytest.mark.gpu

_PARSERS = {}


def parser(config, parts="lexer"):
    from alpacc_b200.native import Parser
    if (config, parts) not in _PARSERS:
        _PARSERS[(config, parts)] = Parser(cases.tables(config, parts))
    return _PARSERS[(config, parts)]


def same(a, b):
    if a.valid != b.valid:
        return False
    return not a.valid or all(np.array_equal(np.asarray(getattr(a, k), dtype=np.int64),
                                             np.asarray(getattr(b, k), dtype=np.int64))
                              for k in ("token_ids", "token_starts", "token_lengths"))


@pytest.mark.parametrize("config", ["json_ext_i32", "sexp_i64", "arithmetic_i64"])
def test_stream_windows_equal_single_call(gpu, config):
    p = parser(config)
    for data in cases.case_inputs(config, sizes=(1, 61, 1000, 14881, 40000), seeds=(0,)):
        want = p.lex(data)
        for w in (64, 997, 15360, 1 << 16):
            if len(data) > 200 * w:
                continue
            got, _ = p.lex_stream(data, window=w)
            assert same(got, want), (config, w, data[:50])


def test_stream_token_longer_than_window(gpu):
    p = parser("json_ext_i32")
    data = b'["' + b"x" * 50000 + b'", 1, "' + b"y" * 3000 + b'"]'
    want = p.lex(data)
    assert want.valid
    got, windows = p.lex_stream(data, window=1000)
    assert same(got, want) and windows >= 2


def test_stream_combined_tables(gpu):
    """On combined tables the stream gives the combined parse's tokens."""
    p = parser("json_ext_i32", "both")
    data = cases.generated("json_ext_i32", 300000, 5)
    full = p.parse(data)
    got, windows = p.lex_stream(data, window=50000)
    assert full.valid and windows >= 6
    for k in ("token_ids", "token_starts", "token_lengths"):
        assert np.array_equal(np.asarray(getattr(got, k)), np.asarray(getattr(full, k)))


class _Summary:
    """Order-sensitive checksum of a lexeme stream plus its first and last lexemes."""

    def __init__(self, n, edge, lay=None):
        import hashlib
        self.n, self.edge = n, edge
        self.lay = lay  # when set: SHA-256 of the lexemes as the lexer-mode record lays them out
        self.sha = hashlib.sha256()
        self.count = 0
        self.h = np.uint64(0)
        self.prev_end = 0
        self.ordered = True
        self.head, self.tail = [], []

    def __call__(self, first, ids, starts, lens):
        assert first == self.count
        # a sum over lexemes of a mix of (index, id, start, length): the same for
        # any split of the stream into windows
        i = np.arange(first, first + len(ids), dtype=np.uint64)
        with np.errstate(over="ignore"):
            v = (starts.astype(np.uint64) * np.uint64(1000003) + lens.astype(np.uint64) * np.uint64(10007)
                 + ids.astype(np.uint64) * np.uint64(131) + i * np.uint64(7919))
            v = v * np.uint64(0x9E3779B97F4A7C15)
            v = v ^ (v >> np.uint64(29))
            self.h = self.h + v.sum(dtype=np.uint64)
        if self.lay is not None:
            from alpacc_b200 import wire
            rec = np.zeros(len(ids), dtype=wire._lexeme_dtype(self.lay))
            rec["id"], rec["start"], rec["length"] = ids, starts, lens
            self.sha.update(rec.tobytes())
        ends = starts + lens
        self.ordered &= bool(starts[0] >= self.prev_end) and bool(np.all(starts[1:] >= ends[:-1]))
        self.ordered &= bool(ends[-1] <= self.n)
        self.prev_end = int(ends[-1])
        self.count += len(ids)
        m = starts < self.edge
        if m.any():
            self.head.append((ids[m], starts[m], lens[m]))
        m = starts >= self.n - self.edge
        if m.any():
            self.tail.append((ids[m], starts[m], lens[m]))

    def cat(self, which):
        parts = self.head if which == "head" else self.tail
        return [np.concatenate([p[i] for p in parts]).astype(np.int64) for i in range(3)]


def test_stream_beyond_2_gib(gpu):
    from alpacc_b200 import workloads as W
    n = (1 << 31) + (1 << 20)
    data = np.frombuffer(W.json_doc(n, 9), dtype=np.uint8)
    p = parser("json_ext_i64")
    edge = 8 << 20
    a, b = _Summary(n, edge, p.layout), _Summary(n, edge)
    p.lex_stream(data, window=1 << 30, on_window=a)
    p.lex_stream(data, window=(768 << 20) + 12345, on_window=b)
    assert a.count == b.count and a.count > 0
    assert a.h == b.h and a.ordered and b.ordered
    # the whole stream against the reference's lexer-mode program
    import struct

    from oracle.ref import RefOracle, available
    if available("json_ext_i64_lexer"):
        want, _, head = RefOracle("json_ext_i64_lexer").record_digest(data, head=9)
        assert head == b"\x01" + struct.pack("<Q", a.count)
        assert a.sha.hexdigest() == want
    # the first lexemes: a single call on the input cut at a token start
    ids, starts, lens = a.cat("head")
    cut = int(starts[-1])
    r = p.lex(data[:cut])
    assert r.valid
    k = len(r.token_ids)
    assert k == len(ids) - 1
    assert np.array_equal(r.token_ids, ids[:k]) and np.array_equal(r.token_starts, starts[:k])
    assert np.array_equal(r.token_lengths, lens[:k])
    # the last lexemes: a single call from a token start to the end
    ids, starts, lens = a.cat("tail")
    cut = int(starts[0])
    r = p.lex(data[cut:])
    assert r.valid and len(r.token_ids) == len(ids)
    assert np.array_equal(r.token_ids, ids) and np.array_equal(r.token_starts + cut, starts)
    assert np.array_equal(r.token_lengths, lens)
