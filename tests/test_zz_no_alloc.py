"""The allocation-free lexer entry point (alpacc_gpu_lex_noalloc).

It serves callers that cannot call cudaMalloc where they lex (a framework
that owns the device memory pool, a real-time loop). Its working memory is a
fixed array inside the library, so these tests call it through the C ABI and
check its tokens against the tokens the ordinary allocating entry point
(alpacc_gpu_parse_device) produces for the same input, on two calls in a row
(the shared array must be cleared between calls); against the lexer-mode
records of the reference's own C program (oracle/_ref) and of the C
restatement oracle; at exactly its 16 MiB limit; on a 124-state keyword lexer
(near the 128-state limit of its per-tile vectors); on a token longer than
length_t holds (reject) and one at the limit (accept); and that its calls make
no device allocation, even the first one on a fresh handle. Oversize inputs
are refused. The file is collected last so a failure here cannot hide
failures elsewhere.
"""

import ctypes

import numpy as np
import pytest

from alpacc_b200 import native, workloads as W
from tests import cases

pytestmark = pytest.mark.gpu


def _lib():
    L = native.lib()
    L.alpacc_gpu_lex_noalloc.restype = ctypes.c_int
    L.alpacc_gpu_lex_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]
    return L


def _tokens_existing(p, d_in, n):
    """Tokens from the allocating entry point (device result -> host)."""
    rc, r = p.parse_device(d_in.data_ptr(), n)
    res = p.device_result(r, rc)
    return rc, res


def _tokens_noalloc(p, d_in, n, lay):
    import torch
    dev = d_in.device
    ids = torch.zeros(max(n, 1) * lay.terminal, dtype=torch.uint8, device=dev)
    starts = torch.zeros(max(n, 1) * lay.index, dtype=torch.uint8, device=dev)
    lens = torch.zeros(max(n, 1) * lay.length, dtype=torch.uint8, device=dev)
    cnt = ctypes.c_uint64(0)
    rc = _lib().alpacc_gpu_lex_noalloc(p._h, d_in.data_ptr(), n, ids.data_ptr(), starts.data_ptr(),
                                       lens.data_ptr(), ctypes.byref(cnt))
    torch.cuda.synchronize()
    T = cnt.value
    dt = lambda k, s: np.dtype(("i" if s else "u") + str(k))  # noqa: E731
    return rc, (ids.cpu().numpy().view(dt(lay.terminal, False))[:T],
                starts.cpu().numpy().view(dt(lay.index, True))[:T],
                lens.cpu().numpy().view(dt(lay.length, False))[:T])


@pytest.mark.parametrize("config", ["json_ext_i32", "arithmetic_i64"])
def test_noalloc_matches_existing_entry_point_twice(gpu, config):
    import torch
    p = native.Parser(cases.tables(config), device=0)
    lay = p.layout
    inputs = [cases.generated(config, 3 << 20, 5), cases.generated(config, 200000, 6)]
    for data in inputs:  # two calls in a row on one handle
        d_in = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
        rc_a, ref = _tokens_existing(p, d_in, len(data))
        rc_b, (ids, starts, lens) = _tokens_noalloc(p, d_in, len(data), lay)
        assert rc_a == native.OK and rc_b == native.OK
        assert np.array_equal(ids.astype(np.int64), ref.token_ids.astype(np.int64))
        assert np.array_equal(starts.astype(np.int64), ref.token_starts.astype(np.int64))
        assert np.array_equal(lens.astype(np.int64), ref.token_lengths.astype(np.int64))
    p.close()


def test_noalloc_reject_empty_and_limit(gpu):
    import torch
    p = native.Parser(cases.tables("json_ext_i32"), device=0)
    lay = p.layout
    bad = b'[1, 2, "unterminated'
    d_in = torch.frombuffer(bytearray(bad), dtype=torch.uint8).cuda()
    rc, _ = _tokens_noalloc(p, d_in, len(bad), lay)
    assert rc == native.REJECT
    rc, (ids, _, _) = _tokens_noalloc(p, d_in, 0, lay)
    assert rc == native.OK and len(ids) == 0
    cnt = ctypes.c_uint64(0)
    rc = _lib().alpacc_gpu_lex_noalloc(p._h, d_in.data_ptr(), (16 << 20) + 1, d_in.data_ptr(), d_in.data_ptr(),
                                       d_in.data_ptr(), ctypes.byref(cnt))
    assert rc == native.E_CAPACITY
    p.close()


def _lex_record(p, data, lay):
    """The lexer-mode response record built from the no-alloc entry point's tokens."""
    import torch

    from alpacc_b200 import wire
    d_in = torch.frombuffer(bytearray(data) or bytearray(1), dtype=torch.uint8).cuda()
    rc, (ids, starts, lens) = _tokens_noalloc(p, d_in, len(data), lay)
    assert rc in (native.OK, native.REJECT), rc
    if rc == native.REJECT:
        return b"\x00"
    return wire.encode_lex_record(wire.LexResult(True, ids, starts, lens), lay)


@pytest.mark.parametrize("config", ["json_ext_i32", "arithmetic_i64", "sexp_i64"])
def test_noalloc_matches_reference_lexer_records(gpu, config):
    """Against the reference's own lexer-mode program (oracle/_ref) and its
    committed records, with a handle holding the lexer-mode tables."""
    import json
    import os

    from oracle.ref import RefOracle, available
    name = cases.mode_name(config, "lexer")
    p = native.Parser(cases.tables(config, "lexer"), device=0)
    lay = p.layout
    try:
        golden = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                             "records_modes.json"))).get(name, [])
        for it in golden:
            data = bytes.fromhex(it["input"])
            assert _lex_record(p, data, lay).hex() == it["record"], data[:40]
        if available(name):
            ref = RefOracle(name)
            for data in cases.case_inputs(config)[:40] + [cases.generated(config, 5 << 20, 21)]:
                assert _lex_record(p, data, lay) == ref.run_case(data), data[:40]
    finally:
        p.close()


def test_noalloc_exactly_at_limit(gpu):
    """An input of exactly 16 MiB (the largest accepted) against the oracle."""
    from oracle.port import PortOracle
    t = cases.tables("json_ext_i32", "lexer")
    data = W.json_doc(16 << 20, 31)
    p = native.Parser(t, device=0)
    try:
        assert _lex_record(p, data, p.layout) == PortOracle(t).run_case(data)
    finally:
        p.close()


def test_noalloc_keyword_lexer_near_state_limit(gpu):
    """A 24-keyword lexer (124 machine states: per-start lanes, per-tile
    transition vectors of 124 entries) against the oracle."""
    from alpacc_b200.grammar.tables import generate_parts
    from oracle.port import PortOracle
    from tests.random_grammars import keyword_grammar, keyword_inputs
    t = generate_parts(keyword_grammar(24), "kw24", False, "lexer")
    p = native.Parser(t, device=0)
    po = PortOracle(t)
    try:
        assert p.info()["M"] > 100
        for data in keyword_inputs(24, seed=5, sizes=(1, 300, 15000, 40000, 400000)):
            assert _lex_record(p, data, p.layout) == po.run_case(data), data[:40]
    finally:
        p.close()


def test_noalloc_length_overflow(gpu):
    """json_ext's length_t is 16 bits: a 70 000-byte string token is rejected
    (lex_string's length check), a 65 535-byte one is accepted with that
    length; both span several lexer tiles."""
    from oracle.port import PortOracle
    t = cases.tables("json_ext_i32", "lexer")
    po = PortOracle(t)
    p = native.Parser(t, device=0)
    try:
        for body, ok in ((70000 - 2, False), (65535 - 2, True), (65536 - 2, False)):
            data = b'[1, "' + b"x" * body + b'", 2]'
            rec = _lex_record(p, data, p.layout)
            assert rec == po.run_case(data)
            assert rec[0] == (1 if ok else 0)
    finally:
        p.close()


def test_noalloc_allocates_nothing(gpu):
    """On a fresh handle, the first and the later calls make no device
    allocation (the library's own counter, and the device's free memory)."""
    import torch
    p = native.Parser(cases.tables("json_ext_i32"), device=0)
    lay = p.layout
    data = cases.generated("json_ext_i32", 2 << 20, 8)
    n = len(data)
    d_in = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
    ids = torch.zeros(n * lay.terminal, dtype=torch.uint8, device="cuda")
    starts = torch.zeros(n * lay.index, dtype=torch.uint8, device="cuda")
    lens = torch.zeros(n * lay.length, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    L = _lib()
    cnt = ctypes.c_uint64(0)

    def call():
        return L.alpacc_gpu_lex_noalloc(p._h, d_in.data_ptr(), n, ids.data_ptr(), starts.data_ptr(),
                                        lens.data_ptr(), ctypes.byref(cnt))

    try:
        allocs0 = native.lib().alpacc_device_allocations()
        assert call() == native.OK  # the first call on this handle
        assert native.lib().alpacc_device_allocations() == allocs0
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        for _ in range(3):
            assert call() == native.OK
        torch.cuda.synchronize()
        assert native.lib().alpacc_device_allocations() == allocs0
        assert torch.cuda.mem_get_info()[0] == free0
        assert cnt.value > 0
    finally:
        p.close()
