"""The allocation-free lexer entry point (alpacc_gpu_lex_noalloc).

It serves callers that cannot call cudaMalloc where they lex (a framework
that owns the device memory pool, a real-time loop). Its working memory is a
fixed array inside the library, so this test calls it through the C ABI on
inputs up to its 16 MiB limit and checks its tokens against the tokens the
ordinary allocating entry point (alpacc_gpu_parse_device) produces for the
same input, on two calls in a row (the shared array must be cleared between
calls), and checks that oversize inputs are refused. It is collected last so a
failure here cannot hide failures elsewhere.
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
