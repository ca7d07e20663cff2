"""The depth-walk tile algorithm of the parser kernels, emulated on the CPU
(tests/native/walk_emu.cpp) and compared with the definition it implements:
for every right bracket / production, the latest earlier element whose depth
is <= h - 1 / h. Inputs span many tiles and super-tiles (256 tiles of 2048
elements), nest thousands deep, and include mismatched and unmatched
brackets, so that the near queries, the warps' queued queries, the staircases
and the resolve's walk back are all exercised."""

import ctypes
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("walk") / "libwalk_emu.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC",
                           os.path.join(HERE, "native", "walk_emu.cpp"), "-o", so])
    L = ctypes.CDLL(so)
    L.walk_emu.restype = ctypes.c_int
    L.walk_emu.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p,
                           ctypes.c_void_p, ctypes.c_void_p]
    return L


def _run(L, mode, elems, arity=None, is_term=None):
    elems = np.ascontiguousarray(elems, dtype=np.uint32)
    parent = np.zeros(max(len(elems), 1), dtype=np.int64)
    mm = np.zeros(2, dtype=np.int64)
    a = np.ascontiguousarray(arity if arity is not None else [0], dtype=np.int32)
    t = np.ascontiguousarray(is_term if is_term is not None else [0], dtype=np.uint8)
    rc = L.walk_emu(mode, elems.ctypes.data, len(elems), a.ctypes.data, t.ctypes.data, parent.ctypes.data,
                    mm.ctypes.data)
    assert rc >= 0, ("emulation and definition disagree", mm.tolist())
    return rc


def _brackets(rng, n, max_depth, types=5):
    """A balanced sequence of n brackets (n even) whose depth wanders up to
    max_depth, in runs (deep nesting), types matched by a stack."""
    out = np.zeros(n, dtype=np.uint32)
    stack = []
    d = 0
    i = 0
    while i < n:
        run = int(rng.integers(1, max(2, max_depth // 4)))
        up = rng.random() < 0.5
        for _ in range(run):
            if i >= n:
                break
            remaining = n - i
            if d == remaining or (not up and d > 0) or d >= max_depth:
                ty = stack.pop()
                out[i] = ty
                d -= 1
            else:
                ty = int(rng.integers(0, types))
                stack.append(ty)
                out[i] = 0x80000000 | ty
                d += 1
            i += 1
    return out


@pytest.mark.parametrize("n,max_depth", [(5000, 40), (300000, 10000), (1200002, 3000), (1100000, 12)])
def test_walk_brackets_balanced(emu, n, max_depth):
    rng = np.random.default_rng(n)
    assert _run(emu, 0, _brackets(rng, n - n % 2, max_depth)) == 0


def test_walk_brackets_rejects(emu):
    rng = np.random.default_rng(5)
    b = _brackets(rng, 400000, 5000)
    m = b.copy()
    i = int(np.nonzero(m >> 31 == 0)[0][150000])
    m[i] ^= 1  # a right bracket of another type
    assert _run(emu, 0, m) != 0
    u = np.concatenate([b[:200001], b[200002:]])  # one bracket dropped: unbalanced
    assert _run(emu, 0, u) != 0
    assert _run(emu, 0, np.concatenate([np.array([5], dtype=np.uint32), b])) != 0  # a right bracket first


@pytest.mark.parametrize("n,deep", [(3000, False), (700000, False), (1300000, True)])
def test_walk_parents(emu, n, deep):
    rng = np.random.default_rng(n)
    arity = np.array([0, 1, 2, 3, 2, 0], dtype=np.int32)
    is_term = (arity == 0).astype(np.uint8)
    if deep:  # long chains of binary productions: depths climb into the thousands, then fall
        p = np.where(rng.random(n) < 0.55, 2, 0).astype(np.uint32)
        p[: n // 3] = 2
    else:
        p = rng.integers(0, len(arity), n).astype(np.uint32)
    assert _run(emu, 1, p, arity, is_term) == 0
