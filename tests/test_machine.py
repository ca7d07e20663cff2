"""The lexer machine the loader derives for the GPU, run on the CPU.

``device_tables.cpp`` turns TO_STATE / COMPOSE / ACCEPT into a minimised Moore
machine over byte classes, which the lexer kernels walk. ``tests/native/
machine_lex.cpp`` walks that machine sequentially with the kernels' boundary
rule; its lexemes must equal the oracle's ``lex_string`` lexemes (lexer-mode
records) for the shipped grammars, random grammars and keyword lexers — a
check of the host-side derivation that needs no GPU.
"""

import ctypes
import os
import subprocess

import numpy as np
import pytest

from alpacc_b200 import native, wire
from alpacc_b200.grammar.tables import generate_parts
from oracle.port import PortOracle
from tests import cases
from tests.random_grammars import fuzz_grammars, keyword_grammar, keyword_inputs

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("machine") / "libmachine_lex.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-shared", "-fPIC",
                           "-I", os.path.join(REPO, "alpacc_b200", "csrc"), "-I", os.path.join(REPO, "include"),
                           os.path.join(HERE, "native", "machine_lex.cpp"),
                           os.path.join(REPO, "alpacc_b200", "csrc", "device_tables.cpp"), "-o", so])
    L = ctypes.CDLL(so)
    L.window_info.restype = ctypes.c_int
    L.window_info.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.machine_lex.restype = ctypes.c_int
    L.machine_lex.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                              ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int)]
    return L


def _compare(L, t, inputs):
    s, keep = native.make_tables(t)
    po = PortOracle(t)
    lay = wire.Layout.of(t)
    states = ctypes.c_int(0)
    for d in inputs:
        cap = len(d) + 1
        out = np.zeros(3 * cap, dtype=np.uint64)
        cnt = ctypes.c_uint64(0)
        rc = L.machine_lex(ctypes.byref(s), d, len(d), out.ctypes.data, cap, ctypes.byref(cnt), ctypes.byref(states))
        assert rc in (native.OK, native.REJECT), rc
        want, _ = wire.decode_lex_record(po.run_case(d), lay)
        assert (rc == native.OK) == want.valid, (t.name, d[:40])
        if want.valid:
            got = out[: 3 * cnt.value].reshape(-1, 3).astype(np.int64)
            assert len(got) == len(want.token_ids), (t.name, d[:40])
            assert np.array_equal(got[:, 0], want.token_ids), (t.name, d[:40])
            assert np.array_equal(got[:, 1], want.token_starts), (t.name, d[:40])
            assert np.array_equal(got[:, 2], want.token_lengths), (t.name, d[:40])
    return states.value


@pytest.mark.parametrize("config", cases.MODE_CONFIGS)
def test_machine_matches_lex_string(harness, config):
    _compare(harness, cases.tables(config, "lexer"), cases.case_inputs(config, sizes=(1, 64, 3000), seeds=(0,)))


def test_machine_random_grammars(harness):
    for name, g, _ in fuzz_grammars(16):
        _compare(harness, generate_parts(g.text(), name, False, "lexer"), g.inputs(0, sentences=(8, 300), noise=(500,)))


@pytest.mark.parametrize("nkw", [8, 24])
def test_machine_keyword_lexers(harness, nkw):
    t = generate_parts(keyword_grammar(nkw), "kw%d" % nkw, False, "lexer")
    states = _compare(harness, t, keyword_inputs(nkw, sizes=(0, 1, 20, 300, 5000)))
    assert states == {8: 50, 24: 124}[nkw]


def _lookup_key(t, key):
    """``lookup_key`` (backends/c/parser.c:17-45): FNV-1a, linear probing up
    to MAX_ITERS, and a found key with a negative span counts as missing."""
    from alpacc_b200.grammar.tables import fnv1a
    H = t.hash_size
    h = fnv1a(key) % H
    for _ in range(t.max_iters):
        if t.ht_valid[h] and all(int(a) == int(b) for a, b in zip(t.ht_keys[h], key)):
            ss, se = (int(x) for x in t.ht_stack_span[h])
            ps, pe = (int(x) for x in t.ht_prod_span[h])
            if min(ss, se, ps, pe) < 0:
                return None
            return (ss, se, ps, pe)
        h = (h + 1) % H
    return None


def _check_pairs(L, t, seed=0):
    import itertools
    s, keep = native.make_tables(t)
    n = t.q + t.k
    nt = t.end_terminal + 1
    space = nt ** n
    if space <= 50000:
        keys = np.array(list(itertools.product(range(nt), repeat=n)), dtype=np.uint64).reshape(-1, n)
    else:
        rng = np.random.default_rng(seed)
        stored = np.array([k for k, v in zip(t.ht_keys, t.ht_valid) if v], dtype=np.uint64).reshape(-1, n)
        keys = np.concatenate([stored, rng.integers(0, nt, (20000, n)).astype(np.uint64)])
    # ids past the terminal range are never a key
    keys = np.concatenate([keys, np.full((1, n), nt, dtype=np.uint64)])
    out = np.zeros((len(keys), 5), dtype=np.int64)
    assert L.pair_lookup(ctypes.byref(s), keys.ctypes.data, len(keys), out.ctypes.data) == native.OK
    found = 0
    for key, o in zip(keys, out):
        want = _lookup_key(t, key)
        assert (o[0] == 1) == (want is not None), (t.name, key)
        if want is not None:
            assert tuple(int(x) for x in o[1:]) == want, (t.name, key)
            found += 1
    return found


@pytest.mark.parametrize("config", sorted(cases.CONFIGS))
def test_pair_table_matches_lookup_key(harness, config):
    L = harness
    L.pair_lookup.restype = ctypes.c_int
    L.pair_lookup.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    assert _check_pairs(L, cases.tables(config)) > 0


@pytest.mark.parametrize("config", ["json_ext_i32", "arithmetic_i64", "sexp_i64", "paper_grammar_i64"])
def test_hashed_pair_table_matches_lookup_key(harness, config, monkeypatch):
    """The hashed form (used for key spaces above 2^26, forced here with
    ALPACC_PAIR_LOOKUP=hashed): the device's probe of the reference's own
    open-addressing table, restated in the harness, against lookup_key."""
    monkeypatch.setenv("ALPACC_PAIR_LOOKUP", "hashed")
    L = harness
    L.pair_lookup.restype = ctypes.c_int
    L.pair_lookup.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    assert _check_pairs(L, cases.tables(config)) > 0
    for name, g, t in list(fuzz_grammars(6)):
        assert _check_pairs(L, t) > 0, name


def test_pair_table_key_space_beyond_dense(harness):
    """A key space above 2^26 keys takes the hashed form without forcing."""
    from tests.random_grammars import big_keyspace_grammar
    L = harness
    L.pair_lookup.restype = ctypes.c_int
    L.pair_lookup.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    name, g, t = big_keyspace_grammar()
    assert (t.end_terminal + 1) ** (t.q + t.k) > (1 << 26)
    assert _check_pairs(L, t) > 0


def test_pair_table_random_grammars(harness):
    L = harness
    L.pair_lookup.restype = ctypes.c_int
    L.pair_lookup.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    for name, g, t in fuzz_grammars(16):
        assert _check_pairs(L, t) > 0, name


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("emu") / "liblexer_emu.so")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-shared", "-fPIC",
                           "-I", os.path.join(REPO, "alpacc_b200", "csrc"), "-I", os.path.join(REPO, "include"),
                           os.path.join(HERE, "native", "lexer_emu.cpp"),
                           os.path.join(REPO, "alpacc_b200", "csrc", "device_tables.cpp"), "-o", so])
    L = ctypes.CDLL(so)
    L.lexer_emu.restype = ctypes.c_int
    L.lexer_emu.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_int,
                            ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p,
                            ctypes.POINTER(ctypes.c_uint64)]
    return L


def _emu_vs_machine(L, M, t, inputs, sets=False, win=16):
    """The tile algorithm of the lexer kernel (emulated) against the machine
    walked byte by byte: status and every lexeme. ``sets``: windows walked as
    explicit state sets instead of in the window machine; ``win``: window
    bytes."""
    s, keep = native.make_tables(t)
    states = ctypes.c_int(0)
    stats = np.zeros(4, dtype=np.int64)
    total = np.zeros(4, dtype=np.int64)
    for d in inputs:
        cap = len(d) + 1
        want = np.zeros(3 * cap, dtype=np.uint64)
        got = np.zeros(3 * cap, dtype=np.uint64)
        cw, cg, lb = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_uint64(0)
        rw = M.machine_lex(ctypes.byref(s), d, len(d), want.ctypes.data, cap, ctypes.byref(cw), ctypes.byref(states))
        rg = L.lexer_emu(ctypes.byref(s), d, len(d), 0, 1 if sets else 0, win, got.ctypes.data, cap,
                         ctypes.byref(cg), stats.ctypes.data, ctypes.byref(lb))
        total += stats
        assert rg == rw, (t.name, len(d), d[:40], rg, rw)
        if rw == native.OK:
            assert cg.value == cw.value, (t.name, len(d))
            assert np.array_equal(got[: 3 * cg.value], want[: 3 * cw.value]), (t.name, len(d), d[:40])
    return total


TILE = 15360


@pytest.mark.parametrize("sets,win", [(False, 16), (True, 16), (False, 32), (True, 24)],
                         ids=["window_machine16", "state_sets16", "window_machine32", "state_sets24"])
@pytest.mark.parametrize("config", sorted(cases.CONFIGS))
def test_lexer_tile_algorithm(harness, emu, config, sets, win):
    ins = cases.case_inputs(config, sizes=(1, 59, 60, 61, 3000, TILE - 1, TILE, TILE + 1, 3 * TILE + 7),
                            seeds=(0,))
    _emu_vs_machine(emu, harness, cases.tables(config, "both"), ins, sets, win)


@pytest.mark.parametrize("sets,win", [(False, 16), (True, 16), (False, 32)],
                         ids=["window_machine16", "state_sets16", "window_machine32"])
def test_lexer_tile_algorithm_open_chunks(harness, emu, sets, win):
    """Inputs whose windows never settle on one state (a numeric array on one
    line is valid both inside and outside a JSON string): per-candidate chunk
    functions and tiles without a known chunk (transition vectors,
    look-back)."""
    t = cases.tables("json_ext_i32")
    rng = np.random.default_rng(7)
    nums = b"[" + b", ".join(str(int(x)).encode() for x in rng.integers(0, 1000, 30000)) + b"]"
    mixed = b'{"a": ' + nums + b', "b": "x y z"}'
    bad = nums[:50000] + b"\x01" + nums[50000:]
    stats = _emu_vs_machine(emu, harness, t, [nums, mixed, bad, nums[:TILE * 2 + 5] + b"]"], sets, win)
    assert stats[0] > 1000 and stats[2] > 0  # open chunks and look-back tiles were exercised


def test_window_machine_tables(harness):
    """The window machine of every shipped grammar is built (its sets fit the
    budget) and each entry's info byte names the next set's one state, the
    dead state for an empty set, or 0xFF for two or more."""
    for config in sorted(cases.CONFIGS):
        t = cases.tables(config, "both")
        s, keep = native.make_tables(t)
        info = np.zeros(4, dtype=np.int64)
        assert harness.window_info(ctypes.byref(s), info.ctypes.data) == 0, config
        sets, singles, opens, bad = info
        assert 0 < sets <= 1024 and singles > 0 and bad == 0, (config, info)


def test_window_machine_tables_random_and_keyword_grammars(harness):
    """The same entry check for 16 random grammars and the keyword lexers of
    8, 24 and 32 keywords (up to 347 sets), all within the budget."""
    grammars = [t for _, _, t in fuzz_grammars(16)]
    grammars += [generate_parts(keyword_grammar(k), "kw%d" % k, False, "both") for k in (8, 24, 32)]
    for t in grammars:
        s, keep = native.make_tables(t)
        info = np.zeros(4, dtype=np.int64)
        assert harness.window_info(ctypes.byref(s), info.ctypes.data) == 0, t.name
        assert info[3] == 0 and 0 < info[0] <= 1024, (t.name, info)


def test_lexer_tile_algorithm_rejects_and_lengths(harness, emu):
    from alpacc_b200 import workloads as W
    t = cases.tables("json_ext_i32")
    docs = [b'[1, "' + b"x" * k + b'", 2]' for k in (65533, 65534, 69998)]
    docs += [b"[1," + b" " * 70000 + b"2]", W.json_doc(200000, 3)[:-3] + b"\x02\x03]", b'"' + b"a" * 40000]
    _emu_vs_machine(emu, harness, t, docs)


@pytest.mark.parametrize("nkw", [8, 24, 32])
def test_lexer_tile_algorithm_keyword_lexers(harness, emu, nkw):
    """Machines above 64 states (256-bit candidate sets) and many candidates;
    both window walks (the window machine, and explicit state sets)."""
    t = generate_parts(keyword_grammar(nkw), "kw%d" % nkw, False, "both")
    ins = keyword_inputs(nkw, seed=nkw, sizes=(0, 1, 20, 300, 15000, 40000))
    _emu_vs_machine(emu, harness, t, ins)
    _emu_vs_machine(emu, harness, t, ins, sets=True)


def test_lexer_tile_algorithm_random_grammars(harness, emu):
    for name, g, t in fuzz_grammars(16):
        _emu_vs_machine(emu, harness, t, g.inputs(0, sentences=(8, 300), noise=(500, 15000)))
