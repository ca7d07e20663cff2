"""ctypes binding of the C ABI (include/alpacc_b200.h) and the host-side mirror
of a generated parser's interface.

``Parser(tables)`` uploads one grammar to the GPU; ``parse(data)`` is the
in-memory form of the generated program's ``run_case`` for combined mode
(src/Alpacc/Generator/C/Generator.hs:114-152): it returns a
``wire.ParseResult`` that is either a reject or the tokens with spans plus the
preorder production tree with parents and token parents. ``run_case(data)``
returns the exact response record bytes.

There is no CPU fallback: constructing a ``Parser`` without the native library
or without a GPU raises.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import wire

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libalpacc_b200.so")

OK, REJECT = 0, 1
E_INVALID, E_CUDA, E_NOMEM, E_CAPACITY, E_TIMEOUT, E_UNSUPPORTED, E_ABORTED = -1, -2, -3, -4, -5, -6, -7
ABI_VERSION = 1


class AlpaccError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        super().__init__("alpacc status %d: %s" % (status, msg))
        self.status = status


class Tables(ctypes.Structure):
    _fields_ = [
        ("abi_version", ctypes.c_uint32), ("terminal_size", ctypes.c_uint32), ("production_size", ctypes.c_uint32),
        ("bracket_size", ctypes.c_uint32), ("state_size", ctypes.c_uint32), ("index_size", ctypes.c_uint32),
        ("length_size", ctypes.c_uint32), ("parts", ctypes.c_uint32),
        ("num_states", ctypes.c_uint64), ("endo_mask", ctypes.c_uint64), ("endo_offset", ctypes.c_uint64),
        ("terminal_mask", ctypes.c_uint64), ("terminal_offset", ctypes.c_uint64), ("produce_mask", ctypes.c_uint64),
        ("produce_offset", ctypes.c_uint64), ("identity", ctypes.c_uint64), ("ignore_token", ctypes.c_int64),
        ("to_state", ctypes.c_void_p), ("compose", ctypes.c_void_p), ("accept", ctypes.c_void_p),
        ("q", ctypes.c_uint64), ("k", ctypes.c_uint64), ("empty_terminal", ctypes.c_uint64),
        ("start_terminal", ctypes.c_uint64), ("end_terminal", ctypes.c_uint64), ("hash_table_size", ctypes.c_uint64),
        ("max_iters", ctypes.c_uint64), ("stacks_size", ctypes.c_uint64), ("productions_size", ctypes.c_uint64),
        ("max_brackets_per_position", ctypes.c_uint64), ("max_prods_per_position", ctypes.c_uint64),
        ("stacks", ctypes.c_void_p), ("productions", ctypes.c_void_p), ("hash_table_is_valid", ctypes.c_void_p),
        ("hash_table_keys", ctypes.c_void_p), ("hash_table_stacks_span", ctypes.c_void_p),
        ("hash_table_productions_span", ctypes.c_void_p), ("number_of_productions", ctypes.c_uint64),
        ("production_to_arity", ctypes.c_void_p), ("production_to_terminal_is_valid", ctypes.c_void_p),
    ]


class Result(ctypes.Structure):
    _fields_ = [
        ("valid", ctypes.c_uint8), ("on_device", ctypes.c_uint8), ("reserved0", ctypes.c_uint16),
        ("reserved1", ctypes.c_uint32), ("num_tokens", ctypes.c_uint64), ("num_nodes", ctypes.c_uint64),
        ("token_ids", ctypes.c_void_p), ("token_starts", ctypes.c_void_p), ("token_lengths", ctypes.c_void_p),
        ("node_productions", ctypes.c_void_p), ("node_parents", ctypes.c_void_p), ("token_parents", ctypes.c_void_p),
        ("internal", ctypes.c_void_p),
    ]


# int sink(void *user, uint64_t first, uint64_t count, const void *ids, const void *starts, const void *lengths)
LEX_SINK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p,
                            ctypes.c_void_p, ctypes.c_void_p)

_lib = None


def lib():
    """The native library; raises when it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AlpaccError(E_INVALID, "native library missing: %s (run python -m alpacc_b200.build)" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        L.alpacc_gpu_load.restype = ctypes.c_void_p
        L.alpacc_gpu_load.argtypes = [ctypes.POINTER(Tables), ctypes.c_int, ctypes.c_uint64,
                                      ctypes.POINTER(ctypes.c_int)]
        L.alpacc_gpu_free.argtypes = [ctypes.c_void_p]
        for name in ("alpacc_gpu_parse", "alpacc_gpu_parse_device"):
            f = getattr(L, name)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Result)]
        L.alpacc_gpu_enqueue.restype = ctypes.c_int
        L.alpacc_gpu_enqueue.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64]
        L.alpacc_gpu_collect.restype = ctypes.c_int
        L.alpacc_gpu_collect.argtypes = [ctypes.c_void_p, ctypes.POINTER(Result)]
        L.alpacc_server_start.restype = ctypes.c_void_p
        L.alpacc_server_start.argtypes = [ctypes.POINTER(Tables), ctypes.c_int, ctypes.c_int, ctypes.c_uint64,
                                          ctypes.POINTER(ctypes.c_int)]
        L.alpacc_server_submit.restype = ctypes.c_int
        L.alpacc_server_submit.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                           ctypes.POINTER(ctypes.c_uint64)]
        L.alpacc_server_wait.restype = ctypes.c_int
        L.alpacc_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Result),
                                         ctypes.POINTER(ctypes.c_double)]
        L.alpacc_server_stats.restype = ctypes.c_int
        L.alpacc_server_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
        L.alpacc_server_stop.restype = None
        L.alpacc_server_stop.argtypes = [ctypes.c_void_p]
        for f in (L.alpacc_server_replay, L.alpacc_gpu_replay):
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        L.alpacc_gpu_geometry.restype = ctypes.c_int
        L.alpacc_gpu_geometry.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
        L.alpacc_gpu_autotune.restype = ctypes.c_int
        L.alpacc_gpu_autotune.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                          ctypes.POINTER(ctypes.c_int)]
        L.alpacc_gpu_parse_batch.restype = ctypes.c_int
        L.alpacc_gpu_parse_batch.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                             ctypes.POINTER(Result)]
        L.alpacc_result_free.argtypes = [ctypes.POINTER(Result)]
        L.alpacc_gpu_lex.restype = ctypes.c_int
        L.alpacc_gpu_lex.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(Result)]
        L.alpacc_gpu_lex_stream.restype = ctypes.c_int
        L.alpacc_gpu_lex_stream.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                            LEX_SINK, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64)]
        L.alpacc_gpu_parse_tokens.restype = ctypes.c_int
        L.alpacc_gpu_parse_tokens.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                              ctypes.POINTER(Result)]
        L.alpacc_gpu_layout.restype = ctypes.c_int
        L.alpacc_gpu_layout.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
        L.alpacc_strerror.restype = ctypes.c_char_p
        L.alpacc_strerror.argtypes = [ctypes.c_int]
        L.alpacc_gpu_last_ms.restype = ctypes.c_double
        L.alpacc_gpu_last_ms.argtypes = [ctypes.c_void_p]
        L.alpacc_gpu_info.restype = ctypes.c_int
        L.alpacc_gpu_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
        L.alpacc_gpu_stage_ms.restype = ctypes.c_int
        L.alpacc_gpu_stage_ms.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
        L.alpacc_gpu_counts.restype = ctypes.c_int
        L.alpacc_gpu_counts.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), ctypes.c_int]
        L.alpacc_gpu_set_diagnostics.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.alpacc_gpu_set_stage_timing.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.alpacc_gpu_stream.restype = ctypes.c_void_p
        L.alpacc_gpu_stream.argtypes = [ctypes.c_void_p]
        L.alpacc_gpu_last_error.restype = ctypes.c_char_p
        L.alpacc_gpu_last_error.argtypes = [ctypes.c_void_p]
        L.alpacc_device_allocations.restype = ctypes.c_uint64
        L.alpacc_device_allocations.argtypes = []
        _lib = L
    return _lib


PARTS = {"both": 0, "lexer": 1, "parser": 2}


def make_tables(t):
    """Fill the C struct from generated tables; returns (struct, keepalive).
    The fields of the part a lexer-mode or parser-mode program lacks stay zero
    / NULL, as that program has no such constants."""
    L = t.lexer
    keep = []
    parts = getattr(t, "parts", "both")

    def arr(a, dtype=None):
        a = np.ascontiguousarray(a if dtype is None else np.asarray(a).astype(dtype))
        keep.append(a)
        return a.ctypes.data

    s = Tables()
    s.abi_version = ABI_VERSION
    s.terminal_size = t.terminal_bits // 8
    s.production_size = t.production_bits // 8
    s.bracket_size = t.bracket_bits // 8
    s.state_size = L.state_bits // 8
    s.index_size = t.index_bits // 8
    s.length_size = t.length_bits // 8
    s.parts = PARTS[parts]
    if parts != "parser":
        _lexer_fields(s, t, arr)
    if parts != "lexer":
        _parser_fields(s, t, arr, tree=parts == "both")
    return s, keep


def _lexer_fields(s, t, arr):
    L = t.lexer
    s.num_states = L.num_states
    s.endo_mask, s.endo_offset = L.index_mask, L.index_offset
    s.terminal_mask, s.terminal_offset = L.token_mask, L.token_offset
    s.produce_mask, s.produce_offset = L.produce_mask, L.produce_offset
    s.identity = L.identity
    s.ignore_token = -1 if t.ignore_token is None else t.ignore_token
    s.to_state = arr(L.to_state)
    s.compose = arr(L.compose)
    s.accept = arr(L.accept, np.uint8)


def _parser_fields(s, t, arr, tree: bool):
    s.q, s.k = t.q, t.k
    s.empty_terminal, s.start_terminal, s.end_terminal = t.empty_terminal, t.start_terminal, t.end_terminal
    s.hash_table_size = t.hash_size
    s.max_iters = t.max_iters
    s.stacks_size, s.productions_size = len(t.stacks), len(t.productions)
    s.max_brackets_per_position, s.max_prods_per_position = t.max_brackets_per_pos, t.max_prods_per_pos
    s.stacks = arr(t.stacks)
    s.productions = arr(t.productions)
    s.hash_table_is_valid = arr(t.ht_valid, np.uint8)
    tw = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[t.terminal_bits // 8]
    s.hash_table_keys = arr(t.ht_keys, tw)
    s.hash_table_stacks_span = arr(t.ht_stack_span, np.int64)
    s.hash_table_productions_span = arr(t.ht_prod_span, np.int64)
    if tree:
        s.number_of_productions = t.num_productions
        s.production_to_arity = arr(t.arity, np.uint64)
        s.production_to_terminal_is_valid = arr(t.prod_is_terminal, np.uint8)


def _np_from(ptr, count, nbytes, signed=False):
    if count == 0:
        return np.zeros(0, dtype=np.dtype(("i" if signed else "u") + str(nbytes)))
    dt = np.dtype(("i" if signed else "u") + str(nbytes))
    buf = (ctypes.c_char * (count * nbytes)).from_address(ptr)
    return np.frombuffer(buf, dtype=dt, count=count).copy()



def _replay(fn, handle, pool: bytes, offsets, doc, arrival_s):
    """Shared body of the trace replays: (latency ms, status, elapsed s)."""
    buf = np.frombuffer(pool, dtype=np.uint8)
    offs = np.ascontiguousarray(offsets, dtype=np.int64)
    doc = np.ascontiguousarray(doc, dtype=np.uint32)
    arr = np.ascontiguousarray(arrival_s, dtype=np.float64)
    n = len(doc)
    lat = np.zeros(n, dtype=np.float64)
    st = np.zeros(n, dtype=np.int32)
    el = ctypes.c_double(0)
    rc = fn(handle, buf.ctypes.data if buf.size else None, offs.ctypes.data, doc.ctypes.data, n, arr.ctypes.data,
            lat.ctypes.data, st.ctypes.data, ctypes.byref(el))
    if rc < 0:
        raise AlpaccError(rc, lib().alpacc_strerror(rc).decode())
    return lat, st, el.value


class Parser:
    """One grammar resident on one GPU (``alpacc_gpu_load``)."""

    def __init__(self, tables, device: int = 0, max_input: int = 0):
        self.tables = tables
        self.layout = wire.Layout.of(tables)
        self._struct, self._keep = make_tables(tables)
        err = ctypes.c_int(0)
        self._lib = lib()
        self._h = self._lib.alpacc_gpu_load(ctypes.byref(self._struct), device, max_input, ctypes.byref(err))
        if not self._h:
            raise AlpaccError(err.value, lib().alpacc_strerror(err.value).decode())

    def close(self):
        if getattr(self, "_h", None):
            # the instance's own reference: module globals may be gone at interpreter exit
            self._lib.alpacc_gpu_free(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def info(self) -> dict:
        vals = (ctypes.c_int64 * 16)()
        n = lib().alpacc_gpu_info(self._h, vals, 16)
        keys = ["M", "C", "max_lanes", "reachable", "dead", "nt", "records", "lex_grid", "lex_reject_reason",
                "parse_reject_reason", "timeout_site", "pair_hashed", "lex_variant", "window_sets"]
        return dict(zip(keys, [vals[i] for i in range(min(n, len(keys)))]))

    def _check(self, rc: int) -> int:
        if rc < 0:
            raise AlpaccError(rc, "%s (%s)" % (lib().alpacc_strerror(rc).decode(),
                                              lib().alpacc_gpu_last_error(self._h).decode()))
        return rc

    def _result(self, r: Result, rc: int) -> wire.ParseResult:
        if rc != OK:
            return wire.ParseResult(False)
        lay = self.layout
        T, N = r.num_tokens, r.num_nodes
        return wire.ParseResult(
            True,
            _np_from(r.token_ids, T, lay.terminal), _np_from(r.token_starts, T, lay.index, True),
            _np_from(r.token_lengths, T, lay.length), _np_from(r.node_productions, N, lay.production),
            _np_from(r.node_parents, N, lay.index, True), _np_from(r.token_parents, T, lay.index, True))

    def parse(self, data) -> wire.ParseResult:
        """Host bytes in, host result out (H2D, device path, D2H)."""
        a = np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data
        a = np.ascontiguousarray(a, dtype=np.uint8)
        r = Result()
        rc = self._check(lib().alpacc_gpu_parse(self._h, a.ctypes.data, a.size, ctypes.byref(r)))
        try:
            return self._result(r, rc)
        finally:
            lib().alpacc_result_free(ctypes.byref(r))

    def lex(self, data) -> wire.LexResult:
        """Lexer-only mode (``alpacc_gpu_lex``): the lexemes of the input, or a
        reject."""
        a = np.ascontiguousarray(np.frombuffer(bytes(data), dtype=np.uint8))
        r = Result()
        rc = self._check(lib().alpacc_gpu_lex(self._h, a.ctypes.data, a.size, ctypes.byref(r)))
        try:
            if rc != OK:
                return wire.LexResult(False)
            lay, T = self.layout, r.num_tokens
            return wire.LexResult(True, _np_from(r.token_ids, T, lay.terminal),
                                  _np_from(r.token_starts, T, lay.index, True),
                                  _np_from(r.token_lengths, T, lay.length))
        finally:
            lib().alpacc_result_free(ctypes.byref(r))

    def lex_stream(self, data, window: int = 0, on_window=None):
        """Chunked lexing (``alpacc_gpu_lex_stream``): the input is lexed in
        windows of ``window`` bytes (0: 1 GiB). Without ``on_window`` the
        windows' lexemes are concatenated into one ``wire.LexResult``; with it,
        ``on_window(first, ids, starts, lengths)`` gets each window's arrays
        and nothing is kept. Returns (result or None, number of windows)."""
        a = data if isinstance(data, np.ndarray) else np.frombuffer(bytes(data), dtype=np.uint8)
        a = np.ascontiguousarray(a, dtype=np.uint8)
        lay = self.layout
        parts = []
        calls = [0]

        def sink(user, first, count, ids, starts, lens):
            calls[0] += 1
            arrs = (_np_from(ids, count, lay.terminal), _np_from(starts, count, lay.index, True),
                    _np_from(lens, count, lay.length))
            if on_window is not None:
                on_window(first, *arrs)
            else:
                parts.append(arrs)
            return 0

        cb = LEX_SINK(sink)
        nt = ctypes.c_uint64(0)
        rc = self._check(lib().alpacc_gpu_lex_stream(self._h, a.ctypes.data if a.size else None, a.size, window,
                                                     cb, None, ctypes.byref(nt)))
        if rc != OK:
            return wire.LexResult(False), calls[0]
        if on_window is not None:
            return None, calls[0]
        cat = [np.concatenate([p[i] for p in parts]) if parts else _np_from(0, 0, w, i == 1)
               for i, w in enumerate((lay.terminal, lay.index, lay.length))]
        return wire.LexResult(True, *cat), calls[0]

    def parse_tokens(self, tokens) -> wire.TokenParseResult:
        """Parser-only mode (``alpacc_gpu_parse_tokens``): terminal ids in, the
        production sequence of the derivation (or a reject) out."""
        lay = self.layout
        a = np.ascontiguousarray(np.asarray(tokens).astype(wire._dt(lay.terminal)))
        r = Result()
        rc = self._check(lib().alpacc_gpu_parse_tokens(self._h, a.ctypes.data if a.size else None, a.size,
                                                       ctypes.byref(r)))
        try:
            if rc != OK:
                return wire.TokenParseResult(False)
            return wire.TokenParseResult(True, _np_from(r.node_productions, r.num_nodes, lay.production))
        finally:
            lib().alpacc_result_free(ctypes.byref(r))

    def autotune(self, dev_ptr: int, n: int) -> int:
        """Tune the launch geometry on a device-resident sample
        (alpacc_gpu_autotune); returns the lexer's CTAs per SM."""
        c = ctypes.c_int(0)
        self._check(lib().alpacc_gpu_autotune(self._h, dev_ptr, n, ctypes.byref(c)))
        return c.value


    def geometry(self) -> dict:
        """The launch geometry (alpacc_gpu_geometry)."""
        v = (ctypes.c_int64 * 6)()
        lib().alpacc_gpu_geometry(self._h, v, 6)
        return {"lex_window_bytes": v[0], "lex_ctas_per_sm": v[1], "pair_ctas_per_sm": v[2],
                "walk_ctas_per_sm": v[3], "from_cache": bool(v[4]), "grammar_digest": "%016x" % (v[5] & (2**64 - 1))}
    def parse_batch(self, docs) -> list:
        """Many independent inputs in one batched call; one ParseResult each."""
        parts = [bytes(d) for d in docs]
        offs = np.zeros(len(parts) + 1, dtype=np.int64)
        offs[1:] = np.cumsum([len(p) for p in parts])
        buf = np.frombuffer(b"".join(parts) or b"\0", dtype=np.uint8)
        outs = (Result * max(len(parts), 1))()
        self._check(lib().alpacc_gpu_parse_batch(self._h, buf.ctypes.data, offs.ctypes.data, len(parts), outs))
        try:
            return [self._result(outs[i], OK if outs[i].valid else REJECT) for i in range(len(parts))]
        finally:
            for i in range(len(parts)):
                lib().alpacc_result_free(ctypes.byref(outs[i]))

    def parse_batch_raw(self, buf_ptr: int, offs_ptr: int, count: int):
        """Batch from raw pointers (bytes, int64 offsets[count+1]); returns the
        Result array; release each with ``free_result``."""
        outs = (Result * max(count, 1))()
        self._check(lib().alpacc_gpu_parse_batch(self._h, buf_ptr, offs_ptr, count, outs))
        return outs

    def parse_device(self, dev_ptr: int, n: int):
        """Bytes already on the device. Returns (status, Result with device pointers)."""
        r = Result()
        rc = self._check(lib().alpacc_gpu_parse_device(self._h, dev_ptr, n, ctypes.byref(r)))
        return rc, r

    def device_result(self, r: Result, rc: int) -> wire.ParseResult:
        """Copy a device result (from ``parse_device``) to host arrays."""
        if rc != OK:
            return wire.ParseResult(False)
        import torch

        lay = self.layout

        def dl(ptr, count, nbytes, signed=False):
            if count == 0:
                return np.zeros(0, dtype=np.dtype(("i" if signed else "u") + str(nbytes)))
            host = np.empty(count * nbytes, dtype=np.uint8)
            torch.cuda.synchronize()
            _cudart_memcpy_d2h(host.ctypes.data, ptr, count * nbytes)
            return host.view(np.dtype(("i" if signed else "u") + str(nbytes)))

        T, N = r.num_tokens, r.num_nodes
        return wire.ParseResult(True, dl(r.token_ids, T, lay.terminal), dl(r.token_starts, T, lay.index, True),
                                dl(r.token_lengths, T, lay.length), dl(r.node_productions, N, lay.production),
                                dl(r.node_parents, N, lay.index, True), dl(r.token_parents, T, lay.index, True))

    def run_case(self, data) -> bytes:
        """The response record bytes ``run_case`` of this grammar's program
        (combined, lexer-mode or parser-mode) would write; for the parser-mode
        program ``data`` is the terminal ids' bytes."""
        parts = getattr(self.tables, "parts", "both")
        if parts == "lexer":
            return wire.encode_lex_record(self.lex(data), self.layout)
        if parts == "parser":
            toks = np.frombuffer(bytes(data), dtype=wire._dt(self.layout.terminal))
            return wire.encode_token_parse_record(self.parse_tokens(toks), self.layout)
        return wire.encode_record(self.parse(data), self.layout)

    def counts(self) -> dict:
        """Tokens, brackets, productions, nodes of the last call; lexer
        diagnostic counters; kernel launches; per-phase SM cycles of the lexer
        and of the two walks' tile kernels (diagnostics on)."""
        vals = (ctypes.c_int64 * 33)()
        lib().alpacc_gpu_counts(self._h, vals, 33)
        walk_phases = ("load_scan", "windows", "near_queries", "queued_queries", "lookback", "staircase",
                       "tree", "next_tile")
        return {"T": vals[0], "B": vals[1], "P": vals[2], "N": vals[3], "lookback_tiles": vals[4],
                "known_chunks": vals[5], "chain_evals": vals[6], "candidate_jobs": vals[7], "launches": vals[8],
                "lexer_phase_cycles": {k: vals[9 + i] for i, k in enumerate(
                    ("load", "window", "walks", "known_scan", "start_states", "open_codes_masks_scan",
                     "count_lookback", "writes"))},
                "bracket_walk_phase_cycles": {k: vals[17 + i] for i, k in enumerate(walk_phases)},
                "parent_walk_phase_cycles": {k: vals[25 + i] for i, k in enumerate(walk_phases)}}

    def set_diagnostics(self, on: bool):
        lib().alpacc_gpu_set_diagnostics(self._h, 1 if on else 0)

    def set_stage_timing(self, on: bool):
        """Record per-stage device times (stage_ms); off by default."""
        lib().alpacc_gpu_set_stage_timing(self._h, 1 if on else 0)

    def stream_handle(self) -> int:
        """The cudaStream_t the handle launches on."""
        return lib().alpacc_gpu_stream(self._h)

    def parse_raw(self, host_ptr: int, n: int):
        """Host pointer in (ideally pinned), host result out; returns (status,
        Result); release it with ``free_result``."""
        r = Result()
        rc = self._check(lib().alpacc_gpu_parse(self._h, host_ptr, n, ctypes.byref(r)))
        return rc, r

    @staticmethod
    def free_result(r: Result):
        lib().alpacc_result_free(ctypes.byref(r))

    def replay(self, pool: bytes, offsets, doc, arrival_s):
        """One plain parse per request of a timed trace (alpacc_gpu_replay):
        request i is input doc[i] of the pool, arriving arrival_s[i] seconds
        after the start. Returns (latency ms, status, elapsed s)."""
        return _replay(self._lib.alpacc_gpu_replay, self._h, pool, offsets, doc, arrival_s)

    def record_digest_raw(self, host_ptr: int, n: int):
        """(status, SHA-256 hex, byte count) of the combined-mode response
        record for the host input at ``host_ptr``: the result arrays are
        hashed in place, in record order (valid byte, T, ids, starts,
        lengths, N, productions, parents, token parents), so a record of
        several GB is never assembled."""
        import hashlib
        import struct

        rc, r = self.parse_raw(host_ptr, n)
        h = hashlib.sha256()
        try:
            if rc != OK:
                h.update(b"\x00")
                return rc, h.hexdigest(), 1
            lay = self.layout
            T, N = r.num_tokens, r.num_nodes
            size = 0
            for ptr, nbytes in ((None, b"\x01" + struct.pack("<Q", T)),
                                (r.token_ids, T * lay.terminal), (r.token_starts, T * lay.index),
                                (r.token_lengths, T * lay.length), (None, struct.pack("<Q", N)),
                                (r.node_productions, N * lay.production), (r.node_parents, N * lay.index),
                                (r.token_parents, T * lay.index)):
                if ptr is None:
                    h.update(nbytes)
                    size += len(nbytes)
                elif nbytes:
                    h.update((ctypes.c_uint8 * nbytes).from_address(ptr))
                    size += nbytes
            return rc, h.hexdigest(), size
        finally:
            self.free_result(r)

    def last_ms(self) -> float:
        return lib().alpacc_gpu_last_ms(self._h)

    STAGES = ("lex", "pairs", "bracket_walk", "bracket_resolve", "parent_walk", "parent_resolve")

    def stage_ms(self) -> dict:
        vals = (ctypes.c_double * 8)()
        lib().alpacc_gpu_stage_ms(self._h, vals, 8)
        return {k: vals[i] for i, k in enumerate(self.STAGES)}


_cudart = None


def _cudart_memcpy_d2h(dst: int, src: int, nbytes: int):
    global _cudart
    if _cudart is None:
        import glob
        cands = glob.glob("/usr/local/cuda/lib64/libcudart.so*")
        _cudart = ctypes.CDLL(cands[0]) if cands else ctypes.CDLL("libcudart.so")
        _cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    rc = _cudart.cudaMemcpy(dst, src, nbytes, 2)
    if rc != 0:
        raise AlpaccError(E_CUDA, "cudaMemcpy failed (%d)" % rc)


class Server:
    """In-process request server with continuous batching (alpacc_server_*)."""

    def __init__(self, tables, device: int = 0, workers: int = 2, budget: int = 8 << 30):
        self._struct, self._keep = make_tables(tables)
        self.layout = wire.Layout.of(tables)
        self._lib = lib()
        err = ctypes.c_int(0)
        self._s = self._lib.alpacc_server_start(ctypes.byref(self._struct), device, workers, budget, ctypes.byref(err))
        if not self._s:
            raise AlpaccError(err.value, self._lib.alpacc_strerror(err.value).decode())

    def submit(self, data) -> int:
        a = np.frombuffer(bytes(data), dtype=np.uint8)
        rid = ctypes.c_uint64(0)
        rc = self._lib.alpacc_server_submit(self._s, a.ctypes.data if a.size else None, a.size, ctypes.byref(rid))
        if rc < 0:
            raise AlpaccError(rc, self._lib.alpacc_strerror(rc).decode())
        return rid.value

    def wait(self, rid: int):
        """(ParseResult, latency ms from submit to completion)."""
        r = Result()
        ms = ctypes.c_double(0)
        rc = self._lib.alpacc_server_wait(self._s, rid, ctypes.byref(r), ctypes.byref(ms))
        if rc < 0:
            raise AlpaccError(rc, self._lib.alpacc_strerror(rc).decode())
        try:
            if rc != OK:
                return wire.ParseResult(False), ms.value
            lay = self.layout
            T, N = r.num_tokens, r.num_nodes
            return wire.ParseResult(
                True,
                _np_from(r.token_ids, T, lay.terminal), _np_from(r.token_starts, T, lay.index, True),
                _np_from(r.token_lengths, T, lay.length), _np_from(r.node_productions, N, lay.production),
                _np_from(r.node_parents, N, lay.index, True), _np_from(r.token_parents, T, lay.index, True)), ms.value
        finally:
            self._lib.alpacc_result_free(ctypes.byref(r))

    def replay(self, pool: bytes, offsets, doc, arrival_s):
        """The trace submitted from a native thread at its arrival times
        (alpacc_server_replay). Returns (latency ms, status, elapsed s)."""
        return _replay(self._lib.alpacc_server_replay, self._s, pool, offsets, doc, arrival_s)

    def stats(self) -> dict:
        v = (ctypes.c_int64 * 6)()
        self._lib.alpacc_server_stats(self._s, v, 6)
        return {"batches": v[0], "served": v[1], "largest_batch": v[2], "queued": v[3], "max_scratch_held": v[4],
                "scratch_share": v[5]}

    def close(self):
        if getattr(self, "_s", None):
            self._lib.alpacc_server_stop(self._s)
            self._s = None

    def __del__(self):
        self.close()
