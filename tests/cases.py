"""Shared test inputs: grammar configurations and seeded input families."""

from __future__ import annotations

import os

import numpy as np

from alpacc_b200 import workloads as W
from alpacc_b200.grammar.cache import load_tables

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GRAMMARS = os.path.join(REPO, "grammars")

# oracle/_ref configuration -> (grammar file, index32)
CONFIGS = {
    "arithmetic_i64": ("arithmetic.alp", False),
    "arithmetic_i32": ("arithmetic.alp", True),
    "json_i32": ("json.alp", True),
    "json_ext_i32": ("json_ext.alp", True),
    "json_ext_i64": ("json_ext.alp", False),
    "sexp_i64": ("sexp.alp", False),
    "sexp_i32": ("sexp.alp", True),
    "paper_grammar_i64": ("paper_grammar.alp", False),
    "list_i64": ("list.alp", False),
    "llp01_i64": ("llp01.alp", False),
}

# configurations whose lexer-mode and parser-mode programs are tested too
MODE_CONFIGS = ("arithmetic_i64", "json_i32", "json_ext_i32", "sexp_i64", "paper_grammar_i64", "llp01_i64")

_TABLES = {}


def tables(config: str, parts: str = "both"):
    """Tables of the combined program of ``config``, or of its lexer-mode /
    parser-mode program."""
    if (config, parts) not in _TABLES:
        g, i32 = CONFIGS[config]
        _TABLES[(config, parts)] = load_tables(os.path.join(GRAMMARS, g), index32=i32, parts=parts)
    return _TABLES[(config, parts)]


def mode_name(config: str, parts: str) -> str:
    """Name of the reference program built for ``config`` in that mode."""
    return config if parts == "both" else "%s_%s" % (config, parts)


FIXED = {
    "arithmetic": [b"", b" ", b"\n\t ", b"1", b"x", b"12+(3*4)", b"12+(3+4)", b"a - 1", b"a-1", b"(((a)))",
                   b"-5*-6", b"1 +", b"()", b"a b", b"1+2+", b"((1)", b"1)", b"9999999999999999999",
                   b"a+b*c/d-e", b"(a+(b*(c-(d/e))))", b"\xff", b"1 2"],
    "json": [b"", b" ", b"0", b"-1.5", b"\"\"", b"\"abc def\"", b"[]", b"{}", b"[1,2,3]", b"{\"a\":1,\"b\":[true,false,null]}",
             b"[[[[[]]]]]", b"[1,]", b"{\"a\"}", b"nul", b"true false", b"[1 2]", b"{\"k\":{\"k\":{\"k\":[]}}}",
             b"  [ 1 , 2 ]  ", b"\"unterminated", b"[\"a\\\"b\", \"\\u00e9\"]", b"1.", b"01", b"[-]"],
    "sexp": [b"", b" ", b"a", b"()", b"(a)", b"(a b c)", b"((a) (b (c d)) e)", b"(", b")", b"(a))", b"((a)",
             b"(a (b) ) (c)", b"  ( x1 y2 )  ", b"(((((((((((a)))))))))))"],
    "paper_grammar": [b"", b"1", b"1+2", b"[1+2]+3", b"[[1]]", b"1+", b"[1", b"1 + [ 2 + 3 ]"],
    "list": [b"", b"[]", b"[a]", b"[a,a,a]", b"[a,]", b"[,a]", b"a"],
    "llp01": [b"", b"[]", b"[][]", b"[[]]", b"[[][]][]", b"[", b"]", b"[]]"],
}


def family(config: str) -> str:
    g = CONFIGS[config][0]
    if g.startswith("json"):
        return "json"
    return g[:-4]


def mutate(data: bytes, rng: np.random.Generator, k: int = 3) -> bytes:
    b = bytearray(data)
    for _ in range(k):
        if not b:
            b.append(int(rng.integers(32, 127)))
            continue
        op = int(rng.integers(0, 3))
        i = int(rng.integers(0, len(b)))
        if op == 0:
            b[i] = int(rng.integers(0, 256)) if rng.random() < 0.2 else int(rng.integers(32, 127))
        elif op == 1:
            del b[i]
        else:
            b.insert(i, int(rng.integers(32, 127)))
    return bytes(b)


def generated(config: str, n: int, seed: int) -> bytes:
    f = family(config)
    if f == "json":
        if config.startswith("json_i32"):
            return simple_json(n, seed)
        return W.json_doc(n, seed)
    if f == "arithmetic":
        return W.arithmetic(n, seed)
    if f == "sexp":
        return W.sexp_doc(n, seed, max_depth=min(200, max(1, n // 64)))
    rng = np.random.default_rng(seed)
    fixed = FIXED[f]
    return fixed[int(rng.integers(0, len(fixed)))]


def simple_json(n: int, seed: int) -> bytes:
    """JSON within the reference json.alp's lexical subset (alnum/space strings,
    no exponents, no escapes)."""
    rng = np.random.default_rng(seed)
    alnum = b"abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ0123456789 "

    def val(d):
        x = rng.random()
        if d < 4 and x < 0.3:
            k = int(rng.integers(0, 5))
            return b"[" + b",".join(val(d + 1) for _ in range(k)) + b"]"
        if d < 4 and x < 0.5:
            k = int(rng.integers(0, 5))
            return b"{" + b",".join(s() + b":" + val(d + 1) for _ in range(k)) + b"}"
        if x < 0.7:
            return s()
        if x < 0.9:
            v = str(int(rng.integers(-1000, 100000))).encode()
            if rng.random() < 0.4:
                v += b"." + str(int(rng.integers(0, 1000))).encode()
            return v
        return (b"true", b"false", b"null")[int(rng.integers(0, 3))]

    def s():
        k = int(rng.integers(0, 12))
        return b'"' + bytes(alnum[int(i)] for i in rng.integers(0, len(alnum), k)) + b'"'

    parts = []
    size = 2
    while size < n:
        e = val(0)
        if size + len(e) + 1 > n and parts:
            break
        parts.append(e)
        size += len(e) + 1
    doc = b"[" + b",".join(parts) + b"]"
    if len(doc) > n:
        doc = b"[]"
    return doc + b" " * (n - len(doc))


# sizes around the lexer's tile geometry: tiles of 15360 bytes (256 chunks of
# 60 bytes, each also reading the 16 bytes before it)
TILE_SIZES = (1, 7, 16, 17, 60, 61, 64, 76, 1000, 15359, 15360, 15361, 15376, 30720, 30721, 40000)


def case_inputs(config: str, sizes=TILE_SIZES, seeds=(0, 1)):
    """Fixed cases, generated documents of several sizes, and mutations."""
    f = family(config)
    out = list(FIXED[f])
    rng = np.random.default_rng(1234)
    for n in sizes:
        for s in seeds:
            d = generated(config, max(n, 2) if f != "sexp" else max(n, 4), 100 + s + n)
            out.append(d)
            out.append(mutate(d, rng, 1 + int(rng.integers(0, 3))))
    return out


def token_inputs(config: str, sizes=(1, 64, 1000, 20000), seeds=(0,)):
    """Parser-mode inputs for ``config`` (see ``token_inputs_for``)."""
    return token_inputs_for(tables(config), case_inputs(config, sizes=sizes, seeds=seeds))


def token_inputs_for(t, inputs, seed: int = 4321):
    """Parser-mode inputs (terminal ids as bytes at terminal_t width): the
    tokens of the accepted inputs under the combined tables ``t``, and
    mutations of them that delete, swap or insert ids, including ids outside
    the grammar's terminal range."""
    from alpacc_b200 import wire
    from oracle.port import PortOracle

    lay = wire.Layout.of(t)
    dt = np.dtype("<u%d" % lay.terminal)
    po = PortOracle(t)
    rng = np.random.default_rng(seed)
    hi = min(256, 1 << t.terminal_bits)
    out = [b""]
    for data in inputs:
        r, _ = wire.decode_record(po.run_case(data), lay)
        if not r.valid:
            continue
        ids = np.asarray(r.token_ids, dtype=np.int64)
        out.append(ids.astype(dt).tobytes())
        for _ in range(2):
            m = list(ids)
            for _ in range(1 + int(rng.integers(0, 3))):
                op = int(rng.integers(0, 3))
                if op == 0 and m:
                    del m[int(rng.integers(0, len(m)))]
                elif op == 1 and len(m) > 1:
                    i, j = rng.integers(0, len(m), 2)
                    m[i], m[j] = m[j], m[i]
                else:
                    m.insert(int(rng.integers(0, len(m) + 1)), int(rng.integers(0, hi)))
            out.append(np.asarray(m, dtype=np.int64).astype(dt).tobytes())
    return out
