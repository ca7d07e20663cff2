"""On-disk cache of generated grammar tables.

Generating the tables of a large lexer (e.g. full JSON strings and numbers:
~3.8k endomorphisms) takes seconds; the result depends only on the grammar text
and the index width, so it is stored as an ``.npz`` under ``_cache/`` next to
this file, keyed by a hash of both and of the generator sources.
"""

from __future__ import annotations

import dataclasses
import hashlib
import json
import os

import numpy as np

from . import lexgen
from .tables import GrammarTables, generate_parts

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE_DIR = os.path.join(HERE, "_cache")
_SOURCES = ("syntax.py", "lexgen.py", "closure.c", "llp.py", "tables.py")

_ARRAYS = ("stacks", "productions", "ht_valid", "ht_keys", "ht_stack_span", "ht_prod_span", "arity",
           "prod_is_terminal")
_LEX_ARRAYS = ("to_state", "compose", "accept")
_SCALARS = ("name", "q", "k", "index32", "terminal_bits", "production_bits", "bracket_bits", "length_bits",
            "ignore_token", "dead_token", "empty_terminal", "start_terminal", "end_terminal", "max_iters",
            "max_brackets_per_pos", "max_prods_per_pos", "terminal_names", "production_names", "parts")
_LEX_SCALARS = ("state_bits", "num_states", "index_mask", "index_offset", "token_mask", "token_offset",
                "produce_mask", "produce_offset", "identity", "num_dfa_states")


def _generator_hash() -> str:
    h = hashlib.sha256()
    for s in _SOURCES:
        p = os.path.join(HERE, s)
        if os.path.exists(p):
            with open(p, "rb") as f:
                h.update(f.read())
    return h.hexdigest()[:16]


def _key(text: str, name: str, index32: bool, parts: str = "both") -> str:
    h = hashlib.sha256()
    h.update(text.encode("utf-8"))
    h.update(b"\0%d\0" % int(index32))
    h.update(_generator_hash().encode())
    suffix = "" if parts == "both" else "_" + parts
    return "%s_%s%s_%s" % (name, "i32" if index32 else "i64", suffix, h.hexdigest()[:16])


def save(t: GrammarTables, path: str) -> None:
    arrays = {a: getattr(t, a) for a in _ARRAYS}
    arrays.update({"lex_" + a: getattr(t.lexer, a) for a in _LEX_ARRAYS})
    meta = {s: getattr(t, s) for s in _SCALARS}
    meta.update({"lex_" + s: getattr(t.lexer, s) for s in _LEX_SCALARS})
    tmp = path + ".tmp.npz"
    np.savez_compressed(tmp, meta=np.array(json.dumps(meta)), **arrays)
    os.replace(tmp, path)


def read(path: str) -> GrammarTables:
    z = np.load(path, allow_pickle=False)
    meta = json.loads(str(z["meta"]))
    lex = lexgen.EncodedLexer(**{s: meta["lex_" + s] for s in _LEX_SCALARS},
                              **{a: z["lex_" + a] for a in _LEX_ARRAYS})
    return GrammarTables(lexer=lex, **{s: meta[s] for s in _SCALARS}, **{a: z[a] for a in _ARRAYS})


def load_tables(path: str, index32: bool = False, parts: str = "both") -> GrammarTables:
    """Tables for the grammar file at ``path`` (of the combined, lexer-mode
    or parser-mode program), generated once and cached."""
    with open(path, "r", encoding="utf-8") as f:
        text = f.read()
    name = os.path.splitext(os.path.basename(path))[0]
    return tables_for_text(text, name, index32, parts)


def tables_for_text(text: str, name: str, index32: bool = False, parts: str = "both") -> GrammarTables:
    if parts == "parser":  # the combined tables' parser part (no cache file of its own)
        t = tables_for_text(text, name, index32, "both")
        return dataclasses.replace(t, parts="parser")
    os.makedirs(CACHE_DIR, exist_ok=True)
    p = os.path.join(CACHE_DIR, _key(text, name, index32, parts) + ".npz")
    if os.path.exists(p):
        try:
            return read(p)
        except Exception:
            pass
    t = generate_parts(text, name=name, index32=index32, parts=parts)
    save(t, p)
    return t
