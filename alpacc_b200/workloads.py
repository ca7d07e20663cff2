"""Seeded synthetic inputs with the shapes of the measured configurations.

* ``arithmetic(n, seed)``  - one expression of the arithmetic grammar padded with
  spaces to exactly ``n`` bytes: numbers of 1-6 digits (20% negative), variables
  of 1-8 letters, operators uniform over ``+ - * /``, parenthesised
  subexpressions with p=0.15 up to depth 8, 0-2 separators from space/\\n/\\t/\\r
  (at least one after a binary ``-`` that precedes a digit, which would
  otherwise lex as a negative number).
* ``json_doc(n, seed)``    - one JSON document (a top-level array) of exactly
  ``n`` bytes: nesting depth geometric(p=0.3) capped at 16, containers of 0-12
  members, strings of printable ASCII of length 0-32 with 5% backslash escapes,
  numbers as ints of up to 10 digits or decimals with optional exponent, one in
  eight separators padded with 1-4 whitespace characters.
* ``sexp_doc(n, seed, unbalanced)`` - one outer list of forms; each form is a
  spine of nested lists with depth drawn from U[1, max_depth], 1-6 children
  per list, atoms ``[a-z0-9]{1,10}``, single spaces; optionally a fraction of
  forms carries one extra ``)``.
* ``json_batch(count, seed)`` / ``json_trace(...)`` - many documents of
  log-normal length (median 8 KiB / 16 KiB) for the batched and served forms.

Large inputs are assembled from a seeded pool of generated elements, so a
256 MiB document takes seconds; every byte sequence is deterministic in the seed.
"""

from __future__ import annotations

import numpy as np

PRINTABLE = [chr(c) for c in range(0x20, 0x7F) if chr(c) not in '"\\']
ESCAPES = ['\\"', "\\\\", "\\/", "\\b", "\\f", "\\n", "\\r", "\\t"]
WS = " \n\t\r"


class _Json:
    def __init__(self, rng: np.random.Generator):
        self.r = rng

    def string(self) -> str:
        r = self.r
        n = int(r.integers(0, 33))
        out = []
        for _ in range(n):
            if r.random() < 0.05:
                if r.random() < 0.2:
                    out.append("\\u%04x" % int(r.integers(0, 0x10000)))
                else:
                    out.append(ESCAPES[int(r.integers(0, len(ESCAPES)))])
            else:
                out.append(PRINTABLE[int(r.integers(0, len(PRINTABLE)))])
        return '"' + "".join(out) + '"'

    def number(self) -> str:
        r = self.r
        digits = int(r.integers(1, 11))
        s = str(int(r.integers(1, 10))) + "".join(str(int(x)) for x in r.integers(0, 10, digits - 1))
        if digits == 1 and r.random() < 0.1:
            s = "0"
        if r.random() < 0.2:
            s = "-" + s
        if r.random() < 0.4:  # decimal
            s += "." + "".join(str(int(x)) for x in r.integers(0, 10, int(r.integers(1, 7))))
            if r.random() < 0.3:
                s += ("e" if r.random() < 0.5 else "E") + ("", "+", "-")[int(r.integers(0, 3))] + str(
                    int(r.integers(0, 400)))
        return s

    def sep(self, s: str) -> str:
        if self.r.random() < 0.125:
            pad = "".join(WS[int(x)] for x in self.r.integers(0, 4, int(self.r.integers(1, 5))))
            return s + pad
        return s

    def scalar(self) -> str:
        x = self.r.random()
        if x < 0.45:
            return self.string()
        if x < 0.9:
            return self.number()
        return ("true", "false", "null")[int(self.r.integers(0, 3))]

    def container(self, depth: int) -> str:
        """A container nested ``depth`` levels deep: one member (at a random
        position) carries the nesting on, the others are scalars or, rarely,
        shallow containers."""
        r = self.r
        n = int(r.integers(1 if depth > 1 else 0, 13))
        spine = int(r.integers(0, n)) if n else -1
        vals = []
        for i in range(n):
            if i == spine and depth > 1:
                vals.append(self.container(depth - 1))
            elif depth > 1 and r.random() < 0.05:
                vals.append(self.container(1))
            else:
                vals.append(self.scalar())
        if r.random() < 0.5:
            return "[" + self.sep(",").join(vals) + "]" if n else "[]"
        items = [self.string() + self.sep(":") + v for v in vals]
        return "{" + self.sep(",").join(items) + "}" if n else "{}"

    def element(self) -> str:
        """A top-level member: nesting depth geometric(p=0.3) capped at 16
        (depth 0 is a scalar)."""
        d = min(16, int(self.r.geometric(0.3)) - 1)
        return self.container(d) if d > 0 else self.scalar()


def _pool_concat(pool, rng, budget: int, sep: bytes):
    """Concatenate pool elements chosen with replacement until ``budget`` bytes."""
    lens = np.array([len(p) for p in pool], dtype=np.int64) + len(sep)
    est = int(budget / lens.mean()) + 16
    picks = rng.integers(0, len(pool), est)
    cum = np.cumsum(lens[picks])
    k = int(np.searchsorted(cum, budget, side="right"))
    picks = picks[:k]
    return sep.join(pool[i] for i in picks)


def json_doc(n: int, seed: int = 2, pool_size: int = 4096) -> bytes:
    """A top-level JSON array of exactly ``n`` bytes (whitespace padded)."""
    rng = np.random.default_rng(seed)
    g = _Json(rng)
    if n < 2:
        raise ValueError("n must be >= 2")
    pool = [g.element().encode() for _ in range(pool_size)]
    body = _pool_concat([p for p in pool if len(p) < max(8, n // 4)] or [b"0"], rng, n - 2, b",")
    doc = b"[" + body + b"]"
    if len(doc) > n:
        doc = b"[]"
    return doc + b" " * (n - len(doc))


def json_small(n: int, seed: int) -> bytes:
    """One JSON value generated to about ``n`` bytes (for batches), padded."""
    rng = np.random.default_rng(seed)
    g = _Json(rng)
    parts = []
    size = 2
    while size < n:
        e = g.element().encode()
        if size + len(e) + 1 > n and parts:
            break
        parts.append(e)
        size += len(e) + 1
    doc = b"[" + b",".join(parts) + b"]"
    if len(doc) > n:
        doc = b"[]"
    return doc + b" " * (n - len(doc))


def _arith_expr(rng, depth: int, out: list, budget: int):
    """E0 := E1 (op E1)* ; E1 := E2 ; E2 := num | var | ( E0 )."""

    def seps(force=False):
        k = int(rng.integers(0, 3))
        if force and k == 0:
            k = 1
        out.append("".join(" \n\t\r"[int(x)] for x in rng.integers(0, 4, k)))

    def operand():
        if depth < 8 and rng.random() < 0.15:
            out.append("(")
            seps()
            _arith_expr(rng, depth + 1, out, max(16, budget // 4))
            seps()
            out.append(")")
            return
        if rng.random() < 0.5:
            d = int(rng.integers(1, 7))
            s = "".join(str(int(x)) for x in rng.integers(0, 10, d))
            out.append(("-" if rng.random() < 0.2 else "") + s)
        else:
            out.append("".join(chr(97 + int(x)) for x in rng.integers(0, 26, int(rng.integers(1, 9)))))

    operand()
    size = 0
    while size < budget:
        op = "+-*/"[int(rng.integers(0, 4))]
        seps()
        out.append(op)
        seps(force=(op == "-"))
        before = len(out)
        operand()
        size += sum(len(x) for x in out[before - 3:]) + 1


def arithmetic(n: int, seed: int = 1) -> bytes:
    rng = np.random.default_rng(seed)
    pool = []
    for _ in range(2048):
        parts = []
        _arith_expr(rng, 0, parts, int(rng.integers(8, 200)))
        pool.append("".join(parts).encode())
    # join sub-expressions with "+" so the whole input is one expression
    body = _pool_concat(pool, rng, n, b" + ")
    if len(body) > n or not body:
        body = b"0"
    return body + b" " * (n - len(body))


_ATOM_CHARS = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz0123456789", dtype=np.uint8)
_OPEN, _ATOM, _CLOSE = 0, 1, 2


def _sexp_form(rng, depth: int, unbalanced: bool) -> bytes:
    """One spine of ``depth`` nested lists. Level i has ``kids`` ~ U[1, 6]
    children: the list that continues the spine sits at position ``pos`` ~
    U[0, kids), the others are atoms ``[a-z0-9]{1,10}``; the innermost list
    holds one atom. Siblings are separated by single spaces.

    Built with array operations: the token sequence (open, atom, close), the
    spaces between siblings (after an atom or a close, before an atom or an
    open), then every token's bytes scattered to its offset."""
    kids = rng.integers(1, 7, depth)
    pos = rng.integers(0, kids)
    post = kids - 1 - pos
    # opening half: per level "(" then pos atoms; then the core atom;
    # closing half, innermost level first: post atoms then ")"
    pre_len = 1 + pos
    types_pre = np.full(int(pre_len.sum()), _ATOM, dtype=np.int8)
    types_pre[np.concatenate(([0], np.cumsum(pre_len)[:-1]))] = _OPEN
    post_r = post[::-1]
    post_len = post_r + 1
    types_post = np.full(int(post_len.sum()), _ATOM, dtype=np.int8)
    types_post[np.cumsum(post_len) - 1] = _CLOSE
    types = np.concatenate((types_pre, np.array([_ATOM], dtype=np.int8), types_post))
    if unbalanced:
        types = np.concatenate((types, np.array([_CLOSE], dtype=np.int8)))
    is_atom = types == _ATOM
    alen = rng.integers(1, 11, int(is_atom.sum()))
    tlen = np.ones(len(types), dtype=np.int64)
    tlen[is_atom] = alen
    left = (types == _ATOM) | (types == _CLOSE)
    right = (types == _ATOM) | (types == _OPEN)
    space = np.zeros(len(types), dtype=bool)
    space[:-1] = left[:-1] & right[1:]
    if unbalanced:
        space[-2] = False  # the extra ")" follows the form directly
    width = tlen + space
    off = np.concatenate(([0], np.cumsum(width)[:-1]))
    out = np.full(int(width.sum()), ord(" "), dtype=np.uint8)
    out[off[types == _OPEN]] = ord("(")
    out[off[types == _CLOSE]] = ord(")")
    # atom characters: each atom's bytes at its offset
    a_off = off[is_atom]
    total = int(alen.sum())
    starts = np.repeat(a_off - np.concatenate(([0], np.cumsum(alen)[:-1])), alen)
    out[starts + np.arange(total)] = _ATOM_CHARS[rng.integers(0, 36, total)]
    return out.tobytes()


def sexp_doc(n: int, seed: int = 3, unbalanced_frac: float = 0.0, max_depth: int = 10000,
             pool_size: int = 512) -> bytes:
    """One outer list ``( form form ... )`` of exactly ``n`` bytes (space padded).

    With ``unbalanced_frac`` > 0 that fraction of forms carries one extra ``)``."""
    rng = np.random.default_rng(seed)
    limit = max(8, n // 4)
    ok = [f for f in (_sexp_form(rng, int(rng.integers(1, max_depth + 1)), False) for _ in range(pool_size))
          if len(f) < limit] or [b"a"]
    bad = [f + b")" for f in ok[: max(1, len(ok) // 8)]]
    lens_ok = np.array([len(f) + 1 for f in ok], dtype=np.int64)
    est = int((n - 2) / lens_ok.mean()) + 16
    pick = rng.integers(0, len(ok), est)
    is_bad = rng.random(est) < unbalanced_frac
    pick_bad = rng.integers(0, len(bad), est)
    forms = [bad[pick_bad[i]] if is_bad[i] else ok[pick[i]] for i in range(est)]
    cum = np.cumsum([len(f) + 1 for f in forms])
    k = int(np.searchsorted(cum, n - 2, side="right"))
    body = b" ".join(forms[:k])
    doc = b"(" + body + b")"
    if len(doc) > n:
        doc = b"()"
    return doc + b" " * (n - len(doc))


def lognormal_lengths(count: int, median: int, lo: int, hi: int, seed: int, sigma: float = 1.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    x = rng.lognormal(np.log(median), sigma, count)
    return np.clip(x, lo, hi).astype(np.int64)


def json_batch(count: int = 4096, median: int = 8192, lo: int = 200, hi: int = 4 << 20, seed: int = 4):
    """(bytes, int64 offsets[count+1]) of ``count`` JSON documents with
    log-normal lengths; each is a top-level array of elements drawn from one
    shared pool (document i uses seed 4_000_000 + i), padded to its length."""
    lens = lognormal_lengths(count, median, lo, hi, seed)
    g = _Json(np.random.default_rng(seed + 1))
    pool = sorted((g.element().encode() for _ in range(8192)), key=len)
    plen = np.array([len(p) for p in pool], dtype=np.int64)
    docs = []
    for i, L in enumerate(lens):
        L = int(L)
        k = max(1, int(np.searchsorted(plen, max(8, L // 4), side="left")))
        body = _pool_concat(pool[:k], np.random.default_rng(4_000_000 + i), L - 2, b",")
        doc = b"[" + body + b"]"
        if len(doc) > L:
            doc = b"[]"
        docs.append(doc + b" " * (L - len(doc)))
    offs = np.zeros(count + 1, dtype=np.int64)
    offs[1:] = np.cumsum([len(d) for d in docs])
    return b"".join(docs), offs


def json_trace(count: int, rate: float, median: int = 16384, lo: int = 64, hi: int = 16 << 20, seed: int = 5):
    """A serving trace: ``count`` JSON requests with log-normal sizes and
    Poisson arrivals at ``rate`` requests/s. Returns (docs, arrival seconds)."""
    buf, offs = json_batch(count, median, lo, hi, seed)
    docs = [buf[offs[i]:offs[i + 1]] for i in range(count)]
    gaps = np.random.default_rng(seed + 7).exponential(1.0 / rate, count)
    return docs, np.cumsum(gaps) - gaps[0]
