"""The windowing rule of chunked lexing, checked on the CPU against the
reference's own algorithm.

``alpacc_gpu_lex_stream`` lexes a window as if it were a whole input, keeps
the lexemes that end at a boundary inside it, and starts the next window at
the last such boundary with the lexer's initial state. This holds if
``lex_string`` (backends/c/lexer.c:39-97) behaves after any boundary exactly
as on a fresh input starting there. Here ``lex_string`` is restated over the
encoded endomorphism tables (TO_STATE, COMPOSE, masks; not the device's
minimised machine), run once on the whole input and once window by window
with that rule, for several grammars (random ones included) and window sizes;
lexemes and accept/reject must agree.
"""

import numpy as np
import pytest

from alpacc_b200.grammar.tables import generate_parts
from tests import cases
from tests.random_grammars import fuzz_grammars


class Lexer:
    """``lex_string`` over the generated tables, with an open-ended mode."""

    def __init__(self, t):
        L = t.lexer
        self.compose = np.asarray(L.compose, dtype=np.int64)
        self.to_state = [int(x) for x in L.to_state]
        self.accept = np.asarray(L.accept, dtype=bool)
        self.N = int(L.num_states)
        self.L = L
        self.identity = int(L.identity)
        self.ignore = t.ignore_token
        self.len_max = (1 << t.length_bits) - 1

    def idx(self, s):
        return (s & self.L.index_mask) >> self.L.index_offset

    def comp(self, a, b):
        return int(self.compose[self.idx(a) * self.N + self.idx(b)])

    def run(self, s: bytes, open_end: bool = False):
        """(ok, lexemes, last boundary). With ``open_end`` the input goes on
        after ``s``: no boundary at its end and no final acceptance check."""
        n = len(s)
        if n == 0:
            return True, [], 0
        L = self.L
        cur = self.comp(self.identity, self.to_state[s[0]])
        start, out, last = 0, [], 0
        for i in range(1, n + 1):
            nxt = self.to_state[s[i]] if i < n else self.identity
            if i < n:
                boundary = bool((self.comp(cur, nxt) & L.produce_mask) >> L.produce_offset)
            else:
                boundary = not open_end
            if boundary:
                term = (cur & L.token_mask) >> L.token_offset
                if term != self.ignore:
                    if i - start > self.len_max:
                        return False, out, last
                    out.append((term, start, i - start))
                start = last = i if i < n else last
            if i < n:
                cur = self.comp(cur, nxt)
        if open_end:
            return True, out, last
        return bool(self.accept[self.idx(cur)]), out, last


def windowed(lx: Lexer, s: bytes, w: int):
    pos, out = 0, []
    while pos < len(s):
        end = min(len(s), pos + w)
        ok, lex, last = lx.run(s[pos:end], open_end=end < len(s))
        if not ok:
            return False, out
        if end < len(s) and last == 0:  # no boundary in the window: widen it
            w *= 2
            continue
        out += [(t, a + pos, ln) for t, a, ln in lex]
        if end == len(s):
            return True, out
        pos += last
    return True, out


def _check(t, inputs, windows=(1, 2, 3, 7, 16, 61)):
    lx = Lexer(t)
    for s in inputs:
        ok, want, _ = lx.run(s)
        for w in windows:
            got_ok, got = windowed(lx, s, w)
            assert got_ok == ok, (t.name, w, s[:40])
            if ok:
                assert got == want, (t.name, w, s[:40])


@pytest.mark.parametrize("config", ["arithmetic_i64", "json_i32", "sexp_i64", "paper_grammar_i64", "llp01_i64"])
def test_windows_restart_at_boundaries(config):
    ins = [d for d in cases.case_inputs(config, sizes=(1, 60, 200), seeds=(0,)) if len(d) <= 400]
    _check(cases.tables(config, "lexer"), ins)


def test_windows_restart_at_boundaries_random_grammars():
    for name, g, t in fuzz_grammars(8):
        ins = [s for s in g.inputs(0, exhaustive=3, sentences=(8, 64), noise=(100,))]
        _check(generate_parts(g.text(), name, False, "lexer"), ins)
