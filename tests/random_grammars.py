"""Random grammars and inputs for differential fuzzing.

A restatement of ``alpacc random`` (src/Alpacc/Random.hs:20-35) with a seeded
numpy generator in place of QuickCheck, so it draws from the same family of
grammars (not the same grammars):

* lexer spec (``genDfaLexerSpec``, src/Alpacc/Lexer/DFA.hs:542-554):
  ``num_terminals`` terminals named ``a, b, c, ...`` in declaration order, each
  a random regex over the first ``num_chars`` letters that does not accept the
  empty string; regexes from ``genRegEx`` (Lexer/RegularExpression.hs:235-259):
  at size <= 1 one of epsilon, a literal or a range of ``size + 1`` picked
  characters; above it also star, concatenation and alternation of two halves;
* grammar (``genGrammar``/``genNtProduction``/``genProduction``,
  src/Alpacc/Grammar.hs:384-445): nonterminals ``A, B, ...``, one production
  per nonterminal plus ``num_productions - num_nonterminals`` with a random
  left side; a right side has 0..6 symbols (QuickCheck's size 30 / 5), the
  first a terminal, the rest terminals or nonterminals; redrawn until every
  nonterminal is productive and reachable from the start (the first rule);
* printed as ``printDfaSpec``/``printGrammar`` (src/Alpacc/CFG.hs:229-265)
  after a ``params`` block with the lookback and lookahead, as
  tests/testc.sh:80-87 of the reference writes it.

Defaults are the reference CLI's (app/Main.hs:200-240): 3 characters, 3
terminals, 2 nonterminals, 3 productions.

Inputs (``inputs``): every string over the grammar's characters up to a small
length (the exhaustive mode of ``alpacc test generate``), plus sentences of
random derivations with each terminal replaced by a random string its regex
matches, at lengths up to several lexer tiles.
"""

from __future__ import annotations

import itertools

import numpy as np

EPS, LIT, RANGE, STAR, CAT, ALT = "eps", "lit", "range", "star", "cat", "alt"


def _alpha(n: int, base: str) -> str:
    """``intToAlpha``: a, b, ..., z, aa, ab, ..."""
    a = base[n % 26]
    return a if n < 26 else _alpha(n // 26 - 1, base) + a


def gen_regex(rng, cs, size):
    kinds = 3 if size <= 1 else 6
    k = int(rng.integers(0, kinds))
    if k == 0:
        return (EPS,)
    if k == 1:
        return (LIT, cs[int(rng.integers(0, len(cs)))])
    if k == 2:
        return (RANGE, [cs[int(rng.integers(0, len(cs)))] for _ in range(size + 1)])
    h = size // 2
    if k == 3:
        return (STAR, gen_regex(rng, cs, h))
    if k == 4:
        return (CAT, gen_regex(rng, cs, h), gen_regex(rng, cs, h))
    return (ALT, gen_regex(rng, cs, h), gen_regex(rng, cs, h))


def nullable(r) -> bool:
    k = r[0]
    if k in (EPS, STAR):
        return True
    if k in (LIT, RANGE):
        return False
    if k == CAT:
        return nullable(r[1]) and nullable(r[2])
    return nullable(r[1]) or nullable(r[2])


def print_regex(r) -> str:
    """``printRegEx`` (CFG.hs:229-238)."""
    k = r[0]
    if k == EPS:
        return ""
    if k == LIT:
        return r[1]
    if k == RANGE:
        lits = [(LIT, c) for c in r[1]]
        alt = lits[-1]
        for x in reversed(lits[:-1]):
            alt = (ALT, x, alt)
        return print_regex(alt)
    if k == STAR:
        return "(" + print_regex(r[1]) + ")*"
    if k == CAT:
        return "(" + print_regex(r[1]) + " " + print_regex(r[2]) + ")"
    return "(" + print_regex(r[1]) + "|" + print_regex(r[2]) + ")"


def sample_regex(rng, r, stars: int = 3) -> str:
    """A random string the regex matches."""
    k = r[0]
    if k == EPS:
        return ""
    if k == LIT:
        return r[1]
    if k == RANGE:
        return r[1][int(rng.integers(0, len(r[1])))]
    if k == STAR:
        return "".join(sample_regex(rng, r[1], stars) for _ in range(int(rng.integers(0, stars + 1))))
    if k == CAT:
        return sample_regex(rng, r[1], stars) + sample_regex(rng, r[2], stars)
    return sample_regex(rng, r[1 + int(rng.integers(0, 2))], stars)


class RandomGrammar:
    def __init__(self, seed: int, q: int = 1, k: int = 1, num_chars: int = 3, num_terminals: int = 3,
                 num_nonterminals: int = 2, num_productions: int = 3, size: int = 30):
        rng = np.random.default_rng(seed)
        self.q, self.k = q, k
        self.chars = [chr(ord("a") + i) for i in range(num_chars)]
        self.terminals = [_alpha(j, "abcdefghijklmnopqrstuvwxyz") for j in range(num_terminals)]
        self.regex = {}
        for t in self.terminals:
            while True:
                r = gen_regex(rng, self.chars, num_terminals)
                if not nullable(r):
                    break
            self.regex[t] = r
        self.nts = [_alpha(j, "ABCDEFGHIJKLMNOPQRSTUVWXYZ") for j in range(max(1, num_nonterminals))]
        while True:
            prods = [(nt, self._rhs(rng, size)) for nt in self.nts]
            for _ in range(max(0, num_productions - len(self.nts))):
                prods.append((self.nts[int(rng.integers(0, len(self.nts)))], self._rhs(rng, size)))
            if self._well_formed(prods):
                break
        self.prods = prods

    def _rhs(self, rng, size):
        n = int(rng.integers(0, size // 5 + 1))
        if n == 0:
            return []
        syms = self.terminals + self.nts
        return [self.terminals[int(rng.integers(0, len(self.terminals)))]] + [
            syms[int(rng.integers(0, len(syms)))] for _ in range(n - 1)]

    def _well_formed(self, prods) -> bool:
        if len(set((a, tuple(b)) for a, b in prods)) != len(prods):
            return False  # duplicate productions are a grammar error
        productive = set()
        changed = True
        while changed:
            changed = False
            for lhs, rhs in prods:
                if lhs not in productive and all(s in self.regex or s in productive for s in rhs):
                    productive.add(lhs)
                    changed = True
        reach = {self.nts[0]}
        changed = True
        while changed:
            changed = False
            for lhs, rhs in prods:
                if lhs in reach:
                    for s in rhs:
                        if s in self.nts and s not in reach:
                            reach.add(s)
                            changed = True
        return productive == set(self.nts) and reach == set(self.nts)

    def text(self) -> str:
        lines = ["params {", "  lookback=%d." % self.q, "  lookahead=%d." % self.k, "}", ""]
        lines += ["%s = /%s/." % (t, print_regex(self.regex[t])) for t in self.terminals]
        spec = "\n".join(lines)
        gram = "".join("%s -> %s.\n" % (lhs, " ".join(rhs)) for lhs, rhs in self.prods)
        return spec + "\n" + gram

    def sentence(self, rng, budget: int) -> str:
        """A random derivation from the start, expanded leftmost with a
        preference for short right sides once the budget is spent."""
        out = []
        length = 0
        stack = [self.nts[0]]
        by_lhs = {nt: [rhs for lhs, rhs in self.prods if lhs == nt] for nt in self.nts}
        steps = 0
        while stack and steps < 200000:
            steps += 1
            s = stack.pop()
            if s in self.regex:
                out.append(sample_regex(rng, self.regex[s]))
                length += len(out[-1])
                continue
            opts = by_lhs[s]
            if length > budget or len(stack) > budget:
                opts = sorted(opts, key=lambda r: sum(x in self.nts for x in r))[:1]
            rhs = opts[int(rng.integers(0, len(opts)))]
            stack.extend(reversed(rhs))
        return "".join(out)

    def token_sentence(self, rng, budget: int) -> list:
        """A random derivation as terminal ids (parser-mode input): the
        terminals are declared first and in order, so terminal i has id i."""
        out = []
        stack = [self.nts[0]]
        by_lhs = {nt: [rhs for lhs, rhs in self.prods if lhs == nt] for nt in self.nts}
        steps = 0
        while stack and steps < 200000:
            steps += 1
            s = stack.pop()
            if s in self.regex:
                out.append(self.terminals.index(s))
                continue
            opts = by_lhs[s]
            if len(out) > budget or len(stack) > budget:
                opts = sorted(opts, key=lambda r: sum(x in self.nts for x in r))[:1]
            stack.extend(reversed(opts[int(rng.integers(0, len(opts)))]))
        return out

    def inputs(self, seed: int = 0, exhaustive: int = 4, sentences=(8, 64, 2000, 20000),
               noise=(100, 15000, 40000)) -> list:
        rng = np.random.default_rng(seed)
        out = [""]
        for n in range(1, exhaustive + 1):
            out += ["".join(p) for p in itertools.product(self.chars, repeat=n)]
        for budget in sentences:
            for _ in range(3):
                out.append(self.sentence(rng, budget))
        # strings of the grammar's characters across lexer tile boundaries
        # (15360 bytes per tile): mostly rejected by the parser, they
        # exercise the lexer's state resolution between tiles
        for n in noise:
            out.append("".join(self.chars[int(i)] for i in rng.integers(0, len(self.chars), n)))
        return [s.encode() for s in out]


# the lookback/lookahead pairs of the reference's random-grammar matrix (Makefile:79-88)
QKS = ((0, 1), (1, 1), (2, 2), (3, 3))


def fuzz_grammars(count: int, first_seed: int = 0):
    """The first ``count`` random grammars (seeds from ``first_seed``, lookback
    and lookahead cycling through ``QKS``) whose tables the generator builds;
    the others are not LLP(q, k) and are skipped, as tests/testc.sh:89-91 of
    the reference skips grammars that fail code generation. Yields
    (name, grammar, combined tables)."""
    from alpacc_b200.grammar.tables import GrammarError, generate_parts

    seed, found = first_seed, 0
    while found < count and seed < first_seed + 100000:
        q, k = QKS[seed % len(QKS)]
        g = RandomGrammar(seed, q, k)
        name = "rand%d_q%dk%d" % (seed, q, k)
        seed += 1
        try:
            t = generate_parts(g.text(), name, False, "both")
        except GrammarError:
            continue
        found += 1
        yield name, g, t


def big_keyspace_grammar():
    """A random LLP(3, 3) grammar with 18 terminals (21 terminal ids with the
    ignore and sentinel ids): its (q + k)-terminal key space, 21^6 = 85.8M
    keys, exceeds the 2^26 keys of the dense pair table, so the loader keeps
    the reference's hash table and the device probes it as lookup_key does.
    Returns (name, grammar, combined tables)."""
    from alpacc_b200.grammar.tables import generate_parts
    g = RandomGrammar(0, 3, 3, num_chars=4, num_terminals=18, num_nonterminals=2, num_productions=3, size=20)
    name = "big0_q3k3"
    return name, g, generate_parts(g.text(), name, False, "both")


def token_sentences(g, seed: int = 0, budgets=(4, 16, 300, 5000)) -> list:
    """Parser-mode inputs of a random grammar: derivations as terminal-id bytes
    (accepted), each also with one id changed (mostly rejected)."""
    rng = np.random.default_rng(seed)
    out = [b""]
    for b in budgets:
        for _ in range(3):
            ids = g.token_sentence(rng, b)
            out.append(bytes(ids))
            if ids:
                m = list(ids)
                m[int(rng.integers(0, len(m)))] = int(rng.integers(0, len(g.terminals) + 3))
                out.append(bytes(m))
    return out


# C's keywords: a lexer whose machine grows with every keyword that shares
# prefixes with the identifier rule
KEYWORDS = ("if", "else", "while", "for", "return", "break", "continue", "int", "float", "char", "void", "struct",
            "switch", "case", "default", "do", "goto", "sizeof", "static", "const", "unsigned", "signed", "long",
            "short", "double", "enum", "union", "typedef", "extern", "register", "volatile", "auto")


def keyword_grammar(nkw: int) -> str:
    """A lexer of ``nkw`` keywords, identifiers, numbers and whitespace under
    an LLP(1, 1) list grammar. The keywords come first, so they win over the
    identifier rule on equal length (the reference's priority by order)."""
    lines = ["params { lookback=1. lookahead=1. }", ""]
    lines += ["kw%d = /%s/." % (i, w) for i, w in enumerate(KEYWORDS[:nkw])]
    lines += ["ident = /[a-z][a-z0-9]*/.", "num = /[0-9]+/.", "ignore = /\\s|\\n|\\t/.", ""]
    lines += ["S -> T S.", "S -> ."]
    lines += ["T -> kw%d." % i for i in range(nkw)] + ["T -> ident.", "T -> num."]
    return "\n".join(lines) + "\n"


def keyword_inputs(nkw: int, seed: int = 0, sizes=(0, 1, 20, 300, 15000, 40000)) -> list:
    """Sequences of keywords, near-keywords (prefixes and extensions, which
    are identifiers), identifiers and numbers with whitespace runs; each size
    once clean and once with a byte no rule accepts."""
    rng = np.random.default_rng(seed)
    kws = KEYWORDS[:nkw]

    def word():
        x = rng.random()
        w = kws[int(rng.integers(0, len(kws)))]
        if x < 0.4:
            return w
        if x < 0.55:
            return w[: max(1, len(w) - 1)]
        if x < 0.7:
            return w + "xyz0"[int(rng.integers(0, 4))]
        if x < 0.85:
            return "".join("abcdefghijklmnopqrstuvwxyz"[int(i)] for i in rng.integers(0, 26, int(rng.integers(1, 9))))
        return str(int(rng.integers(0, 10 ** 6)))

    out = []
    for n in sizes:
        parts, size = [], 0
        while size < n:
            w = word()
            sep = " \n\t"[int(rng.integers(0, 3))] * int(rng.integers(1, 3))
            parts.append(w + sep)
            size += len(w) + len(sep)
        s = "".join(parts)[:n]
        out.append(s.encode())
        if n > 1:
            b = bytearray(s.encode())
            b[int(rng.integers(0, len(b)))] = ord("#")
            out.append(bytes(b))
    return out
