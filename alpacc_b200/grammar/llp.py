"""LL(k) and LLP(q,k) table construction (generator-time, host only).

Restates ``src/Alpacc/Parser/LL.hs`` (FIRST_k / FOLLOW_k with truncated products,
LAST_q / BEFORE_q on the reversed grammar, the LL(k) table) and the LLP
collection of ``src/Alpacc/Parser/LLP.hs`` (Algorithm 8 of Vagner & Melichar,
"Parallel LL parsing", with the reference's items, shortest-prefix LL(k)
configurations, start pairs and bracket homomorphisms).

Grammar symbols are ``(0, nt)`` (Nonterminal) / ``(1, t)`` (Terminal); strings
of terminals are tuples. The results are sets and maps, so iteration order only
matters for which conflict is reported first; items are visited in sorted order
(the order of Haskell's ``Set``).
"""

from __future__ import annotations

from dataclasses import dataclass
from functools import lru_cache

NT, TM = 0, 1


class GrammarError(ValueError):
    pass


@dataclass(frozen=True)
class Grammar:
    start: object
    terminals: tuple
    nonterminals: tuple
    productions: tuple  # ((lhs, rhs_tuple_of_symbols), ...)

    def reversed(self) -> "Grammar":
        """``reverseGrammar`` (Grammar.hs:183-187)."""
        return Grammar(self.start, self.terminals, self.nonterminals,
                       tuple((a, tuple(reversed(w))) for a, w in self.productions))


def trunc_product(k: int, a, b) -> frozenset:
    """``truncatedProduct`` (LL.hs:148-154)."""
    return frozenset((x + y)[:k] for x in a for y in b)


class FirstK:
    """Memoised FIRST_k over strings of symbols (LL.hs:175-285).

    The reference unions the truncated products over every split of the string;
    truncated product is associative, so every split yields the left fold."""

    def __init__(self, k: int, grammar: Grammar):
        self.k = k
        self.g = grammar
        self.fmap = self._first_map()
        self._memo = {}

    def _first_map(self):
        k = self.k
        fm = {nt: frozenset() for nt in self.g.nonterminals}
        changed = True
        while changed:
            changed = False
            for lhs, rhs in self.g.productions:
                s = self._first_with(fm, rhs)
                if not s <= fm[lhs]:
                    fm[lhs] = fm[lhs] | s
                    changed = True
        return fm

    def _first_with(self, fm, syms):
        k = self.k
        acc = frozenset([()])
        for kind, x in syms:
            if all(len(w) >= k for w in acc):
                break
            acc = trunc_product(k, acc, frozenset([(x,)[:k]]) if kind == TM else fm[x])
            if not acc:
                break
        return acc

    def __call__(self, syms) -> frozenset:
        syms = tuple(syms)
        r = self._memo.get(syms)
        if r is None:
            r = self._first_with(self.fmap, syms)
            self._memo[syms] = r
        return r


END = ("$end",)  # ExtendedTerminal End (LL.hs:305-316)
ESTART = ("$start",)  # ExtendedStart


def follow_map(k: int, g: Grammar) -> dict:
    """``followMap`` / ``firstAndFollowMaps`` (LL.hs:355-466): FOLLOW_k on the
    grammar extended by ``S' -> S End^k``, with ``End`` filtered out afterwards."""
    ext_prods = ((ESTART, ((NT, g.start),) + ((TM, END),) * k),) + g.productions
    ext = Grammar(ESTART, g.terminals + (END,), (ESTART,) + g.nonterminals, ext_prods)
    first = FirstK(k, ext)
    fol = {nt: frozenset() for nt in ext.nonterminals}
    fol[g.start] = frozenset([(END,) * k])
    right = []
    for aj, rhs in ext.productions:
        for i, (kind, x) in enumerate(rhs):
            if kind == NT:
                right.append((aj, x, rhs[i + 1:]))
    changed = True
    while changed:
        changed = False
        for aj, ai, rest in right:
            s = trunc_product(k, first(rest), fol[aj])
            if not s <= fol[ai]:
                fol[ai] = fol[ai] | s
                changed = True
    out = {}
    for nt, ss in fol.items():
        if nt == ESTART:
            continue
        out[nt] = frozenset(tuple(t for t in w if t != END) for w in ss)
    return out


class LastQ:
    """LAST_q via FIRST_q of the reversed grammar (``lastMemoized`` LL.hs:249-257)."""

    def __init__(self, q: int, g: Grammar):
        self.first = FirstK(q, g.reversed())
        self._memo = {}

    def __call__(self, syms) -> frozenset:
        syms = tuple(syms)
        r = self._memo.get(syms)
        if r is None:
            r = frozenset(tuple(reversed(w)) for w in self.first(tuple(reversed(syms))))
            self._memo[syms] = r
        return r


def before_map(q: int, g: Grammar) -> dict:
    """BEFORE_q (``lastAndBefore`` LL.hs:418-427)."""
    return {nt: frozenset(tuple(reversed(w)) for w in s) for nt, s in follow_map(q, g.reversed()).items()}


def ll_table(k: int, g: Grammar, first: FirstK, follow: dict) -> dict:
    """``llTableM`` (LL.hs:536-559): (A, y) -> production index; conflicts are an
    error (the grammar is not LL(k))."""
    if k <= 0:
        raise GrammarError("Error: Lookahead must be positive.")
    table = {}
    for i, (nt, rhs) in enumerate(g.productions):
        for y in trunc_product(k, first(rhs), follow[nt]):
            table.setdefault((nt, y), set()).add(i)
    conflicts = {key: v for key, v in table.items() if len(v) > 1}
    if conflicts:
        raise GrammarError("LL(%d) Table Conflicts: %d cells" % (k, len(conflicts)))
    return {key: min(v) for key, v in table.items()}


def ll_parse(k: int, g: Grammar, table: dict, tokens) -> list | None:
    """Sequential LL(k) predictive parse (``llParse`` LL.hs:575-598): the
    production indices of the leftmost derivation, or None."""
    inp = list(tokens)
    pos = 0
    stack = [(NT, g.start)]
    out = []
    while True:
        if not stack:
            return out if pos == len(inp) else None
        kind, x = stack.pop()
        if kind == TM:
            if pos < len(inp) and inp[pos] == x:
                pos += 1
                continue
            return None
        idx = table.get((x, tuple(inp[pos:pos + k])))
        if idx is None:
            return None
        out.append(idx)
        stack.extend(reversed(g.productions[idx][1]))


# ---------------------------------------------------------------------------
# LLP(q,k) (LLP.hs)
# ---------------------------------------------------------------------------


@dataclass(frozen=True, order=True)
class Item:
    """The 4-tuple of Algorithm 8 (``Item`` LLP.hs:60-67): dot production
    ``(lhs, before_dot, after_dot)``, suffix, prefix and the LL(k) configuration
    ``(alpha, omega, pi)``."""

    dot: tuple
    suffix: tuple
    prefix: tuple
    config: tuple


class LLPContext:
    """``LlpContext`` (LLP.hs:116-156, initLlpContext :209-236)."""

    def __init__(self, q: int, k: int, g: Grammar):
        if q < 0:
            raise GrammarError("Error: Lookback must be non-negative.")
        if k < 1:
            raise GrammarError("Error: Lookahead must be positive.")
        self.q, self.k, self.g = q, k, g
        self.first = FirstK(k, g)
        self.follow = follow_map(k, g)
        self.last = LastQ(q, g)
        self.before = before_map(q, g)
        self.table = ll_table(k, g, self.first, self.follow)
        self._prods_of = {}
        for lhs, rhs in g.productions:
            self._prods_of.setdefault(lhs, []).append(rhs)
        self._cfg_memo = {}
        self._before_syms = {nt: [tuple((TM, t) for t in w) for w in sorted(s)] for nt, s in self.before.items()}

    # parseLlpConfig (LLP.hs:470-491)
    def parse_config(self, y, alpha):
        key = (y, alpha)
        if key in self._cfg_memo:
            return self._cfg_memo[key]
        k = self.k
        inp = list(y)
        stack = list(alpha)
        parsed = []
        res = None
        while True:
            if inp and stack and stack[0][0] == TM:
                if inp[0] == stack[0][1]:
                    res = (alpha, tuple(stack[1:]), tuple(parsed))
                break
            if stack and stack[0][0] == NT:
                idx = self.table.get((stack[0][1], tuple(inp[:k])))
                if idx is None:
                    break
                stack = list(self.g.productions[idx][1]) + stack[1:]
                parsed.append(idx)
                continue
            if not inp and not stack:
                res = (alpha, (), tuple(parsed))
            break
        self._cfg_memo[key] = res
        return res

    def shortest_prefix(self, v, x_delta):
        """``solveShortestsPrefix`` (LLP.hs:96-113): first successful config over
        the non-empty prefixes of ``x_delta``, shortest first."""
        for n in range(1, len(x_delta) + 1):
            r = self.parse_config(v, x_delta[:n])
            if r is not None:
                return r
        raise GrammarError("no LL(k) configuration for an LLP item (fromJust)")

    def new_items(self, it: Item) -> set:
        """Step 3(a) (``newLlpItemsMemo`` LLP.hs:241-281)."""
        y, alpha_x, beta = it.dot
        if not alpha_x:
            return set()
        alpha = alpha_x[:-1]
        uj = set()
        for b in self._before_syms[y]:
            uj |= self.last(b + alpha)
        x = (alpha_x[-1],)
        vj = self.first(x + tuple((TM, t) for t in it.prefix))
        x_delta = x + it.config[0]
        dot = (y, alpha, x + beta)
        return {Item(dot, u, v, self.shortest_prefix(v, x_delta)) for u in uj for v in vj}

    def extra_items(self, it: Item) -> set:
        """Step 3(b) for one item (``extraLlpItemMemo`` LLP.hs:283-320)."""
        alpha_y = it.dot[1]
        if not alpha_y or alpha_y[-1][0] == TM:
            return set()
        y = alpha_y[-1][1]
        out = set()
        for delta in self._prods_of.get(y, []):
            for b in self._before_syms[y]:
                for u in self.last(b + delta):
                    out.add(Item((y, delta, ()), u, it.prefix, it.config))
        return out

    def closure(self, items: set) -> frozenset:
        """``extraLlpItemsMemo`` (LLP.hs:324-339)."""
        items = set(items)
        work = list(items)
        while work:
            nxt = []
            for it in work:
                for e in self.extra_items(it):
                    if e not in items:
                        items.add(e)
                        nxt.append(e)
            work = nxt
        return frozenset(items)

    def successors(self, items) -> set:
        """``solveLlpItemsMemo`` (LLP.hs:354-376): group by the symbol before the dot."""
        groups = {}
        for it in items:
            a = it.dot[1]
            if a:
                groups.setdefault(a[-1], []).append(it)
        out = set()
        for _sym, grp in sorted(groups.items()):
            new = set()
            for it in grp:
                new |= self.new_items(it)
            out.add(self.closure(new))
        return out

    def init_items(self) -> frozenset:
        """``initD`` (LLP.hs:84-94)."""
        prods = self._prods_of.get(self.g.start, [])
        if len(prods) != 1:
            return frozenset()
        rhs = prods[0]
        return frozenset(Item((self.g.start, rhs, ()), u, (), ((), (), ())) for u in self.last(rhs))

    def collection(self):
        """``llpCollectionMemo`` (LLP.hs:380-448): returns (table, item sets)."""
        table = {}
        seen = set()
        queue = [self.init_items()]
        head = 0
        while head < len(queue):
            top = queue[head]
            head += 1
            if top in seen:
                continue
            for it in sorted(top):
                a = it.dot[1]
                if not a or a[-1][0] != TM:
                    continue
                key = (it.suffix, it.prefix)
                if key in table and table[key] != it.config:
                    raise GrammarError(
                        "The grammar is not LLP(%d, %d) due to the admissible pair %r" % (self.q, self.k, key))
                table[key] = it.config
            seen.add(top)
            queue.extend(sorted(self.successors(top), key=lambda s: sorted(s)))
        return table, {s for s in seen if s}

    def starts(self) -> dict:
        """``allStarts`` (LLP.hs:495-516)."""
        prods = self._prods_of.get(self.g.start, [])
        s = prods[0] if prods else ()
        tail = s[1:] if s else ()
        return {((), z): (((NT, self.g.start),), tail, ()) for z in self.first(s)}


def llp_table_with_starts(q: int, k: int, g: Grammar) -> dict:
    """``llpParserTableWithStarts`` (LLP.hs:518-541): starts overlaid by the table."""
    ctx = LLPContext(q, k, g)
    table, _ = ctx.collection()
    out = dict(ctx.starts())
    out.update(table)
    return out


LB, RB = 0, 1  # Bracket constructors: LBracket < RBracket


def llp_homomorphisms(q: int, k: int, g: Grammar) -> dict:
    """``llpParserTableWithStartsHomomorphisms`` (LLP.hs:545-574): each pair maps
    to (brackets, productions) with brackets = RBracket alpha ++ LBracket (reverse
    omega); start pairs push only."""
    ctx = LLPContext(q, k, g)
    table, _ = ctx.collection()
    out = {}
    for key, (alpha, omega, pi) in ctx.starts().items():
        out[key] = (tuple((LB, s) for s in reversed(omega)), pi)
    for key, (alpha, omega, pi) in table.items():
        out[key] = (tuple((RB, s) for s in alpha) + tuple((LB, s) for s in reversed(omega)), pi)
    return out


def llp_parse(q: int, k: int, table: dict, tokens) -> list | None:
    """Reference sequential LLP parse by gluing the pairs' stack configurations
    (``llpParse`` LLP.hs:612-654). ``table`` maps pair -> (alpha, omega, pi)."""
    s = [(1,)] + list(tokens) + [(2,)]  # RightTurnstile ++ tokens ++ LeftTurnstile
    pairs = []
    back = []
    for i, x in enumerate(s):
        fwd = tuple(s[i + 1:i + k])
        v = table.get((tuple(back), (x,) + fwd))
        if v is None:
            return None
        pairs.append(v)
        back = (back + [x])[-q:] if q > 0 else []
    acc = None
    for a, o, p in pairs:
        if acc is None:
            acc = (tuple(a), tuple(o), tuple(p))
            continue
        al, ol, pl = acc
        if ol == a:
            acc = (al, o, pl + p)
        elif a[:len(ol)] == ol:
            acc = (al + a[len(ol):], o, pl + p)
        elif ol[:len(a)] == a:
            acc = (al, o + ol[len(a):], pl + p)
        else:
            return None
    return list(acc[2]) if acc is not None else None
