"""Parser for alpacc's ``.alp`` grammar files and its regular-expression dialect.

Restates ``src/Alpacc/CFG.hs:51-227`` (the ``.alp`` syntax: ``params{}``, terminal
rules, nonterminal rules with optional ``[Name]``) and
``src/Alpacc/Lexer/RegularExpression.hs:78-220`` (the regex dialect: ``\\s`` is a
single space, ``.`` is a literal dot, ``\\xHH`` bytes, ``\\uHHHH`` code points,
``[a-z\\x00-\\xFF]`` ranges, postfix ``* + ?``).

Symbols are encoded as tuples whose Python ordering equals the ordering Haskell
derives for the reference's data types, because the reference numbers terminals
and builds sets and maps in that order:

* ``data T = T Text | TLit Text``      -> ``(0, name)`` / ``(1, literal)``
* ``data Symbol nt t = Nonterminal nt | Terminal t`` -> ``(0, nt)`` / ``(1, t)``

Regex ASTs are tuples: ``('eps',)``, ``('lit', bytes)``, ``('range', (bytes, ...))``,
``('star', r)``, ``('alt', a, b)``, ``('cat', a, b)``.
"""

from __future__ import annotations

from dataclasses import dataclass, field

# Symbol constructors (Grammar.hs:87,105-108).
NONTERMINAL = 0
TERMINAL = 1


def T(name: str):
    """Named terminal ``T name`` (Grammar.hs:87)."""
    return (0, name)


def TLit(lit: str):
    """Literal terminal ``TLit lit`` (Grammar.hs:87)."""
    return (1, lit)


def t_pretty(t) -> str:
    return t[1] if t[0] == 0 else '"%s"' % t[1]


class AlpSyntaxError(ValueError):
    pass


@dataclass
class Params:
    """``Params`` record (CFG.hs:51-64): defaults lookback 0, lookahead 1."""

    lookback: int = 0
    lookahead: int = 1
    length: int | None = None


@dataclass
class NTRule:
    nt: str
    name: str | None
    rhs: list  # list of symbols (NONTERMINAL, nt) / (TERMINAL, t)


@dataclass
class CFG:
    """``CFG`` record (CFG.hs:66-71)."""

    params: Params = field(default_factory=Params)
    t_rules: list = field(default_factory=list)  # [(t, regex)]
    nt_rules: list = field(default_factory=list)  # [NTRule]


# ---------------------------------------------------------------------------
# Regular expressions (RegularExpression.hs)
# ---------------------------------------------------------------------------

_ESCAPES = {
    "\\": "\\", "/": "/", "[": "[", "]": "]", "(": "(", ")": ")", "*": "*",
    "+": "+", "|": "|", "s": " ", "t": "\t", "n": "\n", "r": "\r", "?": "?",
}  # RegularExpression.hs:87-103

_SPECIAL = set("\\/[]()*|+?")  # isPrint' exclusions, RegularExpression.hs:132-136


def _char_bytes(c: str) -> bytes:
    return c.encode("utf-8")


def produces_epsilon(r) -> bool:
    """``producesEpsilon`` (RegularExpression.hs:55-61)."""
    tag = r[0]
    if tag == "eps" or tag == "star":
        return True
    if tag in ("lit", "range"):
        return False
    if tag == "alt":
        return produces_epsilon(r[1]) or produces_epsilon(r[2])
    return produces_epsilon(r[1]) and produces_epsilon(r[2])


class _RegexParser:
    """Recursive-descent restatement of ``pRegEx`` (RegularExpression.hs:150-215).

    Whitespace between regex tokens is skipped (``space`` = ``space1`` only,
    RegularExpression.hs:81-85); a literal space must be written ``\\s``.
    """

    def __init__(self, text: str, pos: int):
        self.s = text
        self.i = pos

    def _ws(self):
        while self.i < len(self.s) and self.s[self.i].isspace():
            self.i += 1

    def peek(self):
        return self.s[self.i] if self.i < len(self.s) else ""

    def parse(self):
        self._ws()
        return self.alter()

    def alter(self):
        r = self.concat()
        while self.peek() == "|":
            self.i += 1
            self._ws()
            r = ("alt", r, self.concat())
        return r

    def concat(self):
        r = ("eps",)
        while True:
            t = self.term()
            if t is None:
                return r
            r = ("cat", r, t)

    def term(self):
        c = self.peek()
        if c == "[":
            self.i += 1
            self._ws()
            t = self.range_body()
        elif c == "(":
            self.i += 1
            self._ws()
            t = self.alter()
            if self.peek() != ")":
                raise AlpSyntaxError("expected ')' in regex at %d" % self.i)
            self.i += 1
            self._ws()
        else:
            b = self.char()
            if b is None:
                return None
            t = ("lit", b)
        while True:  # pPostfix
            c = self.peek()
            if c == "*":
                t = ("star", t)
            elif c == "+":
                t = ("cat", t, ("star", t))
            elif c == "?":
                t = ("alt", ("eps",), t)
            else:
                return t
            self.i += 1
            self._ws()

    def _byte(self):
        s, i = self.s, self.i
        if s.startswith("\\x", i) and _ishex(s[i + 2:i + 3]) and _ishex(s[i + 3:i + 4]):
            self.i = i + 4
            self._ws()
            return int(s[i + 2:i + 4], 16)
        return None

    def char(self):
        """``pChar``: escape, ``\\u``, ``\\x`` byte, or printable non-special char."""
        s, i = self.s, self.i
        if i >= len(s):
            return None
        if s[i] == "\\":
            nxt = s[i + 1:i + 2]
            if nxt in _ESCAPES:
                self.i = i + 2
                self._ws()
                return _char_bytes(_ESCAPES[nxt])
            if nxt == "u":
                j = i + 2
                while j < len(s) and _ishex(s[j]):
                    j += 1
                if j > i + 2:
                    self.i = j
                    self._ws()
                    return _char_bytes(chr(int(s[i + 2:j], 16)))
            b = self._byte()
            if b is not None:
                return bytes([b])
            raise AlpSyntaxError("bad escape in regex at %d" % i)
        c = s[i]
        if c in _SPECIAL or c.isspace() or not c.isprintable():
            return None
        self.i = i + 1
        self._ws()
        return _char_bytes(c)

    def _alnum(self):
        c = self.peek()
        if c and c.isalnum():
            self.i += 1
            self._ws()
            return c
        return None

    def range_body(self):
        """``pRange`` (RegularExpression.hs:175-197): alnum ranges, byte ranges,
        single bytes and single alnum chars; at least one item."""
        items: list[bytes] = []
        while self.peek() != "]":
            save = self.i
            a = self._alnum()
            if a is not None and self.peek() == "-":
                self.i += 1
                self._ws()
                b = self._alnum()
                if b is not None:
                    items.extend(_char_bytes(chr(x)) for x in range(ord(a), ord(b) + 1))
                    continue
            self.i = save
            a = self._byte()
            if a is not None:
                save2 = self.i
                if self.peek() == "-":
                    self.i += 1
                    self._ws()
                    b = self._byte()
                    if b is not None:
                        items.extend(bytes([x]) for x in range(a, b + 1))
                        continue
                self.i = save2
                items.append(bytes([a]))
                continue
            self.i = save
            a = self._alnum()
            if a is None:
                raise AlpSyntaxError("bad range item at %d" % self.i)
            items.append(_char_bytes(a))
        if not items:
            raise AlpSyntaxError("empty range at %d" % self.i)
        self.i += 1
        self._ws()
        return ("range", tuple(items))


def _ishex(c: str) -> bool:
    return len(c) == 1 and c in "0123456789abcdefABCDEF"


def parse_regex(text: str):
    """``regExFromText`` (RegularExpression.hs:217-220)."""
    p = _RegexParser(text, 0)
    r = p.parse()
    if p.i != len(text):
        raise AlpSyntaxError("trailing regex input at %d" % p.i)
    return r


def literal_regex(lit: str):
    """Implicit rule of a string literal: ``foldl1 Concat`` of per-char literals
    (CFG.hs:143-145)."""
    parts = [("lit", _char_bytes(c)) for c in lit]
    r = parts[0]
    for p in parts[1:]:
        r = ("cat", r, p)
    return r


# ---------------------------------------------------------------------------
# .alp files (CFG.hs:164-227)
# ---------------------------------------------------------------------------


class _AlpParser:
    def __init__(self, text: str):
        self.s = text
        self.i = 0
        self.space()

    def space(self):
        s = self.s
        while self.i < len(s):
            c = s[self.i]
            if c.isspace():
                self.i += 1
            elif c == "#":
                while self.i < len(s) and s[self.i] != "\n":
                    self.i += 1
            else:
                break

    def peek(self, n=1):
        return self.s[self.i:self.i + n]

    def expect(self, tok: str):
        if not self.s.startswith(tok, self.i):
            raise AlpSyntaxError("expected %r at offset %d" % (tok, self.i))
        self.i += len(tok)
        self.space()

    def accept(self, tok: str) -> bool:
        if self.s.startswith(tok, self.i):
            self.i += len(tok)
            self.space()
            return True
        return False

    def ident(self, first_ok):
        s, i = self.s, self.i
        if i >= len(s) or not first_ok(s[i]):
            return None
        j = i + 1
        while j < len(s) and (s[j] == "_" or (s[j].isascii() and s[j].isalnum())):
            j += 1
        self.i = j
        self.space()
        return s[i:j]

    def decimal(self) -> int:
        s, i = self.s, self.i
        j = i
        while j < len(s) and s[j].isdigit():
            j += 1
        if j == i:
            raise AlpSyntaxError("expected a number at %d" % i)
        self.i = j
        self.space()
        return int(s[i:j])

    def params(self) -> Params:
        p = Params()
        save = self.i
        if not self.accept("params"):
            return p
        if not self.accept("{"):
            self.i = save
            return p
        while not self.accept("}"):
            for name in ("lookback", "lookahead", "length"):
                if self.s.startswith(name, self.i):
                    self.expect(name)
                    self.expect("=")
                    v = self.decimal()
                    self.expect(".")
                    if name == "lookback":
                        p.lookback = v
                    elif name == "lookahead":
                        p.lookahead = v
                    else:
                        if v not in (8, 16, 32, 64):
                            raise AlpSyntaxError("length must be 8, 16, 32, or 64")
                        p.length = v
                    break
            else:
                raise AlpSyntaxError("bad parameter at %d" % self.i)
        return p

    def t_rule(self):
        save = self.i
        name = self.ident(lambda c: c.isascii() and c.islower())
        if name is None or not self.accept("="):
            self.i = save
            return None
        if not self.accept("/"):
            self.i = save
            return None
        rp = _RegexParser(self.s, self.i)
        rp._ws()
        regex = rp.alter()
        self.i = rp.i
        self.expect("/")
        self.expect(".")
        return (T(name), regex)

    def symbol(self):
        c = self.peek()
        if c == '"':
            j = self.s.index('"', self.i + 1)
            lit = self.s[self.i + 1:j]
            if not lit:
                raise AlpSyntaxError("empty string literal at %d" % self.i)
            self.i = j + 1
            self.space()
            return (TERMINAL, TLit(lit))
        if c and c.isascii() and c.islower():
            return (TERMINAL, T(self.ident(lambda ch: True)))
        if c and c.isascii() and c.isupper():
            return (NONTERMINAL, self.ident(lambda ch: True))
        return None

    def nt_rules(self):
        nt = self.ident(lambda c: c.isascii() and c.isupper())
        if nt is None:
            return None
        name = None
        if self.accept("["):
            name = self.ident(lambda c: c.isascii() and c.isupper())
            if name is None:
                raise AlpSyntaxError("bad production name at %d" % self.i)
            self.expect("]")
        self.expect("->")
        alts = [[]]
        while True:
            sym = self.symbol()
            if sym is not None:
                alts[-1].append(sym)
                continue
            if self.accept("|"):
                alts.append([])
                continue
            self.expect(".")
            break
        return [NTRule(nt, name, rhs) for rhs in alts]

    def cfg(self) -> CFG:
        cfg = CFG(params=self.params())
        while True:
            r = self.t_rule()
            if r is None:
                break
            cfg.t_rules.append(r)
        while self.i < len(self.s):
            rules = self.nt_rules()
            if rules is None:
                raise AlpSyntaxError("unexpected input at offset %d" % self.i)
            cfg.nt_rules.extend(rules)
        return cfg


def parse_alp(text: str) -> CFG:
    """``cfgFromText`` (CFG.hs:225-227)."""
    return _AlpParser(text).cfg()


def rule_terminals(cfg: CFG) -> list:
    """Set of terminals used in nonterminal rules, in ``Set`` order (CFG.hs:105-110)."""
    ts = set()
    for r in cfg.nt_rules:
        for kind, s in r.rhs:
            if kind == TERMINAL:
                ts.add(s)
    return sorted(ts)


def lexer_spec(cfg: CFG):
    """``cfgToDFALexerSpec`` (CFG.hs:138-162): implicit literal rules (in ``Set``
    order) first, then the declared rules in file order; the position in this
    list is the lexer priority (``orderMap``)."""
    declared = [t for t, _ in cfg.t_rules]
    implicit = []
    for t in rule_terminals(cfg):
        if t in declared:
            continue
        if t[0] != 1:
            raise AlpSyntaxError("Can not create literal from: %s" % t[1])
        implicit.append((t, literal_regex(t[1])))
    rules = implicit + list(cfg.t_rules)
    for t, r in rules:
        if produces_epsilon(r):
            raise AlpSyntaxError("Error: %s may not produce empty strings." % t_pretty(t))
    if not rules:
        raise AlpSyntaxError("CFG has no lexical rules.")
    return rules
