"""Grammar tables for the combined lex+parse path, as alpacc's generator emits them.

``generate(alp_text)`` restates ``mkLexerParser`` (src/Alpacc/Generator/Analyzer.hs:211-279):
symbol numbering (``encodeSymbols`` src/Alpacc/Encode.hs:289-313), type selection
(``bracketIntType``/``productionIntType``/``symbolTerminalIntType`` Encode.hs:377-418),
the LLP pair table flattened into STACKS / PRODUCTIONS and an open-addressing hash
table (``llpHashTable`` Encode.hs:514-536, ``openAdressing`` src/Alpacc/HashTable.hs:560-585),
arities and terminal-production flags (Analyzer.hs:91-156), and the lexer's
endomorphism tables (see ``lexgen``).

The resulting ``GrammarTables`` is the input contract of the device path: the same
arrays the reference's C backend bakes in as constants
(src/Alpacc/Generator/C/Lexer.hs:16-58, C/Parser.hs:21-95).
"""

from __future__ import annotations

import hashlib
import struct
from dataclasses import dataclass, field

import numpy as np

from . import lexgen
from .llp import NT, TM, Grammar, GrammarError, LB, RB, llp_homomorphisms
from .syntax import CFG, T, lexer_spec, parse_alp, rule_terminals

U64 = (1 << 64) - 1
FNV_OFFSET = 14695981039346656037
FNV_PRIME = 1099511628211

# AugmentedTerminal (Unused T) values (Grammar.hs:60-64, 305-308)
UNUSED = (0, (0,))
RIGHT_TURNSTILE = (1,)  # START
LEFT_TURNSTILE = (2,)  # END
START_NT = (1,)  # AugmentedNonterminal Start


def used(t):
    return (0, (1, t))


def fnv1a(key) -> int:
    """``hash`` (Encode.hs:487-495) / ``hash_key`` (backends/c/parser.c:17-22)."""
    h = FNV_OFFSET
    for a in key:
        h = ((h ^ (int(a) & U64)) * FNV_PRIME) & U64
    return h


def _udtype(bits: int):
    return {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}[bits]


@dataclass
class GrammarTables:
    name: str
    q: int
    k: int
    index32: bool
    terminal_bits: int
    production_bits: int
    bracket_bits: int
    length_bits: int
    # lexer
    lexer: lexgen.EncodedLexer
    ignore_token: int | None
    dead_token: int
    # parser
    empty_terminal: int
    start_terminal: int
    end_terminal: int
    stacks: np.ndarray
    productions: np.ndarray
    ht_valid: np.ndarray  # bool[H]
    ht_keys: np.ndarray  # uint64[H, Q+K]
    ht_stack_span: np.ndarray  # int64[H, 2]
    ht_prod_span: np.ndarray  # int64[H, 2]
    max_iters: int
    max_brackets_per_pos: int
    max_prods_per_pos: int
    arity: np.ndarray  # uint64[P]
    prod_is_terminal: np.ndarray  # bool[P]
    terminal_names: list = field(default_factory=list)
    production_names: list = field(default_factory=list)
    llp_pairs: dict = field(default_factory=dict)  # int key tuple -> (brackets, prods)
    # which program the tables belong to: "both" (combined), "lexer" (lexer
    # constants only, lexer numbering) or "parser" (parser constants, no tree)
    parts: str = "both"

    @property
    def hash_size(self) -> int:
        return int(self.ht_valid.shape[0])

    @property
    def num_productions(self) -> int:
        return int(self.arity.shape[0])

    @property
    def index_bits(self) -> int:
        return 32 if self.index32 else 64

    @property
    def num_terminals(self) -> int:
        return self.end_terminal + 1

    def digest(self) -> str:
        h = hashlib.sha256()
        for a in (self.lexer.to_state, self.lexer.compose, self.lexer.accept, self.stacks, self.productions,
                  self.ht_valid, self.ht_keys, self.ht_stack_span, self.ht_prod_span, self.arity,
                  self.prod_is_terminal):
            h.update(np.ascontiguousarray(a).tobytes())
        h.update(struct.pack("<10q", self.q, self.k, int(self.index32), self.terminal_bits, self.production_bits,
                             self.bracket_bits, self.length_bits, self.lexer.identity, self.max_iters,
                             -1 if self.ignore_token is None else self.ignore_token))
        h.update(self.parts.encode())
        return h.hexdigest()[:16]


def _grammar_error(nts, ts, prods):
    """``grammarError`` (Grammar.hs:264-288): duplicates and nonproductive NTs."""
    seen = set()
    for p in prods:
        if p in seen:
            raise GrammarError("The given grammar contains duplicate productions.")
        seen.add(p)
    productive = set()
    changed = True
    while changed:
        changed = False
        for lhs, rhs in prods:
            if lhs not in productive and all(k == TM or s in productive for k, s in rhs):
                productive.add(lhs)
                changed = True
    bad = set(nts) - productive
    if bad:
        raise GrammarError("The given grammar contains nonproductive productions due to %s" % sorted(bad))


def _nub(xs):
    out = []
    for x in xs:
        if x not in out:
            out.append(x)
    return out


def parsing_grammar(cfg: CFG):
    """``cfgToGrammar`` (CFG.hs:112-136) then ``parsingGrammar`` =
    ``augmentGrammar . addUnusedTerminal . extendByTerminals`` (Grammar.hs:191-381).

    Returns (grammar, user_terminals, names) where names maps user production
    index -> ``[Name]``."""
    if not cfg.nt_rules:
        raise GrammarError("CFG has no production rules.")
    prods = [(r.nt, tuple(r.rhs)) for r in cfg.nt_rules]
    names = {i: r.name for i, r in enumerate(cfg.nt_rules) if r.name}
    nts = _nub([r.nt for r in cfg.nt_rules])
    start = cfg.nt_rules[0].nt
    ts = _nub([t for t, _ in cfg.t_rules] + rule_terminals(cfg))
    _grammar_error(nts, ts, prods)
    # extendByTerminals: every RHS symbol becomes a nonterminal; each terminal t
    # gets the production (Terminal t) -> t.
    ext_nts = [(TM, t) for t in ts] + [(NT, nt) for nt in nts]
    ext_prods = [((NT, lhs), tuple((NT, s) for s in rhs)) for lhs, rhs in prods]
    ext_prods += [((TM, t), ((TM, t),)) for t in ts]
    # addUnusedTerminal + augmentGrammar
    aug_nt = lambda x: (0, x)  # noqa: E731
    aug_prods = []
    for lhs, rhs in ext_prods:
        new_rhs = tuple((NT, aug_nt(s)) if k == NT else (TM, used(s)) for k, s in rhs)
        aug_prods.append((aug_nt(lhs), new_rhs))
    aug_prods.append((START_NT, ((TM, RIGHT_TURNSTILE), (NT, aug_nt((NT, start))), (TM, LEFT_TURNSTILE))))
    terminals = tuple([used(t) for t in ts] + [UNUSED, RIGHT_TURNSTILE, LEFT_TURNSTILE])
    nonterminals = tuple([aug_nt(x) for x in ext_nts] + [START_NT])
    return Grammar(START_NT, terminals, nonterminals, tuple(aug_prods)), ts, names


def encode_symbols(g: Grammar, ignore=T("ignore")) -> dict:
    """``encodeSymbols`` (Encode.hs:289-313): ordinary terminals, then ignore,
    Unused, START (⊢), END (⊣), then nonterminals."""
    special = {LEFT_TURNSTILE, RIGHT_TURNSTILE, UNUSED, used(ignore)}
    fts = [t for t in g.terminals if t not in special]
    tail = [x for x in (used(ignore), UNUSED, RIGHT_TURNSTILE, LEFT_TURNSTILE) if x in g.terminals]
    syms = [(TM, t) for t in fts + tail] + [(NT, nt) for nt in g.nonterminals]
    return {s: i for i, s in enumerate(syms)}


def open_addressing(items):
    """``openAdressing`` (HashTable.hs:560-585): table of 2*len slots, keys
    inserted by ``foldr`` (largest key first), linear probing from the FNV-1a
    hash with the probe offset added before the modulus (Word64 arithmetic)."""
    if not items:
        return [(False, None, None)], 0
    size = 2 * len(items)
    fk, fv = items[0]
    arr = [(False, fk, fv)] * size
    max_iters = 0
    for key, val in reversed(items):
        h = fnv1a(key)
        p = 0
        while True:
            idx = ((p + h) & U64) % size
            if not arr[idx][0]:
                arr[idx] = (True, key, val)
                max_iters = max(max_iters, p + 1)
                break
            p += 1
    return arr, max_iters


def _length_bits(cfg: CFG, index32: bool) -> int:
    if cfg.params.length is not None:
        return cfg.params.length
    return 32 if index32 else 64


def generate_lexer(text: str, name: str = "grammar", index32: bool = False) -> GrammarTables:
    """The lexer-mode program's tables (``mkLexer``, Analyzer.hs:114-150).

    The DFA is the combined program's, but terminals are numbered by the
    lexer's own encoder (``encodeTerminals`` over ``parsingTerminals
    (dfaTerminals spec)``, Encode.hs:144-158, Grammar.hs:321-325): the lexer
    spec's terminals in ``Ord T`` order (``Map.keys`` of its order map,
    DFA.hs:312-313) with ``ignore`` moved behind them, then ``Unused`` (the
    dead token). The combined program numbers them in declaration order
    instead, so the two programs can give one token different ids. Parser
    fields are empty."""
    cfg = parse_alp(text)
    rules = lexer_spec(cfg)
    ign = T("ignore")
    lts = sorted({t for t, _ in rules})
    order = [t for t in lts if t != ign] + ([ign] if ign in lts else [])
    lid = {t: i for i, t in enumerate(order)}
    dead = len(order)
    pl = lexgen.parallel_lexer(lexgen.merged_lexer_dfa(rules))
    enc_lex = lexgen.encode_lexer(pl, lambda r: lid[rules[r][0]], dead + 1, dead)
    # nameTerminals (Analyzer.hs:104-111)
    names = [t[1] if t[0] == 0 else "literal_%d" % i for i, t in enumerate(order)] + ["empty_%d" % dead]
    return GrammarTables(
        name=name, q=0, k=0, index32=index32,
        terminal_bits=lexgen.uint_type_bits(dead), production_bits=8, bracket_bits=8,
        length_bits=_length_bits(cfg, index32),
        lexer=enc_lex, ignore_token=lid.get(ign), dead_token=dead,
        empty_terminal=dead, start_terminal=0, end_terminal=0,
        stacks=np.zeros(0, dtype=np.uint8), productions=np.zeros(0, dtype=np.uint8),
        ht_valid=np.zeros(0, dtype=np.bool_), ht_keys=np.zeros((0, 0), dtype=np.uint64),
        ht_stack_span=np.zeros((0, 2), dtype=np.int64), ht_prod_span=np.zeros((0, 2), dtype=np.int64),
        max_iters=0, max_brackets_per_pos=0, max_prods_per_pos=0,
        arity=np.zeros(0, dtype=np.uint64), prod_is_terminal=np.zeros(0, dtype=np.bool_),
        terminal_names=names, production_names=[], parts="lexer",
    )


def generate_parts(text: str, name: str = "grammar", index32: bool = False, parts: str = "both") -> GrammarTables:
    """Tables of the combined (``both``), lexer-mode (``lexer``) or
    parser-mode (``parser``) program. The parser-mode program (``mkParser``,
    Analyzer.hs:167-209) numbers symbols exactly as the combined one, so its
    tables are the combined tables' parser part."""
    if parts == "lexer":
        return generate_lexer(text, name, index32)
    t = generate(text, name, index32)
    if parts == "parser":
        t.parts = "parser"
    elif parts != "both":
        raise ValueError("parts must be both, lexer or parser")
    return t


def generate(text: str, name: str = "grammar", index32: bool = False) -> GrammarTables:
    """Build every table of the combined program for an ``.alp`` grammar
    (``mkLexerParser``, Analyzer.hs:211-279)."""
    cfg = parse_alp(text)
    q, k = cfg.params.lookback, cfg.params.lookahead
    g, ts, user_names = parsing_grammar(cfg)
    enc = encode_symbols(g)
    term_id = {t: enc[(TM, t)] for t in g.terminals}
    empty_terminal = term_id[UNUSED]
    start_terminal = term_id[RIGHT_TURNSTILE]
    end_terminal = term_id[LEFT_TURNSTILE]
    terminal_bits = lexgen.uint_type_bits(max(term_id.values()))
    bracket_bits = lexgen.uint_type_bits(2 * max(enc.values()))
    production_bits = lexgen.uint_type_bits(len(g.productions))

    # --- LLP pair table (llpHashTable, Encode.hs:514-536)
    hom = llp_homomorphisms(q, k, g)
    top = 1 << (bracket_bits - 1)
    int_table = {}
    for (back, ahead), (brackets, pi) in hom.items():
        back_i = [term_id[t] for t in back][:q]
        back_i = [empty_terminal] * (q - len(back_i)) + back_i
        ahead_i = [term_id[t] for t in ahead][:k]
        ahead_i = ahead_i + [empty_terminal] * (k - len(ahead_i))
        key = tuple(back_i + ahead_i)
        br = tuple((enc[s] | top) if kind == LB else enc[s] for kind, s in brackets)
        int_table[key] = (br, tuple(pi))
    items = sorted(int_table.items())
    stacks, prods, spans = [], [], []
    for key, (br, pi) in items:
        ss = len(stacks)
        stacks.extend(br)
        ps = len(prods)
        prods.extend(pi)
        spans.append((key, ((ss, len(stacks)), (ps, len(prods)))))
    arr, max_iters = open_addressing(spans)
    H = len(arr)
    ht_valid = np.array([a[0] for a in arr], dtype=np.bool_)
    ht_keys = np.array([list(a[1]) if a[1] is not None else [0] * (q + k) for a in arr], dtype=np.uint64).reshape(H, q + k)
    ht_stack_span = np.array([list(a[2][0]) if a[2] is not None else [0, 0] for a in arr], dtype=np.int64).reshape(H, 2)
    ht_prod_span = np.array([list(a[2][1]) if a[2] is not None else [0, 0] for a in arr], dtype=np.int64).reshape(H, 2)
    max_br = max([0] + [int(se - ss) for (ss, se) in ht_stack_span if ss >= 0])
    max_pr = max([0] + [int(pe - ps) for (ps, pe) in ht_prod_span if ps >= 0])

    arity = np.array([sum(1 for kd, _ in rhs if kd == NT) for _, rhs in g.productions], dtype=np.uint64)
    prod_is_terminal = np.array(
        [lhs != START_NT and lhs[1][0] == TM and used(lhs[1][1]) in term_id for lhs, _ in g.productions],
        dtype=np.bool_)

    # --- names (productionNames / nameTerminals, Encode.hs:505-512, Analyzer.hs:104-165)
    prod_names = []
    for i, (lhs, _) in enumerate(g.productions):
        if i in user_names:
            prod_names.append(user_names[i])
        elif lhs == START_NT:
            prod_names.append("start_%d" % i)
        elif lhs[1][0] == NT:
            prod_names.append("%s_%d" % (lhs[1][1], i))
        elif lhs[1][1][0] == 0:
            prod_names.append("%s_%d" % (lhs[1][1][1], i))
        else:
            prod_names.append("Literal_%d" % i)
    lex_terms = sorted((v, t) for t, v in term_id.items() if t[0] == 0)
    term_names = []
    for v, t in lex_terms:
        if t == UNUSED:
            term_names.append("empty_%d" % v)
        elif t[1][1][0] == 0:
            term_names.append(t[1][1][1])
        else:
            term_names.append("literal_%d" % v)

    # --- lexer (DFA + endomorphisms, encoded with the parser's terminal ids)
    rules = lexer_spec(cfg)
    ldfa = lexgen.merged_lexer_dfa(rules)
    pl = lexgen.parallel_lexer(ldfa)
    num_lex_terminals = len(lex_terms)  # AugmentedTerminal entries incl. Unused
    enc_lex = lexgen.encode_lexer(pl, lambda r: term_id[used(rules[r][0])], num_lex_terminals, empty_terminal)
    ignore_token = term_id.get(used(T("ignore")))

    length_bits = _length_bits(cfg, index32)

    return GrammarTables(
        name=name, q=q, k=k, index32=index32,
        terminal_bits=terminal_bits, production_bits=production_bits, bracket_bits=bracket_bits,
        length_bits=length_bits,
        lexer=enc_lex, ignore_token=ignore_token, dead_token=empty_terminal,
        empty_terminal=empty_terminal, start_terminal=start_terminal, end_terminal=end_terminal,
        stacks=np.array(stacks, dtype=_udtype(bracket_bits)),
        productions=np.array(prods, dtype=_udtype(production_bits)),
        ht_valid=ht_valid, ht_keys=ht_keys, ht_stack_span=ht_stack_span, ht_prod_span=ht_prod_span,
        max_iters=max_iters, max_brackets_per_pos=max_br, max_prods_per_pos=max_pr,
        arity=arity, prod_is_terminal=prod_is_terminal,
        terminal_names=term_names, production_names=prod_names,
        llp_pairs=int_table,
    )


def load(path: str, index32: bool = False) -> GrammarTables:
    import os
    with open(path, "r", encoding="utf-8") as f:
        return generate(f.read(), name=os.path.splitext(os.path.basename(path))[0], index32=index32)
