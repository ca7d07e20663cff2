"""Lexer table construction: regexes -> merged lexer DFA -> endomorphism monoid.

Restates the reference generator's lexer half:

* per-terminal minimal DFA (``fromRegExToNFA`` ``src/Alpacc/Lexer/NFA.hs:111-137``,
  ``fromNFAtoDFA``/``minimize``/``removeUselessStates``
  ``src/Alpacc/Lexer/DFA.hs:122-251``);
* the merged lexer DFA over the union of those DFAs, with the token map chosen by
  rule priority and the maximal-munch "producing" transitions
  (``lexerDFA`` ``DFA.hs:322-395``, ``tokenProducingTransitions`` ``DFA.hs:261-299``);
* the byte endomorphisms and their composition closure (``endomorphismTable``
  ``src/Alpacc/Lexer/DFAParallelLexer.hs:45-104``, ``parallelLexer``
  ``src/Alpacc/Lexer/ParallelLexing.hs:265-429``), reproducing the reference's
  discovery order so endomorphism ids match;
* the bit-packed ``state_t`` encoding ``[index | terminal | produce]``
  (``src/Alpacc/Lexer/Encode.hs:33-171``).

Only the language of each per-terminal DFA matters for the merged automaton, and
the merged automaton is used only up to isomorphism (endomorphisms are compared
for equality), so the DFA state numbering here is free; the endomorphism ids,
which are visible in the emitted tables, follow the reference's order exactly.
"""

from __future__ import annotations

import heapq
from dataclasses import dataclass

import numpy as np

# ---------------------------------------------------------------------------
# Regex -> minimal DFA
# ---------------------------------------------------------------------------


class _NFA:
    def __init__(self):
        self.eps = {}  # state -> set
        self.trans = {}  # (state, byte) -> set
        self.n = 0

    def new(self):
        s = self.n
        self.n += 1
        return s

    def add_eps(self, a, b):
        self.eps.setdefault(a, set()).add(b)

    def add(self, a, byte, b):
        self.trans.setdefault((a, byte), set()).add(b)

    def chain(self, a, bs: bytes, b):
        """``newTransitions`` (NFA.hs:84-92): a byte chain a -b0-> . -b1-> ... b."""
        cur = a
        for i, byte in enumerate(bs):
            nxt = b if i == len(bs) - 1 else self.new()
            self.add(cur, byte, nxt)
            cur = nxt

    def build(self, s, e, r):
        """Thompson-style construction following ``auxRegExToNFA`` (NFA.hs:94-109)."""
        tag = r[0]
        if tag == "eps":
            self.add_eps(s, e)
        elif tag == "lit":
            self.chain(s, r[1], e)
        elif tag == "range":
            for bs in r[1]:
                self.chain(s, bs, e)
        elif tag == "cat":
            m = self.new()
            self.build(s, m, r[1])
            self.build(m, e, r[2])
        elif tag == "star":
            m = self.new()
            self.add_eps(s, m)
            self.add_eps(m, e)
            self.build(m, m, r[1])
        elif tag == "alt":
            self.build(s, e, r[1])
            self.build(s, e, r[2])
        else:  # pragma: no cover
            raise ValueError(tag)

    def closure(self, states):
        stack = list(states)
        out = set(states)
        while stack:
            x = stack.pop()
            for y in self.eps.get(x, ()):
                if y not in out:
                    out.add(y)
                    stack.append(y)
        return frozenset(out)


def _regex_bytes(r, acc):
    tag = r[0]
    if tag == "lit":
        acc.update(r[1])
    elif tag == "range":
        for bs in r[1]:
            acc.update(bs)
    elif tag in ("cat", "alt"):
        _regex_bytes(r[1], acc)
        _regex_bytes(r[2], acc)
    elif tag == "star":
        _regex_bytes(r[1], acc)
    return acc


@dataclass
class DFA:
    """Partial DFA: states ``0..n-1``, no dead state, every state useful."""

    n: int
    initial: int
    accepting: frozenset
    trans: dict  # (state, byte) -> state
    alphabet: tuple


def regex_to_min_dfa(regex) -> DFA:
    """Minimal partial DFA of a regex's language (the reference pipeline
    ``minimize . fromNFAtoDFA . fromRegExToNFA`` DFA.hs:338-344)."""
    nfa = _NFA()
    s0, s1 = nfa.new(), nfa.new()
    nfa.build(s0, s1, regex)
    alphabet = tuple(sorted(_regex_bytes(regex, set())))
    # subset construction (DFA.hs:63-147)
    start = nfa.closure({s0})
    index = {start: 0}
    order = [start]
    trans = {}
    i = 0
    while i < len(order):
        cur = order[i]
        i += 1
        for b in alphabet:
            nxt = set()
            for x in cur:
                nxt |= nfa.trans.get((x, b), set())
            if not nxt:
                continue
            nxt = nfa.closure(nxt)
            if nxt not in index:
                index[nxt] = len(order)
                order.append(nxt)
            trans[(index[cur], b)] = index[nxt]
    n = len(order)
    acc = {index[s] for s in order if s1 in s}
    # Moore partition refinement on the total DFA (dead state = n).
    dead = n
    tot = lambda s, b: trans.get((s, b), dead) if s != dead else dead  # noqa: E731
    cls = [1 if s in acc else 0 for s in range(n)] + [0]
    while True:
        sig = {}
        new = []
        for s in range(n + 1):
            key = (cls[s],) + tuple(cls[tot(s, b)] for b in alphabet)
            if key not in sig:
                sig[key] = len(sig)
            new.append(sig[key])
        if len(set(new)) == len(set(cls)):
            cls = new
            break
        cls = new
    dead_cls = cls[dead]
    # renumber the live classes in BFS order from the initial state
    live = {}
    q = [cls[0]]
    live[cls[0]] = 0
    rep = {}
    for s in range(n):
        rep.setdefault(cls[s], s)
    k = 0
    mtrans = {}
    while k < len(q):
        c = q[k]
        k += 1
        s = rep[c]
        for b in alphabet:
            t = cls[tot(s, b)]
            if t == dead_cls:
                continue
            if t not in live:
                live[t] = len(q)
                q.append(t)
            mtrans[(live[c], b)] = live[t]
    macc = frozenset(live[cls[s]] for s in acc)
    return DFA(len(q), 0, macc, mtrans, alphabet)


# ---------------------------------------------------------------------------
# Merged lexer DFA with producing transitions (DFA.hs:261-395)
# ---------------------------------------------------------------------------


@dataclass
class LexerDFA:
    """States ``1..S`` (0 is dead); ``trans`` includes producing transitions."""

    num_states: int  # S
    initial: int
    accepting: frozenset
    trans: dict  # (state, byte) -> state
    producing: frozenset  # {(state, byte)}
    token: dict  # state -> terminal (order index into the rule list)
    alphabet: tuple


def merged_lexer_dfa(rules) -> LexerDFA:
    """``lexerDFA`` (DFA.hs:322-395). ``rules`` is the prioritised rule list
    ``[(terminal, regex)]``; the token of a state is the lowest-index rule whose
    DFA accepts there (``minimumSet`` on ``orderMap``, DFA.hs:360-373)."""
    dfas = [regex_to_min_dfa(r) for _, r in rules]
    alphabet = tuple(sorted(set().union(*[set(d.alphabet) for d in dfas])))
    k = len(dfas)
    init = (True, tuple(d.initial for d in dfas))
    index = {init: 0}
    order = [init]
    trans = {}
    i = 0
    while i < len(order):
        flag, comps = order[i]
        for b in alphabet:
            nxt = tuple(
                (dfas[j].trans.get((c, b)) if c is not None else None) for j, c in enumerate(comps)
            )
            if all(c is None for c in nxt):
                continue
            key = (False, nxt)
            if key not in index:
                index[key] = len(order)
                order.append(key)
            trans[(i, b)] = index[key]
        i += 1
    n = len(order)

    def accepts(st):
        return [j for j, c in enumerate(st[1]) if c is not None and c in dfas[j].accepting]

    acc = {s for s in range(n) if accepts(order[s])}
    # removeUselessStates (DFA.hs:169-183): keep states that reach acceptance
    useful = set(acc)
    changed = True
    while changed:
        changed = False
        for (s, _b), t in trans.items():
            if t in useful and s not in useful:
                useful.add(s)
                changed = True
    keep = [s for s in range(n) if s in useful]
    ren = {s: i + 1 for i, s in enumerate(keep)}  # states 1..S, dead = 0
    trans2 = {(ren[s], b): ren[t] for (s, b), t in trans.items() if s in useful and t in useful}
    acc2 = frozenset(ren[s] for s in acc)
    token = {ren[s]: min(accepts(order[s])) for s in acc}
    initial = ren[0]
    # producing transitions (DFA.hs:261-299): from accepting q on byte t with no
    # transition of its own, jump to where the initial state goes on t.
    producing = set()
    for q in sorted(acc2):
        for b in alphabet:
            if (initial, b) in trans2 and (q, b) not in trans2:
                producing.add((q, b))
    for q, b in producing:
        trans2[(q, b)] = trans2[(initial, b)]
    return LexerDFA(len(keep), initial, acc2, trans2, frozenset(producing), token, alphabet)


# ---------------------------------------------------------------------------
# Endomorphism closure (ParallelLexing.hs, DFAParallelLexer.hs)
# ---------------------------------------------------------------------------


@dataclass
class EndoData:
    e: int
    token: int | None  # rule index or None
    accepting: bool
    producing: bool


@dataclass
class ParallelLexer:
    num_endos: int  # endomorphismsSize
    to_endo: list  # 256 -> EndoData
    comp: np.ndarray  # [N, N] int32 endo id of the composition (default dead=1)
    data: list  # e -> EndoData
    num_dfa_states: int


IDENTITY_E = 0
DEAD_E = 1


def _closure_lib():
    """The C restatement of the closure (closure.c), built in-tree on first use."""
    import ctypes
    import os
    import subprocess
    here = os.path.dirname(os.path.abspath(__file__))
    so = os.path.join(here, "_closure.so")
    src = os.path.join(here, "closure.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-shared", "-fPIC", src, "-o", so])
    lib = ctypes.CDLL(so)
    lib.alpacc_endo_closure.restype = ctypes.c_int
    return lib


def _closure_c(S1, byte_endos, conn0):
    import ctypes
    lib = _closure_lib()
    nb = len(byte_endos)
    ss = np.ascontiguousarray(np.array([e[0] for e in byte_endos], dtype=np.uint16).reshape(nb, S1))
    bs = np.ascontiguousarray(np.array([e[1] for e in byte_endos], dtype=np.uint8).reshape(nb, S1))
    c0 = np.ascontiguousarray(conn0.astype(np.uint8))
    n = ctypes.c_int()
    pss = ctypes.POINTER(ctypes.c_uint16)()
    pbs = ctypes.POINTER(ctypes.c_uint8)()
    pcomp = ctypes.POINTER(ctypes.c_int32)()
    rc = lib.alpacc_endo_closure(
        ctypes.c_int(S1), ctypes.c_int(nb), ss.ctypes.data_as(ctypes.c_void_p), bs.ctypes.data_as(ctypes.c_void_p),
        c0.ctypes.data_as(ctypes.c_void_p), ctypes.byref(n), ctypes.byref(pss), ctypes.byref(pbs), ctypes.byref(pcomp))
    if rc != 0:
        raise RuntimeError("Error: Happend during Parallel Lexing genration, contact a maintainer. (%d)" % rc)
    N = n.value
    images = np.ctypeslib.as_array(pss, shape=(N * S1,)).reshape(N, S1).copy()
    flags = np.ctypeslib.as_array(pbs, shape=(N * S1,)).reshape(N, S1).copy()
    comp = np.ctypeslib.as_array(pcomp, shape=(N * N,)).reshape(N, N).copy()
    for p_ in (pss, pbs, pcomp):
        lib.alpacc_closure_free(ctypes.cast(p_, ctypes.c_void_p))
    comp[comp < 0] = DEAD_E
    return images, flags, comp


def _closure_py(S1, byte_endos, conn0):
    """Pure-Python restatement of ``endoCompositionsTable`` (ParallelLexing.hs:311-403)."""
    nb = len(byte_endos)
    ident = (tuple(range(S1)), (False,) * S1)
    dead = ((0,) * S1, (False,) * S1)
    e_to_endo = {0: ident, 1: dead}
    endo_to_e = {}
    for i, en in enumerate(byte_endos):
        e_to_endo[i + 2] = en
        endo_to_e[en] = i + 2
    comps = {(0, 0): 0}
    for e in list(e_to_endo):
        comps[(0, e)] = e
        comps[(e, 0)] = e
    conn = {i + 2: {j + 2 for j in range(nb) if conn0[i, j]} for i in range(nb)}
    inv = {}
    for e, fs in conn.items():
        for x in fs:
            inv.setdefault(x, set()).add(e)
    max_e = nb + 1
    heap = []
    pending = set()

    def push(e, f):
        if (e, f) not in pending:
            pending.add((e, f))
            heapq.heappush(heap, (e, f))

    for e, fs in conn.items():
        for f in fs:
            push(e, f)
    while heap:
        e, f = heapq.heappop(heap)
        pending.discard((e, f))
        if (e, f) in comps:
            continue
        a_ss = e_to_endo[e][0]
        b_ss, b_bs = e_to_endo[f]
        en = (tuple(b_ss[x] for x in a_ss), tuple(b_bs[x] for x in a_ss))
        g = endo_to_e.get(en)
        if g is None:
            max_e += 1
            g = max_e
            endo_to_e[en] = g
            e_to_endo[g] = en
            comps[(0, g)] = g
            comps[(g, 0)] = g
        comps[(e, f)] = g
        if e not in inv or f not in conn:
            raise RuntimeError("Error: Happend during Parallel Lexing genration, contact a maintainer.")
        pre = inv[e] - inv.get(g, set())
        post = conn[f] - conn.get(g, set())
        new_map = {x: {g} for x in pre}
        new_map.setdefault(g, set()).update(post)
        new_inv = {g: set(pre)}
        for x in post:
            new_inv.setdefault(x, set()).add(g)
        for k_, v in new_map.items():
            conn.setdefault(k_, set()).update(v)
        for k_, v in new_inv.items():
            inv.setdefault(k_, set()).update(v)
        for k_, v in new_map.items():
            for x in v:
                push(k_, x)
    N = max_e + 1
    images = np.array([e_to_endo[e][0] for e in range(N)], dtype=np.uint16)
    flags = np.array([e_to_endo[e][1] for e in range(N)], dtype=np.uint8)
    comp = np.full((N, N), DEAD_E, dtype=np.int32)
    for (a, b), c in comps.items():
        comp[a, b] = c
    return images, flags, comp


def parallel_lexer(ldfa: LexerDFA, use_c: bool = True) -> ParallelLexer:
    """``dfaParallelLexer``/``parallelLexer`` (DFAParallelLexer.hs:97-104,
    ParallelLexing.hs:530-555)."""
    S = ldfa.num_states
    S1 = S + 1
    init = ldfa.initial

    def endo_of(b):  # endomorphismTable (DFAParallelLexer.hs:45-74)
        ss = tuple([0] + [ldfa.trans.get((s, b), 0) for s in range(1, S1)])
        bs = tuple([False] + [((s, b) in ldfa.producing) for s in range(1, S1)])
        return (ss, bs)

    endo_table = {b: endo_of(b) for b in ldfa.alphabet}
    byte_endos = []
    idx_of = {}
    for b in ldfa.alphabet:  # enumerate initE (nub (elems endo_table))
        en = endo_table[b]
        if en not in idx_of:
            idx_of[en] = len(byte_endos)
            byte_endos.append(en)
    # connectedTable (ParallelLexing.hs:405-431): bytes that can follow byte t
    reach, outs = {}, {}
    for (s, b), t in ldfa.trans.items():
        reach.setdefault(b, set()).add(t)
        outs.setdefault(s, set()).add(b)
    nb = len(byte_endos)
    conn0 = np.zeros((nb, nb), dtype=np.bool_)
    for b in ldfa.alphabet:
        i = idx_of[endo_table[b]]
        for s in reach.get(b, ()):
            for x in outs.get(s, ()):
                conn0[i, idx_of[endo_table[x]]] = True
    images, flags, comp = (_closure_c if use_c else _closure_py)(S1, byte_endos, conn0)
    N = images.shape[0]
    data = [EndoData(0, None, False, False), EndoData(1, None, False, False)]
    for e in range(2, N):  # toEndoData (ParallelLexing.hs:194-210)
        s = int(images[e, init])
        data.append(EndoData(e, ldfa.token.get(s), s in ldfa.accepting, bool(flags[e, init])))
    to_endo = [data[idx_of[endo_table[b]] + 2] if b in endo_table else data[DEAD_E] for b in range(256)]
    return ParallelLexer(N, to_endo, comp, data, S)


def find_bit_size(x: int) -> int:
    """``findBitSize`` (Lexer/Encode.hs:33-36): bits to hold ``x`` distinct values."""
    return max(1, x - 1).bit_length()


def uint_type_bits(max_value: int) -> int:
    """``toIntType`` for ``UInt`` (Types.hs:21-26): smallest of 8/16/32/64 bits."""
    for bits in (8, 16, 32, 64):
        if max_value <= (1 << bits) - 1:
            return bits
    raise ValueError("value does not fit in 64 bits")


@dataclass
class EncodedLexer:
    state_bits: int  # width of state_t
    num_states: int  # NUM_STATES (number of endomorphisms)
    index_mask: int
    index_offset: int
    token_mask: int
    token_offset: int
    produce_mask: int
    produce_offset: int
    identity: int
    to_state: np.ndarray  # [256] state_t
    compose: np.ndarray  # [N*N] state_t, row-major by the first argument
    accept: np.ndarray  # [N] bool
    num_dfa_states: int


def encode_lexer(pl: ParallelLexer, terminal_id, num_terminals: int, dead_terminal: int) -> EncodedLexer:
    """``intParallelLexer`` + ``stateIntType`` (Lexer/Encode.hs:38-171).

    ``terminal_id`` maps a rule index to its terminal id; tokens of ``None`` map
    to ``dead_terminal`` (``terminalDead``)."""
    sizes = [pl.num_endos, num_terminals, 1]
    bits = [find_bit_size(s) for s in sizes]
    if sum(bits) > 64:
        raise ValueError("Error: There are too many tokens and/or states to create a data parallel lexer.")
    offs = [0, bits[0], bits[0] + bits[1]]
    masks = [((1 << b) - 1) << o for b, o in zip(bits, offs)]
    state_bits = uint_type_bits((1 << sum(bits)) - 1)

    def enc(d: EndoData) -> int:
        t = dead_terminal if d.token is None else terminal_id(d.token)
        return d.e | (t << offs[1]) | (int(d.producing) << offs[2])

    dt = {8: np.uint8, 16: np.uint16, 32: np.uint32, 64: np.uint64}[state_bits]
    enc_by_e = np.array([enc(d) for d in pl.data], dtype=np.uint64)
    to_state = np.array([enc(d) for d in pl.to_endo], dtype=np.uint64).astype(dt)
    compose = enc_by_e[pl.comp.reshape(-1)].astype(dt)
    accept = np.array([d.accepting for d in pl.data], dtype=np.bool_)
    return EncodedLexer(
        state_bits=state_bits,
        num_states=pl.num_endos,
        index_mask=masks[0],
        index_offset=offs[0],
        token_mask=masks[1],
        token_offset=offs[1],
        produce_mask=masks[2],
        produce_offset=offs[2],
        identity=int(enc(pl.data[IDENTITY_E])),
        to_state=to_state,
        compose=compose,
        accept=accept,
        num_dfa_states=pl.num_dfa_states,
    )
