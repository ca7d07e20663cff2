"""alpacc's binary wire protocol (docs/wire-protocols.md; backends/c/cli.c:1-189).

Request frames are ``u64 frame_len, u64 n, payload``; a batch is ``u64 count``
followed by frames. The combined-mode response record is ``u8 valid`` and, when
valid, the structure-of-arrays sections (Generator/C/Generator.hs:114-152)::

    u64 num_tokens | terminal_t ids | index_t starts | length_t lengths
    u64 num_nodes  | production_t prods | index_t parents | index_t token_parents

The lexer-mode record (Generator.hs:87-102) is ``u8 valid, u64 count`` and per
lexeme ``terminal_t, index_t start, length_t length`` (array of structures);
the parser-mode record (Generator.hs:65-79) is ``u8 valid, u64 count,
production_t[count]``, and its request payload is ``n`` terminal ids
(``frame_len = 8 + n * sizeof(terminal_t)``).

All integers are little-endian at their native widths (``--layout``).
"""

from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np


def _dt(nbytes: int, signed: bool = False):
    return np.dtype(("i" if signed else "u") + str(nbytes)).newbyteorder("<")


@dataclass(frozen=True)
class Layout:
    """Native type sizes in bytes (``print_layout``, C/Generator.hs:153-158)."""

    terminal: int
    production: int
    index: int
    length: int
    parts: str = "both"

    @classmethod
    def of(cls, tables) -> "Layout":
        return cls(tables.terminal_bits // 8, tables.production_bits // 8, tables.index_bits // 8,
                   tables.length_bits // 8, getattr(tables, "parts", "both"))

    def text(self) -> str:
        """``print_layout`` of the program's mode (Generator.hs:80-84, 103-107, 153-158)."""
        if self.parts == "lexer":
            return "terminal_t=%d\nindex_t=%d\nlength_t=%d\n" % (self.terminal, self.index, self.length)
        if self.parts == "parser":
            return "terminal_t=%d\nproduction_t=%d\nindex_t=%d\n" % (self.terminal, self.production, self.index)
        return "terminal_t=%d\nproduction_t=%d\nindex_t=%d\nlength_t=%d\n" % (
            self.terminal, self.production, self.index, self.length)

    def input_bytes(self, n: int) -> int:
        """Payload bytes of a frame for ``n`` (``INPUT_BYTES``, Generator.hs:66, 88)."""
        return n * self.terminal if self.parts == "parser" else n


@dataclass
class ParseResult:
    """A decoded combined-mode record. ``valid`` False means reject."""

    valid: bool
    token_ids: np.ndarray | None = None
    token_starts: np.ndarray | None = None
    token_lengths: np.ndarray | None = None
    productions: np.ndarray | None = None
    parents: np.ndarray | None = None
    token_parents: np.ndarray | None = None

    def equal(self, other: "ParseResult") -> bool:
        if self.valid != other.valid:
            return False
        if not self.valid:
            return True
        for a in ("token_ids", "token_starts", "token_lengths", "productions", "parents", "token_parents"):
            if not np.array_equal(np.asarray(getattr(self, a), dtype=np.int64),
                                  np.asarray(getattr(other, a), dtype=np.int64)):
                return False
        return True


def encode_record(r: ParseResult, lay: Layout) -> bytes:
    """Serialise a result exactly as ``run_case`` does."""
    if not r.valid:
        return b"\x00"
    nt = len(r.token_ids)
    nn = len(r.productions)
    parts = [b"\x01", struct.pack("<Q", nt),
             np.asarray(r.token_ids).astype(_dt(lay.terminal)).tobytes(),
             np.asarray(r.token_starts).astype(_dt(lay.index, True)).tobytes(),
             np.asarray(r.token_lengths).astype(_dt(lay.length)).tobytes(),
             struct.pack("<Q", nn),
             np.asarray(r.productions).astype(_dt(lay.production)).tobytes(),
             np.asarray(r.parents).astype(_dt(lay.index, True)).tobytes(),
             np.asarray(r.token_parents).astype(_dt(lay.index, True)).tobytes()]
    return b"".join(parts)


def decode_record(buf: bytes, lay: Layout, pos: int = 0):
    """Decode one record at ``pos``; returns (ParseResult, next position)."""
    valid = buf[pos]
    pos += 1
    if valid == 0:
        return ParseResult(False), pos
    if valid != 1:
        raise ValueError("bad validity byte %d" % valid)

    def take(count, nbytes, signed=False):
        nonlocal pos
        a = np.frombuffer(buf, dtype=_dt(nbytes, signed), count=count, offset=pos)
        pos += count * nbytes
        return a

    (nt,) = struct.unpack_from("<Q", buf, pos)
    pos += 8
    ids = take(nt, lay.terminal)
    starts = take(nt, lay.index, True)
    lens = take(nt, lay.length)
    (nn,) = struct.unpack_from("<Q", buf, pos)
    pos += 8
    prods = take(nn, lay.production)
    parents = take(nn, lay.index, True)
    tparents = take(nt, lay.index, True)
    return ParseResult(True, ids, starts, lens, prods, parents, tparents), pos


def encode_frame(payload: bytes) -> bytes:
    return struct.pack("<QQ", 8 + len(payload), len(payload)) + payload


def encode_batch(payloads) -> bytes:
    payloads = list(payloads)
    return struct.pack("<Q", len(payloads)) + b"".join(encode_frame(p) for p in payloads)


def decode_batch(buf: bytes, lay: Layout):
    (count,) = struct.unpack_from("<Q", buf, 0)
    pos = 8
    out = []
    for _ in range(count):
        r, pos = decode_any_record(buf, lay, pos)
        out.append(r)
    return out, pos


@dataclass
class LexResult:
    """A decoded lexer-mode record."""

    valid: bool
    token_ids: np.ndarray | None = None
    token_starts: np.ndarray | None = None
    token_lengths: np.ndarray | None = None

    def equal(self, other: "LexResult") -> bool:
        if self.valid != other.valid:
            return False
        return not self.valid or all(
            np.array_equal(np.asarray(getattr(self, a), dtype=np.int64), np.asarray(getattr(other, a), dtype=np.int64))
            for a in ("token_ids", "token_starts", "token_lengths"))


@dataclass
class TokenParseResult:
    """A decoded parser-mode record: the derivation's productions."""

    valid: bool
    productions: np.ndarray | None = None

    def equal(self, other: "TokenParseResult") -> bool:
        if self.valid != other.valid:
            return False
        return not self.valid or np.array_equal(np.asarray(self.productions, dtype=np.int64),
                                                np.asarray(other.productions, dtype=np.int64))


def _lexeme_dtype(lay: Layout):
    return np.dtype([("id", _dt(lay.terminal)), ("start", _dt(lay.index, True)), ("length", _dt(lay.length))])


def encode_lex_record(r: LexResult, lay: Layout) -> bytes:
    if not r.valid:
        return b"\x00"
    a = np.zeros(len(r.token_ids), dtype=_lexeme_dtype(lay))
    a["id"], a["start"], a["length"] = r.token_ids, r.token_starts, r.token_lengths
    return b"\x01" + struct.pack("<Q", len(a)) + a.tobytes()


def decode_lex_record(buf: bytes, lay: Layout, pos: int = 0):
    valid = buf[pos]
    pos += 1
    if valid == 0:
        return LexResult(False), pos
    if valid != 1:
        raise ValueError("bad validity byte %d" % valid)
    (n,) = struct.unpack_from("<Q", buf, pos)
    pos += 8
    dt = _lexeme_dtype(lay)
    a = np.frombuffer(buf, dtype=dt, count=n, offset=pos)
    pos += n * dt.itemsize
    return LexResult(True, a["id"].copy(), a["start"].copy(), a["length"].copy()), pos


def encode_token_parse_record(r: TokenParseResult, lay: Layout) -> bytes:
    if not r.valid:
        return b"\x00"
    p = np.asarray(r.productions).astype(_dt(lay.production))
    return b"\x01" + struct.pack("<Q", len(p)) + p.tobytes()


def decode_token_parse_record(buf: bytes, lay: Layout, pos: int = 0):
    valid = buf[pos]
    pos += 1
    if valid == 0:
        return TokenParseResult(False), pos
    if valid != 1:
        raise ValueError("bad validity byte %d" % valid)
    (n,) = struct.unpack_from("<Q", buf, pos)
    pos += 8
    p = np.frombuffer(buf, dtype=_dt(lay.production), count=n, offset=pos).copy()
    return TokenParseResult(True, p), pos + n * lay.production


def decode_any_record(buf: bytes, lay: Layout, pos: int = 0):
    """Decode one record of the layout's mode."""
    if lay.parts == "lexer":
        return decode_lex_record(buf, lay, pos)
    if lay.parts == "parser":
        return decode_token_parse_record(buf, lay, pos)
    return decode_record(buf, lay, pos)


def encode_mode_frame(payload: bytes, lay: Layout) -> bytes:
    """A request frame whose ``n`` counts the mode's input units (bytes, or
    terminal ids for the parser-mode program)."""
    unit = lay.terminal if lay.parts == "parser" else 1
    if len(payload) % unit:
        raise ValueError("payload is not a whole number of terminal ids")
    return struct.pack("<QQ", 8 + len(payload), len(payload) // unit) + payload
