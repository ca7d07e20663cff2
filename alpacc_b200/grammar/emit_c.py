"""Emission of the generated C program's constant sections.

Restates the text the reference's C emitter writes before each runtime template
(src/Alpacc/Generator/C/Generator.hs:24-60,161-201; C/Lexer.hs:16-58;
C/Parser.hs:21-95): includes, ``terminal_t``/``index_t``/``length_t`` typedefs,
the lexer constants (TO_STATE, COMPOSE, ACCEPT, masks, IDENTITY, IGNORE_TOKEN)
and the parser constants (Q, K, sentinels, hash table, STACKS, PRODUCTIONS,
arities, terminal-production flags). The runtime templates themselves
(lexer.c, parser.c, cli.c) are not part of this module.
"""

from __future__ import annotations

import numpy as np

from .tables import GrammarTables

INCLUDES = [
    "#define _POSIX_C_SOURCE 200809L",
    "#include <stdint.h>",
    "#include <stdbool.h>",
    "#include <stdio.h>",
    "#include <stdlib.h>",
    "#include <string.h>",
    "#include <time.h>",
]


def _uint(bits: int) -> str:
    return "uint%d_t" % bits


def _list(xs) -> str:
    return "{" + ", ".join(xs) + "}"


def _ints(a) -> str:
    return _list([str(int(x)) for x in np.asarray(a).reshape(-1)])


def _bools(a) -> str:
    return _list(["true" if bool(x) else "false" for x in np.asarray(a).reshape(-1)])


def unlines(lines) -> str:
    return "".join(l + "\n" for l in lines)


def index_typedef(t: GrammarTables) -> str:
    """``indexTypedef`` (C/Generator.hs:36-53)."""
    lines = (["#define INDEX32"] if t.index32 else []) + [
        "#ifdef INDEX32",
        "typedef int32_t index_t;",
        "#else",
        "typedef int64_t index_t;",
        "#endif",
        "typedef %s length_t;" % _uint(t.length_bits),
    ]
    return unlines(lines)


def lexer_constants(t: GrammarTables) -> str:
    """``generateLexer`` (C/Lexer.hs:16-58)."""
    L = t.lexer
    st = _uint(L.state_bits)
    ign = "#define IGNORE_TOKEN ((terminal_t) %d)" % t.ignore_token if t.ignore_token is not None else ""
    text = "\n".join([
        "typedef %s state_t;" % st,
        "",
        "#define NUM_STATES %d" % L.num_states,
        "#define NUM_TRANS 256",
        ign,
        "#define ENDO_MASK   ((state_t) %d)" % L.index_mask,
        "#define ENDO_OFFSET ((state_t) %d)" % L.index_offset,
        "#define TERMINAL_MASK   ((state_t) %d)" % L.token_mask,
        "#define TERMINAL_OFFSET ((state_t) %d)" % L.token_offset,
        "#define PRODUCE_MASK   ((state_t) %d)" % L.produce_mask,
        "#define PRODUCE_OFFSET ((state_t) %d)" % L.produce_offset,
        "#define IDENTITY ((state_t) %d)" % L.identity,
        "",
        "static const state_t TO_STATE[NUM_TRANS] =",
        "  " + _ints(L.to_state) + ";",
        "",
        "static const state_t COMPOSE[NUM_STATES * NUM_STATES] =",
        "  " + _ints(L.compose) + ";",
        "",
        "static const bool ACCEPT[NUM_STATES] =",
        "  " + _bools(L.accept) + ";",
    ])
    return text.strip()


def parser_constants(t: GrammarTables, with_tree: bool = True) -> str:
    """``generateParser`` / ``generateParserWithTree`` (C/Parser.hs:21-95)."""
    keys = _list([_list(["(terminal_t) %d" % int(x) for x in row]) for row in t.ht_keys])
    sspan = _list([_list([str(int(a)), str(int(b))]) for a, b in t.ht_stack_span])
    pspan = _list([_list([str(int(a)), str(int(b))]) for a, b in t.ht_prod_span])
    text = "\n".join([
        "typedef %s production_t;" % _uint(t.production_bits),
        "typedef %s bracket_t;" % _uint(t.bracket_bits),
        "#define Q %d" % t.q,
        "#define K %d" % t.k,
        "#define EMPTY_TERMINAL ((terminal_t) %d)" % t.empty_terminal,
        "#define START_TERMINAL ((terminal_t) %d)" % t.start_terminal,
        "#define END_TERMINAL ((terminal_t) %d)" % t.end_terminal,
        "#define HASH_TABLE_SIZE %d" % t.hash_size,
        "#define MAX_ITERS %d" % t.max_iters,
        "#define STACKS_SIZE %d" % len(t.stacks),
        "#define PRODUCTIONS_SIZE %d" % len(t.productions),
        "#define MAX_BRACKETS_PER_POSITION %d" % t.max_brackets_per_pos,
        "#define MAX_PRODS_PER_POSITION %d" % t.max_prods_per_pos,
        "static const bracket_t STACKS[STACKS_SIZE] =",
        "  " + _ints(t.stacks) + ";",
        "static const production_t PRODUCTIONS[PRODUCTIONS_SIZE] =",
        "  " + _ints(t.productions) + ";",
        "static const bool HASH_TABLE_IS_VALID[HASH_TABLE_SIZE] =",
        "  " + _bools(t.ht_valid) + ";",
        "static const terminal_t HASH_TABLE_KEYS[HASH_TABLE_SIZE][Q + K] =",
        "  " + keys + ";",
        "static const int64_t HASH_TABLE_STACKS_SPAN[HASH_TABLE_SIZE][2] =",
        "  " + sspan + ";",
        "static const int64_t HASH_TABLE_PRODUCTIONS_SPAN[HASH_TABLE_SIZE][2] =",
        "  " + pspan + ";",
    ]).strip()
    if with_tree:
        tree = "\n".join([
            "#define ALPACC_WITH_TREE",
            "#define NUMBER_OF_PRODUCTIONS %d" % t.num_productions,
            "static const uint64_t PRODUCTION_TO_ARITY[NUMBER_OF_PRODUCTIONS] =",
            "  " + _ints(t.arity) + ";",
            "static const bool PRODUCTION_TO_TERMINAL_IS_VALID[NUMBER_OF_PRODUCTIONS] =",
            "  " + _bools(t.prod_is_terminal) + ";",
        ]).strip()
        text = text + "\n" + tree
    return text


PROGRAM_KIND = {"both": "combined lexer+parser", "lexer": "lexer", "parser": "parser"}


def program_prefix(t: GrammarTables) -> str:
    """Everything before the lexer or parser constants (C/Generator.hs:161-196)."""
    meta = ["// alpacc %s for grammar %s" % (PROGRAM_KIND[t.parts], t.name)]
    return unlines([
        unlines(meta),
        unlines(INCLUDES),
        "typedef %s terminal_t;" % _uint(t.terminal_bits),
        index_typedef(t),
        unlines(["static void     write_u64le(FILE *f, uint64_t v);"]),
    ])


def constants(t: GrammarTables) -> str:
    """The constant sections of the program ``t.parts`` names: the lexer's for
    the lexer-mode program, the parser's without the tree section for the
    parser-mode one, both (with the tree section) for the combined one."""
    parts = [program_prefix(t)]
    if t.parts != "parser":
        parts.append(lexer_constants(t))
    if t.parts != "lexer":
        parts.append(parser_constants(t, with_tree=t.parts == "both"))
    return unlines(parts)
