/*
 * Glue between a grammar's emitted constants (the C emitter's output,
 * src/Alpacc/Generator/C/{Lexer,Parser}.hs) and the C ABI: builds the
 * alpacc_tables descriptor from the constants in scope (those of the
 * combined, lexer-mode or parser-mode program) and loads the grammar on
 * device 0 on first use.
 */
#include "alpacc_b200.h"

/* Bytes per unit of a frame's n: terminal ids for the parser-mode program
   (INPUT_BYTES, C/Generator.hs:66, 88, 116). */
#if defined(Q) && !defined(NUM_TRANS)
#define WIRE_UNIT ((uint64_t)sizeof(terminal_t))
#else
#define WIRE_UNIT ((uint64_t)1)
#endif

/* print_layout of the program's mode (C/Generator.hs:80-84, 103-107,
   153-158): the same lines alpacc_gpu_layout gives for these tables. */
static void print_layout(FILE *f) {
  fprintf(f, "terminal_t=%zu\n", sizeof(terminal_t));
#ifdef Q
  fprintf(f, "production_t=%zu\n", sizeof(production_t));
#endif
  fprintf(f, "index_t=%zu\n", sizeof(index_t));
#ifdef NUM_TRANS
  fprintf(f, "length_t=%zu\n", sizeof(length_t));
#endif
}

static alpacc_gpu_grammar *gpu_grammar(void) {
  static alpacc_gpu_grammar *g = NULL;
  if (!g) {
    alpacc_tables t;
    memset(&t, 0, sizeof t);
    t.abi_version = ALPACC_ABI_VERSION;
    t.terminal_size = sizeof(terminal_t);
    t.index_size = sizeof(index_t);
    t.length_size = sizeof(length_t);
#if defined(NUM_TRANS) && defined(Q)
    t.parts = ALPACC_PARTS_BOTH;
#elif defined(NUM_TRANS)
    t.parts = ALPACC_PARTS_LEXER;
#else
    t.parts = ALPACC_PARTS_PARSER;
#endif
#ifdef NUM_TRANS /* lexer constants (C/Lexer.hs:16-58) */
    t.state_size = sizeof(state_t);
    t.num_states = NUM_STATES;
    t.endo_mask = ENDO_MASK;
    t.endo_offset = ENDO_OFFSET;
    t.terminal_mask = TERMINAL_MASK;
    t.terminal_offset = TERMINAL_OFFSET;
    t.produce_mask = PRODUCE_MASK;
    t.produce_offset = PRODUCE_OFFSET;
    t.identity = IDENTITY;
#ifdef IGNORE_TOKEN
    t.ignore_token = IGNORE_TOKEN;
#else
    t.ignore_token = -1;
#endif
    t.to_state = TO_STATE;
    t.compose = COMPOSE;
    t.accept = (const uint8_t *)ACCEPT;
#endif
#ifdef Q /* parser constants (C/Parser.hs:21-95) */
    t.production_size = sizeof(production_t);
    t.bracket_size = sizeof(bracket_t);
    t.q = Q;
    t.k = K;
    t.empty_terminal = EMPTY_TERMINAL;
    t.start_terminal = START_TERMINAL;
    t.end_terminal = END_TERMINAL;
    t.hash_table_size = HASH_TABLE_SIZE;
    t.max_iters = MAX_ITERS;
    t.stacks_size = STACKS_SIZE;
    t.productions_size = PRODUCTIONS_SIZE;
    t.max_brackets_per_position = MAX_BRACKETS_PER_POSITION;
    t.max_prods_per_position = MAX_PRODS_PER_POSITION;
    t.stacks = STACKS;
    t.productions = PRODUCTIONS;
    t.hash_table_is_valid = (const uint8_t *)HASH_TABLE_IS_VALID;
    t.hash_table_keys = HASH_TABLE_KEYS;
    t.hash_table_stacks_span = &HASH_TABLE_STACKS_SPAN[0][0];
    t.hash_table_productions_span = &HASH_TABLE_PRODUCTIONS_SPAN[0][0];
#endif
#ifdef ALPACC_WITH_TREE
    t.number_of_productions = NUMBER_OF_PRODUCTIONS;
    t.production_to_arity = PRODUCTION_TO_ARITY;
    t.production_to_terminal_is_valid = (const uint8_t *)PRODUCTION_TO_TERMINAL_IS_VALID;
#endif
    int err = 0;
    g = alpacc_gpu_load(&t, 0, 0, &err);
    if (!g) {
      fprintf(stderr, "error: alpacc_gpu_load: %s\n", alpacc_strerror(err));
      exit(1);
    }
  }
  return g;
}
