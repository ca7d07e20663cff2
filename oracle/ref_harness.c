/*
 * In-memory harness around the reference's generated C program (oracle/_ref).
 *
 * TEST INFRASTRUCTURE ONLY: used by the tests and by bench.py's CPU-baseline
 * leg as the checker / baseline, never by the product path.
 *
 * The generated program (assembled by oracle/build_ref.py from the reference's
 * backends/c/{lexer,parser,cli}.c and its run_case text) is #included with its
 * main() renamed, so its static functions can be called directly:
 *   - ref_run_case: the exact response record bytes that run_case
 *     (src/Alpacc/Generator/C/Generator.hs:114-152) writes, captured with
 *     open_memstream;
 *   - ref_pipeline: lex_string -> parse_test -> compute_parents -> compact_tree
 *     without serialisation, the in-memory timing harness for the CPU baseline;
 *   - ref_layout: the type sizes print_layout reports;
 *   - ref_input_unit: the bytes per unit of run_case's n.
 *   - ref_run_case_sink: the same record streamed to a callback in large
 *     pieces (fopencookie), so records of several GB can be digested without
 *     holding them in memory.
 * The same harness wraps the lexer-mode and parser-mode programs (no
 * ref_pipeline there).
 */
#define _GNU_SOURCE 1 /* fopencookie */
#include <stdio.h>
#include <sys/types.h>
#define main alpacc_generated_main
#include ALPACC_GENERATED
#undef main

int ref_run_case(uint64_t n, const uint8_t *in, uint8_t **out, size_t *out_len) {
  char *buf = NULL;
  size_t len = 0;
  FILE *f = open_memstream(&buf, &len);
  if (!f) return -1;
  run_case(n, in, f);
  fclose(f);
  *out = (uint8_t *)buf;
  *out_len = len;
  return 0;
}

void ref_free(void *p) { free(p); }

typedef void (*ref_sink_fn)(void *user, const char *buf, size_t size);
struct ref_sink_cookie {
  ref_sink_fn fn;
  void *user;
};

static ssize_t ref_sink_write(void *c, const char *buf, size_t size) {
  struct ref_sink_cookie *k = (struct ref_sink_cookie *)c;
  k->fn(k->user, buf, size);
  return (ssize_t)size;
}

int ref_run_case_sink(uint64_t n, const uint8_t *in, ref_sink_fn fn, void *user) {
  struct ref_sink_cookie k = {fn, user};
  cookie_io_functions_t io = {NULL, ref_sink_write, NULL, NULL};
  FILE *f = fopencookie(&k, "w", io);
  if (!f) return -1;
  setvbuf(f, NULL, _IOFBF, (size_t)64 << 20);
  run_case(n, in, f);
  fclose(f);
  return 0;
}

/* Units of run_case's n: bytes, or terminal ids in the parser-mode program
   (INPUT_BYTES, C/Generator.hs:66, 88). */
uint64_t ref_input_unit(void) { return INPUT_BYTES(1); }

#ifdef ALPACC_WITH_TREE
/* Combined programs: returns 1 when accepted (sets the counts), 0 when rejected. */
int ref_pipeline(uint64_t n, const uint8_t *in, uint64_t *num_tokens, uint64_t *num_nodes) {
  lexeme_t *lexemes;
  uint64_t num_lexemes;
  *num_tokens = 0;
  *num_nodes = 0;
  if (!lex_string(in, n, &lexemes, &num_lexemes)) return 0;
  terminal_t *tokens = (terminal_t *)malloc((num_lexemes ? num_lexemes : 1) * sizeof(terminal_t));
  for (uint64_t i = 0; i < num_lexemes; i++) tokens[i] = lexemes[i].terminal;
  production_t *prods;
  uint64_t num_prods;
  if (!parse_test(tokens, num_lexemes, &prods, &num_prods)) {
    free(tokens);
    free(lexemes);
    return 0;
  }
  free(tokens);
  index_t *parents = (index_t *)malloc((num_prods ? num_prods : 1) * sizeof(index_t));
  compute_parents(prods, num_prods, parents);
  production_t *tree_prods = (production_t *)malloc((num_prods ? num_prods : 1) * sizeof(production_t));
  index_t *tree_parents = (index_t *)malloc((num_prods ? num_prods : 1) * sizeof(index_t));
  index_t *token_parents = (index_t *)malloc((num_lexemes ? num_lexemes : 1) * sizeof(index_t));
  int ok = compact_tree(prods, num_prods, parents, num_lexemes, tree_prods, tree_parents, token_parents);
  if (ok) {
    *num_tokens = num_lexemes;
    *num_nodes = num_prods - num_lexemes;
  }
  free(prods);
  free(parents);
  free(lexemes);
  free(tree_prods);
  free(tree_parents);
  free(token_parents);
  return ok ? 1 : 0;
}

#endif

/* Type sizes; production_t is 0 in the lexer-mode program, which has none. */
void ref_layout(uint64_t *sizes) {
  sizes[0] = sizeof(terminal_t);
#ifdef Q
  sizes[1] = sizeof(production_t);
#else
  sizes[1] = 0;
#endif
  sizes[2] = sizeof(index_t);
  sizes[3] = sizeof(length_t);
}
