/*
 * CPU restatement of alpacc's sequential C backend. TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * this library, as the checker; the product path never calls it.
 *
 * It follows the reference algorithm step by step, but takes the grammar
 * tables at run time (through the alpacc_tables struct of
 * include/alpacc_b200.h) instead of as compiled-in constants:
 *   lex_string       backends/c/lexer.c:39-97
 *   lookup_key       backends/c/parser.c:17-45   (FNV-1a + linear probing)
 *   parse_test       backends/c/parser.c:49-98
 *   compute_parents  backends/c/parser.c:103-118
 *   compact_tree     backends/c/parser.c:126-153
 *   run_case         src/Alpacc/Generator/C/Generator.hs:114-152 (record bytes)
 *                    and, by the tables' `parts`, the lexer-mode (:87-102) and
 *                    parser-mode (:65-79) run_case
 *
 * Build: gcc -O2 -std=c99 -shared -fPIC oracle.c -o _port/liboracle_port.so
 */
#define _POSIX_C_SOURCE 200809L
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../include/alpacc_b200.h"

static uint64_t rd(const void *base, uint64_t i, uint32_t w) {
  const uint8_t *p = (const uint8_t *)base + i * w;
  uint64_t v = 0;
  memcpy(&v, p, w); /* little-endian host */
  return v;
}

typedef struct {
  uint64_t terminal, start, length;
} lexeme;

/* lex_string (backends/c/lexer.c:39-97) over encoded endomorphism states. */
static int lex(const alpacc_tables *t, const uint8_t *str, uint64_t n, lexeme **out, uint64_t *num) {
  const uint32_t sw = t->state_size;
  const uint64_t N = t->num_states;
  const uint64_t len_max = t->length_size >= 8 ? ~0ull : ((1ull << (8 * t->length_size)) - 1);
#define IDX(s) (((s)&t->endo_mask) >> t->endo_offset)
#define COMPOSE(a, b) rd(t->compose, IDX(a) * N + IDX(b), sw)
  if (n == 0) {
    *out = NULL;
    *num = 0;
    return 1;
  }
  uint64_t cap = 16, count = 0;
  lexeme *res = (lexeme *)malloc(cap * sizeof(lexeme));
  uint64_t cur = rd(t->to_state, str[0], sw);
  cur = COMPOSE(t->identity, cur); /* lexer.c:52-54 */
  uint64_t tok_start = 0;
  for (uint64_t i = 1; i <= n; i++) {
    uint64_t next = i < n ? rd(t->to_state, str[i], sw) : t->identity;
    int boundary = (i == n) || (((COMPOSE(cur, next) & t->produce_mask) >> t->produce_offset) != 0);
    if (boundary) {
      uint64_t term = (cur & t->terminal_mask) >> t->terminal_offset;
      if (t->ignore_token < 0 || term != (uint64_t)t->ignore_token) {
        uint64_t len = i - tok_start;
        if (len > len_max) { /* lexer.c:68-72 */
          free(res);
          return 0;
        }
        if (count == cap) {
          cap *= 2;
          res = (lexeme *)realloc(res, cap * sizeof(lexeme));
        }
        res[count].terminal = term;
        res[count].start = tok_start;
        res[count].length = len;
        count++;
      }
      tok_start = i;
    }
    if (i < n) cur = COMPOSE(cur, next);
  }
  if (!t->accept[IDX(cur)]) { /* lexer.c:89-92 */
    free(res);
    return 0;
  }
  *out = res;
  *num = count;
  return 1;
#undef COMPOSE
#undef IDX
}

/* lookup_key (backends/c/parser.c:17-45). */
static int lookup(const alpacc_tables *t, const uint64_t *key, int64_t sp[4]) {
  const uint64_t L = t->q + t->k, H = t->hash_table_size;
  uint64_t h = 14695981039346656037ULL;
  for (uint64_t i = 0; i < L; i++) h = (h ^ key[i]) * 1099511628211ULL;
  h %= H;
  for (uint64_t it = 0; it < t->max_iters; it++) {
    int eq = t->hash_table_is_valid[h] != 0;
    for (uint64_t j = 0; eq && j < L; j++) eq = rd(t->hash_table_keys, h * L + j, t->terminal_size) == key[j];
    if (eq) {
      sp[0] = t->hash_table_stacks_span[2 * h];
      sp[1] = t->hash_table_stacks_span[2 * h + 1];
      sp[2] = t->hash_table_productions_span[2 * h];
      sp[3] = t->hash_table_productions_span[2 * h + 1];
      return sp[0] >= 0 && sp[1] >= 0 && sp[2] >= 0 && sp[3] >= 0;
    }
    h = (h + 1) % H;
  }
  return 0;
}

/* parse_test (backends/c/parser.c:49-98): productions of the leftmost
   derivation, checking every stack action against a bracket stack. */
static int parse(const alpacc_tables *t, const uint64_t *tokens, uint64_t n, uint64_t **prods_out, uint64_t *np_out) {
  const uint64_t m = n + 2, Q = t->q, K = t->k;
  const uint32_t bw = t->bracket_size;
  const uint64_t top_bit = 1ull << (8 * bw - 1);
  uint64_t *arr = (uint64_t *)malloc(m * sizeof(uint64_t));
  uint64_t *stack = (uint64_t *)malloc((m * (t->max_brackets_per_position + 1) + 1) * sizeof(uint64_t));
  uint64_t *prods = (uint64_t *)malloc((m * (t->max_prods_per_position + 1) + 1) * sizeof(uint64_t));
  uint64_t key[16];
  uint64_t np = 0;
  if (Q + K > 16) {
    free(arr);
    free(stack);
    free(prods);
    return 0;
  }
  int64_t top = -1;
  int ok = 0;
  arr[0] = t->start_terminal;
  for (uint64_t i = 0; i < n; i++) arr[i + 1] = tokens[i];
  arr[m - 1] = t->end_terminal;
  for (uint64_t i = 0; i < m; i++) {
    for (uint64_t j = 0; j < Q + K; j++) {
      uint64_t idx = i + j;
      key[j] = (idx < Q || idx >= m + Q) ? t->empty_terminal : arr[idx - Q];
    }
    int64_t sp[4];
    if (!lookup(t, key, sp)) goto done;
    for (int64_t j = sp[0]; j < sp[1]; j++) {
      uint64_t b = rd(t->stacks, (uint64_t)j, bw);
      if (b & top_bit) {
        stack[++top] = b;
      } else {
        if (top < 0 || (stack[top] & ~top_bit) != (b & ~top_bit)) goto done;
        top--;
      }
    }
    for (int64_t j = sp[2]; j < sp[3]; j++) prods[np++] = rd(t->productions, (uint64_t)j, t->production_size);
  }
  if (top != -1) goto done;
  *prods_out = prods;
  *np_out = np;
  prods = NULL;
  ok = 1;
done:
  free(arr);
  free(stack);
  free(prods);
  return ok;
}

/* compute_parents (backends/c/parser.c:103-118). */
static void parents_of(const alpacc_tables *t, const uint64_t *prods, uint64_t np, int64_t *parents) {
  uint64_t *remaining = (uint64_t *)malloc((np + 1) * sizeof(uint64_t));
  uint64_t *stk = (uint64_t *)malloc((np + 1) * sizeof(uint64_t));
  int64_t top = -1;
  for (uint64_t i = 0; i < np; i++) {
    uint64_t arity = t->production_to_arity[prods[i]];
    remaining[i] = arity;
    parents[i] = top >= 0 ? (int64_t)stk[top] : 0;
    if (arity > 0) stk[++top] = i;
    while (top >= 0 && remaining[stk[top]] == 0) top--;
    if (top >= 0 && i > 0) remaining[stk[top]]--;
  }
  free(remaining);
  free(stk);
}

static void put(uint8_t **buf, size_t *len, size_t *cap, const void *src, size_t n) {
  if (*len + n > *cap) {
    while (*len + n > *cap) *cap = *cap ? *cap * 2 : 1024;
    *buf = (uint8_t *)realloc(*buf, *cap);
  }
  memcpy(*buf + *len, src, n);
  *len += n;
}

static void put_uint(uint8_t **buf, size_t *len, size_t *cap, uint64_t v, uint32_t w) { put(buf, len, cap, &v, w); }

/* The lexer-mode run_case (src/Alpacc/Generator/C/Generator.hs:87-102):
   u8 valid, u64 count, per lexeme terminal_t, index_t start, length_t length. */
static int lexer_run_case(const alpacc_tables *t, uint64_t n, const uint8_t *in, uint8_t **out, size_t *out_len) {
  uint8_t *buf = NULL;
  size_t len = 0, cap = 0;
  const uint8_t zero = 0, one = 1;
  lexeme *lx = NULL;
  uint64_t nl = 0;
  if (!lex(t, in, n, &lx, &nl)) {
    put(&buf, &len, &cap, &zero, 1);
  } else {
    put(&buf, &len, &cap, &one, 1);
    put_uint(&buf, &len, &cap, nl, 8);
    for (uint64_t i = 0; i < nl; i++) {
      put_uint(&buf, &len, &cap, lx[i].terminal, t->terminal_size);
      put_uint(&buf, &len, &cap, lx[i].start, t->index_size);
      put_uint(&buf, &len, &cap, lx[i].length, t->length_size);
    }
    free(lx);
  }
  *out = buf;
  *out_len = len;
  return 1;
}

/* The parser-mode run_case (src/Alpacc/Generator/C/Generator.hs:65-79): the
   input is n terminal_t ids; u8 valid, u64 count, production_t[count]. */
static int parser_run_case(const alpacc_tables *t, uint64_t n, const uint8_t *in, uint8_t **out, size_t *out_len) {
  uint8_t *buf = NULL;
  size_t len = 0, cap = 0;
  const uint8_t zero = 0, one = 1;
  uint64_t *tokens = (uint64_t *)malloc((n + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < n; i++) tokens[i] = rd(in, i, t->terminal_size);
  uint64_t *prods = NULL, np = 0;
  if (!parse(t, tokens, n, &prods, &np)) {
    put(&buf, &len, &cap, &zero, 1);
  } else {
    put(&buf, &len, &cap, &one, 1);
    put_uint(&buf, &len, &cap, np, 8);
    for (uint64_t i = 0; i < np; i++) put_uint(&buf, &len, &cap, prods[i], t->production_size);
    free(prods);
  }
  free(tokens);
  *out = buf;
  *out_len = len;
  return 1;
}

/* run_case (src/Alpacc/Generator/C/Generator.hs:114-152) into a malloc'd
   buffer; lexer-only and parser-only tables give their mode's record. */
int oracle_run_case(const alpacc_tables *t, uint64_t n, const uint8_t *in, uint8_t **out, size_t *out_len) {
  if (t->parts == ALPACC_PARTS_LEXER) return lexer_run_case(t, n, in, out, out_len);
  if (t->parts == ALPACC_PARTS_PARSER) return parser_run_case(t, n, in, out, out_len);
  uint8_t *buf = NULL;
  size_t len = 0, cap = 0;
  const uint8_t zero = 0, one = 1;
  lexeme *lx = NULL;
  uint64_t nl = 0;
  if (!lex(t, in, n, &lx, &nl)) {
    put(&buf, &len, &cap, &zero, 1);
    *out = buf;
    *out_len = len;
    return 1;
  }
  uint64_t *tokens = (uint64_t *)malloc((nl + 1) * sizeof(uint64_t));
  for (uint64_t i = 0; i < nl; i++) tokens[i] = lx[i].terminal;
  uint64_t *prods = NULL, np = 0;
  if (!parse(t, tokens, nl, &prods, &np)) {
    free(tokens);
    free(lx);
    put(&buf, &len, &cap, &zero, 1);
    *out = buf;
    *out_len = len;
    return 1;
  }
  free(tokens);
  int64_t *parents = (int64_t *)malloc((np + 1) * sizeof(int64_t));
  parents_of(t, prods, np, parents);
  /* compact_tree (backends/c/parser.c:126-153) */
  uint64_t *t_incl = (uint64_t *)malloc((np + 1) * sizeof(uint64_t));
  uint64_t count = 0;
  for (uint64_t i = 0; i < np; i++) {
    if (t->production_to_terminal_is_valid[prods[i]]) count++;
    t_incl[i] = count;
  }
  if (count != nl) {
    put(&buf, &len, &cap, &zero, 1);
  } else {
    uint64_t nn = np - nl;
    uint64_t *tree_prods = (uint64_t *)malloc((np + 1) * sizeof(uint64_t));
    int64_t *tree_parents = (int64_t *)malloc((np + 1) * sizeof(int64_t));
    int64_t *token_parents = (int64_t *)malloc((nl + 1) * sizeof(int64_t));
    for (uint64_t i = 0; i < np; i++) {
      int64_t p_old = parents[i];
      int64_t p_new = p_old - (int64_t)t_incl[p_old];
      if (t->production_to_terminal_is_valid[prods[i]]) {
        token_parents[t_incl[i] - 1] = p_new;
      } else {
        uint64_t j = i - t_incl[i];
        tree_prods[j] = prods[i];
        tree_parents[j] = p_new;
      }
    }
    put(&buf, &len, &cap, &one, 1);
    put_uint(&buf, &len, &cap, nl, 8);
    for (uint64_t i = 0; i < nl; i++) put_uint(&buf, &len, &cap, lx[i].terminal, t->terminal_size);
    for (uint64_t i = 0; i < nl; i++) put_uint(&buf, &len, &cap, lx[i].start, t->index_size);
    for (uint64_t i = 0; i < nl; i++) put_uint(&buf, &len, &cap, lx[i].length, t->length_size);
    put_uint(&buf, &len, &cap, nn, 8);
    for (uint64_t i = 0; i < nn; i++) put_uint(&buf, &len, &cap, tree_prods[i], t->production_size);
    for (uint64_t i = 0; i < nn; i++) put_uint(&buf, &len, &cap, (uint64_t)tree_parents[i], t->index_size);
    for (uint64_t i = 0; i < nl; i++) put_uint(&buf, &len, &cap, (uint64_t)token_parents[i], t->index_size);
    free(tree_prods);
    free(tree_parents);
    free(token_parents);
  }
  free(t_incl);
  free(parents);
  free(prods);
  free(lx);
  *out = buf;
  *out_len = len;
  return 1;
}

void oracle_free(void *p) { free(p); }
