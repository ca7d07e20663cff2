/*
 * Endomorphism composition closure of a lexer DFA, in C for speed.
 *
 * Restates ``parallelLexer`` / ``endoCompositionsTable`` of the reference
 * generator (src/Alpacc/Lexer/ParallelLexing.hs:265-429, 530-555) with the
 * same discovery order, so the endomorphism ids it assigns are the ones the
 * reference assigns:
 *   - E0 = identity, E1 = dead, E2.. = the distinct byte endomorphisms in byte
 *     order (``enumerate initE . nub``);
 *   - the work set of "connected" pairs (e, e') is drained smallest pair first
 *     (``popElement``); a new composition gets id max+1 (``endoNext``);
 *   - the connected / inverse-connected maps are extended by ``preSets`` and
 *     ``postSets`` and the new pairs join the work set.
 * Sets are bitsets; the work set is a binary heap with a pending bitset.
 *
 * Build: gcc -O2 -shared -fPIC closure.c -o _closure.so
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int S1;             /* states incl. dead state 0 */
  int n, cap;         /* endomorphisms, capacity */
  uint16_t *ss;       /* [cap][S1] images */
  uint8_t *bs;        /* [cap][S1] producing flags */
  int words;          /* 64-bit words per bitset row (cap/64) */
  uint64_t *conn;     /* [cap][words] */
  uint64_t *inv;      /* [cap][words] */
  int32_t *comp;      /* [cap][cap], -1 = not computed */
  /* hash of endomorphisms -> id */
  int hcap;
  int32_t *hslot;
} ctx_t;

typedef struct { uint32_t e, f; } pair_t;

typedef struct {
  pair_t *a;
  size_t n, cap;
} heap_t;

static int pair_lt(pair_t x, pair_t y) { return x.e < y.e || (x.e == y.e && x.f < y.f); }

static int heap_push(heap_t *h, pair_t p) {
  if (h->n == h->cap) {
    size_t nc = h->cap ? h->cap * 2 : 1024;
    pair_t *na = (pair_t *)realloc(h->a, nc * sizeof(pair_t));
    if (!na) return -1;
    h->a = na;
    h->cap = nc;
  }
  size_t i = h->n++;
  h->a[i] = p;
  while (i > 0) {
    size_t par = (i - 1) / 2;
    if (!pair_lt(h->a[i], h->a[par])) break;
    pair_t t = h->a[i]; h->a[i] = h->a[par]; h->a[par] = t;
    i = par;
  }
  return 0;
}

static pair_t heap_pop(heap_t *h) {
  pair_t top = h->a[0];
  h->a[0] = h->a[--h->n];
  size_t i = 0;
  for (;;) {
    size_t l = 2 * i + 1, r = l + 1, m = i;
    if (l < h->n && pair_lt(h->a[l], h->a[m])) m = l;
    if (r < h->n && pair_lt(h->a[r], h->a[m])) m = r;
    if (m == i) break;
    pair_t t = h->a[i]; h->a[i] = h->a[m]; h->a[m] = t;
    i = m;
  }
  return top;
}

static uint64_t endo_hash(const ctx_t *c, const uint16_t *ss, const uint8_t *bs) {
  uint64_t h = 1469598103934665603ULL;
  for (int i = 0; i < c->S1; i++) {
    h = (h ^ ss[i]) * 1099511628211ULL;
    h = (h ^ bs[i]) * 1099511628211ULL;
  }
  return h;
}

static int endo_find(const ctx_t *c, const uint16_t *ss, const uint8_t *bs, uint64_t h) {
  uint64_t m = (uint64_t)c->hcap - 1;
  for (uint64_t i = h & m;; i = (i + 1) & m) {
    int32_t id = c->hslot[i];
    if (id < 0) return -1;
    if (!memcmp(c->ss + (size_t)id * c->S1, ss, c->S1 * sizeof(uint16_t)) &&
        !memcmp(c->bs + (size_t)id * c->S1, bs, c->S1))
      return id;
  }
}

static void hash_insert(ctx_t *c, int id) {
  uint64_t h = endo_hash(c, c->ss + (size_t)id * c->S1, c->bs + (size_t)id * c->S1);
  uint64_t m = (uint64_t)c->hcap - 1;
  uint64_t i = h & m;
  while (c->hslot[i] >= 0) i = (i + 1) & m;
  c->hslot[i] = id;
}

static int grow(ctx_t *c, int need) {
  if (need <= c->cap) return 0;
  int ncap = c->cap ? c->cap : 256;
  while (ncap < need) ncap *= 2;
  int nwords = (ncap + 63) / 64;
  uint16_t *nss = (uint16_t *)realloc(c->ss, (size_t)ncap * c->S1 * sizeof(uint16_t));
  uint8_t *nbs = (uint8_t *)realloc(c->bs, (size_t)ncap * c->S1);
  uint64_t *nconn = (uint64_t *)calloc((size_t)ncap * nwords, sizeof(uint64_t));
  uint64_t *ninv = (uint64_t *)calloc((size_t)ncap * nwords, sizeof(uint64_t));
  int32_t *ncomp = (int32_t *)malloc((size_t)ncap * ncap * sizeof(int32_t));
  if (!nss || !nbs || !nconn || !ninv || !ncomp) return -1;
  memset(ncomp, 0xff, (size_t)ncap * ncap * sizeof(int32_t));
  for (int i = 0; i < c->n; i++) {
    if (c->conn) memcpy(nconn + (size_t)i * nwords, c->conn + (size_t)i * c->words, c->words * sizeof(uint64_t));
    if (c->inv) memcpy(ninv + (size_t)i * nwords, c->inv + (size_t)i * c->words, c->words * sizeof(uint64_t));
    if (c->comp) memcpy(ncomp + (size_t)i * ncap, c->comp + (size_t)i * c->cap, c->n * sizeof(int32_t));
  }
  free(c->conn); free(c->inv); free(c->comp);
  c->ss = nss; c->bs = nbs; c->conn = nconn; c->inv = ninv; c->comp = ncomp;
  c->cap = ncap; c->words = nwords;
  /* rehash with a table of at least 4x capacity */
  int hcap = 1;
  while (hcap < 4 * ncap) hcap *= 2;
  free(c->hslot);
  c->hslot = (int32_t *)malloc((size_t)hcap * sizeof(int32_t));
  if (!c->hslot) return -1;
  memset(c->hslot, 0xff, (size_t)hcap * sizeof(int32_t));
  c->hcap = hcap;
  for (int i = 0; i < c->n; i++) hash_insert(c, i);
  return 0;
}

#define BIT_GET(row, x) (((row)[(x) >> 6] >> ((x) & 63)) & 1ULL)
#define BIT_SET(row, x) ((row)[(x) >> 6] |= 1ULL << ((x) & 63))

/*
 * Inputs: S1 = number of DFA states including the dead state 0; nb = number of
 * distinct byte endomorphisms (they become E2..E(nb+1)), given as images
 * ss[nb][S1] and producing flags bs[nb][S1]; conn0[nb][nb] = 1 when byte
 * endomorphism j can follow byte endomorphism i.
 * Outputs (malloc'd, caller frees with alpacc_closure_free): the number of
 * endomorphisms, their images/flags, and the composition table comp[n][n]
 * (-1 where the pair was never composed).
 */
int alpacc_endo_closure(int S1, int nb, const uint16_t *ss, const uint8_t *bs, const uint8_t *conn0,
                        int *out_n, uint16_t **out_ss, uint8_t **out_bs, int32_t **out_comp) {
  ctx_t c;
  memset(&c, 0, sizeof c);
  c.S1 = S1;
  if (grow(&c, nb + 2 + 16) != 0) return -1;
  /* E0 identity, E1 dead */
  for (int s = 0; s < S1; s++) { c.ss[s] = (uint16_t)s; c.bs[s] = 0; }
  for (int s = 0; s < S1; s++) { c.ss[S1 + s] = 0; c.bs[S1 + s] = 0; }
  memcpy(c.ss + 2 * (size_t)S1, ss, (size_t)nb * S1 * sizeof(uint16_t));
  memcpy(c.bs + 2 * (size_t)S1, bs, (size_t)nb * S1);
  c.n = nb + 2;
  /* E0/E1 are never looked up by value (the reference keys its endo map only
     on the byte endomorphisms and their compositions), so only insert E2.. */
  for (int i = 2; i < c.n; i++) hash_insert(&c, i);
  c.comp[0 * c.cap + 0] = 0;
  for (int e = 0; e < c.n; e++) { c.comp[0 * (size_t)c.cap + e] = e; c.comp[(size_t)e * c.cap + 0] = e; }
  heap_t h = {0};
  size_t inv_key_cap = (size_t)c.cap;
  uint8_t *inv_key = (uint8_t *)calloc(inv_key_cap, 1);
  if (!inv_key) return -1;
  uint64_t *pending = NULL;
  size_t pend_cap = 0; /* pending bitset dimension */
  /* pending as a hash-free bitset over cap x cap, resized with cap */
  pend_cap = c.cap;
  pending = (uint64_t *)calloc(((size_t)pend_cap * pend_cap + 63) / 64, sizeof(uint64_t));
  if (!pending) return -1;
#define PEND_IDX(e, f) ((size_t)(e) * pend_cap + (f))
  for (int i = 0; i < nb; i++)
    for (int j = 0; j < nb; j++)
      if (conn0[(size_t)i * nb + j]) {
        int e = i + 2, f = j + 2;
        BIT_SET(c.conn + (size_t)e * c.words, f);
        BIT_SET(c.inv + (size_t)f * c.words, e);
        inv_key[f] = 1;
        size_t pi = PEND_IDX(e, f);
        if (!((pending[pi >> 6] >> (pi & 63)) & 1)) {
          pending[pi >> 6] |= 1ULL << (pi & 63);
          heap_push(&h, (pair_t){(uint32_t)e, (uint32_t)f});
        }
      }
  uint16_t *tmp_ss = (uint16_t *)malloc(S1 * sizeof(uint16_t));
  uint8_t *tmp_bs = (uint8_t *)malloc(S1);
  uint64_t *pre = NULL, *post = NULL;
  int pre_words = 0;
  int rc = 0;
  while (h.n > 0) {
    pair_t p = heap_pop(&h);
    int e = (int)p.e, f = (int)p.f;
    {
      size_t pi = PEND_IDX(e, f);
      pending[pi >> 6] &= ~(1ULL << (pi & 63));
    }
    if (c.comp[(size_t)e * c.cap + f] >= 0) continue;
    const uint16_t *ass = c.ss + (size_t)e * S1;
    const uint16_t *bss = c.ss + (size_t)f * S1;
    const uint8_t *bbs = c.bs + (size_t)f * S1;
    for (int s = 0; s < S1; s++) { tmp_ss[s] = bss[ass[s]]; tmp_bs[s] = bbs[ass[s]]; }
    uint64_t hh = endo_hash(&c, tmp_ss, tmp_bs);
    int g = endo_find(&c, tmp_ss, tmp_bs, hh);
    if (g < 0) {
      if (c.n + 1 > c.cap) {
        int oldcap = c.cap;
        if (grow(&c, c.n + 1) != 0) { rc = -1; break; }
        /* re-layout pending bitset for the new capacity */
        uint64_t *np = (uint64_t *)calloc(((size_t)c.cap * c.cap + 63) / 64, sizeof(uint64_t));
        if (!np) { rc = -1; break; }
        for (int a = 0; a < oldcap; a++)
          for (int b = 0; b < oldcap; b++) {
            size_t oi = (size_t)a * pend_cap + b;
            if ((pending[oi >> 6] >> (oi & 63)) & 1) {
              size_t ni = (size_t)a * c.cap + b;
              np[ni >> 6] |= 1ULL << (ni & 63);
            }
          }
        free(pending);
        pending = np;
        pend_cap = c.cap;
        uint8_t *nk = (uint8_t *)calloc((size_t)c.cap, 1);
        if (!nk) { rc = -1; break; }
        memcpy(nk, inv_key, inv_key_cap);
        free(inv_key);
        inv_key = nk;
        inv_key_cap = (size_t)c.cap;
      }
      g = c.n++;
      memcpy(c.ss + (size_t)g * S1, tmp_ss, S1 * sizeof(uint16_t));
      memcpy(c.bs + (size_t)g * S1, tmp_bs, S1);
      hash_insert(&c, g);
      c.comp[0 * (size_t)c.cap + g] = g;
      c.comp[(size_t)g * c.cap + 0] = g;
    }
    c.comp[(size_t)e * c.cap + f] = g;
    if (pre_words != c.words) {
      free(pre); free(post);
      pre = (uint64_t *)malloc(c.words * sizeof(uint64_t));
      post = (uint64_t *)malloc(c.words * sizeof(uint64_t));
      if (!pre || !post) { rc = -1; break; }
      pre_words = c.words;
    }
    if (!inv_key[e]) { rc = -2; break; } /* IntMap.! on a missing key in preSets */
    inv_key[g] = 1;
    const uint64_t *inv_e = c.inv + (size_t)e * c.words, *inv_g = c.inv + (size_t)g * c.words;
    const uint64_t *conn_f = c.conn + (size_t)f * c.words, *conn_g = c.conn + (size_t)g * c.words;
    for (int w = 0; w < c.words; w++) { pre[w] = inv_e[w] & ~inv_g[w]; post[w] = conn_f[w] & ~conn_g[w]; }
    for (int w = 0; w < c.words; w++) {
      uint64_t m = pre[w];
      while (m) {
        int x = w * 64 + __builtin_ctzll(m);
        m &= m - 1;
        BIT_SET(c.conn + (size_t)x * c.words, g);
        BIT_SET(c.inv + (size_t)g * c.words, x);
        size_t pi = PEND_IDX(x, g);
        if (!((pending[pi >> 6] >> (pi & 63)) & 1)) {
          pending[pi >> 6] |= 1ULL << (pi & 63);
          if (heap_push(&h, (pair_t){(uint32_t)x, (uint32_t)g})) { rc = -1; goto done; }
        }
      }
      m = post[w];
      while (m) {
        int y = w * 64 + __builtin_ctzll(m);
        m &= m - 1;
        BIT_SET(c.conn + (size_t)g * c.words, y);
        BIT_SET(c.inv + (size_t)y * c.words, g);
        inv_key[y] = 1;
        size_t pi = PEND_IDX(g, y);
        if (!((pending[pi >> 6] >> (pi & 63)) & 1)) {
          pending[pi >> 6] |= 1ULL << (pi & 63);
          if (heap_push(&h, (pair_t){(uint32_t)g, (uint32_t)y})) { rc = -1; goto done; }
        }
      }
    }
  }
done:
  free(pre); free(post); free(tmp_ss); free(tmp_bs); free(pending); free(h.a); free(inv_key);
  free(c.conn); free(c.inv); free(c.hslot);
  if (rc != 0) { free(c.ss); free(c.bs); free(c.comp); return rc; }
  /* compact comp to n x n */
  int n = c.n;
  int32_t *comp = (int32_t *)malloc((size_t)n * n * sizeof(int32_t));
  if (!comp) return -1;
  for (int i = 0; i < n; i++) memcpy(comp + (size_t)i * n, c.comp + (size_t)i * c.cap, n * sizeof(int32_t));
  free(c.comp);
  *out_n = n;
  *out_ss = c.ss;
  *out_bs = c.bs;
  *out_comp = comp;
  return 0;
}

void alpacc_closure_free(void *p) { free(p); }
