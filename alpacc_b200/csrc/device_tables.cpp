// Host-side derivation of the device tables from alpacc's generated tables.
#include "device_tables.h"

#include <algorithm>
#include <array>
#include <cstdlib>
#include <cstring>
#include <map>
#include <unordered_map>

namespace alpacc {

namespace {

uint64_t read_uint(const void *base, uint64_t i, uint32_t width) {
  const uint8_t *p = static_cast<const uint8_t *>(base) + i * width;
  switch (width) {
    case 1: return p[0];
    case 2: { uint16_t v; std::memcpy(&v, p, 2); return v; }
    case 4: { uint32_t v; std::memcpy(&v, p, 4); return v; }
    case 8: { uint64_t v; std::memcpy(&v, p, 8); return v; }
  }
  return 0;
}

bool valid_width(uint32_t w) { return w == 1 || w == 2 || w == 4 || w == 8; }

// FNV-1a over the key, as hash_key (backends/c/parser.c:17-22).
uint64_t fnv1a(const uint64_t *key, int len) {
  uint64_t h = 14695981039346656037ULL;
  for (int i = 0; i < len; i++) h = (h ^ key[i]) * 1099511628211ULL;
  return h;
}

}  // namespace

// Minimise the Moore machine of lex_string (backends/c/lexer.c:39-97) over
// the states reachable from IDENTITY.
static int build_lexer(const alpacc_tables *t, int ignore, LexerMachine *lm, std::string *why) {
  const uint64_t N = t->num_states;
  const uint32_t sw = t->state_size;
  auto idx = [&](uint64_t s) { return (s & t->endo_mask) >> t->endo_offset; };
  auto term = [&](uint64_t s) { return (s & t->terminal_mask) >> t->terminal_offset; };
  auto prod = [&](uint64_t s) { return (s & t->produce_mask) >> t->produce_offset; };
  // byte columns: bytes with the same TO_STATE index use the same COMPOSE column
  std::vector<uint64_t> col_of_byte(256);
  std::vector<uint64_t> cols;
  std::vector<int> byte_col(256);
  for (int b = 0; b < 256; b++) {
    uint64_t c = idx(read_uint(t->to_state, b, sw));
    if (c >= N) { *why = "TO_STATE index out of range"; return ALPACC_E_INVALID; }
    auto it = std::find(cols.begin(), cols.end(), c);
    if (it == cols.end()) { byte_col[b] = (int)cols.size(); cols.push_back(c); }
    else byte_col[b] = (int)(it - cols.begin());
  }
  const int C0 = (int)cols.size();
  // reachable encoded states from IDENTITY
  std::unordered_map<uint64_t, int> id;
  std::vector<uint64_t> states;
  id[t->identity] = 0;
  states.push_back(t->identity);
  std::vector<std::vector<int>> nxt;
  for (size_t i = 0; i < states.size(); i++) {
    uint64_t e = idx(states[i]);
    if (e >= N) { *why = "state index out of range"; return ALPACC_E_INVALID; }
    std::vector<int> row(C0);
    for (int c = 0; c < C0; c++) {
      uint64_t s2 = read_uint(t->compose, e * N + cols[c], sw);
      auto it = id.find(s2);
      int j;
      if (it == id.end()) {
        j = (int)states.size();
        id[s2] = j;
        states.push_back(s2);
        if (states.size() > (1u << 22)) { *why = "lexer automaton too large"; return ALPACC_E_UNSUPPORTED; }
      } else {
        j = it->second;
      }
      row[c] = j;
    }
    nxt.push_back(std::move(row));
  }
  const int R = (int)states.size();
  lm->reachable = R;
  // Moore refinement on (terminal, produce, accept) and successor classes.
  std::vector<int> cls(R);
  {
    std::map<std::vector<uint64_t>, int> sig;
    for (int i = 0; i < R; i++) {
      uint64_t e = idx(states[i]);
      std::vector<uint64_t> k = {term(states[i]), prod(states[i]), (uint64_t)(t->accept[e] ? 1 : 0)};
      auto it = sig.find(k);
      if (it == sig.end()) it = sig.emplace(k, (int)sig.size()).first;
      cls[i] = it->second;
    }
  }
  for (;;) {
    std::map<std::vector<uint64_t>, int> sig;
    std::vector<int> ncls(R);
    for (int i = 0; i < R; i++) {
      std::vector<uint64_t> k;
      k.reserve(C0 + 1);
      k.push_back((uint64_t)cls[i]);
      for (int c = 0; c < C0; c++) k.push_back((uint64_t)cls[nxt[i][c]]);
      auto it = sig.find(k);
      if (it == sig.end()) it = sig.emplace(k, (int)sig.size()).first;
      ncls[i] = it->second;
    }
    int before = *std::max_element(cls.begin(), cls.end()) + 1;
    cls.swap(ncls);
    if ((int)sig.size() == before) break;
  }
  const int M = *std::max_element(cls.begin(), cls.end()) + 1;
  // the device keeps machine states in bytes
  if (M > kMaxMachine) { *why = "minimised lexer automaton exceeds 255 states"; return ALPACC_E_UNSUPPORTED; }
  std::vector<std::vector<int>> T(M, std::vector<int>(C0));
  std::vector<uint8_t> sterm(M), sflags(M);
  for (int i = 0; i < R; i++) {
    int m = cls[i];
    for (int c = 0; c < C0; c++) T[m][c] = cls[nxt[i][c]];
    uint64_t tm = term(states[i]);
    if (tm > 255) { *why = "terminal id exceeds 255"; return ALPACC_E_UNSUPPORTED; }
    sterm[m] = (uint8_t)tm;
    uint8_t f = 0;
    if (prod(states[i])) f |= 1;
    if (t->accept[idx(states[i])]) f |= 2;
    if (ignore < 0 || (int64_t)tm != ignore) f |= 4;
    sflags[m] = f;
  }
  // merge byte columns that act identically on the minimised machine
  std::vector<int> col_cls(C0);
  std::vector<std::vector<int>> uniq;
  for (int c = 0; c < C0; c++) {
    std::vector<int> colv(M);
    for (int m = 0; m < M; m++) colv[m] = T[m][c];
    auto it = std::find(uniq.begin(), uniq.end(), colv);
    if (it == uniq.end()) { col_cls[c] = (int)uniq.size(); uniq.push_back(colv); }
    else col_cls[c] = (int)(it - uniq.begin());
  }
  const int C = (int)uniq.size();
  if (C > 255) { *why = "too many byte classes"; return ALPACC_E_UNSUPPORTED; }
  lm->M = M;
  lm->C = C;
  lm->m0 = cls[0];
  lm->cls.resize(256);
  for (int b = 0; b < 256; b++) lm->cls[b] = (uint8_t)col_cls[byte_col[b]];
  lm->trans.assign((size_t)M * C, 0);
  for (int m = 0; m < M; m++)
    for (int c = 0; c < C; c++) lm->trans[(size_t)m * C + c] = (uint8_t)uniq[c][m];
  lm->term = sterm;
  lm->flags = sflags;
  // dead: an absorbing state that is not accepting and never produces
  lm->dead = -1;
  for (int m = 0; m < M; m++) {
    bool absorbing = true;
    for (int c = 0; c < C; c++) absorbing = absorbing && uniq[c][m] == m;
    if (absorbing && !(sflags[m] & 3)) { lm->dead = m; break; }
  }
  // distinct live targets per class and each state's slot
  lm->img.assign((size_t)C * kMaxLanes, 0xff);
  lm->img_cnt.assign(C, 0);
  lm->lane_of.assign((size_t)C * M, 0xff);
  lm->max_lanes = 0;
  for (int c = 0; c < C; c++) {
    std::vector<int> targets;
    for (int m = 0; m < M; m++) {
      if (m == lm->dead) continue;
      int tg = uniq[c][m];
      if (tg == lm->dead) continue;
      auto it = std::find(targets.begin(), targets.end(), tg);
      int slot;
      if (it == targets.end()) { slot = (int)targets.size(); targets.push_back(tg); }
      else slot = (int)(it - targets.begin());
      lm->lane_of[(size_t)c * M + m] = (uint8_t)slot;
    }
    lm->max_lanes = std::max(lm->max_lanes, (int)targets.size());
    if ((int)targets.size() > kMaxLanes) {
      *why = "a byte class reaches more than 32 live states";
      return ALPACC_E_UNSUPPORTED;
    }
    lm->img_cnt[c] = (uint8_t)targets.size();
    for (size_t i = 0; i < targets.size(); i++) lm->img[(size_t)c * kMaxLanes + i] = (uint8_t)targets[i];
  }
  if (M <= 64 && (size_t)C * C <= 65536) {
    lm->img2.assign((size_t)C * C, 0);
    for (int c0 = 0; c0 < C; c0++)
      for (int c1 = 0; c1 < C; c1++) {
        unsigned long long mask = 0;
        for (int i = 0; i < lm->img_cnt[c0]; i++) {
          const int u = uniq[c1][lm->img[(size_t)c0 * kMaxLanes + i]];
          if (u != lm->dead) mask |= 1ull << u;
        }
        lm->img2[(size_t)c0 * C + c1] = mask;
      }
  }
  return ALPACC_OK;
}

int build_lexer_table(const LexerMachine &lm, LexerTable *out, std::string *why) {
  int cp = 1, lg = 0;
  while (cp < lm.C) {
    cp <<= 1;
    lg++;
  }
  const uint32_t swz = (uint32_t)std::min(cp, 32) - 1;
  const int shift = lg + 2;
  const size_t words = (size_t)lm.M * cp;
  if (words * 4 + 512 > 160 * 1024) {
    *why = "lexer table exceeds the shared-memory budget (states x padded byte classes)";
    return ALPACC_E_UNSUPPORTED;
  }
  auto F = [&](uint32_t x) { return (x << shift) | ((x & swz) << 2); };
  out->tab.assign(words, 0);
  for (int s = 0; s < lm.M; s++)
    for (int c = 0; c < cp; c++) {
      uint32_t e = F((uint32_t)s) | (0xFFu << 24);  // columns >= C are never read
      if (c < lm.C) {
        const uint32_t nx = lm.trans[(size_t)s * lm.C + c];
        uint32_t code = 0xFF;
        if (lm.flags[nx] & 1) {
          const bool kept = (lm.flags[s] & 4) != 0;
          if (kept && lm.term[s] >= 0xFE) {
            *why = "terminal id 254 or 255 collides with the lexer's boundary codes";
            return ALPACC_E_UNSUPPORTED;
          }
          code = kept ? lm.term[s] : 0xFE;
        }
        e = F(nx) | (code << 24);
      }
      out->tab[(size_t)s * cp + ((uint32_t)c ^ ((uint32_t)s & swz))] = e;
    }
  out->cls4.resize(256);
  for (int b = 0; b < 256; b++) out->cls4[b] = (uint16_t)(lm.cls[b] * 4);
  out->shift = shift;
  out->swz = (int)swz;
  out->wide_cls = lm.C > 64 ? 1 : 0;

  // ---- the window machine: sets of live states, breadth first from the
  // set of all of them ----
  using Set = std::array<unsigned long long, 4>;
  std::map<Set, int> id;
  std::vector<Set> sets;
  Set full{};
  for (int s = 0; s < lm.M; s++)
    if (s != lm.dead) full[s >> 6] |= 1ull << (s & 63);
  id[full] = 0;
  sets.push_back(full);
  std::vector<int> next;  // [P * C]
  bool fits = true;
  for (size_t i = 0; i < sets.size() && fits; i++) {
    for (int c = 0; c < lm.C; c++) {
      Set ns{};
      for (int s = 0; s < lm.M; s++)
        if (sets[i][s >> 6] >> (s & 63) & 1) {
          const int x = lm.trans[(size_t)s * lm.C + c];
          if (x != lm.dead) ns[x >> 6] |= 1ull << (x & 63);
        }
      auto it = id.find(ns);
      int k;
      if (it != id.end()) {
        k = it->second;
      } else {
        k = (int)sets.size();
        id[ns] = k;
        sets.push_back(ns);
      }
      next.push_back(k);
    }
    if (sets.size() > (size_t)kMaxWindowSets || sets.size() * (size_t)cp * 4 > kWindowBytes) fits = false;
  }
  out->ps_tab.clear();
  out->ps_mask.clear();
  out->ps_sets = 0;
  if (fits) {
    const size_t P = sets.size();
    out->ps_sets = (int)P;
    out->ps_full = F(0);
    out->ps_tab.assign(P * cp, 0);
    out->ps_mask.assign(P * 4, 0);
    for (size_t p = 0; p < P; p++) {
      for (int w = 0; w < 4; w++) out->ps_mask[p * 4 + w] = sets[p][w];
      for (int c = 0; c < cp; c++) {
        uint32_t e = F((uint32_t)p) | (0xFFu << 24);  // columns >= C are never read
        if (c < lm.C) {
          const int k = next[p * lm.C + c];
          int members = 0, one = -1;
          for (int w = 0; w < 4; w++) {
            members += __builtin_popcountll(sets[k][w]);
            if (sets[k][w]) one = 64 * w + __builtin_ctzll(sets[k][w]);
          }
          const uint32_t info = members == 0 ? (uint32_t)lm.dead : members == 1 ? (uint32_t)one : 0xFFu;
          e = F((uint32_t)k) | (info << 24);
        }
        out->ps_tab[p * cp + ((uint32_t)c ^ ((uint32_t)p & swz))] = e;
      }
    }
  }
  return ALPACC_OK;
}

static int build_pairs_hashed(const alpacc_tables *t, PairTable *pt, std::string *why);
static int build_pair_arrays(const alpacc_tables *t, PairTable *pt, std::string *why);

static int build_pairs(const alpacc_tables *t, PairTable *pt, std::string *why) {
  const int q = (int)t->q, k = (int)t->k;
  const int L = q + k;
  const int nt = (int)t->end_terminal + 1;
  pt->nt = nt;
  pt->q = q;
  pt->k = k;
  if (L <= 0 || L > 8) { *why = "q + k must be in 1..8"; return ALPACC_E_UNSUPPORTED; }
  uint64_t dense = 1;
  bool fits = true;
  for (int i = 0; i < L && fits; i++) {
    dense *= (uint64_t)nt;
    fits = dense <= kDenseLimit;
  }
  const uint64_t H = t->hash_table_size;
  const uint32_t tw = t->terminal_size;
  // ALPACC_PAIR_LOOKUP=hashed selects the hashed form for any key space (a
  // diagnostic switch: it lets the probe replay be checked on every grammar)
  const char *force = getenv("ALPACC_PAIR_LOOKUP");
  if (!fits || (force && strcmp(force, "hashed") == 0)) return build_pairs_hashed(t, pt, why);
  pt->dense_size = dense;
  pt->dense.assign(dense, 0xffffffffu);
  // every key the table holds, looked up exactly as lookup_key does
  std::vector<uint64_t> key(L), probe_key(L);
  for (uint64_t slot = 0; slot < H; slot++) {
    if (!t->hash_table_is_valid[slot]) continue;
    bool in_range = true;
    for (int j = 0; j < L; j++) {
      key[j] = read_uint(t->hash_table_keys, slot * L + j, tw);
      if (key[j] >= (uint64_t)nt) in_range = false;
    }
    if (!in_range) continue;  // no input can form this key
    uint64_t h = fnv1a(key.data(), L) % H;
    int64_t found = -1;
    for (uint64_t it = 0; it < t->max_iters; it++) {
      bool eq = t->hash_table_is_valid[h];
      for (int j = 0; eq && j < L; j++) eq = read_uint(t->hash_table_keys, h * L + j, tw) == key[j];
      if (eq) { found = (int64_t)h; break; }
      h = (h + 1) % H;
    }
    if (found < 0) continue;
    const int64_t ss = t->hash_table_stacks_span[2 * found], se = t->hash_table_stacks_span[2 * found + 1];
    const int64_t ps = t->hash_table_productions_span[2 * found], pe = t->hash_table_productions_span[2 * found + 1];
    if (ss < 0 || se < 0 || ps < 0 || pe < 0) continue;  // lookup_key returns false
    if (se < ss || pe < ps || (uint64_t)se > t->stacks_size || (uint64_t)pe > t->productions_size) {
      *why = "hash table span out of range";
      return ALPACC_E_INVALID;
    }
    if (se - ss > 255 || pe - ps > 255) { *why = "more than 255 brackets or productions per pair"; return ALPACC_E_UNSUPPORTED; }
    if (ss >= (1 << 24) || ps >= (1 << 24)) { *why = "stack or production table too large"; return ALPACC_E_UNSUPPORTED; }
    uint64_t d = 0;
    for (int j = 0; j < L; j++) d = d * (uint64_t)nt + key[j];
    if (pt->dense[d] != 0xffffffffu) continue;
    pt->dense[d] = (uint32_t)pt->rec_ss.size();
    pt->rec_ss.push_back((uint32_t)ss);
    pt->rec_ps.push_back((uint32_t)ps);
    pt->rec_nb.push_back((uint8_t)(se - ss));
    pt->rec_np.push_back((uint8_t)(pe - ps));
    pt->max_br = std::max(pt->max_br, (int)(se - ss));
    pt->max_pr = std::max(pt->max_pr, (int)(pe - ps));
  }
  return build_pair_arrays(t, pt, why);
}

// The hashed form: every valid slot of the reference's table, with its own
// record when its spans are usable.
static int build_pairs_hashed(const alpacc_tables *t, PairTable *pt, std::string *why) {
  const int L = pt->q + pt->k;
  const uint64_t H = t->hash_table_size;
  const uint32_t tw = t->terminal_size;
  if (H == 0 || H > (1ull << 31)) { *why = "hash table size out of range"; return ALPACC_E_UNSUPPORTED; }
  pt->hashed = true;
  pt->max_iters = t->max_iters;
  pt->ht_key.assign(H, 0);
  pt->ht_rec.assign(H, kEmptySlot);
  for (uint64_t slot = 0; slot < H; slot++) {
    if (!t->hash_table_is_valid[slot]) continue;
    unsigned long long packed = 0;
    for (int j = 0; j < L; j++) {
      const uint64_t v = read_uint(t->hash_table_keys, slot * L + j, tw);
      if (v > 255) { *why = "terminal ids above 255 are not supported"; return ALPACC_E_UNSUPPORTED; }
      packed |= (unsigned long long)v << (8 * j);
    }
    pt->ht_key[slot] = packed;
    const int64_t ss = t->hash_table_stacks_span[2 * slot], se = t->hash_table_stacks_span[2 * slot + 1];
    const int64_t ps = t->hash_table_productions_span[2 * slot], pe = t->hash_table_productions_span[2 * slot + 1];
    if (ss < 0 || se < 0 || ps < 0 || pe < 0) {  // lookup_key returns false for this key
      pt->ht_rec[slot] = kMissingKey;
      continue;
    }
    if (se < ss || pe < ps || (uint64_t)se > t->stacks_size || (uint64_t)pe > t->productions_size) {
      *why = "hash table span out of range";
      return ALPACC_E_INVALID;
    }
    if (se - ss > 255 || pe - ps > 255) { *why = "more than 255 brackets or productions per pair"; return ALPACC_E_UNSUPPORTED; }
    if (ss >= (1 << 24) || ps >= (1 << 24)) { *why = "stack or production table too large"; return ALPACC_E_UNSUPPORTED; }
    pt->ht_rec[slot] = (uint32_t)pt->rec_ss.size();
    pt->rec_ss.push_back((uint32_t)ss);
    pt->rec_ps.push_back((uint32_t)ps);
    pt->rec_nb.push_back((uint8_t)(se - ss));
    pt->rec_np.push_back((uint8_t)(pe - ps));
    pt->max_br = std::max(pt->max_br, (int)(se - ss));
    pt->max_pr = std::max(pt->max_pr, (int)(pe - ps));
  }
  return build_pair_arrays(t, pt, why);
}

// Stack actions, productions and the per-production arities and flags, for
// either form of the table.
static int build_pair_arrays(const alpacc_tables *t, PairTable *pt, std::string *why) {
  const uint32_t bw = t->bracket_size;
  const uint64_t top = 1ull << (8 * bw - 1);
  pt->stacks.resize(t->stacks_size);
  for (uint64_t i = 0; i < t->stacks_size; i++) {
    uint64_t b = read_uint(t->stacks, i, bw);
    uint64_t sym = b & ~top;
    if (sym >= (1ull << 31)) { *why = "bracket symbol too large"; return ALPACC_E_UNSUPPORTED; }
    pt->stacks[i] = (uint32_t)sym | ((b & top) ? 0x80000000u : 0u);
  }
  // the parser-mode program carries no production count and no arities
  const uint64_t P = t->parts == ALPACC_PARTS_BOTH ? t->number_of_productions : 0;
  pt->prods.resize(t->productions_size);
  for (uint64_t i = 0; i < t->productions_size; i++) {
    uint64_t p = read_uint(t->productions, i, t->production_size);
    if ((t->parts == ALPACC_PARTS_BOTH && p >= P) || p >= (1ull << 31)) {
      *why = "production id out of range";
      return ALPACC_E_INVALID;
    }
    pt->prods[i] = (uint32_t)p;
  }
  pt->arity.resize(P);
  pt->is_term.resize(P);
  for (uint64_t i = 0; i < P; i++) {
    if (t->production_to_arity[i] > (1u << 20)) { *why = "arity too large"; return ALPACC_E_UNSUPPORTED; }
    pt->arity[i] = (int32_t)t->production_to_arity[i];
    pt->is_term[i] = t->production_to_terminal_is_valid[i] ? 1 : 0;
  }
  return ALPACC_OK;
}

int build_host_grammar(const alpacc_tables *t, HostGrammar *out, std::string *why) {
  if (!t || t->abi_version != ALPACC_ABI_VERSION) { *why = "abi_version mismatch"; return ALPACC_E_INVALID; }
  if (t->parts > ALPACC_PARTS_PARSER) { *why = "unknown parts value"; return ALPACC_E_INVALID; }
  const bool lexer = t->parts != ALPACC_PARTS_PARSER, parser = t->parts != ALPACC_PARTS_LEXER;
  if (!valid_width(t->terminal_size) || !(t->index_size == 4 || t->index_size == 8) ||
      (lexer && (!valid_width(t->state_size) || !valid_width(t->length_size))) ||
      (parser && (!valid_width(t->production_size) || !valid_width(t->bracket_size)))) {
    *why = "bad type width";
    return ALPACC_E_INVALID;
  }
  const bool tree = t->parts == ALPACC_PARTS_BOTH;  // arities only in the combined program
  if ((lexer && (!t->to_state || !t->compose || !t->accept || t->num_states == 0)) ||
      (parser && (!t->hash_table_is_valid || !t->hash_table_keys || !t->hash_table_stacks_span ||
                  !t->hash_table_productions_span || (t->stacks_size && !t->stacks) ||
                  (t->productions_size && !t->productions) || t->hash_table_size == 0)) ||
      (tree && (!t->production_to_arity || !t->production_to_terminal_is_valid))) {
    *why = "missing table";
    return ALPACC_E_INVALID;
  }
  if (parser && (t->end_terminal > 255 || t->start_terminal > 255 || t->empty_terminal > 255)) {
    *why = "terminal ids above 255 are not supported";
    return ALPACC_E_UNSUPPORTED;
  }
  out->t = *t;
  out->parts = (int)t->parts;
  out->ignore = lexer && t->ignore_token >= 0 ? (int)t->ignore_token : -1;
  out->len_max = !lexer || t->length_size >= 8 ? ~0ull : ((1ull << (8 * t->length_size)) - 1);
  if (lexer) {
    int rc = build_lexer(t, out->ignore, &out->lex, why);
    if (rc != ALPACC_OK) return rc;
    if (parser)
      for (uint8_t tm : out->lex.term)
        if ((uint64_t)tm > t->end_terminal) {
          *why = "a lexer terminal id is not a parser terminal";
          return ALPACC_E_INVALID;
        }
  }
  return parser ? build_pairs(t, &out->pairs, why) : ALPACC_OK;
}

}  // namespace alpacc
