// Test harness (tests only): runs the minimised lexer machine that
// device_tables.cpp derives for the GPU sequentially on the CPU, with the
// boundary rule of the lexer kernels: a boundary before byte j (j >= 1) when
// the state entered at j produces; the token ending there has the terminal
// and kept flag of the state before it; a dead state rejects; at the end the
// state must accept and the last token is emitted. Comparing its lexemes
// with lex_string's (the oracle) checks the host-side derivation - state
// enumeration, Moore minimisation, byte classes - without a GPU.
#include <cstdint>
#include <string>

#include "device_tables.h"

extern "C" int machine_lex(const alpacc_tables *t, const uint8_t *in, uint64_t n, uint64_t *out, uint64_t cap,
                           uint64_t *count, int *machine_states) {
  alpacc::HostGrammar hg;
  std::string why;
  const int rc = alpacc::build_host_grammar(t, &hg, &why);
  if (rc != ALPACC_OK) return rc;
  const alpacc::LexerMachine &lm = hg.lex;
  *machine_states = lm.M;
  *count = 0;
  if (n == 0) return ALPACC_OK;
  int x = lm.m0;
  uint64_t start = 0, k = 0;
  for (uint64_t j = 0; j < n; j++) {
    const int nx = lm.trans[(size_t)x * lm.C + lm.cls[in[j]]];
    if (j >= 1 && (lm.flags[nx] & 1)) {
      if (lm.flags[x] & 4) {
        if (j - start > hg.len_max) return ALPACC_REJECT;
        if (k < cap) {
          out[3 * k] = lm.term[x];
          out[3 * k + 1] = start;
          out[3 * k + 2] = j - start;
        }
        k++;
      }
      start = j;
    }
    x = nx;
    if (x == lm.dead) return ALPACC_REJECT;
  }
  if (!(lm.flags[x] & 2)) return ALPACC_REJECT;
  if (lm.flags[x] & 4) {
    if (n - start > hg.len_max) return ALPACC_REJECT;
    if (k < cap) {
      out[3 * k] = lm.term[x];
      out[3 * k + 1] = start;
      out[3 * k + 2] = n - start;
    }
    k++;
  }
  *count = k;
  return ALPACC_OK;
}

// The pair record the dense table of device_tables.cpp gives for each of
// `count` keys (q + k terminal ids each): found flag and the stack and
// production spans, as the pair kernel reads them.
extern "C" int pair_lookup(const alpacc_tables *t, const uint64_t *keys, uint64_t count, int64_t *out) {
  alpacc::HostGrammar hg;
  std::string why;
  const int rc = alpacc::build_host_grammar(t, &hg, &why);
  if (rc != ALPACC_OK) return rc;
  const alpacc::PairTable &pt = hg.pairs;
  const int L = pt.q + pt.k;
  for (uint64_t i = 0; i < count; i++) {
    uint64_t d = 0;
    bool bad = false;
    for (int j = 0; j < L; j++) {
      const uint64_t v = keys[i * L + j];
      if (v >= (uint64_t)pt.nt) bad = true;
      d = d * (uint64_t)pt.nt + (bad ? 0 : v);
    }
    uint32_t r = 0xffffffffu;
    if (!pt.hashed) {
      r = bad ? 0xffffffffu : pt.dense[d];
    } else if (!bad) {  // the device's probe of the hashed form
      uint64_t h = 14695981039346656037ull;
      unsigned long long packed = 0;
      for (int j = 0; j < L; j++) {
        h = (h ^ keys[i * L + j]) * 1099511628211ull;
        packed |= (unsigned long long)keys[i * L + j] << (8 * j);
      }
      const uint64_t H = pt.ht_key.size();
      h %= H;
      for (uint64_t it = 0; it < pt.max_iters; it++) {
        const uint32_t rr = pt.ht_rec[h];
        if (rr != alpacc::kEmptySlot && pt.ht_key[h] == packed) {
          r = rr == alpacc::kMissingKey ? 0xffffffffu : rr;
          break;
        }
        h = h + 1 == H ? 0 : h + 1;
      }
    }
    int64_t *o = out + 5 * i;
    if (r == 0xffffffffu) {
      o[0] = 0;
      continue;
    }
    o[0] = 1;
    o[1] = pt.rec_ss[r];
    o[2] = (int64_t)pt.rec_ss[r] + pt.rec_nb[r];
    o[3] = pt.rec_ps[r];
    o[4] = (int64_t)pt.rec_ps[r] + pt.rec_np[r];
  }
  return ALPACC_OK;
}

// The window machine of build_lexer_table, checked against the subset
// construction it encodes: info = {sets, entries naming one state, entries
// naming two or more, entries whose info byte disagrees with the member
// masks}; returns 0, or 1 when no window machine was built.
extern "C" int window_info(const alpacc_tables *t, int64_t *info) {
  alpacc::HostGrammar hg;
  std::string why;
  if (alpacc::build_host_grammar(t, &hg, &why) != ALPACC_OK) return -1;
  const alpacc::LexerMachine &lm = hg.lex;
  alpacc::LexerTable lt;
  if (alpacc::build_lexer_table(lm, &lt, &why) != ALPACC_OK) return -1;
  for (int i = 0; i < 4; i++) info[i] = 0;
  if (lt.ps_tab.empty()) return 1;
  const int P = lt.ps_sets, cp = 1 << (lt.shift - 2);
  info[0] = P;
  for (int p = 0; p < P; p++)
    for (int c = 0; c < lm.C; c++) {
      const uint32_t e = lt.ps_tab[(size_t)p * cp + ((uint32_t)c ^ ((uint32_t)p & (uint32_t)lt.swz))];
      const int k = (int)((e & 0xFFFFFFu) >> lt.shift);
      // the next set from the members of p
      unsigned long long want[4] = {0, 0, 0, 0};
      for (int s = 0; s < lm.M; s++)
        if (lt.ps_mask[(size_t)p * 4 + (s >> 6)] >> (s & 63) & 1) {
          const int x = lm.trans[(size_t)s * lm.C + c];
          if (x != lm.dead) want[x >> 6] |= 1ull << (x & 63);
        }
      int members = 0, one = -1;
      bool same = true;
      for (int w = 0; w < 4; w++) {
        same = same && want[w] == lt.ps_mask[(size_t)k * 4 + w];
        members += __builtin_popcountll(want[w]);
        if (want[w]) one = 64 * w + __builtin_ctzll(want[w]);
      }
      const uint32_t expect = members == 0 ? (uint32_t)lm.dead : members == 1 ? (uint32_t)one : 0xFFu;
      if (!same || (e >> 24) != (expect & 0xFF)) info[3]++;
      if (members == 1) info[1]++;
      if (members > 1) info[2]++;
    }
  return 0;
}
