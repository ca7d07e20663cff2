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
