// Test harness (tests only): a sequential CPU emulation of the tile algorithm
// of alpacc_b200/csrc/lexer.cu - the same shared-memory tables
// (build_lexer_table: the machine and its window machine), tile and chunk
// geometry, the window walk over the 16 to 32 bytes before each chunk (64 for
// a tile's first chunk whose shorter window leaves candidates; in the
// window machine, or as an explicit state set from the first window byte's
// image), the single walk of each chunk whose window left one candidate
// ("known"), per-candidate end states and codes of the other ("open")
// chunks, resolution from the nearest known chunk or the previous tile's
// published outgoing state / transition vector, the boundary and kept masks
// computed with the kernel's byte tricks, the (count, last boundary) carry and
// the token emission with the length check. Its lexemes are compared with
// machine_lex's (the machine walked byte by byte, itself compared with the
// oracle), so the algorithm's logic is checked without a GPU; the parallel
// mechanics (barriers, look-back waits) are not.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "device_tables.h"

namespace {

constexpr int kThreads = 256, kWords = 15, kChunk = 60, kWin = 64;  // kWin: bytes loaded before a tile
constexpr int kData = kThreads * kChunk, kLoad = kWin + kData;
enum { kEmpty = 0, kKnown = 1, kOpen = 2, kOpenTail = 3 };

struct Emu {
  const alpacc::LexerMachine &lm;
  const alpacc::LexerTable &lt;
  uint32_t row_of(uint32_t x) const { return (x << lt.shift) | ((x & (uint32_t)lt.swz) << 2); }
  int state_of(uint32_t f) const { return (int)((f & 0xFFFFFFu) >> lt.shift); }
  uint32_t step(uint32_t f, uint32_t c4) const { return lt.tab[((f & 0xFFFFFFu) ^ c4) >> 2]; }
  uint32_t wstep(uint32_t f, uint32_t c4) const { return lt.ps_tab[((f & 0xFFFFFFu) ^ c4) >> 2]; }
  uint32_t c4(uint8_t b) const { return lt.cls4[b]; }
};

uint32_t nonzero_bytes(uint32_t w) { return (((w & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | w) & 0x80808080u; }
uint32_t movemask4(uint32_t x) { return ((x >> 7) * 0x10204080u) >> 28; }
uint32_t pack_codes(uint32_t e0, uint32_t e1, uint32_t e2, uint32_t e3) {
  return (e0 >> 24) | ((e1 >> 24) << 8) | ((e2 >> 24) << 16) | ((e3 >> 24) << 24);
}

}  // namespace

// sets: walk windows as explicit state sets (the kernel's variant for
// machines without a window machine); win: window bytes (16..32, a multiple
// of 4). stats: [0] open chunks, [1] known chunks, [2] tiles that took the
// look-back, [3] candidate walks.
extern "C" int lexer_emu(const alpacc_tables *t, const uint8_t *in, uint64_t n, int open_end, int sets, int win,
                         uint64_t *out, uint64_t cap, uint64_t *count, int64_t *stats, uint64_t *last_boundary) {
  alpacc::HostGrammar hg;
  std::string why;
  int rc = alpacc::build_host_grammar(t, &hg, &why);
  if (rc != ALPACC_OK) return rc;
  const alpacc::LexerMachine &lm = hg.lex;
  alpacc::LexerTable ltab;
  rc = alpacc::build_lexer_table(lm, &ltab, &why);
  if (rc != ALPACC_OK) return rc;
  if (ltab.ps_tab.empty()) sets = 1;
  const Emu E{lm, ltab};
  const int dead = lm.dead;
  *count = 0;
  *last_boundary = 0;
  for (int i = 0; i < 4; i++) stats[i] = 0;
  if (n == 0) return ALPACC_OK;
  const uint64_t tiles = (n + kData - 1) / kData;
  bool reject = false;
  int error = 0;
  // published per tile: flag 2 + outgoing state, or flag 1 + transition vector
  std::vector<int> flag(tiles, 0), outst(tiles, 0);
  std::vector<std::vector<int>> vec(tiles);
  long long carry_cnt = 0, carry_pos = 0;
  uint64_t k = 0;
  for (uint64_t tile = 0; tile < tiles; tile++) {
    const long long data0 = (long long)tile * kData, load0 = data0 - kWin;
    std::vector<uint8_t> bytes(kLoad, 0);
    for (int i = 0; i < kLoad; i++) {
      const long long p = load0 + i;
      if (p >= 0 && p < (long long)n) bytes[i] = in[p];
    }
    std::vector<int> kind(kThreads, kEmpty), endst(kThreads, 0), nbv(kThreads, 0), start(kThreads, 0);
    std::vector<std::vector<int>> cand(kThreads), lend(kThreads);
    std::vector<std::vector<uint8_t>> lcodes(kThreads);  // open chunks: codes per candidate
    // ---- windows (every chunk's, before any walk writes codes over the
    // bytes: the kernel's barrier), then walks ----
    std::vector<int> x0v(kThreads, -1);
    for (int c = 0; c < kThreads; c++) {
      uint8_t *rb = bytes.data() + kWin + c * kChunk;
      const long long g0 = data0 + (long long)c * kChunk;
      int nb = 0;
      if (g0 < (long long)n) nb = (int)std::min<long long>(kChunk, (long long)n - g0);
      nbv[c] = nb;
      if (nb == 0) continue;
      // the window of `len` bytes ending at the chunk: its one state (the dead
      // state when none), or -1 with the candidates in cv
      auto window = [&](int len, std::vector<int> &cv) -> int {
        const uint8_t *w0 = rb - len;
        cv.clear();
        if (!sets) {
          uint32_t f = ltab.ps_full, e = 0;
          for (int j = 0; j < len; j++) {
            e = E.wstep(f, E.c4(w0[j]));
            f = e;
          }
          const uint32_t info = e >> 24;
          if (info != 0xFF) return (int)info;
          const int p = E.state_of(e);
          for (int s = 0; s < lm.M; s++)
            if (ltab.ps_mask[(size_t)p * 4 + (s >> 6)] >> (s & 63) & 1) cv.push_back(s);
          return -1;
        }
        std::vector<char> set(lm.M, 0);
        const int c0 = lm.cls[w0[0]];
        for (int l = 0; l < lm.img_cnt[c0]; l++) set[lm.img[(size_t)c0 * alpacc::kMaxLanes + l]] = 1;
        for (int j = 1; j < len; j++) {
          std::vector<char> ns(lm.M, 0);
          for (int s = 0; s < lm.M; s++)
            if (set[s]) {
              const int nx = E.state_of(E.step(E.row_of((uint32_t)s), E.c4(w0[j])));
              if (nx != dead) ns[nx] = 1;
            }
          set.swap(ns);
        }
        const int live = (int)std::count(set.begin(), set.end(), 1);
        if (live == 0) return dead;
        if (live == 1) return (int)(std::find(set.begin(), set.end(), 1) - set.begin());
        for (int s = 0; s < lm.M; s++)
          if (set[s]) cv.push_back(s);
        return -1;
      };
      int x0 = -1;
      if (g0 == 0) {
        x0 = lm.m0;
      } else {
        x0 = window(win, cand[c]);
        if (x0 < 0 && c == 0 && win < kWin) x0 = window(kWin, cand[c]);  // the tile's first chunk: the longest window
      }
      x0v[c] = x0;
    }
    for (int c = 0; c < kThreads; c++) {
      uint8_t *rb = bytes.data() + kWin + c * kChunk;
      const long long g0 = data0 + (long long)c * kChunk;
      const int nb = nbv[c];
      if (nb == 0) continue;
      const int x0 = x0v[c];
      if (x0 >= 0) {
        kind[c] = kKnown;
        start[c] = x0;
        if (x0 == dead) {
          reject = true;
          endst[c] = dead;
        } else {
          uint32_t f = E.row_of((uint32_t)x0);
          for (int j = 0; j < nb; j++) {
            const uint32_t e = E.step(f, E.c4(rb[j]));
            rb[j] = (uint8_t)(e >> 24);
            f = e;
          }
          endst[c] = E.state_of(f);
        }
        if (g0 == 0) rb[0] = 0xFF;
        continue;
      }
      if ((int)cand[c].size() > alpacc::kMaxLanes) error = 3;  // more candidates than slots
      kind[c] = nb == kChunk ? kOpen : kOpenTail;
      stats[0]++;
      if (kind[c] == kOpenTail) continue;
      stats[3] += (int64_t)cand[c].size();
      lend[c].resize(cand[c].size());
      lcodes[c].resize(cand[c].size() * kChunk);
      for (size_t l = 0; l < cand[c].size(); l++) {
        uint32_t f = E.row_of((uint32_t)cand[c][l]);
        for (int w = 0; w < kWords; w++) {
          uint32_t e[4];
          for (int q = 0; q < 4; q++) {
            e[q] = E.step(f, E.c4(rb[4 * w + q]));
            f = e[q];
          }
          const uint32_t cw = pack_codes(e[0], e[1], e[2], e[3]);
          std::memcpy(lcodes[c].data() + l * kChunk + 4 * w, &cw, 4);
        }
        lend[c][l] = E.state_of(f);
      }
    }
    for (int c = 0; c < kThreads; c++) stats[1] += kind[c] == kKnown;
    auto slot_of = [&](int c, int x) -> int {
      auto it = std::find(cand[c].begin(), cand[c].end(), x);
      return it == cand[c].end() ? -1 : (int)(it - cand[c].begin());
    };
    auto eval = [&](int c, int x) -> int {
      if (kind[c] == kEmpty) return x;
      if (kind[c] == kKnown) return endst[c];
      if (kind[c] == kOpenTail || x == dead || x < 0) return dead;
      const int slot = slot_of(c, x);
      return slot < 0 ? dead : lend[c][slot];
    };
    // ---- resolution ----
    int ktot = -1;
    std::vector<int> kconst(kThreads);
    for (int c = 0; c < kThreads; c++) {
      kconst[c] = ktot;
      if (kind[c] == kKnown) ktot = c;
    }
    if (ktot >= 0) {
      int x = endst[ktot];
      for (int jj = ktot + 1; jj < kThreads; jj++) x = eval(jj, x);
      flag[tile] = 2;
      outst[tile] = x < 0 ? 0 : x;
    } else if (tile + 1 < tiles) {
      vec[tile].resize(lm.M);
      for (int s = 0; s < lm.M; s++) {
        int x = s;
        for (int jj = 0; jj < kThreads; jj++) x = eval(jj, x);
        vec[tile][s] = x < 0 ? 0 : x;
      }
      flag[tile] = 1;
    }
    int s_in = lm.m0;
    if (kind[0] == kOpen || kind[0] == kOpenTail) {
      stats[2]++;
      if (tile > 0) {
        long long j = (long long)tile - 1;
        int base_state = lm.m0;
        bool have = false;
        while (j >= 0) {
          if (flag[j] >= 2) {
            base_state = outst[j];
            have = true;
            break;
          }
          if (flag[j] == 0) return ALPACC_E_TIMEOUT;  // the kernel would wait forever: a bug
          --j;
        }
        if (!have) j = -1;
        int x = have ? base_state : lm.m0;
        for (long long jj = j + 1; jj < (long long)tile; jj++) {
          if (x == dead || x < 0) break;
          x = vec[jj][x];
        }
        s_in = x;
      }
    }
    for (int c = 0; c < kThreads; c++) {
      if (kind[c] == kKnown) continue;
      int x, from;
      if (kconst[c] >= 0) {
        x = endst[kconst[c]];
        from = kconst[c] + 1;
      } else {
        x = s_in;
        from = 0;
      }
      for (int jj = from; jj < c; jj++) x = eval(jj, x);
      start[c] = x < 0 ? 0 : x;
    }
    if (flag[tile] == 0) {
      flag[tile] = 2;
      const int x = eval(kThreads - 1, start[kThreads - 1]);
      outst[tile] = x < 0 ? 0 : x;
    }
    // ---- open chunks' codes, masks, counts ----
    std::vector<unsigned long long> bmask(kThreads, 0);
    std::vector<long long> cnt(kThreads, 0), lastb(kThreads, 0);
    std::vector<int> final_kept(kThreads, 0), x_endv(kThreads, 0);
    for (int c = 0; c < kThreads; c++) {
      const int nb = nbv[c];
      if (nb == 0) continue;
      uint8_t *rb = bytes.data() + kWin + c * kChunk;
      const long long g0 = data0 + (long long)c * kChunk;
      int x_end = dead;
      if (kind[c] == kKnown) {
        x_end = endst[c];
      } else {
        const int x0 = start[c];
        if (kind[c] == kOpenTail) {
          if (x0 != dead) {
            uint32_t f = E.row_of((uint32_t)x0);
            for (int j = 0; j < nb; j++) {
              const uint32_t e = E.step(f, E.c4(rb[j]));
              rb[j] = (uint8_t)(e >> 24);
              f = e;
            }
            x_end = E.state_of(f);
          }
        } else {
          const int slot = x0 == dead ? -1 : slot_of(c, x0);
          if (slot >= 0) {
            std::memcpy(rb, lcodes[c].data() + slot * kChunk, kChunk);
            x_end = lend[c][slot];
          }
        }
      }
      x_endv[c] = x_end;
      if (x_end == dead) reject = true;
      for (int w = 0; w < kWords; w++) {
        uint32_t cw;
        std::memcpy(&cw, rb + 4 * w, 4);
        bmask[c] |= (unsigned long long)movemask4(nonzero_bytes(~cw)) << (4 * w);
        const uint32_t kb = nonzero_bytes(~(cw | 0x01010101u));
        if (4 * w + 4 <= nb) cnt[c] += __builtin_popcount(kb);
        else if (4 * w < nb) cnt[c] += __builtin_popcount(kb & (0xFFFFFFFFu >> (8 * (4 * w + 4 - nb))));
      }
      if (nb < 64) bmask[c] &= (1ull << nb) - 1;
      if (bmask[c]) lastb[c] = g0 + 63 - __builtin_clzll(bmask[c]);
      if (g0 + nb == (long long)n && !open_end) {
        final_kept[c] = x_end != dead && (lm.flags[x_end] & 4) != 0;
        if (final_kept[c]) ++cnt[c];
        if (x_end == dead || !(lm.flags[x_end] & 2)) reject = true;
      }
    }
    // ---- carry and emission ----
    long long ce = carry_cnt, pe = carry_pos;
    for (int c = 0; c < kThreads; c++) {
      const int nb = nbv[c];
      const long long g0 = data0 + (long long)c * kChunk;
      const uint8_t *rb = bytes.data() + kWin + c * kChunk;
      if (nb > 0) {
        long long prev = pe;
        uint64_t o = (uint64_t)ce;
        for (unsigned long long m = bmask[c]; m; m &= m - 1) {
          const int j = __builtin_ctzll(m);
          const long long p = g0 + j;
          const uint32_t code = rb[j];
          if (code < 0xFE) {
            if ((uint64_t)(p - prev) > hg.len_max) reject = true;
            if (o < cap) {
              out[3 * o] = code;
              out[3 * o + 1] = (uint64_t)prev;
              out[3 * o + 2] = (uint64_t)(p - prev);
            }
            ++o;
          }
          prev = p;
        }
        if (final_kept[c]) {
          if ((uint64_t)((long long)n - prev) > hg.len_max) reject = true;
          if (o < cap) {
            out[3 * o] = lm.term[x_endv[c]];
            out[3 * o + 1] = (uint64_t)prev;
            out[3 * o + 2] = (uint64_t)((long long)n - prev);
          }
          ++o;
        }
        if ((long long)o != ce + cnt[c]) error = 2;  // count and emission disagree
      }
      ce += cnt[c];
      pe = std::max(pe, lastb[c]);
    }
    carry_cnt = ce;
    carry_pos = pe;
    k = (uint64_t)ce;
  }
  if (error) return ALPACC_E_INVALID;
  *count = k;
  *last_boundary = (uint64_t)carry_pos;
  return reject ? ALPACC_REJECT : ALPACC_OK;
}
