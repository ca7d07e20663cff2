// Host driver and C ABI (include/alpacc_b200.h).
//
// One handle = one grammar on one device: its derived tables uploaded once,
// a stream, and scratch buffers that grow to the largest input seen and are
// then reused (the reference allocates and frees device memory per input,
// backends/cuda/cli.cu:747-783).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/alpacc_b200.h"
#include "common.cuh"
#include "device_tables.h"
#include "kernels.h"

using namespace alpacc;

#include "handle.h"
#include "pipeline.h"

namespace {

#define CK(x)                                                   \
  do {                                                          \
    cudaError_t e_ = (x);                                       \
    if (e_ != cudaSuccess) {                                    \
      g->last_error = cudaGetErrorString(e_);                   \
      return ALPACC_E_CUDA;                                     \
    }                                                           \
  } while (0)

#define TRY(x)                 \
  do {                         \
    int r_ = (x);              \
    if (r_ != ALPACC_OK) return r_; \
  } while (0)

int upload_pairs(alpacc_gpu_grammar *g);

// FNV-1a over a byte range, continuing from h (the grammar digest that keys
// the autotuner's cache).
uint64_t fnv_bytes(uint64_t h, const void *p, size_t n) {
  const uint8_t *b = static_cast<const uint8_t *>(p);
  for (size_t i = 0; i < n; i++) h = (h ^ b[i]) * 1099511628211ull;
  return h;
}

// Launch geometry chosen by alpacc_gpu_autotune, cached per (grammar digest,
// device) for the process: handles loaded later for the same grammar and
// device start with it.
struct Geometry {
  int win_words, lex_per_sm, pair_per_sm, pse_per_sm;
};
std::mutex g_geo_mu;
std::map<std::pair<uint64_t, int>, Geometry> g_geo_cache;

void apply_geometry(alpacc_gpu_grammar *g, const Geometry &geo, int sms) {
  g->lex_win_words = geo.win_words;
  g->lex_grid = geo.lex_per_sm * sms;
  g->pair_grid = geo.pair_per_sm * sms;
  g->pse_grid = geo.pse_per_sm * sms;
}

int upload_tables(alpacc_gpu_grammar *g) {
  const LexerMachine &lm = g->hg.lex;
  if (g->hg.parts == ALPACC_PARTS_PARSER) return upload_pairs(g);
  LexerTable lt;
  const int rc = build_lexer_table(lm, &lt, &g->last_error);
  if (rc != ALPACC_OK) return rc;
  g->tab_words = (int)lt.tab.size();
  g->cp_shift = lt.shift;
  g->swz = lt.swz;
  g->wide_cls = lt.wide_cls;
  // ALPACC_LEX_OUTPUT=direct writes the tokens from the lexer kernel itself
  // (counts chained by decoupled look-back) instead of staging boundary codes
  // for the scan and emit kernels
  const char *ov = std::getenv("ALPACC_LEX_OUTPUT");
  g->lex_direct = ov && std::strcmp(ov, "direct") == 0 ? 1 : 0;
  // ALPACC_WALK_PREFIX=pairs: the walks' tile prefixes from the pair kernel's
  // aggregates and walk_prefix_kernel instead of the walks' own look-back
  // (measured slower on json_ext and sexp: the aggregation costs the pair
  // kernel more than the look-back costs the walks)
  const char *pv = std::getenv("ALPACC_WALK_PREFIX");
  g->walk_lookback = pv && std::strcmp(pv, "pairs") == 0 ? 0 : 1;
  // ALPACC_LEX_WINDOW=sets walks windows as explicit state sets even when the
  // window machine exists (tests run that kernel on small machines too)
  const char *wv = std::getenv("ALPACC_LEX_WINDOW");
  const bool force_sets = wv && std::strcmp(wv, "sets") == 0;
  if (!lt.ps_tab.empty() && !force_sets) {
    g->lex_variant = lm.M > 64 ? 1 : 0;
    g->ps_words = (int)lt.ps_tab.size();
    g->ps_full = lt.ps_full;
    g->ps_sets = lt.ps_sets;
    TRY(upload(g->lex_ps, lt.ps_tab));
    TRY(upload(g->lex_psmask, lt.ps_mask));
  } else {
    g->lex_variant = 2;
    g->ps_words = 0;
  }
  if (g->wide_cls) {
    TRY(upload(g->lex_cls4, lt.cls4));
  } else {
    std::vector<uint8_t> c4(lt.cls4.begin(), lt.cls4.end());
    TRY(upload(g->lex_cls4, c4));
  }
  TRY(upload(g->lex_tab, lt.tab));
  TRY(upload(g->img, lm.img));
  TRY(upload(g->img_cnt, lm.img_cnt));
  g->digest = fnv_bytes(g->digest, lt.tab.data(), lt.tab.size() * 4);
  g->digest = fnv_bytes(g->digest, lt.cls4.data(), lt.cls4.size() * 2);
  g->digest = fnv_bytes(g->digest, lm.term.data(), lm.term.size());
  g->digest = fnv_bytes(g->digest, lm.flags.data(), lm.flags.size());
  TRY(upload(g->sterm, lm.term));
  TRY(upload(g->sflags, lm.flags));
  return g->hg.parts == ALPACC_PARTS_LEXER ? ALPACC_OK : upload_pairs(g);
}

int upload_pairs(alpacc_gpu_grammar *g) {
  const PairTable &pt = g->hg.pairs;
  g->digest = fnv_bytes(g->digest, pt.dense.data(), pt.dense.size() * 4);
  g->digest = fnv_bytes(g->digest, pt.ht_key.data(), pt.ht_key.size() * 8);
  g->digest = fnv_bytes(g->digest, pt.stacks.data(), pt.stacks.size() * 4);
  g->digest = fnv_bytes(g->digest, pt.prods.data(), pt.prods.size() * 4);
  g->digest = fnv_bytes(g->digest, pt.arity.data(), pt.arity.size() * 4);
  if (pt.hashed) {
    TRY(upload(g->ht_key, pt.ht_key));
    TRY(upload(g->ht_rec, pt.ht_rec));
  } else {
    TRY(upload(g->dense, pt.dense));
  }
  // records packed as ss | ps << 24 | nb << 48 | np << 56 (spans checked < 2^24 on load)
  std::vector<unsigned long long> rec(pt.rec_ss.size());
  for (size_t i = 0; i < rec.size(); i++)
    rec[i] = (unsigned long long)pt.rec_ss[i] | ((unsigned long long)pt.rec_ps[i] << 24) |
             ((unsigned long long)pt.rec_nb[i] << 48) | ((unsigned long long)pt.rec_np[i] << 56);
  TRY(upload(g->rec, rec));

  TRY(upload(g->stacks, pt.stacks));
  TRY(upload(g->prods, pt.prods));
  TRY(upload(g->arity, pt.arity));
  TRY(upload(g->is_term, pt.is_term));
  return ALPACC_OK;
}

int sync_status(alpacc_gpu_grammar *g) {
  CK(cudaMemcpyAsync(g->h_status, g->d_status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, g->stream));
  CK(cudaStreamSynchronize(g->stream));
  if (g->h_status->error != 0) return g->h_status->error;
  return ALPACC_OK;
}

// Per-stage device times (events around each stage's launches), recorded
// only while stage timing is on: two event records per stage cost host time
// that a small input's call feels.
void stage_begin(alpacc_gpu_grammar *g, int k) {
  if (!g->stage_timing) return;
  cudaEventRecord(g->sev[2 * k], g->stream);
  g->stage_used[k] = true;
}
void stage_end(alpacc_gpu_grammar *g, int k) {
  if (g->stage_timing) cudaEventRecord(g->sev[2 * k + 1], g->stream);
}
void collect_stages(alpacc_gpu_grammar *g) {
  for (int k = 0; k < alpacc_gpu_grammar::kStages; k++) {
    float ms = 0;
    g->stage_ms[k] = (g->stage_used[k] && cudaEventElapsedTime(&ms, g->sev[2 * k], g->sev[2 * k + 1]) == cudaSuccess)
                         ? ms
                         : 0.0;
  }
}

// The dynamic shared-memory attribute of the lexer kernels, per device (the
// caller's current device) and shared by every handle on it: only raised.
int ensure_lex_smem(int device, size_t bytes) {
  static std::mutex mu;
  static std::map<int, size_t> current;
  std::lock_guard<std::mutex> lock(mu);
  size_t &cur = current[device];
  if (bytes <= cur) return ALPACC_OK;
  if (cur == 0 &&
      cudaFuncSetAttribute(lex_emit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kLexEmitSmem) != cudaSuccess) {
    cudaGetLastError();
    return ALPACC_E_CUDA;
  }
  for (auto k : {lex_kernel, lex_kernel_wide, lex_kernel_sets, lex_direct_kernel, lex_direct_kernel_wide,
                 lex_direct_kernel_sets})
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) {
      cudaGetLastError();
      return ALPACC_E_CUDA;
    }
  cur = bytes;
  return ALPACC_OK;
}

constexpr uint64_t kPieceTiles = (16u << 20) / kLexData;  // tiles per host-to-device piece (~16 MiB)

// Token arrays of the current host call: copied on cstream once the lexer
// finished, overlapping the parser's kernels.
int start_token_copy(alpacc_gpu_grammar *g, uint64_t T) {
  const alpacc_tables &tb = g->hg.t;
  const size_t sz[3] = {T * tb.terminal_size, T * tb.index_size, T * tb.length_size};
  size_t total = sizeof(PinnedBlock);
  for (int i = 0; i < 3; i++) {
    g->tok_off[i] = total;
    total += (sz[i] + 15) & ~(size_t)15;
  }
  PinnedBlock *b = acquire_block(g, &g->pinned_cache, &g->pinned_cache_size, total);
  if (!b) return ALPACC_E_NOMEM;
  g->tok_block = b;
  CK(cudaStreamWaitEvent(g->cstream, g->lex_done, 0));
  const void *src[3] = {g->tok_ids.p, g->tok_starts.p, g->tok_lens.p};
  for (int i = 0; i < 3; i++)
    if (sz[i]) CK(cudaMemcpyAsync((char *)b + g->tok_off[i], src[i], sz[i], cudaMemcpyDeviceToHost, g->cstream));
  return ALPACC_OK;
}

// Drop the current call's token block (after a reject or an error).
void abandon_host_result(alpacc_gpu_grammar *g) {
  if (!g->tok_block) return;
  cudaStreamSynchronize(g->cstream);
  release_block(g, reinterpret_cast<PinnedBlock *>(g->tok_block), false);
  g->tok_block = nullptr;
}

// Tree arrays of the current host call, then the whole result.
int finish_host_result(alpacc_gpu_grammar *g, alpacc_result *out) {
  const alpacc_tables &tb = g->hg.t;
  const uint64_t T = g->last_T, N = g->last_N;
  const size_t sz[3] = {N * tb.production_size, N * tb.index_size, T * tb.index_size};
  size_t off[3], total = sizeof(PinnedBlock);
  for (int i = 0; i < 3; i++) {
    off[i] = total;
    total += (sz[i] + 15) & ~(size_t)15;
  }
  PinnedBlock *tree = acquire_block(g, &g->pinned_cache2, &g->pinned_cache2_size, total);
  if (!tree) {
    abandon_host_result(g);
    return ALPACC_E_NOMEM;
  }
  const void *src[3] = {g->node_prods.p, g->node_parents.p, g->token_parents.p};
  for (int i = 0; i < 3; i++)
    if (sz[i]) CK(cudaMemcpyAsync((char *)tree + off[i], src[i], sz[i], cudaMemcpyDeviceToHost, g->stream));
  CK(cudaStreamSynchronize(g->stream));
  CK(cudaStreamSynchronize(g->cstream));
  PinnedBlock *toks = reinterpret_cast<PinnedBlock *>(g->tok_block);
  g->tok_block = nullptr;
  toks->second = tree;
  std::memset(out, 0, sizeof(*out));
  out->valid = 1;
  out->num_tokens = T;
  out->num_nodes = N;
  out->token_ids = (char *)toks + g->tok_off[0];
  out->token_starts = (char *)toks + g->tok_off[1];
  out->token_lengths = (char *)toks + g->tok_off[2];
  out->node_productions = (char *)tree + off[0];
  out->node_parents = (char *)tree + off[1];
  out->token_parents = (char *)tree + off[2];
  out->internal = toks;
  return ALPACC_OK;
}

// What run_device computes: the combined path, the lexer alone (lexer-mode
// program), or the parser alone on token ids already in g->tok_ids
// (parser-mode program: pairs and the bracket walk, no tree).
enum RunMode { kRunBoth = 0, kRunLex = 1, kRunParse = 2 };

// One window of chunked lexing (kRunLex): whether the input continues after
// the window, and the window's offset (added to token starts).
struct LexWindow {
  int open_end;
  uint64_t index_base;
};

// Per-call flags, tickets and counters: one region of the handle's `flags`
// buffer, zeroed by one memset per call (byte offsets, 16-byte aligned).
struct FlagLayout {
  size_t lex_ticket = 0, st1_flag = 0, st2_flags = 0, pair_ticket = 0, pst_flags = 0;
  size_t pse_ticket[2] = {}, pse_flags[2] = {}, super_key[2] = {}, walk_step[2] = {}, walk_term = 0;
  size_t total = 0;
  size_t take(size_t bytes) {
    const size_t off = total;
    total += (std::max<size_t>(bytes, 16) + 15) & ~(size_t)15;
    return off;
  }
};

// Capacity (elements) of a parser-stage array whose exact size only the
// device knows: the full bound when it is small; else the largest exact need
// seen on this handle (with 1/8 slack), at least a floor. A device-side
// overflow makes the call grow to the exact need and run again.
uint64_t plan_cap(uint64_t bound, uint64_t need_seen) {
  constexpr uint64_t kFull = 16ull << 20, kFloor = 16ull << 20;
  if (bound <= kFull) return bound;
  const uint64_t seen = need_seen + need_seen / 8;
  return std::min(bound, std::max(seen, kFloor));
}

// The whole device path for d_in[0..n) (n bytes; n token ids for kRunParse),
// launched without waiting for the host in between: each stage reads the
// counts of the previous one from the device status. Leaves counts in
// g->last_T / last_N.
int run_device_once(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n, int mode, const LexWindow *win) {
  const HostGrammar &hg = g->hg;
  const alpacc_tables &tb = hg.t;
  const LexerMachine &lm = hg.lex;
  const PairTable &pt = hg.pairs;
  const int term_w = (int)tb.terminal_size, idx_w = (int)tb.index_size, len_w = (int)tb.length_size;
  const int prod_w = (int)tb.production_size;
  if (n > (1ull << 31) - 1) return ALPACC_E_CAPACITY;
  g->launches = 0;
  for (int k = 0; k < alpacc_gpu_grammar::kStages; k++) g->stage_used[k] = false;

  // ---- sizes: bounds from n, capacities for what only the device knows ----
  const bool lexing = mode != kRunParse && n > 0;
  const uint64_t lex_tiles = lexing ? (n + kLexData - 1) / kLexData : 0;
  uint64_t piece_tiles = lex_tiles, pieces = lexing ? 1 : 0;
  if (lexing && g->h_in) {  // host input: copied in pieces of ~16 MiB, each lexed as soon as it arrived
    piece_tiles = kPieceTiles;
    pieces = (lex_tiles + piece_tiles - 1) / piece_tiles;
    if (pieces > (uint64_t)alpacc_gpu_grammar::kMaxPieces) {
      piece_tiles = (lex_tiles + alpacc_gpu_grammar::kMaxPieces - 1) / alpacc_gpu_grammar::kMaxPieces;
      pieces = (lex_tiles + piece_tiles - 1) / piece_tiles;
    }
  }
  const bool parsing = mode != kRunLex;
  const uint64_t T_ub = n;  // a token covers at least one byte; parser mode: exactly n ids
  const uint64_t m_ub = T_ub + 2;
  const uint64_t pair_tiles = parsing ? (m_ub + kPairTile - 1) / kPairTile : 0;
  const uint64_t max_br = (uint64_t)std::max(pt.max_br, 1), max_pr = (uint64_t)std::max(pt.max_pr, 1);
  const uint64_t br_cap = parsing ? plan_cap(m_ub * max_br, g->need_br) : 0;
  const uint64_t pr_cap = parsing ? plan_cap(m_ub * max_pr, g->need_pr) : 0;
  const uint64_t e_cap = std::max<uint64_t>(std::max(br_cap, pr_cap), 1);
  const uint64_t pse_tiles = (e_cap + kPseTile - 1) / kPseTile;
  const uint64_t super_n = (pse_tiles >> kPseSuperShift) + 1;

  FlagLayout fl;
  fl.lex_ticket = fl.take(16 + pieces * 4);
  fl.st1_flag = fl.take(lex_tiles * 4);
  fl.st2_flags = fl.take(lex_tiles * 4);
  fl.pair_ticket = fl.take(16);
  fl.pst_flags = fl.take(pair_tiles * 4);
  for (int w = 0; w < 2; ++w) {
    fl.pse_ticket[w] = fl.take(16);
    fl.pse_flags[w] = fl.take(parsing ? pse_tiles * 4 : 0);
    fl.super_key[w] = fl.take(parsing ? super_n * 4 : 0);
    fl.walk_step[w] = fl.take(parsing ? pse_tiles * 4 : 0);
  }
  fl.walk_term = fl.take(parsing ? pse_tiles * 4 : 0);
  TRY(grow(g->flags, fl.total));
  uint8_t *fb = (uint8_t *)g->flags.p;
  if (lexing) {
    TRY(grow(g->codes, lex_tiles * (uint64_t)kLexData));
    TRY(grow(g->tile_cnt, lex_tiles * 4));
    TRY(grow(g->tile_pos, lex_tiles * 4));
    TRY(grow(g->tile_off, lex_tiles * 8));
    TRY(grow(g->tile_prev, lex_tiles * 4));
    TRY(grow(g->st1_state, lex_tiles));
    TRY(grow(g->st1_vec, lex_tiles * (uint64_t)lm.M));
    TRY(grow(g->st2_agg, lex_tiles * 16));
    TRY(grow(g->st2_inc, lex_tiles * 16));
    // tokens: at most one per byte (n + 1 leaves room for what a rejected
    // input's chunks may write before the reject is known)
    TRY(grow(g->tok_ids, (n + 1) * term_w));
    TRY(grow(g->tok_starts, (n + 1) * idx_w));
    TRY(grow(g->tok_lens, (n + 1) * len_w));
  }
  if (parsing) {
    TRY(grow(g->tok_ids, std::max<uint64_t>(T_ub, 1) * term_w));
    TRY(grow(g->pst_agg, pair_tiles * 16));
    TRY(grow(g->pst_inc, pair_tiles * 16));
    TRY(grow(g->br, br_cap * 4));
    TRY(grow(g->pr, pr_cap * 4));
    TRY(grow(g->pse_agg, pse_tiles * 16));
    TRY(grow(g->pse_inc, pse_tiles * 16));
    TRY(grow(g->tile_min, pse_tiles * 4));
    TRY(grow(g->pse_regions, pse_region_bytes(pse_tiles)));
    TRY(grow(g->walk_prefix, std::max<uint64_t>(pse_tiles, 1) * 3 * 8));
    TRY(grow(g->node_prods, std::max<uint64_t>(pr_cap, 1) * prod_w));
    TRY(grow(g->node_parents, std::max<uint64_t>(pr_cap, 1) * idx_w));
    TRY(grow(g->token_parents, std::max<uint64_t>(T_ub, 1) * idx_w));
  }

  CK(cudaMemsetAsync(g->d_status, 0, sizeof(DeviceStatus), g->stream));
  CK(cudaMemsetAsync(fb, 0, fl.total, g->stream));
  if (g->diag) {  // phase cycles: lexer [0, 8), bracket walk [8, 16), parent walk [16, 24)
    TRY(grow(g->diag_cycles, sizeof g->phase_cycles));
    CK(cudaMemsetAsync(g->diag_cycles.p, 0, sizeof g->phase_cycles, g->stream));
  }
  CK(cudaEventRecord(g->ev0, g->stream));

  // ---------------- lexer ----------------
  if (mode == kRunParse) {
    const uint64_t T = n;  // from pageable memory: staged before the call returns
    CK(cudaMemcpyAsync(&g->d_status->num_tokens, &T, 8, cudaMemcpyHostToDevice, g->stream));
  } else if (lexing) {
    LexArgs a = lex_args(g, d_in, n, lex_tiles);
    if (g->diag) a.phase_cycles = (unsigned long long *)g->diag_cycles.p;
    a.st1_flag = (unsigned *)(fb + fl.st1_flag);
    a.st2.flags = (unsigned *)(fb + fl.st2_flags);
    if (win) {
      a.open_end = win->open_end;
      a.index_base = win->index_base;
    }
    stage_begin(g, 0);
    for (uint64_t k = 0; k < pieces; ++k) {
      const uint64_t t0 = k * piece_tiles, t1 = std::min(lex_tiles, t0 + piece_tiles);
      if (g->h_in) {
        const uint64_t b0 = t0 * kLexData, b1 = std::min<uint64_t>(n, t1 * kLexData);
        CK(cudaMemcpyAsync((uint8_t *)d_in + b0, g->h_in + b0, b1 - b0, cudaMemcpyHostToDevice, g->cstream));
        CK(cudaEventRecord(g->piece_ev[k], g->cstream));
        CK(cudaStreamWaitEvent(g->stream, g->piece_ev[k], 0));
      }
      a.tile_begin = t0;
      a.tile_end = t1;
      a.ticket = (unsigned *)(fb + fl.lex_ticket) + 4 + k;
      const unsigned grid = (unsigned)std::min<uint64_t>(t1 - t0, (uint64_t)g->lex_grid);
      CK(g->lex_direct ? launch_lex_direct(g, a, grid, g->stream) : launch_lex(g, a, grid, g->stream));
      ++g->launches;
    }
    if (!g->lex_direct) {
      CK(launch_lex_emit(lex_emit_args(g, a), g->stream));
      g->launches += 2;
    }
    stage_end(g, 0);
  }
  CK(cudaEventRecord(g->lex_done, g->stream));
  // host calls: the lexer's status is read back on the copy stream while the
  // parser runs, so that the token arrays can follow at once
  if (g->host_out && parsing && lexing) {
    CK(cudaStreamWaitEvent(g->cstream, g->lex_done, 0));
    CK(cudaMemcpyAsync(g->h_lex_status, g->d_status, sizeof(DeviceStatus), cudaMemcpyDeviceToHost, g->cstream));
    CK(cudaEventRecord(g->lex_status_ev, g->cstream));
  }

  if (parsing) {
    // ---------------- pair lookup ----------------
    if (n == 0 && mode != kRunParse) CK(cudaMemsetAsync(&g->d_status->num_tokens, 0, 8, g->stream));
    PairArgs a = pair_args(g);
    a.tiles_cap = pair_tiles;
    a.br_cap = br_cap;
    a.pr_cap = pr_cap;
    a.ticket = (unsigned *)(fb + fl.pair_ticket);
    a.st.flags = (unsigned *)(fb + fl.pst_flags);
    // the walks' tile prefixes: their own decoupled look-back, or (selected
    // at load) the pair kernel's aggregates scanned by walk_prefix_kernel
    const bool pfx_on = !g->walk_lookback;
    a.walk_step[0] = pfx_on ? (int *)(fb + fl.walk_step[0]) : nullptr;
    a.walk_step[1] = pfx_on ? (int *)(fb + fl.walk_step[1]) : nullptr;
    a.walk_term = pfx_on ? (int *)(fb + fl.walk_term) : nullptr;
    a.walk_tiles_cap = pse_tiles;
    long long *pfx = (long long *)g->walk_prefix.p;
    const uint64_t pt_n = std::max<uint64_t>(pse_tiles, 1);
    stage_begin(g, 1);
    pair_kernel<<<(unsigned)std::min<uint64_t>(pair_tiles, (uint64_t)g->pair_grid), kPairThreads, 0, g->stream>>>(a);
    ++g->launches;
    CK(cudaGetLastError());
    if (pfx_on) {
      WalkPrefixArgs w{};
      w.walk_step[0] = a.walk_step[0];
      w.walk_step[1] = a.walk_step[1];
      w.walk_term = a.walk_term;
      w.prefix_s[0] = pfx;
      w.prefix_s[1] = pfx + pt_n;
      w.prefix_t = pfx + 2 * pt_n;
      w.tiles_cap = pse_tiles;
      w.status = g->d_status;
      walk_prefix_kernel<<<1, 1024, 0, g->stream>>>(w);
      ++g->launches;
      CK(cudaGetLastError());
    }
    stage_end(g, 1);

    // ------- depth walks (the parent walk also writes the compacted tree) -------
    const int walks = mode == kRunParse ? 1 : 2;  // the parser-mode result has no tree
    for (int walk = 0; walk < walks; ++walk) {
      PseArgs pa = pse_args(g, walk, pse_tiles);
      pa.elem_cap = walk == kPseBrackets ? br_cap : pr_cap;
      pa.ticket = (unsigned *)(fb + fl.pse_ticket[walk]);
      pa.resolve_ticket = pa.ticket + 1;
      pa.st.flags = (unsigned *)(fb + fl.pse_flags[walk]);
      pa.super_key = (uint32_t *)(fb + fl.super_key[walk]);
      pa.prefix_s = pfx_on ? pfx + walk * pt_n : nullptr;
      pa.prefix_t = pfx_on ? pfx + 2 * pt_n : nullptr;
      if (g->diag) pa.phase_cycles = (unsigned long long *)g->diag_cycles.p + 8 + 8 * walk;
      const uint64_t tiles = (pa.elem_cap + kPseTile - 1) / kPseTile;
      stage_begin(g, 2 + 2 * walk);
      pse_tile_kernel<<<(unsigned)std::max<uint64_t>(std::min<uint64_t>(tiles, (uint64_t)g->pse_grid), 1), kPseThreads,
                        0, g->stream>>>(pa);
      ++g->launches;
      stage_end(g, 2 + 2 * walk);
      CK(cudaGetLastError());
      stage_begin(g, 3 + 2 * walk);
      pse_resolve_kernel<<<resolve_blocks(tiles), 256, 0, g->stream>>>(pa);
      ++g->launches;
      stage_end(g, 3 + 2 * walk);
      CK(cudaGetLastError());
    }
    if (mode == kRunParse) {  // parse_test's productions at production_t width
      narrow_u32_kernel<<<(unsigned)std::max<uint64_t>(std::min<uint64_t>((pr_cap + 1023) / 1024, 148 * 8), 1), 256, 0,
                          g->stream>>>((const uint32_t *)g->pr.p, g->node_prods.p, &g->d_status->num_productions,
                                       pr_cap, prod_w);
      ++g->launches;
      CK(cudaGetLastError());
    }
  }
  CK(cudaEventRecord(g->ev1, g->stream));

  // ---- host calls: the token arrays, copied while the parser runs ----
  if (g->host_out && parsing && lexing) {
    CK(cudaEventSynchronize(g->lex_status_ev));
    const DeviceStatus &ls = *g->h_lex_status;
    if (ls.error == 0 && !ls.reject) TRY(start_token_copy(g, ls.num_tokens));
  }
  int rc = sync_status(g);
  if (rc == ALPACC_OK && g->h_status->overflow) rc = ALPACC_E_CAPACITY;  // grown and run again by run_device
  if (g->diag && cudaMemcpy(g->phase_cycles, g->diag_cycles.p, sizeof g->phase_cycles, cudaMemcpyDeviceToHost) !=
                     cudaSuccess)
    cudaGetLastError();
  float ms = 0;
  if (cudaEventElapsedTime(&ms, g->ev0, g->ev1) == cudaSuccess) g->last_ms = ms;
  collect_stages(g);
  const DeviceStatus &st = *g->h_status;
  if (parsing) {  // exact needs of this input, for the capacities of later calls
    g->need_br = std::max<uint64_t>(g->need_br, st.num_brackets);
    g->need_pr = std::max<uint64_t>(g->need_pr, st.num_productions);
  }
  if (rc) return rc;
  if (st.reject) return ALPACC_REJECT;
  const uint64_t T = mode == kRunParse ? n : st.num_tokens;
  if (g->host_out && mode == kRunLex) TRY(start_token_copy(g, T));
  g->last_T = T;
  if (mode == kRunLex) {
    g->last_N = 0;
    return ALPACC_OK;
  }
  if (mode == kRunParse) {
    g->last_N = st.num_productions;
    return ALPACC_OK;
  }
  if (st.num_productions == 0 && T != 0) return ALPACC_REJECT;  // compact_tree: terminal count mismatch
  g->last_N = st.num_nodes;
  return ALPACC_OK;
}

// run_device_once, and once more with capacities grown to the exact needs
// when a parser-stage array overflowed on the device (a first call on an
// input larger than any before).
int run_device(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n, int mode = kRunBoth,
               const LexWindow *win = nullptr) {
  int rc = run_device_once(g, d_in, n, mode, win);
  if (rc == ALPACC_E_CAPACITY && n <= (1ull << 31) - 1) {
    abandon_host_result(g);
    const uint8_t *h_in = g->h_in;
    g->h_in = nullptr;  // the input is on the device already
    rc = run_device_once(g, d_in, n, mode, win);
    g->h_in = h_in;
  }
  return rc;
}

void fill_device_result(alpacc_gpu_grammar *g, alpacc_result *out, int status) {
  std::memset(out, 0, sizeof(*out));
  out->on_device = 1;
  if (status != ALPACC_OK) return;
  out->valid = 1;
  out->num_tokens = g->last_T;
  out->num_nodes = g->last_N;
  out->token_ids = g->tok_ids.p;
  out->token_starts = g->tok_starts.p;
  out->token_lengths = g->tok_lens.p;
  out->node_productions = g->node_prods.p;
  out->node_parents = g->node_parents.p;
  out->token_parents = g->token_parents.p;
}

}  // namespace

extern "C" {

alpacc_gpu_grammar *alpacc_gpu_load(const alpacc_tables *tables, int device, uint64_t max_input, int *err) {
  int dummy;
  if (!err) err = &dummy;
  alpacc_gpu_grammar *g = new (std::nothrow) alpacc_gpu_grammar();
  if (!g) {
    *err = ALPACC_E_NOMEM;
    return nullptr;
  }
  std::string why;
  int rc = build_host_grammar(tables, &g->hg, &why);
  if (rc != ALPACC_OK) {
    g->last_error = why;
    *err = rc;
    delete g;
    return nullptr;
  }
  g->device = device;
  if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&g->ev0) != cudaSuccess || cudaEventCreate(&g->ev1) != cudaSuccess ||
      [&] {
        for (auto &e : g->sev)
          if (cudaEventCreate(&e) != cudaSuccess) return true;
        return false;
      }() ||
      cudaStreamCreateWithFlags(&g->cstream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&g->lex_done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&g->lex_status_ev, cudaEventDisableTiming) != cudaSuccess ||
      [&] {
        for (auto &e : g->piece_ev)
          if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return true;
        return false;
      }() ||
      alpacc::dev_malloc(reinterpret_cast<void **>(&g->d_status), sizeof(DeviceStatus)) != cudaSuccess ||
      cudaMallocHost(&g->h_status, sizeof(DeviceStatus)) != cudaSuccess ||
      cudaMallocHost(&g->h_lex_status, sizeof(DeviceStatus)) != cudaSuccess) {
    cudaGetLastError();
    *err = ALPACC_E_CUDA;
    alpacc_gpu_free(g);
    return nullptr;
  }
  std::memset(g->h_status, 0, sizeof(DeviceStatus));
  rc = upload_tables(g);
  if (rc == ALPACC_OK) rc = ensure_lex_smem(device, lex_dyn_smem(g));
  if (rc == ALPACC_OK) {
    int per_sm = 0, sms = 0;
    int pair_sm = 0, pse_sm = 0;
    if (lex_occupancy(g, &per_sm) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pair_sm, pair_kernel, kPairThreads, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pse_sm, pse_tile_kernel, kPseThreads, 0) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || per_sm < 1 ||
        pair_sm < 1 || pse_sm < 1) {
      cudaGetLastError();
      rc = ALPACC_E_CUDA;
    } else {
      g->lex_grid = per_sm * sms;
      g->pair_grid = pair_sm * sms;
      g->pse_grid = pse_sm * sms;
      g->sms = sms;
      std::lock_guard<std::mutex> lock(g_geo_mu);
      auto it = g_geo_cache.find({g->digest, device});
      if (it != g_geo_cache.end()) {
        apply_geometry(g, it->second, sms);
        g->geo_cached = 1;
      }
    }
  }
  if (rc == ALPACC_OK && max_input > 0) rc = grow(g->in, max_input + 16);
  if (rc != ALPACC_OK) {
    *err = rc;
    alpacc_gpu_free(g);
    return nullptr;
  }
  *err = ALPACC_OK;
  return g;
}

void alpacc_gpu_free(alpacc_gpu_grammar *g) {
  if (!g) return;
  cudaSetDevice(g->device);
  if (g->stream) cudaStreamSynchronize(g->stream);
  DevBuf *bufs[] = {&g->lex_tab, &g->lex_cls4, &g->lex_ps, &g->lex_psmask, &g->img, &g->img_cnt, &g->sterm, &g->sflags,
                    &g->dense, &g->ht_key, &g->ht_rec, &g->rec, &g->stacks, &g->prods,
                    &g->arity, &g->is_term, &g->in, &g->lex_ticket, &g->st1_flag, &g->st1_state, &g->st1_vec,
                    &g->st2_flags, &g->st2_agg, &g->st2_inc, &g->tok_ids, &g->tok_starts, &g->tok_lens,
                    &g->pair_ticket, &g->pst_flags, &g->pst_agg, &g->pst_inc, &g->br, &g->pr, &g->pse_ticket,
                    &g->pse_flags, &g->pse_agg, &g->pse_inc, &g->tile_min, &g->super_key, &g->pse_regions, &g->walk_prefix,
                    &g->node_prods, &g->node_parents,
                    &g->token_parents, &g->flags, &g->diag_cycles, &g->codes, &g->tile_cnt, &g->tile_pos,
                    &g->tile_off, &g->tile_prev, &g->b_arrays, &g->b_desc, &g->b_status,
                    &g->b_pack, &g->b_packed};
  for (DevBuf *b : bufs) release(*b);
  if (g->cstream) cudaStreamSynchronize(g->cstream);
  if (g->pinned_cache) cudaFreeHost(g->pinned_cache);
  if (g->pinned_cache2) cudaFreeHost(g->pinned_cache2);
  if (g->tok_block) cudaFreeHost(g->tok_block);
  if (g->lex_done) cudaEventDestroy(g->lex_done);
  for (auto &e : g->piece_ev)
    if (e) cudaEventDestroy(e);
  if (g->cstream) cudaStreamDestroy(g->cstream);
  if (g->d_status) cudaFree(g->d_status);
  if (g->h_status) cudaFreeHost(g->h_status);
  if (g->h_lex_status) cudaFreeHost(g->h_lex_status);
  if (g->lex_status_ev) cudaEventDestroy(g->lex_status_ev);
  if (g->ev0) cudaEventDestroy(g->ev0);
  if (g->ev1) cudaEventDestroy(g->ev1);
  for (auto &e : g->sev)
    if (e) cudaEventDestroy(e);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

int alpacc_gpu_parse_device(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n, alpacc_result *out) {
  if (!g || !out || (n > 0 && !d_in) || g->hg.parts != ALPACC_PARTS_BOTH) return ALPACC_E_INVALID;
  if (cudaSetDevice(g->device) != cudaSuccess) return ALPACC_E_CUDA;
  int rc = run_device(g, d_in, n);
  g->last_status = rc;
  fill_device_result(g, out, rc);
  return rc;
}

int alpacc_gpu_enqueue(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n) {
  if (!g || (n > 0 && !d_in) || g->hg.parts != ALPACC_PARTS_BOTH) return ALPACC_E_INVALID;
  if (cudaSetDevice(g->device) != cudaSuccess) return ALPACC_E_CUDA;
  int rc = run_device(g, d_in, n);
  g->last_status = rc;
  return rc < 0 ? rc : ALPACC_OK;
}

int alpacc_gpu_collect(alpacc_gpu_grammar *g, alpacc_result *out) {
  if (!g || !out) return ALPACC_E_INVALID;
  fill_device_result(g, out, g->last_status);
  return g->last_status;
}

int alpacc_gpu_parse(alpacc_gpu_grammar *g, const uint8_t *in, uint64_t n, alpacc_result *out) {
  if (!g || !out || (n > 0 && !in)) return ALPACC_E_INVALID;
  std::memset(out, 0, sizeof(*out));
  if (g->hg.parts != ALPACC_PARTS_BOTH) return ALPACC_E_INVALID;
  if (cudaSetDevice(g->device) != cudaSuccess) return ALPACC_E_CUDA;
  int rc = grow(g->in, n + 16);
  if (rc) return rc;
  g->h_in = in;
  g->host_out = true;
  rc = run_device(g, (const uint8_t *)g->in.p, n);
  g->h_in = nullptr;
  g->host_out = false;
  g->last_status = rc;
  if (rc == ALPACC_OK && !g->tok_block) rc = start_token_copy(g, g->last_T);  // empty input: no lexer ran
  if (rc != ALPACC_OK) {
    cudaStreamSynchronize(g->cstream);  // no piece copy may still read the caller's buffer
    abandon_host_result(g);
    return rc;
  }
  return finish_host_result(g, out);
}

void alpacc_result_free(alpacc_result *r) {
  if (!r) return;
  if (r->internal) {
    PinnedBlock *b = reinterpret_cast<PinnedBlock *>(r->internal);
    if (__atomic_sub_fetch(&b->refs, 1, __ATOMIC_ACQ_REL) <= 0) {  // the last result sharing this block
      PinnedBlock *tree = b->second;
      alpacc_gpu_grammar *g = b->owner;
      if (g) {
        release_block(g, b, false);
        release_block(g, tree, true);
      } else {
        cudaFreeHost(b);
        if (tree) cudaFreeHost(tree);
      }
    }
  }
  std::memset(r, 0, sizeof(*r));
}

int alpacc_gpu_lex(alpacc_gpu_grammar *g, const uint8_t *in, uint64_t n, alpacc_result *out) {
  if (!g || !out || (n > 0 && !in)) return ALPACC_E_INVALID;
  std::memset(out, 0, sizeof(*out));
  if (g->hg.parts == ALPACC_PARTS_PARSER) return ALPACC_E_INVALID;
  if (cudaSetDevice(g->device) != cudaSuccess) return ALPACC_E_CUDA;
  int rc = grow(g->in, n + 16);
  if (rc) return rc;
  g->h_in = in;
  g->host_out = true;
  rc = run_device(g, (const uint8_t *)g->in.p, n, kRunLex);
  g->h_in = nullptr;
  g->host_out = false;
  g->last_status = rc;
  if (rc == ALPACC_OK && !g->tok_block) rc = start_token_copy(g, g->last_T);  // empty input: no lexer ran
  if (rc != ALPACC_OK) {
    cudaStreamSynchronize(g->cstream);  // no piece copy may still read the caller's buffer
    abandon_host_result(g);
    return rc;
  }
  if (cudaStreamSynchronize(g->cstream) != cudaSuccess) {
    abandon_host_result(g);
    return ALPACC_E_CUDA;
  }
  PinnedBlock *toks = reinterpret_cast<PinnedBlock *>(g->tok_block);
  g->tok_block = nullptr;
  out->valid = 1;
  out->num_tokens = g->last_T;
  out->token_ids = (char *)toks + g->tok_off[0];
  out->token_starts = (char *)toks + g->tok_off[1];
  out->token_lengths = (char *)toks + g->tok_off[2];
  out->internal = toks;
  return ALPACC_OK;
}

int alpacc_gpu_lex_stream(alpacc_gpu_grammar *g, const uint8_t *in, uint64_t n, uint64_t window,
                          alpacc_lex_sink sink, void *user, uint64_t *num_tokens) {
  if (!g || !sink || (n > 0 && !in)) return ALPACC_E_INVALID;
  if (num_tokens) *num_tokens = 0;
  if (g->hg.parts == ALPACC_PARTS_PARSER) return ALPACC_E_INVALID;
  const alpacc_tables &tb = g->hg.t;
  if (tb.index_size < 8 && n > (1ull << 31) - 1) return ALPACC_E_CAPACITY;  // starts must fit index_t
  if (cudaSetDevice(g->device) != cudaSuccess) return ALPACC_E_CUDA;
  constexpr uint64_t kMaxWindow = (1ull << 31) - 1;  // the lexer kernels' 31-bit positions
  uint64_t w = window ? std::min(window, kMaxWindow) : (1ull << 30);
  uint64_t s = 0, total = 0;
  while (s < n) {
    const uint64_t e = n - s <= w ? n : s + w;
    const LexWindow win{e < n ? 1 : 0, s};
    int rc = grow(g->in, (e - s) + 16);
    if (rc) return rc;
    g->h_in = in + s;
    rc = run_device(g, (const uint8_t *)g->in.p, e - s, kRunLex, &win);
    g->h_in = nullptr;
    if (rc != ALPACC_OK) {
      cudaStreamSynchronize(g->cstream);  // no piece copy may still read the caller's buffer
      return rc;
    }
    const uint64_t T = g->last_T;
    const uint64_t lb = g->h_status->last_boundary;
    if (win.open_end && lb == 0) {  // one token spans the whole window: widen it and lex again
      if (w >= kMaxWindow) return ALPACC_E_CAPACITY;
      w = std::min(2 * w, kMaxWindow);
      continue;
    }
    if (T) {
      const size_t sz[3] = {T * tb.terminal_size, T * tb.index_size, T * tb.length_size};
      size_t off[3], bytes = sizeof(PinnedBlock);
      for (int i = 0; i < 3; i++) {
        off[i] = bytes;
        bytes += (sz[i] + 15) & ~(size_t)15;
      }
      PinnedBlock *b = acquire_block(g, &g->pinned_cache, &g->pinned_cache_size, bytes);
      if (!b) return ALPACC_E_NOMEM;
      const void *src[3] = {g->tok_ids.p, g->tok_starts.p, g->tok_lens.p};
      bool ok = true;
      for (int i = 0; i < 3 && ok; i++)
        ok = cudaMemcpyAsync((char *)b + off[i], src[i], sz[i], cudaMemcpyDeviceToHost, g->stream) == cudaSuccess;
      ok = ok && cudaStreamSynchronize(g->stream) == cudaSuccess;
      const int stop = ok ? sink(user, total, T, (char *)b + off[0], (char *)b + off[1], (char *)b + off[2]) : 0;
      release_block(g, b, false);
      if (!ok) return ALPACC_E_CUDA;
      if (stop) return ALPACC_E_ABORTED;
    }
    total += T;
    if (num_tokens) *num_tokens = total;
    if (!win.open_end) break;
    s += lb;
  }
  return ALPACC_OK;
}

int alpacc_gpu_parse_tokens(alpacc_gpu_grammar *g, const void *tokens, uint64_t n, alpacc_result *out) {
  if (!g || !out || (n > 0 && !tokens)) return ALPACC_E_INVALID;
  std::memset(out, 0, sizeof(*out));
  if (g->hg.parts == ALPACC_PARTS_LEXER) return ALPACC_E_INVALID;
  if (n > (1ull << 31) - 1) return ALPACC_E_CAPACITY;
  if (cudaSetDevice(g->device) != cudaSuccess) return ALPACC_E_CUDA;
  const alpacc_tables &tb = g->hg.t;
  int rc = grow(g->tok_ids, std::max<uint64_t>(n, 1) * tb.terminal_size);
  if (rc) return rc;
  if (n) CK(cudaMemcpyAsync(g->tok_ids.p, tokens, n * tb.terminal_size, cudaMemcpyHostToDevice, g->stream));
  rc = run_device(g, nullptr, n, kRunParse);
  g->last_status = rc;
  if (rc != ALPACC_OK) {
    cudaStreamSynchronize(g->stream);  // the token copy may still read the caller's buffer
    return rc;
  }
  const uint64_t P = g->last_N;
  const size_t bytes = P * tb.production_size;
  PinnedBlock *b = acquire_block(g, &g->pinned_cache, &g->pinned_cache_size, sizeof(PinnedBlock) + bytes);
  if (!b) return ALPACC_E_NOMEM;
  if (bytes && (cudaMemcpyAsync(b + 1, g->node_prods.p, bytes, cudaMemcpyDeviceToHost, g->stream) != cudaSuccess ||
                cudaStreamSynchronize(g->stream) != cudaSuccess)) {
    release_block(g, b, false);
    return ALPACC_E_CUDA;
  }
  out->valid = 1;
  out->num_nodes = P;
  out->node_productions = b + 1;
  out->internal = b;
  return ALPACC_OK;
}

}  // extern "C"

namespace {

// The lexer-mode record's lexemes (terminal_t, index_t, length_t each),
// interleaved in a bounded buffer and written in large pieces.
void write_lexemes(FILE *out, const alpacc_tables &tb, const alpacc_result &r) {
  const size_t tw = tb.terminal_size, iw = tb.index_size, lw = tb.length_size, rec = tw + iw + lw;
  const size_t per = 1 << 16;
  std::vector<uint8_t> buf(per * rec);
  for (uint64_t i0 = 0; i0 < r.num_tokens; i0 += per) {
    const uint64_t cnt = std::min<uint64_t>(per, r.num_tokens - i0);
    uint8_t *p = buf.data();
    for (uint64_t i = i0; i < i0 + cnt; i++) {
      std::memcpy(p, (const uint8_t *)r.token_ids + i * tw, tw);
      std::memcpy(p + tw, (const uint8_t *)r.token_starts + i * iw, iw);
      std::memcpy(p + tw + iw, (const uint8_t *)r.token_lengths + i * lw, lw);
      p += rec;
    }
    fwrite(buf.data(), rec, cnt, out);
  }
}

}  // namespace

extern "C" {

int alpacc_gpu_run_case(alpacc_gpu_grammar *g, uint64_t n, const uint8_t *in, FILE *out) {
  if (!g || !out) return ALPACC_E_INVALID;
  alpacc_result r;
  const int parts = g->hg.parts;
  int rc = parts == ALPACC_PARTS_LEXER    ? alpacc_gpu_lex(g, in, n, &r)
           : parts == ALPACC_PARTS_PARSER ? alpacc_gpu_parse_tokens(g, in, n, &r)
                                          : alpacc_gpu_parse(g, in, n, &r);
  if (rc == ALPACC_REJECT) {
    fputc(0, out);
    return rc;
  }
  if (rc != ALPACC_OK) return rc;
  const alpacc_tables &tb = g->hg.t;
  fputc(1, out);
  uint64_t T = r.num_tokens, N = r.num_nodes;
  if (parts == ALPACC_PARTS_LEXER) {  // C/Generator.hs:87-102
    fwrite(&T, 8, 1, out);
    write_lexemes(out, tb, r);
  } else if (parts == ALPACC_PARTS_PARSER) {  // C/Generator.hs:65-79
    fwrite(&N, 8, 1, out);
    fwrite(r.node_productions, tb.production_size, N, out);
  } else {  // C/Generator.hs:114-152
    fwrite(&T, 8, 1, out);
    fwrite(r.token_ids, tb.terminal_size, T, out);
    fwrite(r.token_starts, tb.index_size, T, out);
    fwrite(r.token_lengths, tb.length_size, T, out);
    fwrite(&N, 8, 1, out);
    fwrite(r.node_productions, tb.production_size, N, out);
    fwrite(r.node_parents, tb.index_size, N, out);
    fwrite(r.token_parents, tb.index_size, T, out);
  }
  alpacc_result_free(&r);
  return rc;
}

// print_layout of each mode (C/Generator.hs:80-84, 103-107, 153-158)
int alpacc_gpu_layout(const alpacc_gpu_grammar *g, char *buf, size_t len) {
  if (!g) return ALPACC_E_INVALID;
  const alpacc_tables &tb = g->hg.t;
  if (g->hg.parts == ALPACC_PARTS_LEXER)
    return snprintf(buf, len, "terminal_t=%u\nindex_t=%u\nlength_t=%u\n", tb.terminal_size, tb.index_size,
                    tb.length_size);
  if (g->hg.parts == ALPACC_PARTS_PARSER)
    return snprintf(buf, len, "terminal_t=%u\nproduction_t=%u\nindex_t=%u\n", tb.terminal_size,
                    tb.production_size, tb.index_size);
  return snprintf(buf, len, "terminal_t=%u\nproduction_t=%u\nindex_t=%u\nlength_t=%u\n", tb.terminal_size,
                  tb.production_size, tb.index_size, tb.length_size);
}

const char *alpacc_strerror(int status) {
  switch (status) {
    case ALPACC_OK: return "ok";
    case ALPACC_REJECT: return "input rejected";
    case ALPACC_E_INVALID: return "invalid argument or tables";
    case ALPACC_E_CUDA: return "CUDA error";
    case ALPACC_E_NOMEM: return "out of memory";
    case ALPACC_E_CAPACITY: return "input exceeds capacity";
    case ALPACC_E_TIMEOUT: return "device wait timed out";
    case ALPACC_E_UNSUPPORTED: return "tables exceed the supported limits";
    case ALPACC_E_ABORTED: return "stopped by the caller's callback";
  }
  return "unknown status";
}

double alpacc_gpu_last_ms(alpacc_gpu_grammar *g) { return g ? g->last_ms : -1.0; }

int alpacc_gpu_autotune(alpacc_gpu_grammar *g, const uint8_t *d_sample, uint64_t n, int *choice) {
  if (!g || (n > 0 && !d_sample) || g->hg.parts == ALPACC_PARTS_PARSER) return ALPACC_E_INVALID;
  const bool both = g->hg.parts == ALPACC_PARTS_BOTH;
  if (cudaSetDevice(g->device) != cudaSuccess) return ALPACC_E_CUDA;
  int lex_max = 0, pair_max = 0, pse_max = 0;
  const int sms = g->sms;
  if (lex_occupancy(g, &lex_max) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pair_max, pair_kernel, kPairThreads, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pse_max, pse_tile_kernel, kPseThreads, 0) != cudaSuccess ||
      lex_max < 1 || pair_max < 1 || pse_max < 1 || sms < 1) {
    cudaGetLastError();
    return ALPACC_E_CUDA;
  }
  // mean time of stages [k0, k1) over two runs after one warm-up, or < 0
  auto timed = [&](int mode, int k0, int k1) -> double {
    double ms = 0;
    for (int rep = 0; rep < 3; ++rep) {
      if (run_device(g, d_sample, n, mode) < 0) return -1.0;
      if (rep > 0)
        for (int k = k0; k < k1; ++k) ms += g->stage_ms[k];
    }
    return ms / 2;
  };
  Geometry geo{g->lex_win_words, g->lex_grid / sms, g->pair_grid / sms, g->pse_grid / sms};
  struct TimingOn {  // stage times while tuning; the caller's setting afterwards
    alpacc_gpu_grammar *g;
    int was;
    ~TimingOn() { g->stage_timing = was; }
  } timing_on{g, g->stage_timing};
  g->stage_timing = 1;
  double best = -1.0;
  // lexer: window length x resident CTAs per SM (fewer CTAs: less contention
  // for shared-memory banks and the look-back; more: more latency hidden)
  const int wins[3] = {4, 6, 8};
  for (int wi = 0; wi < 3; ++wi)
    for (int c = lex_max; c >= 1 && c >= lex_max - 2; --c) {
      Geometry t = geo;
      t.win_words = wins[wi];
      t.lex_per_sm = c;
      apply_geometry(g, t, sms);
      const double ms = timed(kRunLex, 0, 1);
      if (ms >= 0 && (best < 0 || ms < best)) {
        best = ms;
        geo.win_words = t.win_words;
        geo.lex_per_sm = c;
      }
    }
  if (best < 0) {
    apply_geometry(g, geo, sms);
    return ALPACC_E_CUDA;
  }
  if (both) {  // the pair kernel's and the walks' resident CTAs per SM
    best = -1.0;
    for (int c = pair_max; c >= 1 && c >= pair_max - 2; --c) {
      Geometry t = geo;
      t.pair_per_sm = c;
      apply_geometry(g, t, sms);
      const double ms = timed(kRunBoth, 1, 2);
      if (ms >= 0 && (best < 0 || ms < best)) {
        best = ms;
        geo.pair_per_sm = c;
      }
    }
    best = -1.0;
    for (int c = pse_max; c >= 1 && c >= pse_max - 2; --c) {
      Geometry t = geo;
      t.pse_per_sm = c;
      apply_geometry(g, t, sms);
      const double ms = timed(kRunBoth, 2, 6);
      if (ms >= 0 && (best < 0 || ms < best)) {
        best = ms;
        geo.pse_per_sm = c;
      }
    }
  }
  apply_geometry(g, geo, sms);
  {
    std::lock_guard<std::mutex> lock(g_geo_mu);
    g_geo_cache[{g->digest, g->device}] = geo;
  }
  g->geo_cached = 0;
  if (choice) *choice = geo.lex_per_sm;
  return ALPACC_OK;
}

int alpacc_gpu_geometry(const alpacc_gpu_grammar *g, int64_t *vals, int n) {
  if (!g || !vals || g->sms < 1) return ALPACC_E_INVALID;
  const int64_t v[6] = {4 * g->lex_win_words, g->lex_grid / g->sms, g->pair_grid / g->sms, g->pse_grid / g->sms,
                        g->geo_cached, (int64_t)g->digest};
  for (int i = 0; i < n && i < 6; i++) vals[i] = v[i];
  return 6;
}

void *alpacc_gpu_stream(alpacc_gpu_grammar *g) { return g ? (void *)g->stream : nullptr; }

// Diagnostics for tests: derived machine sizes and the last error text.
int alpacc_gpu_info(const alpacc_gpu_grammar *g, int64_t *vals, int nvals) {
  if (!g || !vals) return ALPACC_E_INVALID;
  const int64_t v[] = {g->hg.lex.M, g->hg.lex.C, g->hg.lex.max_lanes, g->hg.lex.reachable, g->hg.lex.dead,
                       g->hg.pairs.nt, (int64_t)g->hg.pairs.rec_ss.size(), g->lex_grid,
                       g->h_status ? g->h_status->lex_reject_reason : 0,
                       g->h_status ? g->h_status->parse_reject_reason : 0,
                       g->h_status ? g->h_status->timeout_site : 0, g->hg.pairs.hashed ? 1 : 0, g->lex_variant,
                       g->ps_sets};
  const int nv = (int)(sizeof(v) / sizeof(v[0]));
  for (int i = 0; i < nvals && i < nv; i++) vals[i] = v[i];
  return nv;
}

const char *alpacc_gpu_last_error(const alpacc_gpu_grammar *g) { return g ? g->last_error.c_str() : ""; }

uint64_t alpacc_device_allocations(void) { return alpacc::g_device_allocs.load(std::memory_order_relaxed); }

int alpacc_gpu_counts(const alpacc_gpu_grammar *g, int64_t *vals, int n) {
  if (!g || !vals || !g->h_status) return ALPACC_E_INVALID;
  int64_t v[9 + 24] = {(int64_t)g->h_status->num_tokens, (int64_t)g->h_status->num_brackets,
                       (int64_t)g->h_status->num_productions, (int64_t)g->h_status->num_nodes,
                       (int64_t)g->h_status->scratch[0], (int64_t)g->h_status->scratch[1],
                       (int64_t)g->h_status->scratch[2], (int64_t)g->h_status->scratch[3],
                       (int64_t)g->launches};
  for (int i = 0; i < 24; i++) v[9 + i] = (int64_t)g->phase_cycles[i];
  const int nv = (int)(sizeof v / sizeof v[0]);
  for (int i = 0; i < n && i < nv; i++) vals[i] = v[i];
  return nv;
}

void alpacc_gpu_set_diagnostics(alpacc_gpu_grammar *g, int on) {
  if (g) g->diag = on;
}

void alpacc_gpu_set_stage_timing(alpacc_gpu_grammar *g, int on) {
  if (g) g->stage_timing = on ? 1 : 0;
}

int alpacc_gpu_stage_ms(const alpacc_gpu_grammar *g, double *out, int n) {
  if (!g || !out) return ALPACC_E_INVALID;
  for (int k = 0; k < n && k < alpacc_gpu_grammar::kStages; k++) out[k] = g->stage_ms[k];
  return alpacc_gpu_grammar::kStages;
}

}  // extern "C"
