// The grammar handle behind the C ABI (shared by the .cu files of the library).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/alpacc_b200.h"
#include "common.cuh"
#include "device_tables.h"

#include <atomic>

namespace alpacc {

// Device allocations this library has made in the process (every cudaMalloc
// goes through dev_malloc); read by alpacc_device_allocations.
inline std::atomic<unsigned long long> g_device_allocs{0};

inline cudaError_t dev_malloc(void **p, size_t bytes) {
  g_device_allocs.fetch_add(1, std::memory_order_relaxed);
  return cudaMalloc(p, bytes);
}

struct DevBuf {
  void *p = nullptr;
  size_t cap = 0;
};

// Grow-only device buffer (contents are not preserved when it grows).
inline int grow(DevBuf &b, size_t bytes) {
  if (bytes <= b.cap && b.p) return ALPACC_OK;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  size_t want = std::max<size_t>(bytes, 256);
  if (dev_malloc(&b.p, want) != cudaSuccess) {
    cudaGetLastError();
    return ALPACC_E_NOMEM;
  }
  b.cap = want;
  return ALPACC_OK;
}

inline void release(DevBuf &b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}

template <typename T>
int upload(DevBuf &b, const std::vector<T> &v) {
  size_t bytes = std::max<size_t>(v.size() * sizeof(T), 16);
  int rc = grow(b, bytes);
  if (rc) return rc;
  if (!v.empty() && cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return ALPACC_E_CUDA;
  return ALPACC_OK;
}

}  // namespace alpacc

using alpacc::DevBuf;
using alpacc::DeviceStatus;
using alpacc::HostGrammar;

struct alpacc_gpu_grammar {
  int device = 0;
  HostGrammar hg;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  double last_ms = -1.0;
  // per-kernel timing: event pairs around each launch of the last call
  static constexpr int kStages = 8;
  cudaEvent_t sev[2 * kStages] = {};
  bool stage_used[kStages] = {};
  double stage_ms[kStages] = {};
  // tables
  DevBuf lex_tab, lex_cls4, lex_ps, lex_psmask, img, img_cnt, sterm, sflags;
  DevBuf dense, ht_key, ht_rec, rec, stacks, prods, arity, is_term;
  // lexer table shape (build_lexer_table): entries, rows of 1 << (cp_shift - 2),
  // column swizzle mask, u16 class table when classes exceed 64
  int tab_words = 0, cp_shift = 2, swz = 0, wide_cls = 0;
  // lexer kernel variant: 0 window machine, at most 64 states; 1 window
  // machine, more states; 2 windows walked as explicit state sets
  int lex_variant = 0;
  int ps_words = 0;        // window machine entries in shared memory (0: none)
  uint32_t ps_full = 0;
  int ps_sets = 0;
  int lex_win_words = 4;   // window before each chunk (words; 4..8)
  int lex_direct = 0;      // tokens written by the lexer kernel (look-back) instead of staged codes
  int stage_timing = 0;    // record per-stage events (alpacc_gpu_set_stage_timing)
  int walk_lookback = 1;   // walks find their tile prefixes by look-back (else walk_prefix_kernel)
  int sms = 0;             // SMs of the device
  uint64_t digest = 14695981039346656037ull;  // FNV-1a of the device tables (autotuner cache key)
  int geo_cached = 0;      // the launch geometry came from the autotuner's cache
  int lex_grid = 0;  // persistent grid of lex_kernel
  int pair_grid = 0, pse_grid = 0;  // resident CTAs of pair_kernel / pse_tile_kernel
  // parser-stage capacities: the largest exact needs seen (brackets, productions)
  uint64_t need_br = 0, need_pr = 0;
  int launches = 0;  // kernel launches of the last call
  int diag = 0;
  // status
  DeviceStatus *d_status = nullptr;
  DeviceStatus *h_status = nullptr;  // pinned
  DeviceStatus *h_lex_status = nullptr;  // pinned: the status after the lexer (host calls)
  cudaEvent_t lex_status_ev = nullptr;
  // scratch
  DevBuf in;                                   // device copy of host input
  DevBuf flags;                                // per-call flags, tickets, counters (zeroed each call)
  DevBuf diag_cycles;                          // diagnostics: lexer and walk phase cycles
  unsigned long long phase_cycles[24] = {};    // of the last call
  DevBuf lex_ticket, st1_flag, st1_state, st1_vec, st2_flags, st2_agg, st2_inc;
  DevBuf codes, tile_cnt, tile_pos, tile_off, tile_prev;  // staged lexer output
  DevBuf tok_ids, tok_starts, tok_lens;
  DevBuf pair_ticket, pst_flags, pst_agg, pst_inc, br, pr;
  DevBuf pse_ticket, pse_flags, pse_agg, pse_inc, tile_min, super_key;
  DevBuf pse_regions;  // per walk tile: staircase and queries (pse_region_bytes)
  DevBuf walk_prefix;  // per walk tile: depth prefixes of both walks, terminal-count prefix (i64)
  DevBuf node_prods, node_parents, token_parents;
  // batches: descriptor arrays, per-document statuses, packing ranges, packed results
  DevBuf b_arrays, b_desc, b_status, b_pack, b_packed;
  // pinned host result buffers kept for reuse (released results come back
  // here): the token arrays' block and the tree arrays' block
  std::mutex cache_mu;  // results may be released from other threads than the one parsing
  void *pinned_cache = nullptr;
  size_t pinned_cache_size = 0;
  void *pinned_cache2 = nullptr;
  size_t pinned_cache2_size = 0;
  // host-buffer calls (alpacc_gpu_parse): the input is copied in pieces on
  // cstream, each piece's lexer launch waits for its copy; the token arrays
  // are copied back on cstream while the parser runs
  cudaStream_t cstream = nullptr;
  static constexpr int kMaxPieces = 64;
  cudaEvent_t piece_ev[kMaxPieces] = {};
  cudaEvent_t lex_done = nullptr;
  const uint8_t *h_in = nullptr;  // host input of the current call, or null
  bool host_out = false;          // copy the tokens back as soon as they exist
  void *tok_block = nullptr;      // pinned block receiving the tokens of the current call
  size_t tok_off[3] = {};
  // last result (device)
  uint64_t last_T = 0, last_N = 0;
  int last_status = ALPACC_E_INVALID;
  std::string last_error;
};

// Header of a pinned host result block; the arrays follow it. A single
// document's result owns two blocks (the token arrays, copied while the parser
// runs, and the tree arrays in `second`); the results of a batch share one
// block, released when the last of them is (`refs`).
struct PinnedBlock {
  alpacc_gpu_grammar *owner;
  size_t size;
  PinnedBlock *second;
  int refs;
  int pad0;
  size_t pad[4];
};

// A pinned block of at least `total` bytes, from the handle's cache when it
// is large enough.
inline PinnedBlock *acquire_block(alpacc_gpu_grammar *g, void **cache, size_t *cache_size, size_t total) {
  void *host = nullptr;
  void *stale = nullptr;
  {
    std::lock_guard<std::mutex> lock(g->cache_mu);
    if (*cache && *cache_size >= total) host = *cache;
    else stale = *cache;
    *cache = nullptr;
  }
  if (!host) {
    if (stale) cudaFreeHost(stale);
    const size_t want = total + total / 8;
    if (cudaMallocHost(&host, want) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    reinterpret_cast<PinnedBlock *>(host)->size = want;
  }
  PinnedBlock *b = reinterpret_cast<PinnedBlock *>(host);
  b->owner = g;
  b->second = nullptr;
  b->refs = 1;
  return b;
}

inline void release_block(alpacc_gpu_grammar *g, PinnedBlock *b, bool tree) {
  if (!b) return;
  void **cache = tree ? &g->pinned_cache2 : &g->pinned_cache;
  size_t *size = tree ? &g->pinned_cache2_size : &g->pinned_cache_size;
  {
    std::lock_guard<std::mutex> lock(g->cache_mu);
    if (!*cache) {
      *cache = b;
      *size = b->size;
      return;
    }
  }
  cudaFreeHost(b);
}

// Dynamic shared memory of the lexer kernels for this handle's tables: the
// class table, the entries, the window machine's entries.
inline size_t lex_dyn_smem(const alpacc_gpu_grammar *g) {
  return (g->wide_cls ? 512 : 256) + (size_t)g->tab_words * 4 + (size_t)g->ps_words * 4;
}
