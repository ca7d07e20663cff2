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

int upload_tables(alpacc_gpu_grammar *g) {
  const LexerMachine &lm = g->hg.lex;
  if (lm.M > 128) return ALPACC_E_UNSUPPORTED;  // 7-bit states in the transition entries
  // transition entries at class * M + state: next state | produce(next) << 7
  const size_t mc = (size_t)lm.M * lm.C;
  std::vector<uint32_t> trw((mc + 3) / 4, 0);
  for (int c = 0; c < lm.C; c++)
    for (int m = 0; m < lm.M; m++) {
      const size_t i = (size_t)c * lm.M + m;
      const uint32_t nx = lm.trans[(size_t)m * lm.C + c];
      const uint32_t e = nx | ((lm.flags[nx] & 1u) << 7);
      trw[i >> 2] |= e << ((i & 3) * 8);
    }
  g->trans_word_count = (int)trw.size();
  // copies of the byte-class and transition tables in shared memory: more
  // copies mean fewer bank conflicts on data-dependent lookups, but fewer
  // resident CTAs; measured on json_ext, occupancy wins - keep a CTA's tables
  // within ~12 KB
  int copies = 32;
  while (copies > 1 && (size_t)copies * (trw.size() * 4 + 512) > 12 * 1024) copies >>= 1;
  if (const char *e = getenv("ALPACC_LEX_COPIES")) {
    int v = atoi(e);
    if (v >= 1 && v <= 32 && (v & (v - 1)) == 0) copies = v;
  }
  g->trans_rep = copies;
  TRY(upload(g->cls_id, lm.cls));
  TRY(upload(g->trans_words, trw));
  TRY(upload(g->lane_of, lm.lane_of));
  TRY(upload(g->img, lm.img));
  TRY(upload(g->img_cnt, lm.img_cnt));
  TRY(upload(g->sterm, lm.term));
  TRY(upload(g->sflags, lm.flags));
  const PairTable &pt = g->hg.pairs;
  TRY(upload(g->dense, pt.dense));
  TRY(upload(g->rec_ss, pt.rec_ss));
  TRY(upload(g->rec_ps, pt.rec_ps));
  TRY(upload(g->rec_nb, pt.rec_nb));
  TRY(upload(g->rec_np, pt.rec_np));
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

void stage_begin(alpacc_gpu_grammar *g, int k) {
  cudaEventRecord(g->sev[2 * k], g->stream);
  g->stage_used[k] = true;
}
void stage_end(alpacc_gpu_grammar *g, int k) { cudaEventRecord(g->sev[2 * k + 1], g->stream); }
void collect_stages(alpacc_gpu_grammar *g) {
  for (int k = 0; k < alpacc_gpu_grammar::kStages; k++) {
    float ms = 0;
    g->stage_ms[k] = (g->stage_used[k] && cudaEventElapsedTime(&ms, g->sev[2 * k], g->sev[2 * k + 1]) == cudaSuccess)
                         ? ms
                         : 0.0;
  }
}

size_t lex_smem_bytes(const alpacc_gpu_grammar *g) { return lex_dyn_smem(g); }

// The kernel attribute is per function, shared by every handle: only raise it.
int ensure_lex_smem(size_t bytes) {
  static std::mutex mu;
  static size_t current = 0;
  std::lock_guard<std::mutex> lock(mu);
  if (bytes <= current) return ALPACC_OK;
  if (cudaFuncSetAttribute(lex_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) {
    cudaGetLastError();
    return ALPACC_E_CUDA;
  }
  current = bytes;
  return ALPACC_OK;
}

// The whole device path for d_in[0..n). Leaves counts in g->last_T / last_N.
int run_device(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n) {
  const HostGrammar &hg = g->hg;
  const alpacc_tables &tb = hg.t;
  const LexerMachine &lm = hg.lex;
  const PairTable &pt = hg.pairs;
  const int term_w = (int)tb.terminal_size, idx_w = (int)tb.index_size, len_w = (int)tb.length_size;
  const int prod_w = (int)tb.production_size;
  if (n > (1ull << 31) - 1) return ALPACC_E_CAPACITY;
  CK(cudaMemsetAsync(g->d_status, 0, sizeof(DeviceStatus), g->stream));
  for (int k = 0; k < alpacc_gpu_grammar::kStages; k++) g->stage_used[k] = false;
  CK(cudaEventRecord(g->ev0, g->stream));

  // ---------------- lexer ----------------
  uint64_t T = 0;
  if (n > 0) {
    const uint64_t tiles = (n + kLexData - 1) / kLexData;
    TRY(grow(g->lex_ticket, 16));
    TRY(grow(g->st1_flag, tiles * 4));
    TRY(grow(g->st1_state, tiles));
    TRY(grow(g->st1_vec, tiles * (uint64_t)lm.M));
    TRY(grow(g->st2_flags, tiles * 4));
    TRY(grow(g->st2_agg, tiles * 16));
    TRY(grow(g->st2_inc, tiles * 16));
    TRY(grow(g->tok_ids, n * term_w));
    TRY(grow(g->tok_starts, n * idx_w));
    TRY(grow(g->tok_lens, n * len_w));
    CK(cudaMemsetAsync(g->lex_ticket.p, 0, 16, g->stream));
    CK(cudaMemsetAsync(g->st1_flag.p, 0, tiles * 4, g->stream));
    CK(cudaMemsetAsync(g->st2_flags.p, 0, tiles * 4, g->stream));
    LexArgs a{};
    a.in = d_in;
    a.n = n;
    a.num_tiles = tiles;
    a.cls_id = (const uint8_t *)g->cls_id.p;
    a.trans_words_ptr = (const uint32_t *)g->trans_words.p;
    a.trans_words = g->trans_word_count;
    a.copies = g->trans_rep;
    a.lane_of = (const uint8_t *)g->lane_of.p;
    a.img = (const uint8_t *)g->img.p;
    a.img_cnt = (const uint8_t *)g->img_cnt.p;
    a.sterm = (const uint8_t *)g->sterm.p;
    a.sflags = (const uint8_t *)g->sflags.p;
    a.M = lm.M;
    a.C = lm.C;
    a.dead = lm.dead;
    a.m0 = lm.m0;
    a.ignore = hg.ignore;
    a.len_max = hg.len_max;
    a.tok_ids = g->tok_ids.p;
    a.tok_starts = g->tok_starts.p;
    a.tok_lens = g->tok_lens.p;
    a.term_w = term_w;
    a.idx_w = idx_w;
    a.len_w = len_w;
    a.ticket = (unsigned *)g->lex_ticket.p;
    a.st1_flag = (unsigned *)g->st1_flag.p;
    a.st1_state = (uint8_t *)g->st1_state.p;
    a.st1_vec = (uint8_t *)g->st1_vec.p;
    a.st2 = PairTileState{(unsigned *)g->st2_flags.p, (unsigned long long *)g->st2_agg.p,
                          (unsigned long long *)g->st2_inc.p};
    a.status = g->d_status;
    a.diag = g->diag;
    stage_begin(g, 0);
    const unsigned grid = (unsigned)std::min<uint64_t>(tiles, (uint64_t)g->lex_grid);
    lex_kernel<<<grid, kLexThreads, lex_smem_bytes(g), g->stream>>>(a);
    stage_end(g, 0);
    CK(cudaGetLastError());
    int rc = sync_status(g);
    if (rc) return rc;
    if (g->h_status->reject) return ALPACC_REJECT;
    T = g->h_status->num_tokens;
  }

  // ---------------- pair lookup ----------------
  const uint64_t m = T + 2;
  const uint64_t br_cap = m * (uint64_t)std::max(pt.max_br, 1);
  const uint64_t pr_cap = m * (uint64_t)std::max(pt.max_pr, 1);
  {
    const uint64_t tiles = (m + kPairTile - 1) / kPairTile;
    TRY(grow(g->pair_ticket, 16));
    TRY(grow(g->pst_flags, tiles * 4));
    TRY(grow(g->pst_agg, tiles * 16));
    TRY(grow(g->pst_inc, tiles * 16));
    TRY(grow(g->br, br_cap * 4));
    TRY(grow(g->pr, pr_cap * 4));
    TRY(grow(g->tok_ids, std::max<uint64_t>(T, 1) * term_w));
    CK(cudaMemsetAsync(g->pair_ticket.p, 0, 16, g->stream));
    CK(cudaMemsetAsync(g->pst_flags.p, 0, tiles * 4, g->stream));
    if (n == 0) CK(cudaMemsetAsync(&g->d_status->num_tokens, 0, 8, g->stream));
    PairArgs a{};
    a.tok_ids = g->tok_ids.p;
    a.term_w = term_w;
    a.num_tokens = &g->d_status->num_tokens;
    a.num_tiles = tiles;
    a.q = pt.q;
    a.k = pt.k;
    a.nt = pt.nt;
    a.empty_t = (int)tb.empty_terminal;
    a.start_t = (int)tb.start_terminal;
    a.end_t = (int)tb.end_terminal;
    a.dense = (const uint32_t *)g->dense.p;
    a.rec_ss = (const uint32_t *)g->rec_ss.p;
    a.rec_ps = (const uint32_t *)g->rec_ps.p;
    a.rec_nb = (const uint8_t *)g->rec_nb.p;
    a.rec_np = (const uint8_t *)g->rec_np.p;
    a.stacks = (const uint32_t *)g->stacks.p;
    a.prods = (const uint32_t *)g->prods.p;
    a.br_out = (uint32_t *)g->br.p;
    a.pr_out = (uint32_t *)g->pr.p;
    a.br_cap = br_cap;
    a.pr_cap = pr_cap;
    a.ticket = (unsigned *)g->pair_ticket.p;
    a.st = PairTileState{(unsigned *)g->pst_flags.p, (unsigned long long *)g->pst_agg.p,
                         (unsigned long long *)g->pst_inc.p};
    a.status = g->d_status;
    stage_begin(g, 1);
    pair_kernel<<<(unsigned)tiles, kPairThreads, 0, g->stream>>>(a);
    stage_end(g, 1);
    CK(cudaGetLastError());
    int rc = sync_status(g);
    if (rc) return rc;
    if (g->h_status->reject) return ALPACC_REJECT;
  }
  const uint64_t B = g->h_status->num_brackets;
  const uint64_t P = g->h_status->num_productions;

  // ---------------- depth walks (the parent walk also writes the compacted tree) ----------------
  const uint64_t Emax = std::max<uint64_t>(std::max(B, P), 1);
  const uint64_t pse_tiles_max = (Emax + kPseTile - 1) / kPseTile;
  TRY(grow(g->pse_ticket, 16));
  TRY(grow(g->pse_flags, pse_tiles_max * 4));
  TRY(grow(g->pse_agg, pse_tiles_max * 16));
  TRY(grow(g->pse_inc, pse_tiles_max * 16));
  TRY(grow(g->ch_h0, pse_tiles_max * kPseThreads * 4));
  TRY(grow(g->ch_tc, pse_tiles_max * kPseThreads * 4));
  TRY(grow(g->tile_min, pse_tiles_max * 4));
  TRY(grow(g->chunk_min, pse_tiles_max * kPseThreads * 4));
  TRY(grow(g->super_min, ((pse_tiles_max >> kPseSuperShift) + 1) * 4));
  TRY(grow(g->queue, Emax * 8));
  TRY(grow(g->queue_len, 16));
  TRY(grow(g->node_prods, std::max<uint64_t>(P, 1) * prod_w));
  TRY(grow(g->node_parents, std::max<uint64_t>(P, 1) * idx_w));
  TRY(grow(g->token_parents, std::max<uint64_t>(T, 1) * idx_w));
  for (int mode = 0; mode < 2; ++mode) {
    const uint64_t E = mode == kPseBrackets ? B : P;
    if (E == 0) continue;
    const uint64_t tiles = (E + kPseTile - 1) / kPseTile;
    CK(cudaMemsetAsync(g->pse_ticket.p, 0, 16, g->stream));
    CK(cudaMemsetAsync(g->pse_flags.p, 0, tiles * 4, g->stream));
    CK(cudaMemsetAsync(g->queue_len.p, 0, 16, g->stream));
    CK(cudaMemsetAsync(g->super_min.p, 0x7f, ((tiles >> kPseSuperShift) + 1) * 4, g->stream));
    PseArgs a{};
    a.mode = mode;
    a.elems = (const uint32_t *)(mode == kPseBrackets ? g->br.p : g->pr.p);
    a.count = mode == kPseBrackets ? &g->d_status->num_brackets : &g->d_status->num_productions;
    a.num_tokens = &g->d_status->num_tokens;
    a.num_tiles = tiles;
    a.arity = (const int32_t *)g->arity.p;
    a.is_term = (const uint8_t *)g->is_term.p;
    a.ch_h0 = (int32_t *)g->ch_h0.p;
    a.ch_min = (int32_t *)g->chunk_min.p;
    a.ch_tc = (int32_t *)g->ch_tc.p;
    a.tile_min = (int32_t *)g->tile_min.p;
    a.super_min = (int32_t *)g->super_min.p;
    a.queue = (unsigned long long *)g->queue.p;
    a.queue_cap = Emax;
    a.queue_len = (unsigned long long *)g->queue_len.p;
    a.node_prods = g->node_prods.p;
    a.node_parents = g->node_parents.p;
    a.token_parents = g->token_parents.p;
    a.prod_w = prod_w;
    a.idx_w = idx_w;
    a.ticket = (unsigned *)g->pse_ticket.p;
    a.st = PairTileState{(unsigned *)g->pse_flags.p, (unsigned long long *)g->pse_agg.p,
                         (unsigned long long *)g->pse_inc.p};
    a.status = g->d_status;
    stage_begin(g, 2 + 2 * mode);
    pse_tile_kernel<<<(unsigned)tiles, kPseThreads, 0, g->stream>>>(a);
    stage_end(g, 2 + 2 * mode);
    CK(cudaGetLastError());
    stage_begin(g, 3 + 2 * mode);
    pse_resolve_kernel<<<148 * 4, 256, 0, g->stream>>>(a);
    stage_end(g, 3 + 2 * mode);
    CK(cudaGetLastError());
  }
  if (P == 0) CK(cudaMemsetAsync(&g->d_status->num_nodes, 0, 8, g->stream));
  CK(cudaEventRecord(g->ev1, g->stream));
  int rc = sync_status(g);
  if (rc) return rc;
  float ms = 0;
  if (cudaEventElapsedTime(&ms, g->ev0, g->ev1) == cudaSuccess) g->last_ms = ms;
  collect_stages(g);
  if (g->h_status->reject) return ALPACC_REJECT;
  if (P == 0 && T != 0) return ALPACC_REJECT;  // compact_tree: terminal count mismatch
  g->last_T = T;
  g->last_N = g->h_status->num_nodes;
  return ALPACC_OK;
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

// Header of a pinned host result block; the arrays follow it.
struct PinnedBlock {
  alpacc_gpu_grammar *owner;
  size_t size;
  size_t pad[6];
};

// Copy a device result to one pinned host block (reused across calls once the
// caller frees the previous result).
int copy_result_to_host(alpacc_gpu_grammar *g, alpacc_result *out) {
  const alpacc_tables &tb = g->hg.t;
  const uint64_t T = g->last_T, N = g->last_N;
  const size_t sz[6] = {T * tb.terminal_size, T * tb.index_size, T * tb.length_size,
                        N * tb.production_size, N * tb.index_size, T * tb.index_size};
  size_t off[6], total = sizeof(PinnedBlock);
  for (int i = 0; i < 6; i++) {
    off[i] = total;
    total += (sz[i] + 15) & ~(size_t)15;
  }
  void *host = nullptr;
  if (g->pinned_cache && g->pinned_cache_size >= total) {
    host = g->pinned_cache;
    g->pinned_cache = nullptr;
  } else {
    if (g->pinned_cache) cudaFreeHost(g->pinned_cache);
    g->pinned_cache = nullptr;
    size_t want = total + total / 8;
    if (cudaMallocHost(&host, want) != cudaSuccess) {
      cudaGetLastError();
      return ALPACC_E_NOMEM;
    }
    reinterpret_cast<PinnedBlock *>(host)->size = want;
  }
  reinterpret_cast<PinnedBlock *>(host)->owner = g;
  const void *src[6] = {g->tok_ids.p, g->tok_starts.p, g->tok_lens.p, g->node_prods.p, g->node_parents.p,
                        g->token_parents.p};
  for (int i = 0; i < 6; i++)
    if (sz[i]) CK(cudaMemcpyAsync((char *)host + off[i], src[i], sz[i], cudaMemcpyDeviceToHost, g->stream));
  CK(cudaStreamSynchronize(g->stream));
  std::memset(out, 0, sizeof(*out));
  out->valid = 1;
  out->num_tokens = T;
  out->num_nodes = N;
  out->token_ids = (char *)host + off[0];
  out->token_starts = (char *)host + off[1];
  out->token_lengths = (char *)host + off[2];
  out->node_productions = (char *)host + off[3];
  out->node_parents = (char *)host + off[4];
  out->token_parents = (char *)host + off[5];
  out->internal = host;
  return ALPACC_OK;
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
      cudaMalloc(&g->d_status, sizeof(DeviceStatus)) != cudaSuccess ||
      cudaMallocHost(&g->h_status, sizeof(DeviceStatus)) != cudaSuccess) {
    cudaGetLastError();
    *err = ALPACC_E_CUDA;
    alpacc_gpu_free(g);
    return nullptr;
  }
  std::memset(g->h_status, 0, sizeof(DeviceStatus));
  rc = upload_tables(g);
  if (rc == ALPACC_OK) rc = ensure_lex_smem(lex_smem_bytes(g));
  if (rc == ALPACC_OK) {
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lex_kernel, kLexThreads, lex_smem_bytes(g)) !=
            cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || per_sm < 1) {
      cudaGetLastError();
      rc = ALPACC_E_CUDA;
    } else {
      g->lex_grid = per_sm * sms;
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
  DevBuf *bufs[] = {&g->cls_id, &g->trans_words, &g->lane_of, &g->img, &g->img_cnt, &g->sterm, &g->sflags,
                    &g->dense, &g->rec_ss, &g->rec_ps, &g->rec_nb, &g->rec_np, &g->stacks, &g->prods,
                    &g->arity, &g->is_term, &g->in, &g->lex_ticket, &g->st1_flag, &g->st1_state, &g->st1_vec,
                    &g->st2_flags, &g->st2_agg, &g->st2_inc, &g->tok_ids, &g->tok_starts, &g->tok_lens,
                    &g->pair_ticket, &g->pst_flags, &g->pst_agg, &g->pst_inc, &g->br, &g->pr, &g->pse_ticket,
                    &g->pse_flags, &g->pse_agg, &g->pse_inc, &g->ch_h0, &g->ch_tc, &g->tile_min,
                    &g->chunk_min, &g->super_min, &g->queue, &g->queue_len, &g->node_prods, &g->node_parents,
                    &g->token_parents};
  for (DevBuf *b : bufs) release(*b);
  if (g->pinned_cache) cudaFreeHost(g->pinned_cache);
  if (g->d_status) cudaFree(g->d_status);
  if (g->h_status) cudaFreeHost(g->h_status);
  if (g->ev0) cudaEventDestroy(g->ev0);
  if (g->ev1) cudaEventDestroy(g->ev1);
  for (auto &e : g->sev)
    if (e) cudaEventDestroy(e);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

int alpacc_gpu_parse_device(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n, alpacc_result *out) {
  if (!g || !out || (n > 0 && !d_in)) return ALPACC_E_INVALID;
  if (cudaSetDevice(g->device) != cudaSuccess) return ALPACC_E_CUDA;
  int rc = run_device(g, d_in, n);
  g->last_status = rc;
  fill_device_result(g, out, rc);
  return rc;
}

int alpacc_gpu_enqueue(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n) {
  if (!g || (n > 0 && !d_in)) return ALPACC_E_INVALID;
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
  if (cudaSetDevice(g->device) != cudaSuccess) return ALPACC_E_CUDA;
  int rc = grow(g->in, n + 16);
  if (rc) return rc;
  if (n > 0 && cudaMemcpyAsync(g->in.p, in, n, cudaMemcpyHostToDevice, g->stream) != cudaSuccess)
    return ALPACC_E_CUDA;
  rc = run_device(g, (const uint8_t *)g->in.p, n);
  g->last_status = rc;
  if (rc != ALPACC_OK) return rc;
  return copy_result_to_host(g, out);
}

int alpacc_gpu_parse_batch(alpacc_gpu_grammar *g, const uint8_t *bytes, const int64_t *offsets, uint32_t count,
                           alpacc_result *outs) {
  if (!g || !offsets || !outs) return ALPACC_E_INVALID;
  for (uint32_t i = 0; i < count; i++) {
    const int64_t a = offsets[i], b = offsets[i + 1];
    if (b < a) return ALPACC_E_INVALID;
    int rc = alpacc_gpu_parse(g, bytes + a, (uint64_t)(b - a), &outs[i]);
    if (rc < 0) return rc;
    outs[i].valid = rc == ALPACC_OK ? 1 : 0;
  }
  return ALPACC_OK;
}

void alpacc_result_free(alpacc_result *r) {
  if (!r) return;
  if (r->internal) {
    PinnedBlock *b = reinterpret_cast<PinnedBlock *>(r->internal);
    alpacc_gpu_grammar *g = b->owner;
    if (g && !g->pinned_cache) {
      g->pinned_cache = b;
      g->pinned_cache_size = b->size;
    } else {
      cudaFreeHost(b);
    }
  }
  std::memset(r, 0, sizeof(*r));
}

int alpacc_gpu_run_case(alpacc_gpu_grammar *g, uint64_t n, const uint8_t *in, FILE *out) {
  alpacc_result r;
  int rc = alpacc_gpu_parse(g, in, n, &r);
  if (rc == ALPACC_REJECT) {
    fputc(0, out);
    return rc;
  }
  if (rc != ALPACC_OK) return rc;
  const alpacc_tables &tb = g->hg.t;
  fputc(1, out);
  uint64_t T = r.num_tokens, N = r.num_nodes;
  fwrite(&T, 8, 1, out);
  fwrite(r.token_ids, tb.terminal_size, T, out);
  fwrite(r.token_starts, tb.index_size, T, out);
  fwrite(r.token_lengths, tb.length_size, T, out);
  fwrite(&N, 8, 1, out);
  fwrite(r.node_productions, tb.production_size, N, out);
  fwrite(r.node_parents, tb.index_size, N, out);
  fwrite(r.token_parents, tb.index_size, T, out);
  alpacc_result_free(&r);
  return rc;
}

int alpacc_gpu_layout(const alpacc_gpu_grammar *g, char *buf, size_t len) {
  if (!g) return ALPACC_E_INVALID;
  const alpacc_tables &tb = g->hg.t;
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
  }
  return "unknown status";
}

double alpacc_gpu_last_ms(alpacc_gpu_grammar *g) { return g ? g->last_ms : -1.0; }

void *alpacc_gpu_stream(alpacc_gpu_grammar *g) { return g ? (void *)g->stream : nullptr; }

// Diagnostics for tests: derived machine sizes and the last error text.
int alpacc_gpu_info(const alpacc_gpu_grammar *g, int64_t *vals, int nvals) {
  if (!g || !vals) return ALPACC_E_INVALID;
  const int64_t v[] = {g->hg.lex.M, g->hg.lex.C, g->hg.lex.max_lanes, g->hg.lex.reachable, g->hg.lex.dead,
                       g->hg.pairs.nt, (int64_t)g->hg.pairs.rec_ss.size(), g->trans_rep,
                       g->h_status ? g->h_status->lex_reject_reason : 0,
                       g->h_status ? g->h_status->parse_reject_reason : 0,
                       g->h_status ? g->h_status->timeout_site : 0};
  const int nv = (int)(sizeof(v) / sizeof(v[0]));
  for (int i = 0; i < nvals && i < nv; i++) vals[i] = v[i];
  return nv;
}

const char *alpacc_gpu_last_error(const alpacc_gpu_grammar *g) { return g ? g->last_error.c_str() : ""; }

int alpacc_gpu_counts(const alpacc_gpu_grammar *g, int64_t *vals, int n) {
  if (!g || !vals || !g->h_status) return ALPACC_E_INVALID;
  const int64_t v[8] = {(int64_t)g->h_status->num_tokens, (int64_t)g->h_status->num_brackets,
                        (int64_t)g->h_status->num_productions, (int64_t)g->h_status->num_nodes,
                        (int64_t)g->h_status->scratch[0], (int64_t)g->h_status->scratch[1],
                        (int64_t)g->h_status->scratch[2], (int64_t)g->h_status->scratch[3]};
  for (int i = 0; i < n && i < 8; i++) vals[i] = v[i];
  return 8;
}

void alpacc_gpu_set_diagnostics(alpacc_gpu_grammar *g, int on) {
  if (g) g->diag = on;
}

int alpacc_gpu_stage_ms(const alpacc_gpu_grammar *g, double *out, int n) {
  if (!g || !out) return ALPACC_E_INVALID;
  for (int k = 0; k < n && k < alpacc_gpu_grammar::kStages; k++) out[k] = g->stage_ms[k];
  return alpacc_gpu_grammar::kStages;
}

}  // extern "C"
