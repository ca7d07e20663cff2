// Many independent documents through one launch per stage
// (alpacc_gpu_parse_batch).
//
// The reference parses one input per run_case call (C/Generator.hs:114-152);
// its CUDA backend sets up and launches per input (backends/cuda/cli.cu:739-792).
// Here a batch is laid out as per-document regions of the same scratch arrays
// the single-document path uses, every stage is launched once for all
// documents (kernels map virtual tiles to (document, local tile), see
// BatchDesc), the tile counts of the parser stages are planned on the device
// from the counts the previous stage left in each document's status, and the
// host synchronises once to read the statuses and once for the packed
// results. Each document's result is bit-identical to parsing it alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/alpacc_b200.h"
#include "handle.h"
#include "kernels.h"
#include "pipeline.h"
#include "scratch.h"

using namespace alpacc;

namespace {

#define BCK(x)                                \
  do {                                        \
    cudaError_t e_ = (x);                     \
    if (e_ != cudaSuccess) {                  \
      g->last_error = cudaGetErrorString(e_); \
      return ALPACC_E_CUDA;                   \
    }                                         \
  } while (0)

#define BTRY(x)                     \
  do {                              \
    int r_ = (x);                   \
    if (r_ != ALPACC_OK) return r_; \
  } while (0)

// Byte ranges (src offset, dst offset, length) copied by one CTA each.
__global__ void pack_ranges_kernel(const uint8_t *src, uint8_t *dst, const unsigned long long *r, int count) {
  for (int i = blockIdx.x; i < count; i += gridDim.x) {
    const unsigned long long so = r[3 * i], dof = r[3 * i + 1], len = r[3 * i + 2];
    for (unsigned long long k = threadIdx.x; k < len; k += blockDim.x) dst[dof + k] = src[so + k];
  }
}


}  // namespace

namespace alpacc {

void BatchSizes::add(const alpacc_gpu_grammar *g, uint64_t n) {
  const uint64_t max_br = (uint64_t)std::max(g->hg.pairs.max_br, 1), max_pr = (uint64_t)std::max(g->hg.pairs.max_pr, 1);
  docs += 1;
  bytes += n;
  tokens += n + 1;
  brackets += (n + 3) * max_br;
  productions += (n + 3) * max_pr;
  lex_tiles += (n + kLexData - 1) / kLexData;
  pair_tiles += (n + 3 + kPairTile - 1) / kPairTile;
  br_tiles += ((n + 3) * max_br + kPseTile - 1) / kPseTile;
  pr_tiles += ((n + 3) * max_pr + kPseTile - 1) / kPseTile;
}

int batch_needs(alpacc_gpu_grammar *g, const BatchSizes &z, BufNeed *out) {
  const alpacc_tables &tb = g->hg.t;
  const uint64_t D = z.docs, lt = std::max<uint64_t>(z.lex_tiles, 1);
  const uint64_t walk = std::max<uint64_t>(std::max(z.br_tiles, z.pr_tiles), 1);
  const uint64_t words = 2 * D + 7 * (D + 1);
  const uint64_t T = z.tokens, B = z.brackets, P = z.productions;
  const uint64_t tw = tb.terminal_size, iw = tb.index_size, lw = tb.length_size, pw = tb.production_size;
  const BufNeed v[] = {
      {&g->b_arrays, words * 8}, {&g->b_desc, sizeof(BatchDesc)}, {&g->b_status, D * sizeof(DeviceStatus)},
      {&g->in, z.bytes + 16}, {&g->lex_ticket, 16}, {&g->st1_flag, lt * 4}, {&g->st1_state, lt},
      {&g->st1_vec, lt * (uint64_t)g->hg.lex.M}, {&g->st2_flags, lt * 4}, {&g->codes, lt * (uint64_t)kLexData},
      {&g->tile_cnt, lt * 4}, {&g->tile_pos, lt * 4}, {&g->tile_off, lt * 8}, {&g->tile_prev, lt * 4},
      {&g->st2_agg, lt * 16}, {&g->st2_inc, lt * 16}, {&g->tok_ids, T * tw}, {&g->tok_starts, T * iw},
      {&g->tok_lens, T * lw}, {&g->pair_ticket, 16}, {&g->pst_flags, z.pair_tiles * 4},
      {&g->pst_agg, z.pair_tiles * 16}, {&g->pst_inc, z.pair_tiles * 16}, {&g->br, B * 4}, {&g->pr, P * 4},
      {&g->pse_ticket, 16}, {&g->pse_flags, walk * 4}, {&g->pse_agg, walk * 16}, {&g->pse_inc, walk * 16},
      {&g->tile_min, walk * 4}, {&g->super_key, ((walk >> kPseSuperShift) + 1) * 4},
      {&g->pse_regions, pse_region_bytes(walk)}, {&g->node_prods, P * pw}, {&g->node_parents, P * iw},
      {&g->token_parents, T * iw},
      // result packing: at most 6 ranges per document and every array packed
      {&g->b_pack, std::max<uint64_t>(18 * D, 3) * 8},
      {&g->b_packed, T * (tw + iw + lw + iw) + P * (pw + iw) + 6 * 16}};
  constexpr int k = (int)(sizeof v / sizeof v[0]);
  static_assert(k <= kBatchBufs, "batch buffer list");
  for (int i = 0; i < k; i++) out[i] = BufNeed{v[i].buf, std::max<uint64_t>(v[i].bytes, 256)};
  return k;
}

uint64_t batch_scratch_bytes(alpacc_gpu_grammar *g, const BatchSizes &z) {
  BufNeed need[kBatchBufs];
  const int k = batch_needs(g, z, need);
  uint64_t sum = 0;
  for (int i = 0; i < k; i++) sum += need[i].bytes;
  return sum;
}

uint64_t fit_batch_scratch(alpacc_gpu_grammar *g, const BatchSizes &z, uint64_t budget) {
  BufNeed need[kBatchBufs];
  const int k = batch_needs(g, z, need);
  uint64_t held = 0;
  for (int i = 0; i < k; i++) held += std::max<uint64_t>(need[i].buf->cap, need[i].bytes);
  if (held > budget) {
    held = 0;
    for (int i = 0; i < k; i++) {
      if (need[i].buf->cap > need[i].bytes) {
        if (g->stream) cudaStreamSynchronize(g->stream);
        release(*need[i].buf);
      }
      held += need[i].bytes;
    }
  }
  return held;
}

uint64_t batch_scratch_held(alpacc_gpu_grammar *g) {
  BufNeed need[kBatchBufs];
  const int k = batch_needs(g, BatchSizes{}, need);
  uint64_t held = 0;
  for (int i = 0; i < k; i++) held += need[i].buf->cap;
  return held;
}

}  // namespace alpacc

namespace {

int run_batch(alpacc_gpu_grammar *g, const uint8_t *bytes, const int64_t *offsets, uint32_t count,
              alpacc_result *outs) {
  const HostGrammar &hg = g->hg;
  const alpacc_tables &tb = hg.t;
  const PairTable &pt = hg.pairs;
  const int D = (int)count;
  const uint64_t base = (uint64_t)offsets[0];
  const uint64_t total = (uint64_t)offsets[count] - base;
  const uint64_t max_br = (uint64_t)std::max(pt.max_br, 1), max_pr = (uint64_t)std::max(pt.max_pr, 1);

  // ---- per-document regions and tile ranges (host) ----
  // device layout of the u64 arrays: in_off[D] n[D] tok_off[D+1] br_off[D+1]
  // pr_off[D+1] lex_tile0[D+1] pair_tile0[D+1] br_tile0[D+1] pr_tile0[D+1]
  const size_t words = 2 * (size_t)D + 7 * ((size_t)D + 1);
  std::vector<unsigned long long> h(words, 0);
  unsigned long long *in_off = h.data(), *nd = in_off + D, *tok_off = nd + D, *br_off = tok_off + D + 1,
                     *pr_off = br_off + D + 1, *lex_tile0 = pr_off + D + 1;
  BatchSizes z;
  for (int d = 0; d < D; d++) {
    const uint64_t n = (uint64_t)(offsets[d + 1] - offsets[d]);
    in_off[d] = (uint64_t)offsets[d] - base;
    nd[d] = n;
    tok_off[d + 1] = tok_off[d] + n + 1;
    br_off[d + 1] = br_off[d] + (n + 3) * max_br;
    pr_off[d + 1] = pr_off[d] + (n + 3) * max_pr;
    lex_tile0[d + 1] = lex_tile0[d] + (n + kLexData - 1) / kLexData;
    z.add(g, n);
  }
  const uint64_t lex_tiles = lex_tile0[D];
  const uint64_t pair_ub = z.pair_tiles, br_ub = z.br_tiles, pr_ub = z.pr_tiles;
  const uint64_t walk_ub = std::max<uint64_t>(std::max(br_ub, pr_ub), 1);
  const int term_w = (int)tb.terminal_size, idx_w = (int)tb.index_size, len_w = (int)tb.length_size;
  const int prod_w = (int)tb.production_size;

  // ---- device buffers (exactly batch_needs: the server admits by it) ----
  {
    BufNeed need[kBatchBufs];
    const int k = batch_needs(g, z, need);
    for (int i = 0; i < k; i++)
      if (need[i].buf != &g->b_pack && need[i].buf != &g->b_packed) BTRY(grow(*need[i].buf, need[i].bytes));
  }

  unsigned long long *da = (unsigned long long *)g->b_arrays.p;
  BatchDesc bd{};
  bd.docs = D;
  bd.in_off = da;
  bd.n = da + D;
  bd.tok_off = da + 2 * D;
  bd.br_off = bd.tok_off + D + 1;
  bd.pr_off = bd.br_off + D + 1;
  bd.lex_tile0 = bd.pr_off + D + 1;
  bd.pair_tile0 = const_cast<unsigned long long *>(bd.lex_tile0) + D + 1;
  bd.br_tile0 = bd.pair_tile0 + D + 1;
  bd.pr_tile0 = bd.br_tile0 + D + 1;
  bd.status = (DeviceStatus *)g->b_status.p;
  const BatchDesc *d_bd = (const BatchDesc *)g->b_desc.p;
  cudaStream_t s = g->stream;
  BCK(cudaMemcpyAsync(g->b_arrays.p, h.data(), (2 * (size_t)D + 4 * ((size_t)D + 1)) * 8, cudaMemcpyHostToDevice, s));
  BCK(cudaMemcpyAsync(g->b_desc.p, &bd, sizeof bd, cudaMemcpyHostToDevice, s));
  BCK(cudaMemsetAsync(g->b_status.p, 0, (size_t)D * sizeof(DeviceStatus), s));
  if (total) BCK(cudaMemcpyAsync(g->in.p, bytes + base, total, cudaMemcpyHostToDevice, s));
  BCK(cudaMemsetAsync(g->lex_ticket.p, 0, 16, s));
  BCK(cudaMemsetAsync(g->st1_flag.p, 0, std::max<uint64_t>(lex_tiles, 1) * 4, s));
  BCK(cudaMemsetAsync(g->st2_flags.p, 0, std::max<uint64_t>(lex_tiles, 1) * 4, s));
  BCK(cudaMemsetAsync(g->pair_ticket.p, 0, 16, s));
  BCK(cudaMemsetAsync(g->pst_flags.p, 0, pair_ub * 4, s));
  g->launches = 0;

  // ---- lexer: one launch over every document's tiles ----
  if (lex_tiles) {
    LexArgs a = lex_args(g, (const uint8_t *)g->in.p, total, lex_tiles);
    a.batch = d_bd;
    a.status = bd.status;
    BCK(launch_lex(g, a, (unsigned)std::min<uint64_t>(lex_tiles, (uint64_t)g->lex_grid), s));
    BCK(launch_lex_emit(lex_emit_args(g, a), s));
    g->launches += 3;
  }
  // ---- pairs ----
  batch_plan_kernel<<<1, 1024, 0, s>>>(bd, kPlanPairs, bd.pair_tile0, kPairTile);
  {
    PairArgs pa = pair_args(g);
    pa.batch = d_bd;
    pa.status = bd.status;
    pair_kernel<<<(unsigned)std::min<uint64_t>(pair_ub, (uint64_t)g->pair_grid), kPairThreads, 0, s>>>(pa);
  }
  batch_plan_kernel<<<1, 1024, 0, s>>>(bd, kPlanBrackets, bd.br_tile0, kPseTile);
  batch_plan_kernel<<<1, 1024, 0, s>>>(bd, kPlanParents, bd.pr_tile0, kPseTile);
  g->launches += 4;
  BCK(cudaGetLastError());
  // ---- depth walks ----
  for (int mode = 0; mode < 2; ++mode) {
    const uint64_t ub = mode == kPseBrackets ? br_ub : pr_ub;
    if (!ub) continue;
    BCK(cudaMemsetAsync(g->pse_ticket.p, 0, 16, s));
    BCK(cudaMemsetAsync(g->pse_flags.p, 0, ub * 4, s));
    BCK(cudaMemsetAsync(g->super_key.p, 0, ((ub >> kPseSuperShift) + 1) * 4, s));
    PseArgs pa = pse_args(g, mode, walk_ub);
    pa.batch = d_bd;
    pa.status = bd.status;
    pse_tile_kernel<<<(unsigned)std::min<uint64_t>(ub, (uint64_t)g->pse_grid), kPseThreads, 0, s>>>(pa);
    pse_resolve_kernel<<<resolve_blocks(ub), 256, 0, s>>>(pa);
    g->launches += 2;
    BCK(cudaGetLastError());
  }
  std::vector<DeviceStatus> st(D);
  BCK(cudaMemcpyAsync(st.data(), g->b_status.p, (size_t)D * sizeof(DeviceStatus), cudaMemcpyDeviceToHost, s));
  BCK(cudaStreamSynchronize(s));

  // ---- statuses, packed results ----
  std::vector<char> valid(D, 0);
  std::vector<uint64_t> T(D, 0), N(D, 0);
  uint64_t Tt = 0, Nt = 0;
  for (int d = 0; d < D; d++) {
    if (st[d].error != 0 || st[d].overflow) {  // the regions are upper bounds: an overflow is an internal error
      g->last_error = "batch document failed";
      return st[d].error != 0 ? st[d].error : ALPACC_E_CAPACITY;
    }
    const uint64_t P = st[d].num_productions;
    T[d] = st[d].num_tokens;
    N[d] = st[d].num_nodes;
    valid[d] = !st[d].reject && !(P == 0 && T[d] != 0);  // compact_tree: terminal count mismatch
    if (valid[d]) {
      Tt += T[d];
      Nt += N[d];
    }
  }
  struct Arr {
    const DevBuf *buf;
    int w;
    const unsigned long long *reg;  // region offsets (elements)
    bool tokens;                    // counted by T (else N)
  };
  const Arr arrs[6] = {{&g->tok_ids, term_w, tok_off, true},        {&g->tok_starts, idx_w, tok_off, true},
                       {&g->tok_lens, len_w, tok_off, true},        {&g->node_prods, prod_w, pr_off, false},
                       {&g->node_parents, idx_w, pr_off, false},    {&g->token_parents, idx_w, tok_off, true}};
  size_t sec[6], packed = 0;
  for (int i = 0; i < 6; i++) {
    sec[i] = packed;
    packed += ((arrs[i].tokens ? Tt : Nt) * (uint64_t)arrs[i].w + 15) & ~(uint64_t)15;
  }
  std::vector<unsigned long long> ranges;
  ranges.reserve((size_t)D * 18);
  int nr[6];
  for (int i = 0; i < 6; i++) {
    nr[i] = 0;
    uint64_t o = 0;
    for (int d = 0; d < D; d++) {
      if (!valid[d]) continue;
      const uint64_t c = arrs[i].tokens ? T[d] : N[d];
      ranges.push_back(arrs[i].reg[d] * (uint64_t)arrs[i].w);
      ranges.push_back(sec[i] + o * (uint64_t)arrs[i].w);
      ranges.push_back(c * (uint64_t)arrs[i].w);
      o += c;
      nr[i]++;
    }
  }
  BTRY(grow(g->b_pack, std::max<size_t>(ranges.size(), 3) * 8));
  BTRY(grow(g->b_packed, std::max<size_t>(packed, 16)));
  if (!ranges.empty())
    BCK(cudaMemcpyAsync(g->b_pack.p, ranges.data(), ranges.size() * 8, cudaMemcpyHostToDevice, s));
  size_t r0 = 0;
  for (int i = 0; i < 6; i++) {
    if (nr[i]) {
      pack_ranges_kernel<<<std::min(nr[i], 148 * 8), 256, 0, s>>>((const uint8_t *)arrs[i].buf->p,
                                                                  (uint8_t *)g->b_packed.p,
                                                                  (const unsigned long long *)g->b_pack.p + 3 * r0, nr[i]);
      ++g->launches;
    }
    r0 += nr[i];
  }
  BCK(cudaGetLastError());
  int nvalid = 0;
  for (int d = 0; d < D; d++) nvalid += valid[d];
  PinnedBlock *blk = nullptr;
  if (nvalid) {
    blk = acquire_block(g, &g->pinned_cache, &g->pinned_cache_size, sizeof(PinnedBlock) + packed);
    if (!blk) return ALPACC_E_NOMEM;
    if (packed)
      BCK(cudaMemcpyAsync((char *)blk + sizeof(PinnedBlock), g->b_packed.p, packed, cudaMemcpyDeviceToHost, s));
    BCK(cudaStreamSynchronize(s));
    blk->refs = nvalid;
  }
  uint64_t to = 0, no = 0;
  char *hb = blk ? (char *)blk + sizeof(PinnedBlock) : nullptr;
  for (int d = 0; d < D; d++) {
    alpacc_result &r = outs[d];
    std::memset(&r, 0, sizeof r);
    if (!valid[d]) continue;
    r.valid = 1;
    r.num_tokens = T[d];
    r.num_nodes = N[d];
    r.token_ids = hb + sec[0] + to * term_w;
    r.token_starts = hb + sec[1] + to * idx_w;
    r.token_lengths = hb + sec[2] + to * len_w;
    r.node_productions = hb + sec[3] + no * prod_w;
    r.node_parents = hb + sec[4] + no * idx_w;
    r.token_parents = hb + sec[5] + to * idx_w;
    r.internal = blk;
    to += T[d];
    no += N[d];
  }
  return ALPACC_OK;
}

}  // namespace

extern "C" int alpacc_gpu_parse_batch(alpacc_gpu_grammar *g, const uint8_t *bytes, const int64_t *offsets,
                                      uint32_t count, alpacc_result *outs) {
  if (!g || !offsets || (count && !outs)) return ALPACC_E_INVALID;
  if (g->hg.parts != ALPACC_PARTS_BOTH) return ALPACC_E_INVALID;  // the batch path is the combined one
  for (uint32_t i = 0; i < count; i++) {
    if (offsets[i + 1] < offsets[i] || offsets[i + 1] - offsets[i] > (int64_t)(1ll << 31) - 1)
      return ALPACC_E_INVALID;
    std::memset(&outs[i], 0, sizeof outs[i]);
  }
  if (count == 0) return ALPACC_OK;
  if (offsets[count] > offsets[0] && !bytes) return ALPACC_E_INVALID;
  if (cudaSetDevice(g->device) != cudaSuccess) return ALPACC_E_CUDA;
  return run_batch(g, bytes, offsets, count, outs);
}
