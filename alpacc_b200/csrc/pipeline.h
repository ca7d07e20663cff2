// Kernel argument blocks filled from a grammar handle's tables and scratch
// buffers, shared by the single-document path (api.cu) and the batch path
// (batch.cu). The caller grows the scratch buffers first and then sets the
// per-call fields (sizes, tickets, capacities, batch descriptor).
#pragma once

#include <algorithm>

#include "handle.h"
#include "kernels.h"

namespace alpacc {

inline LexArgs lex_args(alpacc_gpu_grammar *g, const uint8_t *d_in, uint64_t n, uint64_t tiles) {
  const HostGrammar &hg = g->hg;
  const LexerMachine &lm = hg.lex;
  LexArgs a{};
  a.in = d_in;
  a.n = n;
  a.num_tiles = tiles;
  a.tab = (const uint32_t *)g->lex_tab.p;
  a.tab_words = g->tab_words;
  a.cls4 = (const uint8_t *)g->lex_cls4.p;
  a.wide_cls = g->wide_cls;
  a.cp_shift = g->cp_shift;
  a.swz = g->swz;
  a.ps_tab = g->ps_words ? (const uint32_t *)g->lex_ps.p : nullptr;
  a.ps_words = g->ps_words;
  a.ps_full = g->ps_full;
  a.ps_mask = (const unsigned long long *)g->lex_psmask.p;
  a.win_words = g->lex_win_words;
  a.img = (const uint8_t *)g->img.p;
  a.img_cnt = (const uint8_t *)g->img_cnt.p;
  a.sterm = (const uint8_t *)g->sterm.p;
  a.sflags = (const uint8_t *)g->sflags.p;
  a.M = lm.M;
  a.C = lm.C;
  a.dead = lm.dead;
  a.m0 = lm.m0;
  a.len_max = hg.len_max;
  a.tok_ids = g->tok_ids.p;
  a.tok_starts = g->tok_starts.p;
  a.tok_lens = g->tok_lens.p;
  a.term_w = (int)hg.t.terminal_size;
  a.idx_w = (int)hg.t.index_size;
  a.len_w = (int)hg.t.length_size;
  a.ticket = (unsigned *)g->lex_ticket.p;
  a.st1_flag = (unsigned *)g->st1_flag.p;
  a.st1_state = (uint8_t *)g->st1_state.p;
  a.st1_vec = (uint8_t *)g->st1_vec.p;
  a.st2 = PairTileState{(unsigned *)g->st2_flags.p, (unsigned long long *)g->st2_agg.p,
                        (unsigned long long *)g->st2_inc.p};
  a.status = g->d_status;
  a.diag = g->diag;
  a.codes = (uint8_t *)g->codes.p;
  a.tile_cnt = (uint32_t *)g->tile_cnt.p;
  a.tile_pos = (uint32_t *)g->tile_pos.p;
  return a;
}

// The lexer kernels by variant (alpacc_gpu_grammar::lex_variant).
using LexKernel = void (*)(LexArgs);
inline LexKernel lex_staged_kernel(const alpacc_gpu_grammar *g) {
  static const LexKernel k[3] = {lex_kernel, lex_kernel_wide, lex_kernel_sets};
  return k[g->lex_variant];
}
inline LexKernel lex_direct_kernel_of(const alpacc_gpu_grammar *g) {
  static const LexKernel k[3] = {lex_direct_kernel, lex_direct_kernel_wide, lex_direct_kernel_sets};
  return k[g->lex_variant];
}

// The staged lexer kernel for this handle's machine (codes and tile totals).
inline cudaError_t launch_lex(const alpacc_gpu_grammar *g, const LexArgs &a, unsigned grid, cudaStream_t s) {
  lex_staged_kernel(g)<<<grid, kLexThreads, lex_dyn_smem(g), s>>>(a);
  return cudaGetLastError();
}

// The direct lexer kernel (tokens written by the kernel itself).
inline cudaError_t launch_lex_direct(const alpacc_gpu_grammar *g, const LexArgs &a, unsigned grid, cudaStream_t s) {
  lex_direct_kernel_of(g)<<<grid, kLexThreads, lex_dyn_smem(g), s>>>(a);
  return cudaGetLastError();
}

// Arguments of the scan and emit kernels of the staged lexer.
inline LexEmitArgs lex_emit_args(const alpacc_gpu_grammar *g, const LexArgs &a) {
  LexEmitArgs e{};
  e.codes = a.codes;
  e.n = a.n;
  e.num_tiles = a.num_tiles;
  e.tile_cnt = a.tile_cnt;
  e.tile_pos = a.tile_pos;
  e.tile_off = (unsigned long long *)g->tile_off.p;
  e.tile_prev = (uint32_t *)g->tile_prev.p;
  e.tok_ids = a.tok_ids;
  e.tok_starts = a.tok_starts;
  e.tok_lens = a.tok_lens;
  e.term_w = a.term_w;
  e.idx_w = a.idx_w;
  e.len_w = a.len_w;
  e.len_max = a.len_max;
  e.index_base = a.index_base;
  e.open_end = a.open_end;
  e.status = a.status;
  e.batch = a.batch;
  return e;
}

// The scan and emit kernels after the staged lexer's launches.
inline cudaError_t launch_lex_emit(const LexEmitArgs &e, cudaStream_t s) {
  lex_scan_kernel<<<1, kLexScanThreads, 0, s>>>(e);
  lex_emit_kernel<<<(unsigned)std::min<unsigned long long>(e.num_tiles, 148ull * 4), 256, kLexEmitSmem, s>>>(e);
  return cudaGetLastError();
}

// Resident CTAs of the staged lexer kernel per SM.
inline cudaError_t lex_occupancy(const alpacc_gpu_grammar *g, int *per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, lex_staged_kernel(g), kLexThreads, lex_dyn_smem(g));
}

inline PairArgs pair_args(alpacc_gpu_grammar *g) {
  const alpacc_tables &tb = g->hg.t;
  const PairTable &pt = g->hg.pairs;
  PairArgs a{};
  a.tok_ids = g->tok_ids.p;
  a.term_w = (int)tb.terminal_size;
  a.num_tokens = &g->d_status->num_tokens;
  a.q = pt.q;
  a.k = pt.k;
  a.nt = pt.nt;
  a.empty_t = (int)tb.empty_terminal;
  a.start_t = (int)tb.start_terminal;
  a.end_t = (int)tb.end_terminal;
  a.dense = pt.hashed ? nullptr : (const uint32_t *)g->dense.p;
  a.ht_key = (const unsigned long long *)g->ht_key.p;
  a.ht_rec = (const uint32_t *)g->ht_rec.p;
  a.ht_size = pt.ht_key.size();
  a.max_iters = pt.max_iters;
  a.rec = (const unsigned long long *)g->rec.p;
  a.stacks = (const uint32_t *)g->stacks.p;
  a.prods = (const uint32_t *)g->prods.p;
  a.br_out = (uint32_t *)g->br.p;
  a.pr_out = (uint32_t *)g->pr.p;
  a.ticket = (unsigned *)g->pair_ticket.p;
  a.st = PairTileState{(unsigned *)g->pst_flags.p, (unsigned long long *)g->pst_agg.p,
                       (unsigned long long *)g->pst_inc.p};
  a.status = g->d_status;
  a.arity = (const int32_t *)g->arity.p;
  a.is_term = (const uint8_t *)g->is_term.p;
  return a;
}

// CTAs of pse_resolve_kernel for a walk of at most `tiles` tiles: one warp
// per tile (8 per CTA), at most 8 CTAs per SM.
inline unsigned resolve_blocks(uint64_t tiles) {
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(148 * 8, (tiles + 7) / 8));
}

// Bytes of the walk's per-tile regions for `tiles` tiles: staircase depths,
// query values, their terminal counts (4 bytes each per entry), staircase and
// query offsets (2 bytes each), then the two per-tile counts.
inline uint64_t pse_region_bytes(uint64_t tiles) {
  return std::max<uint64_t>(tiles, 1) * ((uint64_t)kPseTile * 20 + 8);
}

inline PseArgs pse_args(alpacc_gpu_grammar *g, int mode, uint64_t tiles) {
  const alpacc_tables &tb = g->hg.t;
  PseArgs a{};
  a.mode = mode;
  a.elems = (const uint32_t *)(mode == kPseBrackets ? g->br.p : g->pr.p);
  a.count = mode == kPseBrackets ? &g->d_status->num_brackets : &g->d_status->num_productions;
  a.num_tokens = &g->d_status->num_tokens;
  a.arity = (const int32_t *)g->arity.p;
  a.is_term = (const uint8_t *)g->is_term.p;
  a.num_prods = (int)g->hg.pairs.arity.size();
  a.tile_min = (int32_t *)g->tile_min.p;
  a.super_key = (uint32_t *)g->super_key.p;
  const uint64_t entries = std::max<uint64_t>(tiles, 1) * kPseTile;
  uint8_t *r = (uint8_t *)g->pse_regions.p;
  a.stair_val = (int32_t *)r;
  a.q_val = a.stair_val + entries;
  a.stair_tc = a.q_val + entries;
  a.q_tc = a.stair_tc + entries;
  a.stair_off = (uint16_t *)(a.q_tc + entries);
  a.q_off = a.stair_off + entries;
  a.stair_cnt = (uint32_t *)(a.q_off + entries);
  a.q_cnt = a.stair_cnt + std::max<uint64_t>(tiles, 1);
  a.node_prods = g->node_prods.p;
  a.node_parents = g->node_parents.p;
  a.token_parents = g->token_parents.p;
  a.prod_w = (int)tb.production_size;
  a.idx_w = (int)tb.index_size;
  a.ticket = (unsigned *)g->pse_ticket.p;
  a.resolve_ticket = a.ticket + 1;
  a.st = PairTileState{(unsigned *)g->pse_flags.p, (unsigned long long *)g->pse_agg.p,
                       (unsigned long long *)g->pse_inc.p};
  a.status = g->d_status;
  return a;
}

}  // namespace alpacc
