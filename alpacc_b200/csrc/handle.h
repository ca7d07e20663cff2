// The grammar handle behind the C ABI (shared by the .cu files of the library).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/alpacc_b200.h"
#include "common.cuh"
#include "device_tables.h"

namespace alpacc {

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
  if (cudaMalloc(&b.p, want) != cudaSuccess) {
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
  DevBuf cls_id, trans_words, lane_of, img, img_cnt, sterm, sflags;
  DevBuf dense, rec_ss, rec_ps, rec_nb, rec_np, stacks, prods, arity, is_term;
  int trans_word_count = 0, trans_rep = 32;
  int lex_grid = 0;
  int diag = 0;
  // status
  DeviceStatus *d_status = nullptr;
  DeviceStatus *h_status = nullptr;  // pinned
  // scratch
  DevBuf in;                                   // device copy of host input
  DevBuf lex_ticket, st1_flag, st1_state, st1_vec, st2_flags, st2_agg, st2_inc;
  DevBuf tok_ids, tok_starts, tok_lens;
  DevBuf pair_ticket, pst_flags, pst_agg, pst_inc, br, pr;
  DevBuf pse_ticket, pse_flags, pse_agg, pse_inc, ch_h0, ch_tc, tile_min, chunk_min, super_min, queue, queue_len;
  DevBuf node_prods, node_parents, token_parents;
  // pinned host result buffers kept for reuse (released results come back here)
  void *pinned_cache = nullptr;
  size_t pinned_cache_size = 0;
  // last result (device)
  uint64_t last_T = 0, last_N = 0;
  int last_status = ALPACC_E_INVALID;
  std::string last_error;
};

// Dynamic shared memory of lex_kernel for this handle's tables.
inline size_t lex_dyn_smem(const alpacc_gpu_grammar *g) {
  return ((256 * (size_t)g->trans_rep * 2 + 15) & ~(size_t)15) + (size_t)g->trans_word_count * g->trans_rep * 4;
}
