// Exact device scratch of a batch (alpacc_gpu_parse_batch), shared by the
// batch path, which grows the handle's buffers to these sizes, and by the
// server's admission, which keeps what a worker's handle holds within its
// share of the scratch budget.
#pragma once

#include <cstdint>

struct alpacc_gpu_grammar;

namespace alpacc {

struct DevBuf;

// Upper bounds the batch path sizes its regions by, summed over documents.
struct BatchSizes {
  uint64_t docs = 0, bytes = 0, tokens = 0, brackets = 0, productions = 0;
  uint64_t lex_tiles = 0, pair_tiles = 0, br_tiles = 0, pr_tiles = 0;
  void add(const alpacc_gpu_grammar *g, uint64_t n);  // one more document of n bytes
};

struct BufNeed {
  DevBuf *buf;
  uint64_t bytes;  // what grow() allocates for it
};

constexpr int kBatchBufs = 40;

// Every scratch buffer of the batch path with its size for a batch of z
// (result packing at its bound); returns the count (<= kBatchBufs).
int batch_needs(alpacc_gpu_grammar *g, const BatchSizes &z, BufNeed *out);
// Sum of batch_needs.
uint64_t batch_scratch_bytes(alpacc_gpu_grammar *g, const BatchSizes &z);
// Bytes the handle's batch buffers will hold after running z: each buffer
// keeps the larger of its capacity and its need; when that sum exceeds
// `budget`, the buffers larger than their need are released first (after the
// handle's stream is idle), so the handle then holds exactly
// batch_scratch_bytes(z). Returns the bytes held afterwards.
uint64_t fit_batch_scratch(alpacc_gpu_grammar *g, const BatchSizes &z, uint64_t budget);
// Bytes the handle's batch buffers hold now.
uint64_t batch_scratch_held(alpacc_gpu_grammar *g);

}  // namespace alpacc
