// Kernel argument blocks and launch geometry shared by the host driver.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "device_tables.h"

namespace alpacc {

// ---- lexer tiles: 256 chunks x 15 words (60 bytes); the first 8 chunks are
// a halo repeating the end of the previous tile ----
constexpr int kLexThreads = 256;
constexpr int kLexWords = 15;
constexpr int kLexChunk = kLexWords * 4;
constexpr int kLexHalo = 8;
constexpr int kLexLoad = kLexThreads * kLexChunk;               // bytes loaded per tile
constexpr int kLexData = (kLexThreads - kLexHalo) * kLexChunk;  // new bytes per tile

struct LexArgs {
  const uint8_t *in;
  unsigned long long n;
  unsigned long long num_tiles;
  // minimised machine
  const uint8_t *cls_id;            // [256] byte -> class
  const uint32_t *trans_words_ptr;  // [trans_words] u8 entries (next | produce << 7) at class * M + state
  int trans_words;
  int copies;                       // table copies in shared memory (power of two <= 32)
  const uint8_t *lane_of;           // [C*M]
  const uint8_t *img;               // [C*kMaxLanes]
  const uint8_t *img_cnt;           // [C]
  const uint8_t *sterm;             // [M]
  const uint8_t *sflags;            // [M] bit0 produce, bit1 accept, bit2 kept
  int M, C, dead, m0, ignore;
  unsigned long long len_max;
  // outputs (native widths)
  void *tok_ids, *tok_starts, *tok_lens;
  int term_w, idx_w, len_w;
  // look-back state (zeroed before launch)
  unsigned *ticket;
  unsigned *st1_flag;   // [tiles] 1 = transition vector published, 2 = outgoing state published
  uint8_t *st1_state;   // [tiles]
  uint8_t *st1_vec;     // [tiles * M]
  PairTileState st2;    // (kept-token count, last boundary position)
  DeviceStatus *status;
  int diag;             // 1: accumulate diagnostic counters in status->scratch
};

__global__ void lex_kernel(LexArgs args);

// ---- pair lookup / stack-action expansion: 256 threads x 8 positions ----
constexpr int kPairThreads = 256;
constexpr int kPairItems = 8;
constexpr int kPairTile = kPairThreads * kPairItems;

struct PairArgs {
  const void *tok_ids;      // lexer output, terminal ids (term_w bytes each)
  int term_w;
  const unsigned long long *num_tokens;  // device: T
  unsigned long long num_tiles;          // tiles launched (upper bound)
  int q, k, nt;
  int empty_t, start_t, end_t;
  const uint32_t *dense;    // [nt^(q+k)] record index or 0xffffffff
  const uint32_t *rec_ss, *rec_ps;
  const uint8_t *rec_nb, *rec_np;
  const uint32_t *stacks;   // bit31 left
  const uint32_t *prods;
  uint32_t *br_out;         // brackets (capacity br_cap)
  uint32_t *pr_out;         // productions (capacity pr_cap)
  unsigned long long br_cap, pr_cap;
  unsigned *ticket;
  PairTileState st;         // (brackets, productions)
  DeviceStatus *status;
};

__global__ void pair_kernel(PairArgs args);

// ---- previous-smaller search over depth walks: 256 threads x 8 elements ----
constexpr int kPseThreads = 256;
constexpr int kPseItems = 8;
constexpr int kPseTile = kPseThreads * kPseItems;

constexpr int kPseSuperShift = 8;  // 256 tiles per super-tile

enum PseMode : int { kPseBrackets = 0, kPseParents = 1 };

struct PseArgs {
  int mode;
  const uint32_t *elems;          // brackets or productions
  const unsigned long long *count;  // device: number of elements
  unsigned long long num_tiles;
  const int32_t *arity;           // parents: per production
  const uint8_t *is_term;         // parents: terminal production flags
  int32_t *h;                     // [E] depth before each element
  int32_t *answer;                // [E] matched / parent position (-1 pending)
  int32_t *tinc;                  // parents: [E] inclusive terminal-production count
  int32_t *tile_min;              // [tiles]
  int32_t *chunk_min;             // [tiles * kPseThreads]
  int32_t *super_min;             // [ceil(tiles / 256)] minimum over each run of 256 tiles
  unsigned long long *queue;      // pending (element) indices
  unsigned long long queue_cap;
  unsigned long long *queue_len;  // device counter
  unsigned *ticket;
  PairTileState st;               // (sum of steps, terminal count)
  DeviceStatus *status;
};

__global__ void pse_tile_kernel(PseArgs args);
__global__ void pse_resolve_kernel(PseArgs args);

// ---- tree compaction (compact_tree) ----
struct CompactArgs {
  const uint32_t *prods;
  const unsigned long long *count;   // P
  const unsigned long long *num_tokens;
  const int32_t *parent;
  const int32_t *tinc;
  const uint8_t *is_term;
  void *node_prods, *node_parents, *token_parents;
  int prod_w, idx_w;
  DeviceStatus *status;
};

__global__ void compact_kernel(CompactArgs args);

}  // namespace alpacc
