// Kernel argument blocks and launch geometry shared by the host driver.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "device_tables.h"

namespace alpacc {

// ---- batches: many independent documents through one launch per stage ----
// Each stage's tiles form one virtual tile space in which document d owns
// tiles [tile0[d], tile0[d+1]); a ticketed tile is mapped to (document, local
// tile) by binary search. Per-document data lives in per-document regions of
// every array and each document has its own status, so documents never see
// each other: each behaves exactly as if it had been parsed alone.
struct BatchDesc {
  int docs;
  const unsigned long long *in_off;   // [docs] byte offset of document d in the input
  const unsigned long long *n;        // [docs] bytes of document d
  const unsigned long long *tok_off;  // [docs+1] token region (capacity n_d + 1)
  const unsigned long long *br_off;   // [docs+1] bracket region (capacity (n_d + 3) * max brackets per position)
  const unsigned long long *pr_off;   // [docs+1] production and tree-node region
  const unsigned long long *lex_tile0;  // [docs+1] lexer tiles (host: from n_d)
  unsigned long long *pair_tile0;       // [docs+1] pair tiles (planned on the device from T_d)
  unsigned long long *br_tile0;         // [docs+1] bracket-walk tiles (from B_d)
  unsigned long long *pr_tile0;         // [docs+1] parent-walk tiles (from P_d)
  DeviceStatus *status;                 // [docs]
};

// Document owning virtual tile vt: the last d with tile0[d] <= vt (documents
// without tiles share their successor's tile0 and are skipped by the search).
__device__ __forceinline__ int batch_doc(const unsigned long long *tile0, int docs, unsigned long long vt) {
  int lo = 0, hi = docs;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (tile0[mid] <= vt) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Per-document tile counts of the next stage from the counts the previous
// stage left in each document's status (one CTA): tile0[d] = sum over earlier
// documents of ceil((count_d + extra) / tile).
enum PlanKind : int { kPlanPairs = 0, kPlanBrackets = 1, kPlanParents = 2 };
__global__ void batch_plan_kernel(BatchDesc b, int kind, unsigned long long *tile0, unsigned long long tile);

// ---- lexer tiles: 256 chunks x 15 words (60 bytes), loaded with the 64
// bytes before the tile (the first chunk's longest window) ----
constexpr int kLexThreads = 256;
constexpr int kLexWords = 15;
constexpr int kLexChunk = kLexWords * 4;
constexpr int kLexWin = 64;                                     // bytes loaded before a tile
constexpr int kLexData = kLexThreads * kLexChunk;               // bytes per tile
constexpr int kLexLoad = kLexWin + kLexData;                    // bytes loaded per tile
constexpr int kLexLanes = kMaxLanes;                            // candidate starts of an open chunk

struct LexArgs {
  const uint8_t *in;
  unsigned long long n;
  unsigned long long num_tiles;
  // minimised machine in the form of build_lexer_table: entries
  // F(next) | code << 24 in rows of 1 << (cp_shift - 2), columns swizzled by
  // (state & swz)
  const uint32_t *tab;              // [tab_words]
  int tab_words;
  const uint8_t *cls4;              // byte -> class * 4: u8[256], or u16[256] when wide_cls
  int wide_cls;
  int cp_shift, swz;
  // window machine (build_lexer_table): entries in the same row format,
  // F of the set of all live states, member states of each set (4 words)
  const uint32_t *ps_tab;           // [ps_words], null: windows walked as explicit state sets
  int ps_words;
  uint32_t ps_full;
  const unsigned long long *ps_mask;
  int win_words;                    // window before each chunk: 4..8 words (16..32 bytes)
  const uint8_t *img;               // [C*kLexLanes] live targets of each class (explicit set walks)
  const uint8_t *img_cnt;           // [C]
  const uint8_t *sterm;             // [M]
  const uint8_t *sflags;            // [M] bit0 produce, bit1 accept, bit2 kept
  int M, C, dead, m0;
  unsigned long long len_max;
  // outputs (native widths)
  void *tok_ids, *tok_starts, *tok_lens;
  int term_w, idx_w, len_w;
  // look-back state (zeroed before launch)
  unsigned *ticket;
  unsigned *st1_flag;   // [tiles] 1 = transition vector published, 2 = outgoing state published
  uint8_t *st1_state;   // [tiles]
  uint8_t *st1_vec;     // [tiles * M]
  unsigned long long tile_begin, tile_end;  // this launch's tiles (tile_end 0: all num_tiles)
  PairTileState st2;    // (kept-token count, last boundary)
  DeviceStatus *status;
  int diag;             // 1: accumulate diagnostic counters in status->scratch
  // diagnostics: SM cycles of each barrier-delimited phase summed over tiles
  // (thread 0's clock): 0 load, 1 window walk, 2 chunk walks + candidate
  // jobs, 3 known-chunk scan, 4 start states, 5 open chunks' codes + masks +
  // count scan, 6 count look-back, 7 token / code writes; null when off
  unsigned long long *phase_cycles;
  const BatchDesc *batch;  // null: one document (in, n, status); else tiles are virtual (lex_tile0)
  // One window of a longer input (chunked lexing): the input continues after
  // byte n, so the token in progress at n is neither emitted nor judged; the
  // window's last boundary is left in status->last_boundary.
  int open_end;
  unsigned long long index_base;  // added to every token start (a window's offset in chunked lexing)
  // Staged output (lex_kernel*): each tile writes the codes of
  // its data bytes to codes[tile * kLexData ...] and its (kept-token count,
  // last boundary) to tile_cnt / tile_pos; lex_scan_kernel and lex_emit_kernel
  // then write the tokens, so no tile waits for another's count. The direct
  // kernels (lex_direct_kernel*) chain the counts by
  // decoupled look-back (st2) and write the tokens themselves.
  uint8_t *codes;
  uint32_t *tile_cnt, *tile_pos;
};

// Staged and direct output, each for: machines of at most 64 states with a
// window machine (one 64-bit candidate set), of up to 255 states with one
// (four words), and any machine whose window machine was not built (windows
// walked as explicit state sets).
__global__ void lex_kernel(LexArgs args);
__global__ void lex_kernel_wide(LexArgs args);
__global__ void lex_kernel_sets(LexArgs args);
__global__ void lex_direct_kernel(LexArgs args);
__global__ void lex_direct_kernel_wide(LexArgs args);
__global__ void lex_direct_kernel_sets(LexArgs args);

struct LexEmitArgs {
  const uint8_t *codes;             // [tiles * kLexData] codes of every data byte (lex_kernel)
  unsigned long long n;
  unsigned long long num_tiles;
  const uint32_t *tile_cnt, *tile_pos;
  unsigned long long *tile_off;     // exclusive prefix of tile_cnt (token index, in the document's region)
  uint32_t *tile_prev;              // last boundary before each tile (0: none)
  void *tok_ids, *tok_starts, *tok_lens;
  int term_w, idx_w, len_w;
  unsigned long long len_max;
  unsigned long long index_base;
  int open_end;
  DeviceStatus *status;
  const BatchDesc *batch;           // null: one document; else counts restart at each document's first tile
};

constexpr int kLexScanThreads = 1024;
__global__ void lex_scan_kernel(LexEmitArgs args);  // one CTA
__global__ void lex_emit_kernel(LexEmitArgs args);  // CTAs over tiles
constexpr int kLexEmitSmem = 2 * kLexData + 9 * 2048;  // its dynamic shared memory (bytes)

// ---- pair lookup / stack-action expansion: 256 threads x 8 positions ----
constexpr int kPairThreads = 256;
constexpr int kPairItems = 8;
constexpr int kPairTile = kPairThreads * kPairItems;
constexpr int kPairOut = 6144;  // output window of pair_kernel (elements)

struct PairArgs {
  const void *tok_ids;      // lexer output, terminal ids (term_w bytes each)
  int term_w;
  const unsigned long long *num_tokens;  // device: T
  unsigned long long tiles_cap;          // pair tiles the look-back state holds (ALPACC_E_CAPACITY beyond)
  int q, k, nt;
  int empty_t, start_t, end_t;
  const uint32_t *dense;    // [nt^(q+k)] record index or 0xffffffff; null: the hashed form below
  const unsigned long long *ht_key;  // hashed form: [ht_size] key terminals packed 8 bits each
  const uint32_t *ht_rec;            // hashed form: [ht_size] record, kEmptySlot or kMissingKey
  unsigned long long ht_size, max_iters;
  const unsigned long long *rec;  // ss | ps << 24 | nb << 48 | np << 56
  const uint32_t *stacks;   // bit31 left
  const uint32_t *prods;
  uint32_t *br_out;         // brackets (capacity br_cap)
  uint32_t *pr_out;         // productions (capacity pr_cap)
  unsigned long long br_cap, pr_cap;
  unsigned *ticket;
  PairTileState st;         // (brackets, productions)
  DeviceStatus *status;
  const BatchDesc *batch;   // null: one document; else virtual tiles (pair_tile0) and per-document regions
  // one document: per depth-walk tile (kPseTile elements of the output) the
  // sum of the depth steps of its brackets / productions and the number of
  // its terminal productions, accumulated as the elements are written (zeroed
  // before launch; null: not accumulated)
  int *walk_step[2];
  int *walk_term;
  unsigned long long walk_tiles_cap;
  const int32_t *arity;     // per production
  const uint8_t *is_term;
};

__global__ void pair_kernel(PairArgs args);

// Exclusive prefixes of the depth walks' tile aggregates (one CTA): per walk
// tile the depth and (parents) the terminal-production count before it, so
// that the walk kernels need no look-back.
struct WalkPrefixArgs {
  const int *walk_step[2];
  const int *walk_term;
  long long *prefix_s[2];
  long long *prefix_t;
  unsigned long long tiles_cap;
  DeviceStatus *status;
};
__global__ void walk_prefix_kernel(WalkPrefixArgs args);

// ---- previous-smaller search over depth walks: 256 threads x 8 elements ----
// A chunk is one thread's 8 consecutive elements; a tile is 256 chunks. Per
// tile the walk keeps its minimum depth, its staircase and its unanswered
// queries (PseArgs) for the resolve kernel.
constexpr int kPseThreads = 256;
constexpr int kPseItems = 8;
constexpr int kPseTile = kPseThreads * kPseItems;

constexpr int kPseSuperShift = 8;  // 256 tiles per super-tile

enum PseMode : int { kPseBrackets = 0, kPseParents = 1 };

struct PseArgs {
  int mode;
  const uint32_t *elems;            // brackets (bit 31 = left) or productions
  const unsigned long long *count;  // device: number of elements
  const unsigned long long *num_tokens;
  unsigned long long elem_cap;      // elements the walk's arrays hold (ALPACC_E_CAPACITY beyond)
  const int32_t *arity;             // parents: per production
  const uint8_t *is_term;           // parents: terminal production flags
  int num_prods;                    // entries of arity / is_term
  int32_t *tile_min;                // [tiles] minimum depth of each tile
  uint32_t *super_key;              // [ceil(tiles / 256)] INT_MAX - minimum over each run of 256 tiles (0: none)
  // per tile (regions of kPseTile entries): the staircase - the tile's
  // right-to-left strict minima, in position order (their depths increase):
  // offset in the tile, depth, (parents) inclusive terminal-production count -
  // and the queries the tile could not answer, in position order (their query
  // values decrease): offset, query value, (parents) inclusive terminal count
  uint16_t *stair_off, *q_off;
  int32_t *stair_val, *stair_tc, *q_val, *q_tc;
  uint32_t *stair_cnt, *q_cnt;      // [tiles]
  // parents: the compacted tree (compact_tree), written as answers are found
  void *node_prods, *node_parents, *token_parents;
  int prod_w, idx_w;
  unsigned *ticket;                 // tiles of the walk
  unsigned *resolve_ticket;         // tiles with queries, taken by the resolve kernel's warps
  PairTileState st;                 // (sum of steps, terminal count)
  DeviceStatus *status;
  const BatchDesc *batch;           // null: one document; else virtual tiles (br_tile0 / pr_tile0)
  // one document: the tile's depth and terminal-count prefixes from
  // walk_prefix_kernel (null: decoupled look-back over the tiles, st)
  const long long *prefix_s, *prefix_t;
  // diagnostics: SM cycles of each phase of pse_tile_kernel summed over tiles
  // (thread 0's clock): 0 load + steps + scan, 1 depths + windows, 2 own and
  // previous chunk queries, 3 the warps' queued queries, 4 look-back,
  // 5 staircase + unanswered queries, 6 tree entries, 7 next tile; null when off
  unsigned long long *phase_cycles;
};

__global__ void pse_tile_kernel(PseArgs args);
__global__ void pse_resolve_kernel(PseArgs args);
__global__ void narrow_u32_kernel(const uint32_t *src, void *dst, const unsigned long long *count,
                                  unsigned long long cap, int width);

}  // namespace alpacc
