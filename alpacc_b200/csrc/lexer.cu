// Data-parallel lexer for sm_100a: the sequential semantics of lex_string
// (backends/c/lexer.c:39-97) computed tile-parallel.
//
// The lexer runs a Moore machine over byte classes that device_tables.cpp
// derives from TO_STATE / COMPOSE / ACCEPT. Its transition table lives in
// shared memory as 32-bit entries (build_lexer_table): entry(s, c) =
// F(next) | code << 24, where F(x) is the byte offset of state x's row (rows
// of CP >= C entries, CP a power of two, columns swizzled by the row's low
// state bits so that threads reading one class in different states meet in
// different banks) and code says what happens before the byte: 0xFF no token
// boundary, 0xFE the token that ends here is ignored, else its terminal id.
// One step of the machine is then a class lookup, one LOP3 (address =
// (entry & 0xFFFFFF) ^ class * 4) and one shared-memory load.
//
// A tile is 256 chunks of 60 bytes (15 words: an odd word stride, so per-thread
// rows are bank-conflict free), loaded with the 64 bytes before it.
//
// Window: each chunk walks the 16 (up to 32: a per-grammar choice of the
// autotuner) bytes before it in the window machine (the
//   subset automaton of the live states, same row format, from the set of all
//   of them), which yields the set of states the chunk can start in. On JSON
//   that set is one state for ~95% of chunks, on s-expressions for all: the
//   chunk's start is then known without looking at any other chunk
//   ("known"). A tile's first chunk whose window leaves several candidates
//   walks the whole 64 bytes loaded before the tile once more, so that the
//   tile rarely needs its predecessor's state. The window walk is the same fixed number of steps in every
//   thread.
//   Machines whose subset automaton is too large walk the window as an
//   explicit state set instead.
// Walk: a known chunk walks its 60 bytes once from its start (fully unrolled),
//   writing each byte's code over the consumed input word. A chunk whose
//   window left two or more candidates ("open") has each candidate walked on
//   its own - one job per candidate, spread over the whole CTA - keeping the
//   end state per candidate and, for the first 64 jobs, the codes.
// Resolution: an open chunk's start is the end of the nearest known chunk
//   before it carried through the open chunks in between; only when the
//   tile's first chunk is open does the tile read its predecessor's published
//   outgoing state (bounded look-back). The open chunk then takes its true
//   candidate's codes (or walks again when that candidate had no code slot).
// Output, staged (lex_kernel*): each tile writes the codes of its bytes
//   (16-byte stores from shared memory) and its (kept-token count, last
//   boundary); lex_scan_kernel scans the tile totals and lex_emit_kernel turns
//   each tile's codes into tokens at their final places, with the length_t
//   check of lexer.c:68-72. No tile waits for another tile's count.
// Output, direct (lex_direct_kernel*, for the allocation-free entry point):
//   boundary masks from the code words, a (token count, last boundary) block
//   scan, a decoupled look-back over tiles (Merrill & Garland 2016) and the
//   kept tokens written by the kernel itself.
//
// Reference equivalents: backends/cuda/lexer.cu:437-760 (``lexer`` kernel) and
// backends/cuda/scan.cu:181-400 (look-back).
#include <cstdint>

#include "common.cuh"
#include "kernels.h"

namespace alpacc {

namespace {

__device__ __forceinline__ void store_uint(void *base, unsigned long long i, int w, unsigned long long v) {
  switch (w) {
    case 1: static_cast<uint8_t *>(base)[i] = (uint8_t)v; break;
    case 2: static_cast<uint16_t *>(base)[i] = (uint16_t)v; break;
    case 4: static_cast<uint32_t *>(base)[i] = (uint32_t)v; break;
    default: static_cast<unsigned long long *>(base)[i] = v; break;
  }
}

// kOpenTail: an open chunk holding the input's last byte (no candidate jobs:
// walked once its start is known; nothing after it reads its end state)
enum ChunkKind : uint8_t { kEmpty = 0, kKnown = 1, kOpen = 2, kOpenTail = 3 };

constexpr uint32_t kAddrMask = 0xFFFFFFu;  // F(next) bits of an entry
constexpr uint8_t kNoBoundary = 0xFF, kIgnored = 0xFE;
constexpr uint32_t kOpenInfo = 0xFFu;        // window machine: two or more candidates
constexpr int kWinWords = kLexWin / 4;  // words loaded before the tile
// Candidate walks of open chunks run as jobs spread over the CTA (rounds of
// one job per thread); the first kCodeJobs keep their codes, so the chunk's
// second pass copies the true candidate's codes instead of walking again.
constexpr int kCodeJobs = 64;
// Tokens staged per window by lex_emit_kernel before consecutive threads
// write them out.
constexpr int kTokWin = 2048;
static_assert(kLexEmitSmem == 2 * kLexData + 9 * kTokWin, "emit kernel shared memory");

// The set of states an open chunk can start in, W 64-bit words.
template <int W>
struct StateSet {
  unsigned long long w[W];
  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int i = 0; i < W; i++) w[i] = 0;
  }
  __device__ __forceinline__ void add(int s) {
#pragma unroll
    for (int i = 0; i < W; i++)
      if ((s >> 6) == i) w[i] |= 1ull << (s & 63);
  }
  __device__ __forceinline__ bool many() const {
    if (W == 1) return (w[0] & (w[0] - 1)) != 0;
    return count() > 1;
  }
  __device__ __forceinline__ bool empty() const {
    unsigned long long o = 0;
#pragma unroll
    for (int i = 0; i < W; i++) o |= w[i];
    return o == 0;
  }
  __device__ __forceinline__ int count() const {
    int c = 0;
#pragma unroll
    for (int i = 0; i < W; i++) c += __popcll(w[i]);
    return c;
  }
  __device__ __forceinline__ int first() const {
#pragma unroll
    for (int i = 0; i < W; i++)
      if (w[i]) return 64 * i + __ffsll((long long)w[i]) - 1;
    return -1;
  }
};

template <int W>
struct LexSmem {
  uint32_t bytes[kLexLoad / 4];             // window + tile; codes replace the consumed words
  uint8_t lend[kLexLanes * kLexThreads];    // open chunks: end state per candidate (candidate-major)
  unsigned long long cand[W][kLexThreads];  // open chunks: their candidate start states
  uint8_t kind[kLexThreads];
  uint8_t endst[kLexThreads];  // known chunks: end state
  uint8_t start[kLexThreads];  // every chunk's true start state
  uint16_t jfirst[kLexThreads];  // first candidate job of each chunk (jobs of earlier chunks)
  uint32_t jcodes[kCodeJobs * kLexWords];  // codes of the first candidate jobs
  uint8_t sterm[256];          // per machine state: terminal id
  uint8_t sflags[256];         // bit1 accept, bit2 kept
  int kconst[kLexThreads];
  int scan_a[kLexThreads / 32], scan_b[kLexThreads / 32];
  unsigned tile;
  int s_in;
  int out_published;
  long long cnt_prefix, pos_prefix;
};

// A machine in shared memory (the lexer's or the window machine): class
// table and entries, plus the shape parameters that turn a state into its row
// offset and back.
struct Tab {
  const uint8_t *cls;  // [256] class * 4 (u8), or [512] bytes of u16 when wide
  const uint8_t *ent;  // entries, addressed by byte offset
  int wide;
  int shift;           // F(x) >> shift == x
  uint32_t swz;        // K - 1
};

__device__ __forceinline__ uint32_t cls4_of(const Tab &tb, uint32_t b) {
  return tb.wide ? (uint32_t) reinterpret_cast<const uint16_t *>(tb.cls)[b] : (uint32_t)tb.cls[b];
}

__device__ __forceinline__ uint32_t row_of(const Tab &tb, uint32_t x) { return (x << tb.shift) | ((x & tb.swz) << 2); }

__device__ __forceinline__ int state_of(const Tab &tb, uint32_t f) { return (int)((f & kAddrMask) >> tb.shift); }

// One machine step: the entry for (state of f, class c4 / 4).
__device__ __forceinline__ uint32_t step(const Tab &tb, uint32_t f, uint32_t c4) {
  return *reinterpret_cast<const uint32_t *>(tb.ent + ((f & kAddrMask) ^ c4));
}

// The four bytes' codes of a word walked from f (entries e0..e3 of its bytes)
// packed into one word.
__device__ __forceinline__ uint32_t pack_codes(uint32_t e0, uint32_t e1, uint32_t e2, uint32_t e3) {
  return __byte_perm(__byte_perm(e0, e1, 0x0073), __byte_perm(e2, e3, 0x0073), 0x5410);
}

// A full chunk (15 words of src) walked from state x: the codes of its bytes
// into dst (may be src), returns the end state.
__device__ __forceinline__ int walk_chunk(const Tab &tb, const uint32_t *src, uint32_t *dst, int x) {
  uint32_t f = row_of(tb, (uint32_t)x);
#pragma unroll
  for (int w = 0; w < kLexWords; ++w) {
    const uint32_t word = src[w];
    const uint32_t e0 = step(tb, f, cls4_of(tb, __byte_perm(word, 0, 0x4440)));
    const uint32_t e1 = step(tb, e0, cls4_of(tb, __byte_perm(word, 0, 0x4441)));
    const uint32_t e2 = step(tb, e1, cls4_of(tb, __byte_perm(word, 0, 0x4442)));
    const uint32_t e3 = step(tb, e2, cls4_of(tb, __byte_perm(word, 0, 0x4443)));
    f = e3;
    dst[w] = pack_codes(e0, e1, e2, e3);
  }
  return state_of(tb, f);
}

// The first nb bytes of a row walked from state x, codes written over them;
// returns the end state.
__device__ __forceinline__ int walk_bytes(const Tab &tb, uint8_t *rb, int nb, int x) {
  uint32_t f = row_of(tb, (uint32_t)x);
  for (int j = 0; j < nb; ++j) {
    const uint32_t e = step(tb, f, cls4_of(tb, rb[j]));
    rb[j] = (uint8_t)(e >> 24);
    f = e;
  }
  return state_of(tb, f);
}

// The window of chunk t (the nw words before its row, `win` pointing at the
// first): the one state the chunk can start in (the dead state when none), or
// -1 with the candidates in *cand. kPs: walked in the window machine; else as
// an explicit state set from the first window byte's image.
template <int W, bool kPs>
__device__ __forceinline__ int window_start(const LexArgs &a, const Tab &tb, const Tab &tw, const uint32_t *win,
                                            int nw, StateSet<W> *cand) {
  if (kPs) {
    uint32_t f = a.ps_full, e = 0;
#pragma unroll 4
    for (int w = 0; w < nw; ++w) {
      const uint32_t word = win[w];
      e = step(tw, f, cls4_of(tb, __byte_perm(word, 0, 0x4440)));
      e = step(tw, e, cls4_of(tb, __byte_perm(word, 0, 0x4441)));
      e = step(tw, e, cls4_of(tb, __byte_perm(word, 0, 0x4442)));
      e = step(tw, e, cls4_of(tb, __byte_perm(word, 0, 0x4443)));
      f = e;
    }
    const uint32_t info = e >> 24;
    if (info != kOpenInfo) return (int)info;
    const int p = state_of(tw, e);
#pragma unroll
    for (int i = 0; i < W; i++) cand->w[i] = __ldg(a.ps_mask + 4 * p + i);
    return -1;
  } else {
    const uint8_t *wb = reinterpret_cast<const uint8_t *>(win);
    StateSet<W> set;
    set.clear();
    const int c0 = (int)(cls4_of(tb, wb[0]) >> 2);
    const int cnt = __ldg(a.img_cnt + c0);
    for (int l = 0; l < cnt; l++) set.add(__ldg(a.img + c0 * kLexLanes + l));
    for (int j = 1; j < 4 * nw; ++j) {
      const uint32_t c4 = cls4_of(tb, wb[j]);
      StateSet<W> ns;
      ns.clear();
#pragma unroll
      for (int i = 0; i < W; i++)
        for (unsigned long long m = set.w[i]; m; m &= m - 1) {
          const int s = 64 * i + __ffsll((long long)m) - 1;
          const int nx = state_of(tb, step(tb, row_of(tb, (uint32_t)s), c4));
          if (nx != a.dead) ns.add(nx);
        }
      set = ns;
    }
    if (set.empty()) return a.dead;  // (a machine without a dead state never empties a set)
    if (!set.many()) return set.first();
    *cand = set;
    return -1;
  }
}

// Candidate slot of state x among an open chunk's candidates (its rank in the
// set), or -1 when x is not one of them.
template <int W>
__device__ __forceinline__ int cand_slot(const LexSmem<W> *sm, int t, int x) {
  int r = 0;
#pragma unroll
  for (int i = 0; i < W; i++) {
    const unsigned long long m = sm->cand[i][t];
    if ((x >> 6) == i) return (m >> (x & 63) & 1) ? r + __popcll(m & ((1ull << (x & 63)) - 1)) : -1;
    r += __popcll(m);
  }
  return -1;
}

// The l-th candidate (in state order) of open chunk t.
template <int W>
__device__ __forceinline__ int cand_state(const LexSmem<W> *sm, int t, int l) {
#pragma unroll
  for (int i = 0; i < W; i++) {
    unsigned long long m = sm->cand[i][t];
    const int c = __popcll(m);
    if (l < c) {
      for (int k = 0; k < l; k++) m &= m - 1;
      return 64 * i + __ffsll((long long)m) - 1;
    }
    l -= c;
  }
  return 0;
}

// f_t(x): the state after chunk t when it starts in state x: a known chunk's
// end state (its start is fixed), an open chunk's end for candidate x (dead
// when x is not a candidate: the true state always is one while the input is
// valid). A chunk holding the input's last byte is never followed by a
// non-empty chunk.
template <int W>
__device__ __forceinline__ int eval_chunk(const LexArgs &a, const LexSmem<W> *sm, int t, int x) {
  const int kind = sm->kind[t];
  if (kind == kEmpty) return x;
  const int dead = a.dead;
  if (kind == kKnown) return sm->endst[t];
  if (kind == kOpenTail || x == dead || x < 0) return dead;
  const int slot = cand_slot(sm, t, x);
  return slot < 0 ? dead : sm->lend[slot * kLexThreads + t];
}

struct CntPosOp {
  __device__ Pair64 operator()(Pair64 e, Pair64 l) const { return Pair64{e.a + l.a, e.b > l.b ? e.b : l.b}; }
};

// Bytes of `w` that differ from 0: 0x80 in such a byte, 0 elsewhere (exact, no
// borrow between bytes).
__device__ __forceinline__ uint32_t nonzero_bytes(uint32_t w) {
  return (((w & 0x7F7F7F7Fu) + 0x7F7F7F7Fu) | w) & 0x80808080u;
}

// The four 0x80 flags of nonzero_bytes as a 4-bit mask (byte i -> bit i).
__device__ __forceinline__ uint32_t movemask4(uint32_t x) { return ((x >> 7) * 0x10204080u) >> 28; }

template <int W, bool kPs, bool kStaged>
__device__ __forceinline__ void lex_body(const LexArgs &a, unsigned char *dyn_smem, LexSmem<W> *sm) {
  const int t = threadIdx.x;
  const int lane = t & 31;

  // ---- tables, once per CTA ----
  const int cls_bytes = a.wide_cls ? 512 : 256;
  uint8_t *s_cls = dyn_smem;
  uint8_t *s_ent = dyn_smem + cls_bytes;
  uint8_t *s_win = s_ent + a.tab_words * 4;
  for (int i = t; i < cls_bytes / 4; i += kLexThreads)
    reinterpret_cast<uint32_t *>(s_cls)[i] = __ldg(reinterpret_cast<const uint32_t *>(a.cls4) + i);
  for (int i = t; i < a.tab_words; i += kLexThreads) reinterpret_cast<uint32_t *>(s_ent)[i] = __ldg(a.tab + i);
  if (kPs)
    for (int i = t; i < a.ps_words; i += kLexThreads) reinterpret_cast<uint32_t *>(s_win)[i] = __ldg(a.ps_tab + i);
  for (int i = t; i < 256; i += kLexThreads) {
    sm->sterm[i] = i < a.M ? __ldg(a.sterm + i) : 0;
    sm->sflags[i] = i < a.M ? __ldg(a.sflags + i) : 0;
  }
  const Tab tb{s_cls, s_ent, a.wide_cls, a.cp_shift, (uint32_t)a.swz};
  const Tab tw{s_cls, s_win, a.wide_cls, a.cp_shift, (uint32_t)a.swz};
  const int dead = a.dead;
  const unsigned long long num_tiles = a.num_tiles;
  const unsigned long long tile_end = a.tile_end ? a.tile_end : num_tiles;
  unsigned long long *pcyc = a.phase_cycles;
  long long tp = clock64();
// diagnostics: thread 0 adds the cycles since the previous mark to phase k
#define LEX_PHASE(k)                                                  \
  if (pcyc && t == 0) {                                               \
    const long long now_ = clock64();                                 \
    atomicAdd(pcyc + (k), (unsigned long long)(now_ - tp));           \
    tp = now_;                                                        \
  }

  for (unsigned long long round = 0;; ++round) {
    if (round > tile_end - a.tile_begin) {  // every round takes a new ticket: cannot happen
      if (t == 0) record_timeout(a.status, kSiteLexTiles);
      break;
    }
    __syncthreads();  // tables ready / previous tile fully consumed
    LEX_PHASE(7);
    if (t == 0) sm->tile = atomicAdd(a.ticket, 1u);
    __syncthreads();
    const unsigned long long tile = a.tile_begin + sm->tile;
    if (tile >= tile_end) break;
    if (t == 0 && !a.batch && tile + gridDim.x < tile_end) {
      // warm L2 with the bytes of the tile a CTA takes about one tile time
      // from now (tickets go out in order)
      const long long p0 = (long long)(tile + gridDim.x) * kLexData - kLexWin;
      const long long p1 = min((long long)a.n, p0 + (long long)kLexLoad);
      if (p1 > p0) prefetch_l2(a.in + p0, (unsigned long long)(p1 - p0));
    }
    // this tile's document: the whole input, or one document of a batch
    // (virtual tile `tile` is local tile `lt` of `tiles_t`)
    const uint8_t *in_base = a.in;
    long long n = (long long)a.n;
    unsigned long long lt = tile, tiles_t = num_tiles, tok_base = 0;
    DeviceStatus *st = a.status;
    if (a.batch) {
      const BatchDesc &b = *a.batch;
      const int d = batch_doc(b.lex_tile0, b.docs, tile);
      lt = tile - b.lex_tile0[d];
      tiles_t = b.lex_tile0[d + 1] - b.lex_tile0[d];
      in_base = a.in + b.in_off[d];
      n = (long long)b.n[d];
      st = b.status + d;
      tok_base = b.tok_off[d];  // the document's token region
    }
    const long long data0 = (long long)lt * kLexData;
    const long long load0 = data0 - (long long)kLexWin;

    // ---- load window + tile ----
    {
      const uint8_t *in = in_base;
      uint8_t *dst = reinterpret_cast<uint8_t *>(sm->bytes);
      const bool aligned = ((reinterpret_cast<uintptr_t>(in) & 15) == 0);
      for (int v = t; v < kLexLoad / 16; v += kLexThreads) {
        const long long g = load0 + 16ll * v;
        if (aligned && g >= 0 && g + 16 <= n) {
          reinterpret_cast<uint4 *>(dst)[v] = __ldg(reinterpret_cast<const uint4 *>(in + g));
        } else {
          uint32_t wv[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            uint32_t x = 0;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              const long long p = g + 4 * q + k;
              if (p >= 0 && p < n) x |= (uint32_t)in[p] << (8 * k);
            }
            wv[q] = x;
          }
          reinterpret_cast<uint4 *>(dst)[v] = make_uint4(wv[0], wv[1], wv[2], wv[3]);
        }
      }
    }
    const long long g0 = data0 + (long long)t * kLexChunk;  // this chunk's first byte
    int nb = 0;
    if (g0 < n) nb = (int)min((long long)kLexChunk, n - g0);
    uint32_t *row = sm->bytes + kWinWords + t * kLexWords;
    uint8_t *rb = reinterpret_cast<uint8_t *>(row);
    __syncthreads();
    LEX_PHASE(0);

    // ---- window: the states the chunk can start in ----
    int x0 = -1;  // known start state
    int kind = kEmpty;
    if (nb > 0) {
      if (g0 == 0) {
        x0 = a.m0;  // the document's first chunk
      } else {
        StateSet<W> cand;
        x0 = window_start<W, kPs>(a, tb, tw, row - a.win_words, a.win_words, &cand);
        if (x0 < 0 && t == 0 && a.win_words < kWinWords)  // the tile's first chunk: the longest window
          x0 = window_start<W, kPs>(a, tb, tw, row - kWinWords, kWinWords, &cand);
        if (x0 < 0) {
#pragma unroll
          for (int i = 0; i < W; i++) sm->cand[i][t] = cand.w[i];
        }
      }
      kind = x0 >= 0 ? kKnown : nb == kLexChunk ? kOpen : kOpenTail;
    }
    sm->kind[t] = (uint8_t)kind;
    const int lanes = kind == kOpen ? [&] {
      int c = 0;
#pragma unroll
      for (int i = 0; i < W; i++) c += __popcll(sm->cand[i][t]);
      return c;
    }() : 0;
    int njobs;
    // (the scan's barriers also end every window read before the walks
    // below overwrite rows with codes)
    const int jex = block_exclusive_scan<int>(lanes, AddI32(), 0, sm->scan_a, &njobs);
    sm->jfirst[t] = (uint16_t)jex;  // non-decreasing over the chunks (at most 256 x 32 jobs)
    LEX_PHASE(1);

    // ---- walks: known chunks from their start; candidates of open chunks
    // as jobs spread over the CTA ----
    int x_end = dead;
    if (kind == kKnown) {
      if (x0 == dead) {
        record_reject(st, &st->lex_reject_reason, 1);  // no state survives the window: invalid input
      } else if (nb == kLexChunk) {
        x_end = walk_chunk(tb, row, row, x0);
      } else {
        x_end = walk_bytes(tb, rb, nb, x0);
      }
      if (g0 == 0) rb[0] = kNoBoundary;
      sm->endst[t] = (uint8_t)(x_end < 0 ? 0 : x_end);
      sm->start[t] = (uint8_t)(x0 < 0 ? 0 : x0);
    }
    __syncthreads();  // jfirst complete
    if (a.diag && t == 0 && njobs) atomicAdd(&st->scratch[3], (unsigned long long)njobs);
    for (int job = t; job < njobs; job += kLexThreads) {
      // the job's chunk: the last chunk whose first job is <= job (a chunk
      // without jobs shares its successor's first job, so it is skipped)
      int lo = 0, hi = kLexThreads - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((int)sm->jfirst[mid] <= job) lo = mid;
        else hi = mid - 1;
      }
      const int l = job - (int)sm->jfirst[lo];
      const uint32_t *src = sm->bytes + kWinWords + lo * kLexWords;  // an open chunk's row: still its bytes
      uint32_t *dst = job < kCodeJobs ? sm->jcodes + job * kLexWords : nullptr;
      uint32_t f = row_of(tb, (uint32_t)cand_state(sm, lo, l));
#pragma unroll 3
      for (int w = 0; w < kLexWords; ++w) {
        const uint32_t word = src[w];
        const uint32_t e0 = step(tb, f, cls4_of(tb, __byte_perm(word, 0, 0x4440)));
        const uint32_t e1 = step(tb, e0, cls4_of(tb, __byte_perm(word, 0, 0x4441)));
        const uint32_t e2 = step(tb, e1, cls4_of(tb, __byte_perm(word, 0, 0x4442)));
        const uint32_t e3 = step(tb, e2, cls4_of(tb, __byte_perm(word, 0, 0x4443)));
        f = e3;
        if (dst) dst[w] = pack_codes(e0, e1, e2, e3);
      }
      sm->lend[l * kLexThreads + lo] = (uint8_t)state_of(tb, f);
    }
    __syncthreads();
    LEX_PHASE(2);

    // ---- resolution: nearest known chunk before each chunk ----
    int ktot;
    const int kex = block_exclusive_scan<int>(kind == kKnown ? t : -1, MaxI32(), -1, sm->scan_a, &ktot);
    sm->kconst[t] = kex;
    if (t == 0) sm->out_published = 0;
    if (a.diag) {
      const int nknown = __syncthreads_count(kind == kKnown);
      if (t == 0) atomicAdd(&st->scratch[1], (unsigned long long)nknown);
    }
    __syncthreads();
    LEX_PHASE(3);
    if (ktot >= 0) {
      // the outgoing state does not depend on the incoming one: publish now
      if (t == 0) {
        int x = sm->endst[ktot];
        for (int jj = ktot + 1; jj < kLexThreads; ++jj) x = eval_chunk(a, sm, jj, x);
        a.st1_state[tile] = (uint8_t)(x < 0 ? 0 : x);
        __threadfence();
        st_release_u32(a.st1_flag + tile, 2u);
        sm->out_published = 1;
      }
    } else if (lt + 1 < tiles_t) {
      // no known chunk at all: publish the tile's transition vector
      for (int s = t; s < a.M; s += kLexThreads) {
        int x = s;
        for (int jj = 0; jj < kLexThreads; ++jj) x = eval_chunk(a, sm, jj, x);
        a.st1_vec[tile * (unsigned long long)a.M + s] = (uint8_t)(x < 0 ? 0 : x);
      }
      __syncthreads();
      if (t == 0) {
        __threadfence();
        st_release_u32(a.st1_flag + tile, 1u);
      }
    }
    __syncthreads();
    if (sm->kind[0] == kOpen || sm->kind[0] == kOpenTail) {  // the tile's incoming state: look back
      if (t == 0) {
        if (a.diag) atomicAdd(&st->scratch[0], 1ull);
        int s_in = a.m0;
        if (lt > 0) {
          long long j = (long long)tile - 1;
          const long long jfirst = (long long)(tile - lt);  // the document's first tile
          int base_state = a.m0;
          bool have = false;
          while (j >= jfirst) {
            const unsigned f = wait_flag(a.st1_flag + j, 1u, st, kSiteLexState);
            if (f == 0) break;
            if (f >= 2) {
              base_state = *reinterpret_cast<volatile uint8_t *>(a.st1_state + j);
              have = true;
              break;
            }
            --j;
          }
          if (!have) j = jfirst - 1;
          int x = have ? base_state : a.m0;
          for (long long jj = j + 1; jj < (long long)tile; ++jj) {
            if (x == dead || x < 0) break;
            x = *reinterpret_cast<volatile uint8_t *>(a.st1_vec + jj * (unsigned long long)a.M + x);
          }
          s_in = x;
        }
        sm->s_in = s_in;
      }
      __syncthreads();
    }
    // ---- the start state of every chunk that is not known ----
    unsigned chain = 0;
    if (kind != kKnown) {
      const int k = sm->kconst[t];
      int x, from;
      if (k >= 0) {
        x = sm->endst[k];
        from = k + 1;
      } else {
        x = sm->s_in;
        from = 0;
      }
      for (int jj = from; jj < t; ++jj) x = eval_chunk(a, sm, jj, x);
      sm->start[t] = (uint8_t)(x < 0 ? 0 : x);
      x0 = x;
      chain = (unsigned)(t - from);
    }
    if (a.diag) {  // every lane of the warp takes part
      const unsigned w = __reduce_add_sync(0xffffffffu, chain);
      if (lane == 0) atomicAdd(&st->scratch[2], (unsigned long long)w);
    }
    __syncthreads();
    LEX_PHASE(4);
    if (t == 0 && !sm->out_published) {
      const int x = eval_chunk(a, sm, kLexThreads - 1, sm->start[kLexThreads - 1]);
      a.st1_state[tile] = (uint8_t)(x < 0 ? 0 : x);
      __threadfence();
      st_release_u32(a.st1_flag + tile, 2u);
    }

    // ---- open chunks: the true candidate's codes (or a walk from it) ----
    long long cnt = 0, lastb = 0;
    unsigned long long bmask = 0;
    bool final_kept = false;
    if (kind == kOpenTail) {
      x_end = x0 == dead || x0 < 0 ? dead : walk_bytes(tb, rb, nb, x0);
    } else if (kind == kOpen) {
      // (a start that is not a candidate: the true state died before the chunk)
      const int slot = x0 == dead || x0 < 0 ? -1 : cand_slot(sm, t, x0);
      if (slot >= 0) {
        const int job = (int)sm->jfirst[t] + slot;
        if (job < kCodeJobs) {
          const uint32_t *src = sm->jcodes + job * kLexWords;
#pragma unroll
          for (int w = 0; w < kLexWords; ++w) row[w] = src[w];
          x_end = sm->lend[slot * kLexThreads + t];
        } else {
          x_end = walk_chunk(tb, row, row, x0);
        }
      }
    }
    if (nb > 0) {
      if (x_end == dead) record_reject(st, &st->lex_reject_reason, 1);
      // ---- boundaries (all) and kept boundaries (code < 0xFE, i.e.
      // (code | 1) != 0xFF) from the code words ----
      unsigned long long kmask = 0;
#pragma unroll
      for (int w = 0; w < kLexWords; ++w) {
        const uint32_t cw = row[w];
        bmask |= (unsigned long long)movemask4(nonzero_bytes(~cw)) << (4 * w);
        kmask |= (unsigned long long)movemask4(nonzero_bytes(~(cw | 0x01010101u))) << (4 * w);
      }
      if (nb < 64) {  // bytes past the input do not count
        bmask &= (1ull << nb) - 1;
        kmask &= (1ull << nb) - 1;
      }
      cnt = __popcll(kmask);
      if (bmask) lastb = g0 + 63 - __clzll((long long)bmask);
      if (g0 + nb == n && !a.open_end) {  // this chunk holds the last byte of the input
        final_kept = x_end != dead && (sm->sflags[x_end] & 4) != 0;
        if (final_kept) ++cnt;
        if (x_end == dead || !(sm->sflags[x_end] & 2)) record_reject(st, &st->lex_reject_reason, 2);
      }
    }
    // ---- (count, last boundary) carry: block scan, then across tiles ----
    int cnt_tot, pos_tot, cnt_ex, pos_ex;
    block_exclusive_scan2(sm->scan_a, sm->scan_b, (int)cnt, (int)lastb, &cnt_ex, &pos_ex, &cnt_tot, &pos_tot);
    LEX_PHASE(5);
    if (kStaged) {
      // the tile's totals and the codes of its data bytes, for the scan and
      // emit kernels (the block scan above ended with a barrier: every row
      // holds its final codes)
      if (t == 0) {
        a.tile_cnt[tile] = (uint32_t)cnt_tot;
        a.tile_pos[tile] = (uint32_t)pos_tot;
      }
      if (final_kept) {  // one chunk of the document holds its last byte
        st->final_term = sm->sterm[x_end];
        st->final_kept = 1;
      }
      uint4 *dst = reinterpret_cast<uint4 *>(a.codes + tile * (unsigned long long)kLexData);
      const uint4 *src = reinterpret_cast<const uint4 *>(reinterpret_cast<const uint8_t *>(sm->bytes) +
                                                         kLexWin);
      for (int v = t; v < kLexData / 16; v += kLexThreads) dst[v] = src[v];
      LEX_PHASE(7);
      continue;
    }
    if (t < kWarp) {
      const Pair64 agg{cnt_tot, pos_tot};
      Pair64 prefix{0, 0};
      if (lt > 0) {
        if (t == 0) publish_pair(a.st2, (long long)tile, agg, false);
        prefix = warp_lookback_pair(a.st2, (long long)tile, Pair64{0, 0}, CntPosOp(), st, kSiteLexCount);
      }
      if (t == 0) {
        const Pair64 inc = CntPosOp()(prefix, agg);
        publish_pair(a.st2, (long long)tile, inc, true);
        sm->cnt_prefix = prefix.a;
        sm->pos_prefix = prefix.b;
        if (lt + 1 == tiles_t) {
          st->num_tokens = (unsigned long long)inc.a;
          st->last_boundary = (unsigned long long)inc.b;
        }
      }
    }
    __syncthreads();
    LEX_PHASE(6);

    // ---- the kept tokens, straight into the outputs ----
    if (nb > 0) {
      unsigned long long out = tok_base + (unsigned long long)(sm->cnt_prefix + cnt_ex);
      long long prev = sm->pos_prefix > pos_ex ? sm->pos_prefix : pos_ex;  // 0: the token starts at byte 0
      const unsigned long long len_max = a.len_max;
      const unsigned long long base = a.index_base;
      bool too_long = false;
      for (unsigned long long m = bmask; m; m &= m - 1) {
        const int j = __ffsll((long long)m) - 1;
        const long long p = g0 + j;
        const uint32_t code = rb[j];
        if (code < kIgnored) {
          const unsigned long long len = (unsigned long long)(p - prev);
          too_long |= len > len_max;
          store_uint(a.tok_ids, out, a.term_w, code);
          store_uint(a.tok_starts, out, a.idx_w, base + (unsigned long long)prev);
          store_uint(a.tok_lens, out, a.len_w, len);
          ++out;
        }
        prev = p;
      }
      if (final_kept) {
        const unsigned long long len = (unsigned long long)(n - prev);
        too_long |= len > len_max;
        store_uint(a.tok_ids, out, a.term_w, sm->sterm[x_end]);
        store_uint(a.tok_starts, out, a.idx_w, base + (unsigned long long)prev);
        store_uint(a.tok_lens, out, a.len_w, len);
      }
      if (too_long) record_reject(st, &st->lex_reject_reason, 3);
    }
  }
}

}  // namespace

#undef LEX_PHASE

#define LEX_KERNEL(name, W, PS, STAGED)                          \
  __global__ void __launch_bounds__(kLexThreads, 4) name(LexArgs args) { \
    extern __shared__ __align__(16) unsigned char dyn_smem[];   \
    __shared__ __align__(16) LexSmem<W> sm;                    \
    lex_body<W, PS, STAGED>(args, dyn_smem, &sm);              \
  }

LEX_KERNEL(lex_kernel, 1, true, true)
LEX_KERNEL(lex_kernel_wide, 4, true, true)
LEX_KERNEL(lex_kernel_sets, 4, false, true)
LEX_KERNEL(lex_direct_kernel, 1, true, false)
LEX_KERNEL(lex_direct_kernel_wide, 4, true, false)
LEX_KERNEL(lex_direct_kernel_sets, 4, false, false)

#undef LEX_KERNEL

// ---------------------------------------------------------------------------
// Scan and token writes of the staged lexer
// ---------------------------------------------------------------------------

namespace {

// (count, last boundary) with segment starts: the prefix restarts at a batch
// document's first tile (flag kSeg in the position word).
constexpr long long kSeg = 1ll << 62;

struct SegCntPosOp {
  __device__ Pair64 operator()(Pair64 l, Pair64 r) const {
    if (r.b & kSeg) return r;
    const long long lp = l.b & ~kSeg;
    return Pair64{l.a + r.a, (lp > r.b ? lp : r.b) | (l.b & kSeg)};
  }
};

}  // namespace

// Exclusive (count, last boundary) prefix over the tiles, by one CTA: each
// tile's first token index (in its document's token region) and the last
// boundary before it; each document's token count and last boundary.
__global__ void __launch_bounds__(kLexScanThreads) lex_scan_kernel(LexEmitArgs a) {
  __shared__ Pair64 tmp[kLexScanThreads / 32];
  const int t = threadIdx.x;
  constexpr int kPer = 16;
  const BatchDesc *bd = a.batch;
  auto seg_doc = [&](unsigned long long i, bool *start) -> int {
    if (!bd) {
      *start = i == 0;
      return 0;
    }
    const int d = batch_doc(bd->lex_tile0, bd->docs, i);
    *start = bd->lex_tile0[d] == i;
    return d;
  };
  Pair64 carry{0, 0};
  for (unsigned long long base = 0; base < a.num_tiles; base += (unsigned long long)kLexScanThreads * kPer) {
    const unsigned long long i0 = base + (unsigned long long)t * kPer;
    Pair64 loc{0, 0};
    for (int k = 0; k < kPer && i0 + k < a.num_tiles; ++k) {
      bool start;
      seg_doc(i0 + k, &start);
      const Pair64 v{(long long)a.tile_cnt[i0 + k], (long long)a.tile_pos[i0 + k] | (start ? kSeg : 0)};
      loc = SegCntPosOp()(loc, v);
    }
    Pair64 tot;
    const Pair64 ex = block_exclusive_scan_pair(loc, SegCntPosOp(), Pair64{0, 0}, tmp, &tot);
    Pair64 run = SegCntPosOp()(carry, ex);
    for (int k = 0; k < kPer && i0 + k < a.num_tiles; ++k) {
      bool start;
      const int d = seg_doc(i0 + k, &start);
      if (start) run = Pair64{0, 0};
      const unsigned long long region = bd ? bd->tok_off[d] : 0;
      a.tile_off[i0 + k] = region + (unsigned long long)run.a;
      a.tile_prev[i0 + k] = (uint32_t)(run.b & ~kSeg);
      const long long rp = run.b & ~kSeg, tp = (long long)a.tile_pos[i0 + k];
      run = Pair64{run.a + (long long)a.tile_cnt[i0 + k], rp > tp ? rp : tp};
      if (bd && i0 + k + 1 == bd->lex_tile0[d + 1]) {  // the document's last tile
        bd->status[d].num_tokens = (unsigned long long)run.a;
        bd->status[d].last_boundary = (unsigned long long)run.b;
      }
    }
    carry = SegCntPosOp()(carry, tot);
  }
  if (t == 0 && !bd) {
    a.status->num_tokens = (unsigned long long)carry.a;
    a.status->last_boundary = (unsigned long long)(carry.b & ~kSeg);
  }
}

// The tokens of each tile from its codes: per 60-byte chunk the boundary and
// kept masks, a block scan of (count, last boundary) on top of the tile's
// prefix, then each chunk's kept tokens written at their final places with
// the length_t check (lexer.c:68-72); the input's last token (kept, ending at
// byte n) after the last chunk's.
__global__ void __launch_bounds__(256) lex_emit_kernel(LexEmitArgs a) {
  // dynamic shared memory (kLexEmitSmem bytes): two buffers of a tile's
  // codes (the next tile's are copied in while this one's are turned into
  // tokens), then a window of the tile's tokens written out by consecutive
  // threads
  extern __shared__ __align__(16) unsigned char emit_smem[];
  uint32_t(*rows2)[kLexThreads * kLexWords] = reinterpret_cast<uint32_t(*)[kLexThreads * kLexWords]>(emit_smem);
  uint32_t *s_start = reinterpret_cast<uint32_t *>(emit_smem + 2 * kLexData);
  uint32_t *s_len = s_start + kTokWin;
  uint8_t *s_id = reinterpret_cast<uint8_t *>(s_len + kTokWin);
  __shared__ int sa[8], sb[8];
  const int t = threadIdx.x;
  auto fetch = [&](unsigned long long tl, uint32_t *dst) {
    const uint8_t *src = a.codes + tl * (unsigned long long)kLexData;
    for (int v = t; v < kLexData / 16; v += kLexThreads) cp_async16(dst + 4 * v, src + 16 * v);
  };
  if (blockIdx.x < a.num_tiles) fetch(blockIdx.x, rows2[0]);
  cp_async_commit();
  int buf = 0;
  for (unsigned long long tile = blockIdx.x; tile < a.num_tiles; tile += gridDim.x, buf ^= 1) {
    long long n = (long long)a.n;
    unsigned long long lt = tile;
    DeviceStatus *st = a.status;
    if (a.batch) {
      const int d = batch_doc(a.batch->lex_tile0, a.batch->docs, tile);
      lt = tile - a.batch->lex_tile0[d];
      n = (long long)a.batch->n[d];
      st = a.batch->status + d;
    }
    // the next tile's codes into the other buffer (read by everyone for the
    // tile before this one: the barrier that ended it has passed)
    if (tile + gridDim.x < a.num_tiles) fetch(tile + gridDim.x, rows2[buf ^ 1]);
    cp_async_commit();
    cp_async_wait<1>();  // this tile's copies (all but the group just issued)
    __syncthreads();
    const uint32_t *rows = rows2[buf];
    const long long g0 = (long long)lt * kLexData + (long long)t * kLexChunk;
    int nb = 0;
    if (g0 < n) nb = (int)min((long long)kLexChunk, n - g0);
    const uint32_t *row = rows + t * kLexWords;
    const uint8_t *rb = reinterpret_cast<const uint8_t *>(row);
    unsigned long long bmask = 0, kmask = 0;
    if (nb > 0) {
#pragma unroll
      for (int w = 0; w < kLexWords; ++w) {
        const uint32_t cw = row[w];
        bmask |= (unsigned long long)movemask4(nonzero_bytes(~cw)) << (4 * w);
        kmask |= (unsigned long long)movemask4(nonzero_bytes(~(cw | 0x01010101u))) << (4 * w);
      }
      if (nb < 64) {
        bmask &= (1ull << nb) - 1;
        kmask &= (1ull << nb) - 1;
      }
    }
    const bool last = nb > 0 && g0 + nb == n;  // holds the input's last byte
    const bool final_kept = last && !a.open_end && st->final_kept;
    const int cnt = __popcll(kmask) + (final_kept ? 1 : 0);
    const int lastb = bmask ? (int)(g0 + 63 - __clzll((long long)bmask)) : 0;
    int cnt_ex, pos_ex, cnt_tot, pos_tot;
    block_exclusive_scan2(sa, sb, cnt, lastb, &cnt_ex, &pos_ex, &cnt_tot, &pos_tot);
    const unsigned long long out0 = a.tile_off[tile];
    const long long tp = (long long)a.tile_prev[tile];
    const unsigned long long len_max = a.len_max;
    const unsigned long long base = a.index_base;
    const uint32_t final_term = final_kept ? (uint32_t)st->final_term : 0u;
    bool too_long = false;
    // the tile's tokens in windows of kTokWin: each thread puts its chunk's
    // tokens that fall in the window at their places, then consecutive
    // threads write the window out (positions are < 2^31: 32-bit staging)
    for (int w0 = 0; w0 < cnt_tot; w0 += kTokWin) {
      if (nb > 0 && cnt_ex < w0 + kTokWin && cnt_ex + cnt > w0) {
        int o = cnt_ex - w0;
        long long prev = tp > pos_ex ? tp : pos_ex;  // 0: the token starts at byte 0
        for (unsigned long long m = bmask; m; m &= m - 1) {
          const int j = __ffsll((long long)m) - 1;
          const long long p = g0 + j;
          const uint32_t code = rb[j];
          if (code < kIgnored) {
            if (o >= 0 && o < kTokWin) {
              const unsigned long long len = (unsigned long long)(p - prev);
              too_long |= len > len_max;
              s_id[o] = (uint8_t)code;
              s_start[o] = (uint32_t)prev;
              s_len[o] = (uint32_t)len;
            }
            ++o;
          }
          prev = p;
        }
        if (final_kept && o >= 0 && o < kTokWin) {
          const unsigned long long len = (unsigned long long)(n - prev);
          too_long |= len > len_max;
          s_id[o] = (uint8_t)final_term;
          s_start[o] = (uint32_t)prev;
          s_len[o] = (uint32_t)len;
        }
      }
      __syncthreads();
      const int wn = cnt_tot - w0 < kTokWin ? cnt_tot - w0 : kTokWin;
      const unsigned long long ob = out0 + (unsigned long long)w0;
      for (int i = t; i < wn; i += kLexThreads) {
        store_uint(a.tok_ids, ob + i, a.term_w, s_id[i]);
        store_uint(a.tok_starts, ob + i, a.idx_w, base + s_start[i]);
        store_uint(a.tok_lens, ob + i, a.len_w, s_len[i]);
      }
      __syncthreads();
    }
    if (too_long) record_reject(st, &st->lex_reject_reason, 3);
    __syncthreads();  // this tile's rows and window are consumed
  }
  cp_async_wait<0>();
}

}  // namespace alpacc
