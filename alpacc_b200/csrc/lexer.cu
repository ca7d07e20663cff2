// Data-parallel lexer for sm_100a: the sequential semantics of lex_string
// (backends/c/lexer.c:39-97) computed tile-parallel in one kernel.
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
// rows are bank-conflict free); the first 8 chunks are a halo repeating the
// 480 bytes before the tile's 14880 data bytes, walked again so that the tile
// can almost always derive its incoming state by itself.
//
// Pass 1 (each chunk, start state unknown): the set of live states after its
//   first bytes is walked until it is one state (typically 1-4 bytes on JSON)
//   and word aligned; from there a fully unrolled single-lane walk writes each
//   byte's code over the consumed input word. Such a chunk maps every live
//   start to one end state ("constant"). A chunk whose set is not one state
//   after 16 bytes ("open") instead has each of its first byte's targets
//   walked on its own - one job per lane, spread over the whole CTA so that no
//   thread walks several lanes while the others wait - keeping the end state
//   per start lane and, for the first 64 jobs, the lane's codes.
// Resolution: each chunk's start state follows from the nearest constant chunk
//   before it; only when no halo chunk is constant does the tile read its
//   predecessor's published outgoing state (bounded look-back).
// Pass 2: each data chunk re-walks the bytes before its walk converged from
//   its true start, writing their codes; an open chunk copies its true lane's
//   codes (or walks the chunk again when its lanes had no code slots), a
//   partial chunk (the input's last) is walked whole.
// Output, staged (lex_kernel): each tile writes the codes of its data bytes
//   (16-byte stores from shared memory) and its (kept-token count, last
//   boundary); lex_scan_kernel scans the tile totals and lex_emit_kernel turns
//   each tile's codes into tokens at their final places, with the length_t
//   check of lexer.c:68-72. No tile waits for another tile's count.
// Output, direct (lex_direct_kernel, for the allocation-free entry point):
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

enum ChunkKind : uint8_t { kEmpty = 0, kConst = 1, kOpen = 2, kPartial = 3 };

constexpr uint32_t kAddrMask = 0xFFFFFFu;  // F(next) bits of an entry
constexpr uint8_t kNoBoundary = 0xFF, kIgnored = 0xFE;
// Bytes a chunk walks as a state set before it counts as open: bounds how long
// one late-converging chunk can hold its warp in the set walk.
constexpr int kSetWalk = 16;
// Lane walks of open chunks run as jobs spread over the CTA (rounds of one
// lane per thread); the first kCodeJobs keep their codes, so the chunk's
// pass 2 copies the true lane's codes instead of walking again.
constexpr int kCodeJobs = 64;

struct LexSmem {
  uint32_t bytes[kLexThreads * kLexWords];  // the tile; codes replace the consumed words
  uint8_t lend[kLexLanes * kLexThreads];    // open chunks: end state per start lane (lane-major)
  uint8_t kind[kLexThreads];
  uint8_t endst[kLexThreads];  // constant chunks: end state
  uint8_t c0[kLexThreads];     // class of the chunk's first byte
  uint8_t start[kLexThreads];  // true start state of data chunks
  uint16_t jfirst[kLexThreads];  // first lane job of each chunk (jobs of earlier chunks; none for closed ones)
  uint32_t jcodes[kCodeJobs * kLexWords];  // codes of bytes 1..59 of the first lane jobs
  uint8_t sterm[256];          // per machine state: terminal id
  uint8_t sflags[256];         // bit1 accept, bit2 kept
  int kconst[kLexThreads];
  int scan_a[kLexThreads / 32], scan_b[kLexThreads / 32];
  unsigned tile;
  int s_in;
  int need_lookback;
  int out_published;
  long long cnt_prefix, pos_prefix;
};

// The machine in shared memory: class table and entries, plus the shape
// parameters that turn a state into its row offset and back.
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

// f_t(x): the state after chunk t when it starts in state x. A constant chunk
// maps every live start to its one end state (a start whose lane died instead
// is caught when the chunk is re-walked from its true start, which then
// rejects the input); an open chunk keeps the end state of each start lane.
// A partial chunk (the input's last) is never followed by a non-empty chunk.
__device__ __forceinline__ int eval_chunk(const LexArgs &a, const LexSmem *sm, int t, int x) {
  const int kind = sm->kind[t];
  if (kind == kEmpty) return x;
  const int dead = a.dead;
  if (x == dead || x < 0) return dead;
  if (kind == kConst) return sm->endst[t];
  if (kind == kPartial) return dead;
  const int slot = __ldg(a.lane_of + (size_t)sm->c0[t] * a.M + x);
  if (slot == 0xff) return dead;
  return sm->lend[slot * kLexThreads + t];
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

// The set walk of pass 1 over W 64-bit words of states.
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
  // more than one state (no population count for a single word)
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

// Pass 1 for a full chunk: returns the chunk kind; sets *jw_out (bytes walked
// as a set, a multiple of 4: pass 2 re-walks them), the converged state at
// that point (or -1), and the end state (constant) or the per-lane end states
// in lend (open).
template <int W>
__device__ __forceinline__ int pass1_chunk(const LexArgs &a, const Tab &tb, LexSmem *sm, int t, int *jw_out,
                                           int *end_out, int *conv_out) {
  uint32_t *row = sm->bytes + t * kLexWords;
  const uint8_t *rb = reinterpret_cast<const uint8_t *>(row);
  const int dead = a.dead;
  const int c0 = (int)(cls4_of(tb, rb[0]) >> 2);
  sm->c0[t] = (uint8_t)c0;
  StateSet<W> set;
  set.clear();
  int j;
  if (W == 1 && a.img2) {  // the first two bytes at once
    set.w[0] = __ldg(a.img2 + c0 * a.C + (int)(cls4_of(tb, rb[1]) >> 2));
    j = 2;
  } else {
    const int cnt = __ldg(a.img_cnt + c0);
    for (int l = 0; l < cnt; l++) set.add(__ldg(a.img + c0 * kLexLanes + l));
    j = 1;
  }
  // walk the set until it is one state and the position is word aligned, at
  // most kSetWalk bytes
  bool many = set.many();
  while (j < kSetWalk && (many || (j & 3))) {
    const uint32_t c4 = cls4_of(tb, rb[j]);
    StateSet<W> ns;
    ns.clear();
#pragma unroll
    for (int i = 0; i < W; i++)
      for (unsigned long long m = set.w[i]; m; m &= m - 1) {
        const int s = 64 * i + __ffsll((long long)m) - 1;
        const int nx = state_of(tb, step(tb, row_of(tb, (uint32_t)s), c4));
        if (nx != dead) ns.add(nx);
      }
    set = ns;
    many = set.many();
    ++j;
  }
  *conv_out = -1;
  if (set.empty()) {  // every live start dies in this chunk
    *jw_out = j;
    *end_out = dead;
    return kConst;
  }
  if (many) {  // open: its start lanes are walked one by one as CTA-wide jobs
    *jw_out = kLexChunk;
    *end_out = -1;
    return kOpen;
  }
  const int s_conv = set.first();
  *conv_out = s_conv;
  *jw_out = j;
  if (j >= kLexChunk) {
    *end_out = s_conv;
    return kConst;
  }
  // the unrolled walk from the converged state: codes of words >= j / 4
  const uint32_t fconv = row_of(tb, (uint32_t)s_conv);
  const int jw4 = j >> 2;
  uint32_t f = fconv;
#pragma unroll
  for (int w = 0; w < kLexWords; ++w) {
    if (w == jw4) f = fconv;
    const uint32_t word = row[w];
    const uint32_t e0 = step(tb, f, cls4_of(tb, __byte_perm(word, 0, 0x4440)));
    const uint32_t e1 = step(tb, e0, cls4_of(tb, __byte_perm(word, 0, 0x4441)));
    const uint32_t e2 = step(tb, e1, cls4_of(tb, __byte_perm(word, 0, 0x4442)));
    const uint32_t e3 = step(tb, e2, cls4_of(tb, __byte_perm(word, 0, 0x4443)));
    f = e3;
    if (w >= jw4) row[w] = __byte_perm(__byte_perm(e0, e1, 0x0073), __byte_perm(e2, e3, 0x0073), 0x5410);
  }
  *end_out = state_of(tb, f);
  return kConst;
}

// One lane of an open chunk: bytes 1..59 of chunk tc's row walked from lane
// l's state (the state byte 0 leads to), end state into lend; with `codes`,
// the codes of bytes 1..59 (byte 0 left 0xFF).
__device__ __forceinline__ void walk_lane(const LexArgs &a, const Tab &tb, LexSmem *sm, int tc, int l,
                                          uint32_t *codes) {
  const uint32_t *row = sm->bytes + tc * kLexWords;
  uint32_t f = row_of(tb, __ldg(a.img + sm->c0[tc] * kLexLanes + l));
  {
    const uint32_t word = row[0];
    const uint32_t e1 = step(tb, f, cls4_of(tb, __byte_perm(word, 0, 0x4441)));
    const uint32_t e2 = step(tb, e1, cls4_of(tb, __byte_perm(word, 0, 0x4442)));
    const uint32_t e3 = step(tb, e2, cls4_of(tb, __byte_perm(word, 0, 0x4443)));
    f = e3;
    if (codes) codes[0] = __byte_perm(__byte_perm(0xFF000000u, e1, 0x0073), __byte_perm(e2, e3, 0x0073), 0x5410);
  }
#pragma unroll 2
  for (int w = 1; w < kLexWords; ++w) {
    const uint32_t word = row[w];
    const uint32_t e0 = step(tb, f, cls4_of(tb, __byte_perm(word, 0, 0x4440)));
    const uint32_t e1 = step(tb, e0, cls4_of(tb, __byte_perm(word, 0, 0x4441)));
    const uint32_t e2 = step(tb, e1, cls4_of(tb, __byte_perm(word, 0, 0x4442)));
    const uint32_t e3 = step(tb, e2, cls4_of(tb, __byte_perm(word, 0, 0x4443)));
    f = e3;
    if (codes) codes[w] = __byte_perm(__byte_perm(e0, e1, 0x0073), __byte_perm(e2, e3, 0x0073), 0x5410);
  }
  sm->lend[l * kLexThreads + tc] = (uint8_t)state_of(tb, f);
}

template <int W, bool kStaged>
__device__ __forceinline__ void lex_body(const LexArgs &a, unsigned char *dyn_smem, LexSmem *sm) {
  const int t = threadIdx.x;
  const int lane = t & 31;

  // ---- tables, once per CTA ----
  const int cls_bytes = a.wide_cls ? 512 : 256;
  uint8_t *s_cls = dyn_smem;
  uint8_t *s_ent = dyn_smem + cls_bytes;
  for (int i = t; i < cls_bytes / 4; i += kLexThreads)
    reinterpret_cast<uint32_t *>(s_cls)[i] = __ldg(reinterpret_cast<const uint32_t *>(a.cls4) + i);
  for (int i = t; i < a.tab_words; i += kLexThreads) reinterpret_cast<uint32_t *>(s_ent)[i] = __ldg(a.tab + i);
  for (int i = t; i < 256; i += kLexThreads) {
    sm->sterm[i] = i < a.M ? __ldg(a.sterm + i) : 0;
    sm->sflags[i] = i < a.M ? __ldg(a.sflags + i) : 0;
  }
  const Tab tb{s_cls, s_ent, a.wide_cls, a.cp_shift, (uint32_t)a.swz};
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
    const long long load0 = data0 - (long long)kLexHalo * kLexChunk;

    // ---- load halo + data ----
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
    const long long g0 = load0 + (long long)t * kLexChunk;
    int nb = 0;
    if (g0 >= 0 && g0 < n) nb = (int)min((long long)kLexChunk, n - g0);
    __syncthreads();
    LEX_PHASE(0);

    // ---- pass 1 ----
    int jw = nb, end = -1, conv = -1, kind = kEmpty;
    if (nb == kLexChunk) {
      kind = pass1_chunk<W>(a, tb, sm, t, &jw, &end, &conv);
    } else if (nb > 0) {
      kind = kPartial;  // the input's last chunk: walked whole in pass 2
    }
    sm->kind[t] = (uint8_t)kind;
    sm->endst[t] = (uint8_t)(end < 0 ? 0 : end);
    if (a.diag) {
      const unsigned w = __reduce_add_sync(0xffffffffu, (unsigned)(kind == kConst ? jw : nb));
      if (lane == 0) atomicAdd(&st->scratch[3], (unsigned long long)w);
    }
    // ---- open chunks: one job per start lane, spread over the CTA ----
    {
      const int lanes = kind == kOpen ? (int)__ldg(a.img_cnt + sm->c0[t]) : 0;
      int njobs;
      const int jex = block_exclusive_scan<int>(lanes, AddI32(), 0, sm->scan_a, &njobs);
      LEX_PHASE(1);
      sm->jfirst[t] = (uint16_t)jex;  // non-decreasing over the chunks (at most 256 x 32 jobs)
      __syncthreads();
      for (int job = t; job < njobs; job += kLexThreads) {
        // the job's chunk: the last chunk whose first job is <= job (a chunk
        // without lanes shares its successor's first job, so it is skipped)
        int lo = 0, hi = kLexThreads - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if ((int)sm->jfirst[mid] <= job) lo = mid;
          else hi = mid - 1;
        }
        walk_lane(a, tb, sm, lo, job - (int)sm->jfirst[lo], job < kCodeJobs ? sm->jcodes + job * kLexWords : nullptr);
      }
    }
    __syncthreads();
    LEX_PHASE(2);

    // ---- resolution: nearest constant chunk before each chunk ----
    const bool is_const = kind == kConst;
    int ktot;
    const int kex = block_exclusive_scan<int>(is_const ? t : -1, MaxI32(), -1, sm->scan_a, &ktot);
    sm->kconst[t] = kex;
    if (t == kLexHalo) sm->need_lookback = kex < 0 ? 1 : 0;
    if (t == 0) sm->out_published = 0;
    if (a.diag) {
      const int nconst = __syncthreads_count(is_const);
      if (t == 0) atomicAdd(&st->scratch[1], (unsigned long long)nconst);
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
      // no constant chunk at all: publish the data region's transition vector
      for (int s = t; s < a.M; s += kLexThreads) {
        int x = s;
        for (int jj = kLexHalo; jj < kLexThreads; ++jj) x = eval_chunk(a, sm, jj, x);
        a.st1_vec[tile * (unsigned long long)a.M + s] = (uint8_t)(x < 0 ? 0 : x);
      }
      __syncthreads();
      if (t == 0) {
        __threadfence();
        st_release_u32(a.st1_flag + tile, 1u);
      }
    }
    __syncthreads();
    if (sm->need_lookback) {
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
    // ---- each data chunk's start state ----
    unsigned chain = 0;
    if (t >= kLexHalo) {
      const int k = sm->kconst[t];
      int x, from;
      if (k >= 0) {
        x = sm->endst[k];
        from = k + 1;
      } else {
        x = sm->s_in;
        from = kLexHalo;
      }
      for (int jj = from; jj < t; ++jj) x = eval_chunk(a, sm, jj, x);
      sm->start[t] = (uint8_t)(x < 0 ? 0 : x);
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

    // ---- pass 2: the bytes walked as a set (all of an open or partial
    // chunk) again from the true start, writing their codes ----
    long long cnt = 0, lastb = 0;
    unsigned long long bmask = 0;
    bool final_kept = false;
    int x_end = 0;
    uint32_t *row = sm->bytes + t * kLexWords;
    uint8_t *rb = reinterpret_cast<uint8_t *>(row);
    if (t >= kLexHalo && nb > 0) {
      const int x0 = sm->start[t];
      bool died = x0 == dead;
      uint32_t f = row_of(tb, (uint32_t)(x0 < 0 ? 0 : x0));
      int slot = 0xff;
      if (kind == kOpen && !died) {
        slot = __ldg(a.lane_of + (size_t)sm->c0[t] * a.M + x0);
        const int job = slot == 0xff ? kCodeJobs : (int)sm->jfirst[t] + slot;
        if (job < kCodeJobs) {  // the true lane's codes, walked already: copy them
          const uint32_t e0 = step(tb, f, cls4_of(tb, rb[0]));
          const uint32_t *src = sm->jcodes + job * kLexWords;
#pragma unroll
          for (int w = 0; w < kLexWords; ++w) row[w] = src[w];
          rb[0] = g0 >= 1 ? (uint8_t)(e0 >> 24) : kNoBoundary;
          jw = 0;  // nothing left to walk
        }
      }
      if (!died) {
        for (int j = 0; j < jw; ++j) {
          const uint32_t e = step(tb, f, cls4_of(tb, rb[j]));
          rb[j] = (g0 + j >= 1) ? (uint8_t)(e >> 24) : kNoBoundary;
          f = e;
        }
        died = state_of(tb, f) == dead;
      }
      if (kind == kConst) {
        // the walk from the true start must meet the converged lane
        if (!died && conv >= 0 && state_of(tb, f) != conv) atomicCAS(&st->error, 0, -1 /* internal error */);
        x_end = died ? dead : end;
      } else if (kind == kOpen && jw == 0) {
        x_end = slot == 0xff ? dead : sm->lend[slot * kLexThreads + t];
      } else {
        x_end = died ? dead : state_of(tb, f);
      }
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
                                                         kLexHalo * kLexChunk);
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
    if (t >= kLexHalo && nb > 0) {
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

__global__ void __launch_bounds__(kLexThreads, 5) lex_kernel(LexArgs args) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ __align__(16) LexSmem sm;
  lex_body<1, true>(args, dyn_smem, &sm);
}

__global__ void __launch_bounds__(kLexThreads, 5) lex_kernel_wide(LexArgs args) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ __align__(16) LexSmem sm;
  lex_body<4, true>(args, dyn_smem, &sm);
}

__global__ void __launch_bounds__(kLexThreads, 5) lex_direct_kernel(LexArgs args) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ __align__(16) LexSmem sm;
  lex_body<1, false>(args, dyn_smem, &sm);
}

__global__ void __launch_bounds__(kLexThreads, 5) lex_direct_kernel_wide(LexArgs args) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ __align__(16) LexSmem sm;
  lex_body<4, false>(args, dyn_smem, &sm);
}

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
  __shared__ __align__(16) uint32_t rows[kLexThreads * kLexWords];
  __shared__ int sa[8], sb[8];
  const int t = threadIdx.x;
  constexpr int kChunks = kLexThreads - kLexHalo;  // data chunks per tile
  for (unsigned long long tile = blockIdx.x; tile < a.num_tiles; tile += gridDim.x) {
    long long n = (long long)a.n;
    unsigned long long lt = tile;
    DeviceStatus *st = a.status;
    if (a.batch) {
      const int d = batch_doc(a.batch->lex_tile0, a.batch->docs, tile);
      lt = tile - a.batch->lex_tile0[d];
      n = (long long)a.batch->n[d];
      st = a.batch->status + d;
    }
    __syncthreads();  // the previous tile's rows are consumed
    const uint4 *src = reinterpret_cast<const uint4 *>(a.codes + tile * (unsigned long long)kLexData);
    for (int v = t; v < kLexData / 16; v += kLexThreads) reinterpret_cast<uint4 *>(rows)[v] = src[v];
    __syncthreads();
    const long long g0 = (long long)lt * kLexData + (long long)t * kLexChunk;
    int nb = 0;
    if (t < kChunks && g0 < n) nb = (int)min((long long)kLexChunk, n - g0);
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
    if (nb > 0) {
      unsigned long long out = a.tile_off[tile] + (unsigned long long)cnt_ex;
      const long long tp = (long long)a.tile_prev[tile];
      long long prev = tp > pos_ex ? tp : pos_ex;  // 0: the token starts at byte 0
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
        store_uint(a.tok_ids, out, a.term_w, (unsigned long long)st->final_term);
        store_uint(a.tok_starts, out, a.idx_w, base + (unsigned long long)prev);
        store_uint(a.tok_lens, out, a.len_w, len);
      }
      if (too_long) record_reject(st, &st->lex_reject_reason, 3);
    }
  }
}

}  // namespace alpacc
