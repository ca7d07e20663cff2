// Data-parallel LLP parser for sm_100a: the semantics of parse_test,
// compute_parents and compact_tree (backends/c/parser.c:49-153).
//
// pair_kernel     per token position: the (q, k) key around it, a dense-table
//                 lookup of its stack actions and productions, and the scatter
//                 of both into flat arrays at offsets from a decoupled
//                 look-back scan (backends/c/parser.c:60-84; the reference's
//                 CUDA form: backends/cuda/parser.cu:378-449, phases A-C).
// pse_tile_kernel depth walk over brackets (+1 left, -1 right) or productions
//                 (+arity-1), with the match of each right bracket / the parent
//                 of each production found as the previous element whose depth
//                 is <= a query value, inside the tile; parents found are
//                 written straight into the compacted tree (compact_tree). Each
//                 tile stores its staircase (the elements a later query can
//                 find) and the queries it could not answer
//                 (backends/c/parser.c:74-87,103-118,126-153).
// pse_resolve     one warp per tile with queries: 32 queries at a time walk
//                 back over tile minima (super-tile minima skip long runs) and
//                 binary-search the answering tile's staircase, then emit the
//                 same outputs.
#include <climits>
#include <cstdint>

#include "common.cuh"
#include "kernels.h"

namespace alpacc {

namespace {

__device__ __forceinline__ unsigned long long load_uint(const void *base, unsigned long long i, int w) {
  switch (w) {
    case 1: return static_cast<const uint8_t *>(base)[i];
    case 2: return static_cast<const uint16_t *>(base)[i];
    case 4: return static_cast<const uint32_t *>(base)[i];
    default: return static_cast<const unsigned long long *>(base)[i];
  }
}

__device__ __forceinline__ void store_uint(void *base, unsigned long long i, int w, unsigned long long v) {
  switch (w) {
    case 1: static_cast<uint8_t *>(base)[i] = (uint8_t)v; break;
    case 2: static_cast<uint16_t *>(base)[i] = (uint16_t)v; break;
    case 4: static_cast<uint32_t *>(base)[i] = (uint32_t)v; break;
    default: static_cast<unsigned long long *>(base)[i] = v; break;
  }
}

struct AddPair {
  __device__ Pair64 operator()(Pair64 e, Pair64 l) const { return Pair64{e.a + l.a, e.b + l.b}; }
};

}  // namespace

// ---------------------------------------------------------------------------
// Pair lookup and expansion
// ---------------------------------------------------------------------------

// The tile's terminals (with the q before and k - 1 after it) are staged in
// shared memory once; keys are formed there with positions strided across the
// threads (conflict-free), the per-position counts are scanned in blocked
// order (one packed 64-bit scan of (brackets, productions)), and the tile's
// stack actions, then its productions, are assembled in a shared-memory
// window and written with consecutive threads (a thread's own runs would
// cost one memory transaction per element).
__global__ void __launch_bounds__(kPairThreads, 5) pair_kernel(PairArgs a) {
  __shared__ unsigned s_tile;
  __shared__ long long s_tmp[kPairThreads / 32];
  __shared__ long long s_prefix_b, s_prefix_p;
  __shared__ uint16_t s_term[kPairTile + 8];             // window of terminals; 0xffff = out of range
  __shared__ __align__(16) uint32_t s_rec[kPairTile];    // record per position
  __shared__ __align__(16) uint16_t s_cnt[kPairTile];    // brackets | productions << 8
  __shared__ __align__(16) uint32_t s_out[kPairOut];     // output window
  __shared__ int s_wstep[8], s_wterm[8];                 // the window's walk-tile aggregates
  const int t = threadIdx.x;
  const int lane = t & (kWarp - 1);
  const int L = a.q + a.k;
  const unsigned long long *rec = a.rec;
  const uint32_t *stacks = a.stacks, *prods = a.prods;
  unsigned long long total;
  if (a.batch) {
    total = a.batch->pair_tile0[a.batch->docs];
  } else {
    // the lexer rejected: nothing to expand (one read, shared by the CTA:
    // this kernel's own rejects may land meanwhile)
    if (__syncthreads_or(t == 0 && *reinterpret_cast<volatile int *>(&a.status->reject) != 0)) return;
    total = (*a.num_tokens + 2 + kPairTile - 1) / kPairTile;
    if (total > a.tiles_cap) {
      if (t == 0 && blockIdx.x == 0) record_overflow(a.status);
      return;
    }
  }
  for (;;) {
  __syncthreads();  // the previous tile's shared data is consumed
  if (t == 0) s_tile = atomicAdd(a.ticket, 1u);
  __syncthreads();
  const unsigned long long tile = s_tile;  // virtual tile in a batch
  if (tile >= total) break;
  // this tile's document
  unsigned long long lt = tile;
  const void *tok_ids = a.tok_ids;
  uint32_t *br_base = a.br_out, *pr_base = a.pr_out;
  unsigned long long br_cap = a.br_cap, pr_cap = a.pr_cap;
  DeviceStatus *st = a.status;
  long long T;
  if (a.batch) {
    const BatchDesc &b = *a.batch;
    const int d = batch_doc(b.pair_tile0, b.docs, tile);
    lt = tile - b.pair_tile0[d];
    st = b.status + d;
    T = (long long)st->num_tokens;
    tok_ids = static_cast<const uint8_t *>(a.tok_ids) + b.tok_off[d] * (unsigned long long)a.term_w;
    br_base = a.br_out + b.br_off[d];
    pr_base = a.pr_out + b.pr_off[d];
    br_cap = b.br_off[d + 1] - b.br_off[d];
    pr_cap = b.pr_off[d + 1] - b.pr_off[d];
  } else {
    T = (long long)*a.num_tokens;
  }
  const long long m = T + 2;
  const long long tile0 = (long long)lt * kPairTile;
  if (tile0 >= m) continue;  // beyond the data: nobody waits on this tile

  // ---- terminals of positions tile0 - q .. tile0 + kPairTile + k - 2 ----
  for (int i = t; i < kPairTile + L - 1; i += kPairThreads) {
    const long long pos = tile0 - a.q + i;
    int term;
    if (pos < 0 || pos >= m) term = a.empty_t;
    else if (pos == 0) term = a.start_t;
    else if (pos == m - 1) term = a.end_t;
    else term = (int)load_uint(tok_ids, (unsigned long long)(pos - 1), a.term_w);
    s_term[i] = (unsigned)term < (unsigned)a.nt ? (uint16_t)term : (uint16_t)0xffff;
  }
  __syncthreads();

  // ---- keys and records, positions strided over the threads ----
  bool missing = false;
#pragma unroll
  for (int j = 0; j < kPairItems; ++j) {
    const int li = j * kPairThreads + t;
    uint32_t r = 0xffffffffu;
    if (tile0 + li < m) {
      bool bad = false;
      if (a.dense) {
        unsigned long long d = 0;
        for (int x = 0; x < L; ++x) {
          const unsigned term = s_term[li + x];
          bad |= term == 0xffffu;  // keeps the table index in bounds
          d = d * (unsigned long long)a.nt + term;
        }
        r = bad ? 0xffffffffu : __ldg(a.dense + d);
      } else {
        // lookup_key (parser.c:30-45): FNV-1a over the key's terminals, linear
        // probing from hash % size for at most MAX_ITERS slots; the first slot
        // holding the key decides
        unsigned long long h = 14695981039346656037ull, key = 0;
        for (int x = 0; x < L; ++x) {
          const unsigned term = s_term[li + x];
          bad |= term == 0xffffu;  // an id outside the grammar is never a key
          h = (h ^ (unsigned long long)term) * 1099511628211ull;
          key |= (unsigned long long)(term & 0xffu) << (8 * x);
        }
        if (!bad) {
          h %= a.ht_size;
          for (unsigned long long it = 0; it < a.max_iters; ++it) {
            const uint32_t rr = __ldg(a.ht_rec + h);
            if (rr != kEmptySlot && __ldg(a.ht_key + h) == key) {
              r = rr == kMissingKey ? 0xffffffffu : rr;
              break;
            }
            h = h + 1 == a.ht_size ? 0 : h + 1;
          }
        }
      }
      if (r == 0xffffffffu) missing = true;
    }
    s_rec[li] = r;
    s_cnt[li] = r == 0xffffffffu ? (uint16_t)0 : (uint16_t)(rec[r] >> 48);
  }
  if (missing) record_reject(st, &st->parse_reject_reason, 1);
  __syncthreads();

  // ---- blocked counts: thread t owns positions t*8 .. t*8+7 ----
  uint16_t cnt[kPairItems];
  {
    const uint4 cv = reinterpret_cast<const uint4 *>(s_cnt)[t];
    cnt[0] = cv.x & 0xffff; cnt[1] = cv.x >> 16; cnt[2] = cv.y & 0xffff; cnt[3] = cv.y >> 16;
    cnt[4] = cv.z & 0xffff; cnt[5] = cv.z >> 16; cnt[6] = cv.w & 0xffff; cnt[7] = cv.w >> 16;
  }
  long long sb = 0, sp = 0;
#pragma unroll
  for (int j = 0; j < kPairItems; ++j) {
    sb += cnt[j] & 0xff;
    sp += cnt[j] >> 8;
  }
  long long tot;
  const long long ex = block_exclusive_scan<long long>((sb << 32) + sp, AddI64(), 0ll, s_tmp, &tot);
  const long long tb = tot >> 32, tp = tot & 0xffffffffll;
  if (t < kWarp) {
    const Pair64 agg{tb, tp};
    Pair64 prefix{0, 0};
    if (lt > 0) {
      if (t == 0) publish_pair(a.st, (long long)tile, agg, false);
      prefix = warp_lookback_pair(a.st, (long long)tile, Pair64{0, 0}, AddPair(), st, kSitePairs);
    }
    if (t == 0) {
      const Pair64 inc{prefix.a + agg.a, prefix.b + agg.b};
      publish_pair(a.st, (long long)tile, inc, true);
      s_prefix_b = prefix.a;
      s_prefix_p = prefix.b;
      if (tile0 + kPairTile >= m) {  // last data tile
        st->num_brackets = (unsigned long long)inc.a;
        st->num_productions = (unsigned long long)inc.b;
      }
    }
  }
  __syncthreads();
  const long long pre_b = s_prefix_b, pre_p = s_prefix_p;
  if ((unsigned long long)(pre_b + tb) > br_cap || (unsigned long long)(pre_p + tp) > pr_cap) {
    if (t == 0) record_overflow(st);
    continue;
  }
  // ---- brackets (pass 0) and productions (pass 1) through the output window ----
  for (int pass = 0; pass < 2; ++pass) {
    const long long total = pass == 0 ? tb : tp;
    const long long base = pass == 0 ? (ex >> 32) : (ex & 0xffffffffll);
    const uint32_t *src = pass == 0 ? stacks : prods;
    uint32_t *dst = pass == 0 ? br_base + pre_b : pr_base + pre_p;
    for (long long w0 = 0; w0 < total; w0 += kPairOut) {
      long long o = base;
#pragma unroll
      for (int j = 0; j < kPairItems; ++j) {
        const int c = pass == 0 ? (cnt[j] & 0xff) : (cnt[j] >> 8);
        if (c == 0) continue;
        const unsigned long long rc = rec[s_rec[t * kPairItems + j]];
        const uint32_t sidx = (uint32_t)((pass == 0 ? rc : rc >> 24) & 0xffffffu);
        for (int x = 0; x < c; ++x) {
          const long long q = o + x - w0;
          if (q >= 0 && q < kPairOut) s_out[q] = src[sidx + x];
        }
        o += c;
      }
      if (t < 8) {
        s_wstep[t] = 0;
        s_wterm[t] = 0;
      }
      __syncthreads();
      const int wn = (int)(total - w0 < kPairOut ? total - w0 : kPairOut);
      int *wstep = a.walk_step[pass];
      if (!wstep) {
        for (int i = t; i < wn; i += kPairThreads) dst[w0 + i] = s_out[i];
      } else {
        // also the walk tiles' aggregates: a warp's 32 consecutive elements
        // lie in at most two walk tiles (reduced per tile in the warp, then
        // added in shared memory: slots of the window's at most 4 tiles)
        const long long gbase = (pass == 0 ? pre_b : pre_p) + w0;  // element index of s_out[0]
        const long long tfirst = gbase / kPseTile;
        for (int i0 = 0; i0 < wn; i0 += kPairThreads) {
          const int i = i0 + t;
          const bool in = i < wn;
          int stp = 0, trm = 0, slot = 0;
          if (in) {
            const uint32_t v = s_out[i];
            dst[w0 + i] = v;
            if (pass == 0) {
              stp = (v >> 31) ? 1 : -1;
            } else {
              stp = __ldg(a.arity + v) - 1;
              trm = __ldg(a.is_term + v) ? 1 : 0;
            }
            slot = (int)((gbase + i) / kPseTile - tfirst);
          }
          const int s0 = __shfl_sync(0xffffffffu, slot, 0);
          const bool same = slot == s0;
          const int sa = __reduce_add_sync(0xffffffffu, same ? stp : 0);
          const int sb = __reduce_add_sync(0xffffffffu, same ? 0 : stp);
          const int ta = __reduce_add_sync(0xffffffffu, same ? trm : 0);
          const int tb2 = __reduce_add_sync(0xffffffffu, same ? 0 : trm);
          const bool two = __any_sync(0xffffffffu, in && !same);
          if (lane == 0) {
            atomicAdd(&s_wstep[s0], sa);
            atomicAdd(&s_wterm[s0], ta);
            if (two) {
              atomicAdd(&s_wstep[s0 + 1], sb);
              atomicAdd(&s_wterm[s0 + 1], tb2);
            }
          }
        }
        __syncthreads();
        if (t < 8 && tfirst + t < (long long)a.walk_tiles_cap && (s_wstep[t] != 0 || s_wterm[t] != 0)) {
          atomicAdd(wstep + tfirst + t, s_wstep[t]);
          if (pass == 1) atomicAdd(a.walk_term + tfirst + t, s_wterm[t]);
        }
      }
      __syncthreads();
    }
  }
  }  // tiles
}

// Exclusive prefixes of the walk tiles' aggregates, both walks, by one CTA.
__global__ void __launch_bounds__(1024) walk_prefix_kernel(WalkPrefixArgs a) {
  __shared__ long long tmp[32];
  const int t = threadIdx.x;
  if (*reinterpret_cast<volatile int *>(&a.status->reject) || *reinterpret_cast<volatile int *>(&a.status->overflow))
    return;  // the walks do not run
  constexpr int kPer = 16;
  for (int walk = 0; walk < 2; ++walk) {
    const unsigned long long E = walk == 0 ? a.status->num_brackets : a.status->num_productions;
    const unsigned long long tiles = (E + kPseTile - 1) / kPseTile;
    if (tiles > a.tiles_cap) continue;  // the walk kernel records the overflow
    const int *stp = a.walk_step[walk];
    long long carry = 0;
    for (unsigned long long base = 0; base < tiles; base += 1024ull * kPer) {
      const unsigned long long i0 = base + (unsigned long long)t * kPer;
      // (step sum, terminal count) packed: the count is non-negative and < 2^32
      long long loc = 0;
      for (int k = 0; k < kPer && i0 + k < tiles; ++k)
        loc += (long long)stp[i0 + k] * (1ll << 32) + (walk == 1 ? (long long)a.walk_term[i0 + k] : 0);
      long long tot;
      long long run = carry + block_exclusive_scan<long long>(loc, AddI64(), 0ll, tmp, &tot);
      for (int k = 0; k < kPer && i0 + k < tiles; ++k) {
        const long long tc = run & 0xffffffffll;  // exact while the running count stays below 2^32
        a.prefix_s[walk][i0 + k] = (run - tc) >> 32;
        if (walk == 1) a.prefix_t[i0 + k] = tc;
        run += (long long)stp[i0 + k] * (1ll << 32) + (walk == 1 ? (long long)a.walk_term[i0 + k] : 0);
      }
      carry += tot;
    }
  }
}

// ---------------------------------------------------------------------------
// Previous-smaller search over depth walks
// ---------------------------------------------------------------------------

namespace {

constexpr int kPseStride = kPseItems + 1;  // odd word stride: conflict-free per-thread rows
constexpr int kPseWarps = kPseThreads / kWarp;
constexpr long long kPack = 1ll << 32;     // (step sum, terminal count) packed in one scan value

struct PseSmem {
  uint32_t v[kPseThreads * kPseStride];
  int32_t h[kPseThreads * kPseStride];   // depth before each element, relative to the tile start
  int32_t tc[kPseThreads * kPseStride];  // parents: inclusive terminal count, relative to the tile start
  int32_t lv[6][kPseThreads];            // lv[k][i]: minimum of chunk minima over (i - 2^k, i] within i's warp
  int32_t wmin[kPseWarps];               // minimum of each warp's chunk minima
  union {
    struct {
      uint16_t wq[kPseTile];    // per warp: its pending queries (element index in the tile)
      int16_t wans[kPseTile];   // answer of a pending query (element index), or -1
    };
    int32_t pnew[kPseTile];     // parents, after the queries: each element's tree parent, or kNoParent
  };
  long long tmp[kPseWarps];
  long long prefix_a, prefix_b;
};

constexpr int kPseSmemProds = 1024;  // production tables copied to shared memory up to this size
constexpr int32_t kNoParent = INT_MIN;  // the element's parent is found by the resolve kernel

// compact_tree's output for production e (parser.c:126-153): terminal
// productions give their token's parent, the others a tree node; parents are
// renumbered by subtracting the terminal productions before them.
// One document's view of the walk's arrays (a batch document, or the input).
struct PseDoc {
  const uint32_t *elems;
  long long E, T;
  unsigned long long tile_first;  // virtual index of the document's first tile
  void *node_prods, *node_parents, *token_parents;
  DeviceStatus *st;
};

__device__ __forceinline__ PseDoc pse_doc(const PseArgs &a, unsigned long long vt, int *doc) {
  PseDoc v;
  if (!a.batch) {
    *doc = 0;
    v.elems = a.elems;
    v.E = (long long)*a.count;
    v.T = (long long)*a.num_tokens;
    v.tile_first = 0;
    v.node_prods = a.node_prods;
    v.node_parents = a.node_parents;
    v.token_parents = a.token_parents;
    v.st = a.status;
    return v;
  }
  const BatchDesc &b = *a.batch;
  const bool parents = a.mode == kPseParents;
  const unsigned long long *tile0 = parents ? b.pr_tile0 : b.br_tile0;
  const int d = batch_doc(tile0, b.docs, vt);
  *doc = d;
  v.st = b.status + d;
  v.E = (long long)(parents ? v.st->num_productions : v.st->num_brackets);
  v.T = (long long)v.st->num_tokens;
  v.elems = a.elems + (parents ? b.pr_off[d] : b.br_off[d]);
  v.tile_first = tile0[d];
  v.node_prods = static_cast<uint8_t *>(a.node_prods) + b.pr_off[d] * (unsigned long long)a.prod_w;
  v.node_parents = static_cast<uint8_t *>(a.node_parents) + b.pr_off[d] * (unsigned long long)a.idx_w;
  v.token_parents = static_cast<uint8_t *>(a.token_parents) + b.tok_off[d] * (unsigned long long)a.idx_w;
  return v;
}

__device__ __forceinline__ void emit_node(const PseArgs &a, const PseDoc &dv, uint32_t prod, bool term, long long e,
                                          long long tinc_e, long long p_new) {
  if (term) {
    if (tinc_e >= 1 && tinc_e <= dv.T)
      store_uint(dv.token_parents, (unsigned long long)(tinc_e - 1), a.idx_w, (unsigned long long)p_new);
  } else {
    const long long o = e - tinc_e;
    if (o >= 0) {
      store_uint(dv.node_prods, (unsigned long long)o, a.prod_w, prod);
      store_uint(dv.node_parents, (unsigned long long)o, a.idx_w, (unsigned long long)p_new);
    }
  }
}

}  // namespace

// One tile of 2048 elements: depth walk, then each query (a right bracket's
// match, a production's parent) searched as the latest earlier element whose
// depth is <= the query value - first in the thread's own chunk and the
// previous one, then (the warp's pending queries through a shared queue, 32
// at a time) in earlier chunks of the warp by binary descent over window
// minima, then in earlier warps. The tile's prefix (global depth and terminal
// count before it) comes from a decoupled look-back over the preceding tiles,
// or from walk_prefix_kernel. The tile then stores its staircase and the
// queries it could not answer for pse_resolve_kernel; parents found here are
// written straight into the compacted tree.
__global__ void __launch_bounds__(kPseThreads, 4) pse_tile_kernel(PseArgs a) {
  __shared__ unsigned s_tile;
  __shared__ PseSmem sm;
  __shared__ int32_t s_arity[kPseSmemProds];
  __shared__ uint8_t s_is_term[kPseSmemProds];
  const int t = threadIdx.x;
  const int lane = t & (kWarp - 1);
  const int warp = t >> 5;
  const bool parents = a.mode == kPseParents;
  const bool prod_smem = parents && a.num_prods <= kPseSmemProds;
  if (prod_smem)
    for (int i = t; i < a.num_prods; i += kPseThreads) {
      s_arity[i] = __ldg(a.arity + i);
      s_is_term[i] = __ldg(a.is_term + i);
    }
  unsigned long long *pcyc = a.phase_cycles;
  long long tp = clock64();
// diagnostics: thread 0 adds the cycles since the previous mark to phase k
#define PSE_PHASE(k)                                        \
  if (pcyc && t == 0) {                                     \
    const long long now_ = clock64();                       \
    atomicAdd(pcyc + (k), (unsigned long long)(now_ - tp)); \
    tp = now_;                                              \
  }
  unsigned long long total;
  if (a.batch) {
    total = (parents ? a.batch->pr_tile0 : a.batch->br_tile0)[a.batch->docs];
  } else {
    // already rejected, or the pair stage overflowed: nothing to find (one
    // read, shared by the CTA)
    if (__syncthreads_or(t == 0 && (*reinterpret_cast<volatile int *>(&a.status->reject) != 0 ||
                                    *reinterpret_cast<volatile int *>(&a.status->overflow) != 0)))
      return;
    const unsigned long long E = *a.count;
    if (E > a.elem_cap) {
      if (t == 0 && blockIdx.x == 0) record_overflow(a.status);
      return;
    }
    total = (E + kPseTile - 1) / kPseTile;
  }
  for (;;) {
  __syncthreads();  // the previous tile's shared data is consumed
  PSE_PHASE(7);
  if (t == 0) s_tile = atomicAdd(a.ticket, 1u);
  __syncthreads();
  const unsigned long long tile = s_tile;  // virtual tile in a batch
  if (tile >= total) break;
  int doc;
  const PseDoc dv = pse_doc(a, tile, &doc);
  DeviceStatus *st = dv.st;
  const long long E = dv.E;
  const unsigned long long lt = tile - dv.tile_first;
  const long long tile0 = (long long)lt * kPseTile;  // elements are indexed within the document
  if (tile0 >= E) continue;
  if (t == 0 && !a.batch && tile0 + (long long)gridDim.x * kPseTile < E) {
    // warm L2 with the elements of the tile a CTA takes about one tile time
    // from now (tickets go out in order)
    const long long e0 = tile0 + (long long)gridDim.x * kPseTile;
    const long long e1 = min(E, e0 + (long long)kPseTile);
    prefetch_l2(dv.elems + e0, (unsigned long long)(e1 - e0) * 4);
  }
  const long long c0 = tile0 + (long long)t * kPseItems;  // first element of this thread's chunk

  // ---- load ----
  uint32_t v[kPseItems];
  const bool vec = ((reinterpret_cast<uintptr_t>(dv.elems + c0) & 15) == 0);
  if (c0 + kPseItems <= E && vec) {
    const uint4 x0 = __ldg(reinterpret_cast<const uint4 *>(dv.elems + c0));
    const uint4 x1 = __ldg(reinterpret_cast<const uint4 *>(dv.elems + c0) + 1);
    v[0] = x0.x; v[1] = x0.y; v[2] = x0.z; v[3] = x0.w;
    v[4] = x1.x; v[5] = x1.y; v[6] = x1.z; v[7] = x1.w;
  } else {
#pragma unroll
    for (int j = 0; j < kPseItems; ++j) v[j] = c0 + j < E ? dv.elems[c0 + j] : 0u;
  }

  // ---- local steps, one packed scan ----
  int hr[kPseItems], tcr[kPseItems];
  int ssum = 0, tsum = 0;
#pragma unroll
  for (int j = 0; j < kPseItems; ++j) {
    hr[j] = ssum;
    if (c0 + j < E) {
      if (!parents) {
        ssum += (v[j] >> 31) ? 1 : -1;
      } else if (prod_smem && v[j] < kPseSmemProds) {
        ssum += s_arity[v[j]] - 1;
        tsum += s_is_term[v[j]];
      } else {
        ssum += __ldg(a.arity + v[j]) - 1;
        tsum += __ldg(a.is_term + v[j]) ? 1 : 0;
      }
    }
    tcr[j] = tsum;
  }
  long long tot;
  const long long ex = block_exclusive_scan<long long>((long long)ssum * kPack + tsum, AddI64(), 0ll, sm.tmp, &tot);
  const int ex_t = (int)(ex & 0xffffffffll);
  const int ex_s = (int)((ex - ex_t) >> 32);
  const long long tot_t = tot & 0xffffffffll;
  const long long tot_s = (tot - tot_t) >> 32;
  // publish the aggregate at once; tile 0's aggregate is its inclusive prefix
  if (t == 0 && !a.prefix_s) publish_pair(a.st, (long long)tile, Pair64{tot_s, tot_t}, lt == 0);
  PSE_PHASE(0);

  // ---- relative depths, chunk minimum, warp windows ----
  int cmin = INT_MAX;
#pragma unroll
  for (int j = 0; j < kPseItems; ++j) {
    hr[j] += ex_s;
    if (c0 + j < E && hr[j] < cmin) cmin = hr[j];
    sm.v[t * kPseStride + j] = v[j];
    sm.h[t * kPseStride + j] = hr[j];
    if (parents) sm.tc[t * kPseStride + j] = ex_t + tcr[j];
  }
  int L[6];
  L[0] = cmin;
#pragma unroll
  for (int k = 1; k < 6; ++k) {
    const int o = __shfl_up_sync(0xffffffffu, L[k - 1], 1 << (k - 1));
    L[k] = (lane >= (1 << (k - 1)) && o < L[k - 1]) ? o : L[k - 1];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) sm.lv[k][t] = L[k];
  if (lane == kWarp - 1) sm.wmin[warp] = L[5];
  __syncthreads();
  PSE_PHASE(1);

  // ---- queries: own chunk, then the previous chunk ----
  // ans: local index of the answer; -1 pending; -2 no query; -3 the root
  int ans[kPseItems];
  unsigned need = 0;
  const int prev_min = t > 0 ? sm.lv[0][t - 1] : INT_MAX;  // minimum depth of the previous chunk
#pragma unroll
  for (int j = 0; j < kPseItems; ++j) {
    ans[j] = -2;
    const long long e = c0 + j;
    if (e >= E) continue;
    int qv;
    if (parents) {
      if (e == 0) {
        ans[j] = -3;
        continue;
      }
      qv = hr[j];
    } else {
      if (v[j] >> 31) continue;  // left bracket: no query
      qv = hr[j] - 1;
    }
    int f = 0;
    bool got = false;
    uint32_t pv = 0;
#pragma unroll
    for (int jj = 0; jj < j; ++jj)
      if (hr[jj] <= qv) {
        f = jj;
        pv = v[jj];
        got = true;
      }
    if (!got && prev_min <= qv) {  // the latest candidate lies in the previous chunk
#pragma unroll
      for (int jj = kPseItems - 1; jj >= 0; --jj)
        if (!got && sm.h[(t - 1) * kPseStride + jj] <= qv) {
          f = jj - kPseItems;
          pv = sm.v[(t - 1) * kPseStride + jj];
          got = true;
        }
    }
    if (got) {
      ans[j] = t * kPseItems + f;
      if (!parents && ((pv ^ v[j]) & 0x7fffffffu)) record_reject(st, &st->parse_reject_reason, 2);
    } else {
      ans[j] = -1;
      need |= 1u << j;
    }
  }
  PSE_PHASE(2);
  // ---- earlier chunks of the tile: the warp's pending queries, 32 at a
  // time (one per lane, whichever thread they came from) ----
  {
    const int pend = __popc(need);
    const int incl = warp_inclusive_scan(pend, [](int x, int y) { return x + y; });
    const int total_w = __shfl_sync(0xffffffffu, incl, kWarp - 1);
    if (total_w) {  // warp-uniform
      uint16_t *q = sm.wq + warp * (kWarp * kPseItems);
      int slot = incl - pend;
      for (unsigned m = need; m; m &= m - 1) q[slot++] = (uint16_t)(t * kPseItems + __ffs(m) - 1);
      __syncwarp();
      for (int i = lane; i < total_w; i += kWarp) {
        const int e = q[i];
        const int ct = e / kPseItems;  // its chunk (thread)
        const int qv = sm.h[ct * kPseStride + e % kPseItems] - (parents ? 0 : 1);
        int found = -1;
        // chunks of this warp before the previous one (checked already): the
        // latest whose minimum is <= qv, by binary descent over the windows
        int pos = ct - warp * kWarp - 2;
        if (pos >= 0 && sm.lv[5][warp * kWarp + pos] <= qv) {
#pragma unroll
          for (int k = 4; k >= 0; --k)
            if (pos >= (1 << k) && sm.lv[k][warp * kWarp + pos] > qv) pos -= 1 << k;
          const int pl = warp * kWarp + pos;
#pragma unroll
          for (int jj = kPseItems - 1; jj >= 0; --jj)
            if (found < 0 && sm.h[pl * kPseStride + jj] <= qv) found = pl * kPseItems + jj;
        }
        // then earlier warps of the tile
        for (int w = warp - 1; w >= 0 && found < 0; --w) {
          if (sm.wmin[w] > qv) continue;
          int p = w * kWarp + kWarp - 1;
#pragma unroll
          for (int k = 4; k >= 0; --k)
            if (sm.lv[k][p] > qv && p - (1 << k) >= w * kWarp) p -= 1 << k;
#pragma unroll
          for (int jj = kPseItems - 1; jj >= 0; --jj)
            if (found < 0 && sm.h[p * kPseStride + jj] <= qv) found = p * kPseItems + jj;
        }
        if (found >= 0 && !parents) {
          const uint32_t pv = sm.v[(found / kPseItems) * kPseStride + found % kPseItems];
          if ((pv ^ sm.v[ct * kPseStride + e % kPseItems]) & 0x7fffffffu)
            record_reject(st, &st->parse_reject_reason, 2);
        }
        sm.wans[e] = (int16_t)found;
      }
      __syncwarp();
#pragma unroll
      for (int j = 0; j < kPseItems; ++j)
        if (need >> j & 1u) ans[j] = sm.wans[t * kPseItems + j];
    }
  }

  PSE_PHASE(3);
  // ---- the tile's prefix: look-back by warp 0, now that predecessors had time ----
  // (or read from walk_prefix_kernel's output)
  if (t < kWarp) {
    Pair64 prefix{0, 0};
    if (a.prefix_s) {
      if (t == 0) prefix = Pair64{a.prefix_s[tile], parents ? a.prefix_t[tile] : 0ll};
    } else if (lt > 0) {
      prefix = warp_lookback_pair(a.st, (long long)tile, Pair64{0, 0}, AddPair(), st, kSitePse);
    }
    if (t == 0) {
      const Pair64 inc{prefix.a + tot_s, prefix.b + tot_t};
      if (lt > 0 && !a.prefix_s) publish_pair(a.st, (long long)tile, inc, true);
      sm.prefix_a = prefix.a;
      sm.prefix_b = prefix.b;
      if (tile0 + kPseTile >= E) {  // last tile: global checks
        if (!parents) {
          if (inc.a != 0) record_reject(st, &st->parse_reject_reason, 3);
        } else {
          if (inc.b != dv.T) record_reject(st, &st->parse_reject_reason, 4);
          st->num_nodes = (unsigned long long)(E - inc.b);
        }
      }
    }
  }
  __syncthreads();

  PSE_PHASE(4);
  // ---- staircase, unanswered queries, tile minimum ----
  // An element is on the staircase when every later element of the tile is
  // deeper: only those can answer a later tile's query. In position order the
  // stairs' depths increase and the unanswered queries' values decrease.
  const int32_t off = (int32_t)((parents ? 1 : 0) + sm.prefix_a);
  const long long pb = sm.prefix_b;
  {
    int suf = cmin;  // minimum over this warp's chunks from this one on
#pragma unroll
    for (int d = 1; d < kWarp; d <<= 1) {
      const int o = __shfl_down_sync(0xffffffffu, suf, d);
      if (lane + d < kWarp && o < suf) suf = o;
    }
    int later = __shfl_down_sync(0xffffffffu, suf, 1);  // minimum over the later chunks of the tile
    if (lane == kWarp - 1) later = INT_MAX;
    for (int w = warp + 1; w < kPseWarps; ++w) later = sm.wmin[w] < later ? sm.wmin[w] : later;
    // (depths, values and terminal counts are read back from shared memory:
    // fewer registers live across the look-back)
    const int row = t * kPseStride;
    unsigned smask = 0, qmask = 0;
#pragma unroll
    for (int j = kPseItems - 1; j >= 0; --j) {
      const int h = sm.h[row + j];
      if (c0 + j < E && h < later) {
        smask |= 1u << j;
        later = h;
      }
      if (ans[j] == -1) qmask |= 1u << j;
    }
    long long ctot;
    const long long cex = block_exclusive_scan<long long>((long long)__popc(smask) * kPack + __popc(qmask), AddI64(),
                                                          0ll, sm.tmp, &ctot);
    const unsigned long long base = tile * (unsigned long long)kPseTile;
    unsigned long long si = base + (unsigned long long)(cex >> 32);
    unsigned long long qi = base + (unsigned long long)(cex & 0xffffffffll);
#pragma unroll
    for (int j = 0; j < kPseItems; ++j) {
      if (smask >> j & 1u) {
        a.stair_off[si] = (uint16_t)(t * kPseItems + j);
        a.stair_val[si] = sm.h[row + j] + off;
        if (parents) a.stair_tc[si] = (int32_t)(pb + sm.tc[row + j]);
        ++si;
      }
      if (qmask >> j & 1u) {
        a.q_off[qi] = (uint16_t)(t * kPseItems + j);
        a.q_val[qi] = sm.h[row + j] + off - (parents ? 0 : 1);
        if (parents) a.q_tc[qi] = (int32_t)(pb + sm.tc[row + j]);
        ++qi;
      }
    }
    if (t == 0) {
      int32_t r = sm.wmin[0];
#pragma unroll
      for (int w = 1; w < kPseWarps; ++w) r = sm.wmin[w] < r ? sm.wmin[w] : r;
      const int32_t tm = r + off;  // the tile holds at least one element
      a.tile_min[tile] = tm;
      atomicMax(a.super_key + (tile >> kPseSuperShift), (uint32_t)((long long)INT_MAX - (long long)tm));
      a.stair_cnt[tile] = (uint32_t)(ctot >> 32);
      a.q_cnt[tile] = (uint32_t)(ctot & 0xffffffffll);
    }
  }
  PSE_PHASE(5);
  if (parents) {
    // each element's parent (answered in this tile) into shared memory, then
    // the tree entries written by consecutive threads for consecutive
    // elements (their places in each output array are consecutive)
#pragma unroll
    for (int j = 0; j < kPseItems; ++j) {
      const int an = ans[j];
      int32_t pn = kNoParent;
      if (an == -3) {  // the root: compute_parents gives it parent 0
        pn = (int32_t)(0 - (pb + sm.tc[0]));
      } else if (an >= 0) {
        pn = (int32_t)(tile0 + an - (pb + sm.tc[(an / kPseItems) * kPseStride + an % kPseItems]));
      }
      sm.pnew[t * kPseItems + j] = pn;
    }
    __syncthreads();
    for (int i = t; i < kPseTile; i += kPseThreads) {
      const long long e = tile0 + i;
      const int32_t pn = sm.pnew[i];
      if (e >= E || pn == kNoParent) continue;
      const int r = (i / kPseItems) * kPseStride + i % kPseItems;
      const int tc = sm.tc[r];
      const int tprev = i == 0 ? 0 : sm.tc[i % kPseItems ? r - 1 : r - kPseStride + kPseItems - 1];
      emit_node(a, dv, sm.v[r], tc != tprev, e, pb + tc, pn);
    }
  }
  PSE_PHASE(6);
  }  // tiles
#undef PSE_PHASE
}

namespace {

// Latest index in [lo, hi] whose value is <= qv, or -1; one warp, 32 values
// per step, highest index first.
__device__ __forceinline__ long long warp_latest_le(const int32_t *arr, long long hi, long long lo, int32_t qv,
                                                    int lane) {
  for (long long base = hi; base >= lo; base -= 32) {
    const long long idx = base - lane;
    const int32_t v = idx >= lo ? arr[idx] : INT_MAX;
    const unsigned b = __ballot_sync(0xffffffffu, v <= qv);
    if (b) return base - (__ffs(b) - 1);
  }
  return -1;
}

// The same over super-tile keys (INT_MAX - minimum; 0: no tile).
__device__ __forceinline__ long long warp_latest_le_key(const uint32_t *keys, long long hi, long long lo, int32_t qv,
                                                        int lane) {
  for (long long base = hi; base >= lo; base -= 32) {
    const long long idx = base - lane;
    const long long v = idx >= lo ? (long long)INT_MAX - (long long)keys[idx] : (long long)INT_MAX;
    const unsigned b = __ballot_sync(0xffffffffu, v <= qv);
    if (b) return base - (__ffs(b) - 1);
  }
  return -1;
}

// Latest tile in [first, hi] whose minimum is <= qv, or -1: the tiles of
// hi's super-tile first, then the super-tile minima before it, then the tiles
// of the super-tile found (never before the document's first tile).
__device__ __forceinline__ long long latest_tile_le(const PseArgs &a, long long hi, long long first, int32_t qv,
                                                    int lane) {
  const long long sup0 = (hi >> kPseSuperShift) << kPseSuperShift;
  long long tt = warp_latest_le(a.tile_min, hi, sup0 > first ? sup0 : first, qv, lane);
  if (tt < 0 && sup0 > first) {
    const long long sp =
        warp_latest_le_key(a.super_key, (sup0 >> kPseSuperShift) - 1, first >> kPseSuperShift, qv, lane);
    if (sp >= 0) {
      const long long lo = sp << kPseSuperShift;
      tt = warp_latest_le(a.tile_min, ((sp + 1) << kPseSuperShift) - 1, lo > first ? lo : first, qv, lane);
    }
  }
  return tt;
}

}  // namespace

// One warp per tile with unanswered queries. The queries (values decreasing
// in position order) are taken 32 at a time: the latest earlier tile whose
// minimum is <= the first query's value answers that query and every later
// one whose value is still >= that minimum (the tiles in between are deeper
// than all of them); each such lane binary-searches the tile's staircase for
// its last stair of depth <= its value. The walk back goes on from that tile
// for the rest. Queries no tile answers: an unmatched right bracket, or
// compute_parents' parent 0 of an empty stack.
__global__ void __launch_bounds__(256) pse_resolve_kernel(PseArgs a) {
  const bool parents = a.mode == kPseParents;
  unsigned long long total;
  if (a.batch) {
    total = (parents ? a.batch->pr_tile0 : a.batch->br_tile0)[a.batch->docs];
  } else {
    // the walk stopped early or not at all (no kernel sets these words while
    // this one runs; the tile kernel checks the same words before it starts)
    if (*reinterpret_cast<volatile int *>(&a.status->error) || *reinterpret_cast<volatile int *>(&a.status->reject) ||
        *reinterpret_cast<volatile int *>(&a.status->overflow))
      return;
    const unsigned long long E = *a.count;
    if (E > a.elem_cap) return;
    total = (E + kPseTile - 1) / kPseTile;
  }
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned long long tile = 0;
    if (lane == 0) tile = atomicAdd(a.resolve_ticket, 1u);
    tile = __shfl_sync(0xffffffffu, tile, 0);
    if (tile >= total) break;
    int doc;
    const PseDoc dv = pse_doc(a, tile, &doc);
    const long long first = (long long)dv.tile_first;
    if ((long long)(tile - first) * kPseTile >= dv.E) continue;
    const unsigned nq = a.q_cnt[tile];
    if (nq == 0) continue;
    DeviceStatus *st = dv.st;
    const unsigned long long qb = tile * (unsigned long long)kPseTile;
    const long long ebase = (long long)(tile - first) * kPseTile;
    long long j = (long long)tile - 1;  // answering tiles are at most this one
    unsigned q = 0;
    while (q < nq) {
      const unsigned qi = q + lane;
      const bool have = qi < nq;
      const int32_t qv = have ? a.q_val[qb + qi] : INT_MIN;
      j = j >= first ? latest_tile_le(a, j, first, __shfl_sync(0xffffffffu, qv, 0), lane) : -1;
      if (j < 0) break;
      const int32_t tm = a.tile_min[j];
      const bool ok = have && qv >= tm;
      if (ok) {
        const unsigned long long sb = (unsigned long long)j * kPseTile;
        int lo = 0, hi = (int)a.stair_cnt[j] - 1;  // stair_val[sb] == tm <= qv
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (a.stair_val[sb + mid] <= qv) lo = mid;
          else hi = mid - 1;
        }
        const long long e = ebase + a.q_off[qb + qi];
        const long long p = (j - first) * kPseTile + a.stair_off[sb + lo];
        const uint32_t v = dv.elems[e];
        if (parents) {
          emit_node(a, dv, v, __ldg(a.is_term + v) != 0, e, a.q_tc[qb + qi], p - a.stair_tc[sb + lo]);
        } else if ((dv.elems[p] ^ v) & 0x7fffffffu) {
          record_reject(st, &st->parse_reject_reason, 2);
        }
      }
      q += __popc(__ballot_sync(0xffffffffu, ok));  // lane 0 is answered: progress
    }
    if (q < nq) {  // no earlier tile answers the rest
      if (!parents) {
        if (lane == 0) record_reject(st, &st->parse_reject_reason, 3);
        continue;
      }
      const long long tinc0 = __ldg(a.is_term + dv.elems[0]) ? 1 : 0;  // inclusive terminal count at element 0
      for (unsigned qi = q + lane; qi < nq; qi += kWarp) {
        const long long e = ebase + a.q_off[qb + qi];
        const uint32_t v = dv.elems[e];
        emit_node(a, dv, v, __ldg(a.is_term + v) != 0, e, a.q_tc[qb + qi], 0 - tinc0);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Batch planning
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(1024) batch_plan_kernel(BatchDesc b, int kind, unsigned long long *tile0,
                                                          unsigned long long tile) {
  __shared__ long long tmp[32];
  const int t = threadIdx.x;
  long long carry = 0;
  for (int base = 0; base < b.docs; base += 1024) {
    const int d = base + t;
    long long cnt = 0;
    if (d < b.docs) {
      const DeviceStatus &s = b.status[d];
      const unsigned long long c = kind == kPlanPairs ? s.num_tokens + 2
                                   : kind == kPlanBrackets ? s.num_brackets : s.num_productions;
      cnt = (long long)((c + tile - 1) / tile);
    }
    long long tot;
    const long long ex = block_exclusive_scan<long long>(cnt, AddI64(), 0ll, tmp, &tot);
    if (d < b.docs) tile0[d] = (unsigned long long)(carry + ex);
    carry += tot;
  }
  if (t == 0) tile0[b.docs] = (unsigned long long)carry;
}

// ---------------------------------------------------------------------------
// Parser-mode output: the u32 production ids of the pair stage narrowed to
// production_t (the width parse_test writes). Each thread converts 4
// consecutive ids per step.
// ---------------------------------------------------------------------------

__global__ void narrow_u32_kernel(const uint32_t *src, void *dst, const unsigned long long *count_p,
                                  unsigned long long cap, int width) {
  const unsigned long long count = *count_p < cap ? *count_p : cap;
  const unsigned long long quads = (count + 3) / 4;
  for (unsigned long long q = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; q < quads;
       q += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long i0 = 4 * q;
    const int k = count - i0 < 4 ? (int)(count - i0) : 4;
    for (int j = 0; j < k; ++j) store_uint(dst, i0 + j, width, __ldg(src + i0 + j));
  }
}

}  // namespace alpacc
