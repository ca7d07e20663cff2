// Data-parallel lexer for sm_100a: the sequential semantics of lex_string
// (backends/c/lexer.c:39-97) computed tile-parallel.
//
// The lexer runs a Moore machine over byte classes that device_tables.cpp
// derives from TO_STATE / COMPOSE / ACCEPT: a transition entry holds the next
// state (7 bits) and that state's produce flag (bit 7), indexed by
// class * M + state. Persistent CTAs load the tables into shared memory once
// - the byte-class table and the transition table are replicated (`copies`
// of each, lane l reading copy l % copies) so data-dependent lookups from one
// warp rarely meet in a bank - and then take tiles by ticket.
//
// A tile is 256 chunks of 60 bytes (15 words: an odd stride, so per-thread
// walks are bank-conflict free). The first 8 chunks are a halo - the 480
// bytes before the tile's 14880 data bytes - walked again so that the tile
// can almost always derive its incoming state by itself.
//
// Pass 1: every chunk computes its transition function without knowing its
//   start state by running the machine from every live state its first byte
//   can lead to ("lanes") and merging lanes that meet. Once one lane is left
//   (after a few bytes) the walk costs one lookup per byte and records the
//   token boundaries it passes: a 64-bit mask, and the state before each
//   boundary written over the consumed byte. Such a chunk maps every live
//   start state to one end state ("constant").
// Resolution: a chunk's start state follows from the nearest constant chunk
//   before it; only when no halo chunk is constant does the tile read its
//   predecessor's published outgoing state (decoupled look-back, bounded).
// Pass 2: each data chunk re-walks only the bytes before its lanes merged,
//   from its true start, then counts kept tokens over the recorded
//   boundaries; a (count, last boundary) carry is scanned across the tile and
//   across tiles by decoupled look-back; tokens are written structure-of-arrays.
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

constexpr int kNotConverged = 255;

struct LexSmem {
  uint32_t bytes[kLexThreads * kLexWords];  // the tile; recorded boundary states overwrite consumed bytes
  uint8_t lst[kMaxLanes * kLexThreads];     // lane states, slot-major
  uint8_t lrm[kMaxLanes * kLexThreads];     // original slot -> merged slot
  uint16_t active[kLexThreads];
  uint8_t c0[kLexThreads];      // class id of the chunk's first byte
  uint8_t nbytes[kLexThreads];
  uint8_t start[kLexThreads];   // true start state of data chunks
  uint8_t cstate[kLexThreads];  // lane state just before the recorded part
  uint8_t exact[kLexThreads];   // 1: lanes tracked per start state (lst/lrm valid)
  uint8_t sterm[256];           // per machine state: terminal id
  uint8_t sflags[256];          // bit1 accept, bit2 kept
  uint8_t cls_id[256];          // byte -> class id (first byte of a chunk)
  long long scan_tmp[kLexThreads / 32];
  Pair64 pair_tmp[kLexThreads / 32];
  int kconst[kLexThreads];
  unsigned tile;
  int s_in;
  int need_lookback;
  int out_published;
  long long cnt_prefix, pos_prefix;
};

struct Tabs {
  const uint16_t *cls;    // [256 * copies] class * M
  const uint32_t *trans;  // [words * copies] packed u8 entries
  int copies;
  int lane_copy;
};

__device__ __forceinline__ uint32_t cls_pre(const Tabs &tb, uint32_t b) {
  return tb.cls[b * (uint32_t)tb.copies + (uint32_t)tb.lane_copy];
}

// entry of (class premultiplied cp, state s): next state | produce << 7
__device__ __forceinline__ uint32_t entry(const Tabs &tb, uint32_t cp, uint32_t s) {
  const uint32_t i = cp + s;
  const uint32_t w = tb.trans[(i >> 2) * (uint32_t)tb.copies + (uint32_t)tb.lane_copy];
  return __byte_perm(w, 0, i & 3);
}

// f_t(x): the state after chunk t when it starts in state x. A chunk walked as
// a state set is constant: every live start ends in its one state (a start
// whose lane died instead is caught when the chunk is re-walked from its true
// start, which then rejects the input).
__device__ __forceinline__ int eval_chunk(const LexArgs &a, const LexSmem *sm, int t, int x) {
  if (sm->nbytes[t] == 0) return x;
  const int dead = a.dead;
  if (x == dead) return dead;
  if (!sm->exact[t]) return sm->active[t] ? sm->lst[t] : dead;
  const int slot = __ldg(a.lane_of + (size_t)sm->c0[t] * a.M + x);
  if (slot == 0xff) return dead;
  const int r = sm->lrm[slot * kLexThreads + t];
  if (!((sm->active[t] >> r) & 1)) return dead;
  return sm->lst[r * kLexThreads + t];
}

__device__ __forceinline__ int const_value(const LexArgs &a, const LexSmem *sm, int k) {
  const uint32_t act = sm->active[k];
  if (!act) return a.dead;
  return sm->lst[(__ffs(act) - 1) * kLexThreads + k];
}

struct CntPosOp {
  __device__ Pair64 operator()(Pair64 e, Pair64 l) const { return Pair64{e.a + l.a, e.b > l.b ? e.b : l.b}; }
};

}  // namespace

__global__ void __launch_bounds__(kLexThreads, 6) lex_kernel(LexArgs args) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ __align__(16) LexSmem sm_static;
  LexSmem *sm = &sm_static;
  const LexArgs &a = args;
  const int t = threadIdx.x;
  const int lane = t & 31;
  const int copies = a.copies;

  // ---- tables, once per CTA ----
  uint16_t *s_cls = reinterpret_cast<uint16_t *>(dyn_smem);
  uint32_t *s_trans = reinterpret_cast<uint32_t *>(dyn_smem + ((256 * copies * 2 + 15) & ~15));
  for (int i = t; i < 256 * copies; i += kLexThreads) s_cls[i] = (uint16_t)(__ldg(a.cls_id + i / copies) * a.M);
  for (int i = t; i < a.trans_words * copies; i += kLexThreads) s_trans[i] = __ldg(a.trans_words_ptr + i / copies);
  for (int i = t; i < 256; i += kLexThreads) {
    sm->sterm[i] = i < a.M ? __ldg(a.sterm + i) : 0;
    sm->sflags[i] = i < a.M ? __ldg(a.sflags + i) : 0;
    sm->cls_id[i] = __ldg(a.cls_id + i);
  }
  const Tabs tb{s_cls, s_trans, copies, lane & (copies - 1)};
  const int dead = a.dead;
  const unsigned long long num_tiles = a.num_tiles;
  const unsigned long long tile_end = a.tile_end ? a.tile_end : num_tiles;

  for (unsigned long long round = 0;; ++round) {
    if (round > tile_end - a.tile_begin) {  // every round takes a new ticket: cannot happen
      if (t == 0) record_timeout(a.status, kSiteLexTiles);
      break;
    }
    __syncthreads();  // tables ready / previous tile fully consumed
    if (t == 0) sm->tile = atomicAdd(a.ticket, 1u);
    __syncthreads();
    const unsigned long long tile = a.tile_begin + sm->tile;
    if (tile >= tile_end) break;
    // this tile's document: the whole input, or one document of a batch
    // (virtual tile `tile` is local tile `lt` of `tiles_t`)
    const uint8_t *in_base = a.in;
    long long n = (long long)a.n;
    unsigned long long lt = tile, tiles_t = num_tiles;
    DeviceStatus *st = a.status;
    if (a.batch) {
      const BatchDesc &b = *a.batch;
      const int d = batch_doc(b.lex_tile0, b.docs, tile);
      lt = tile - b.lex_tile0[d];
      tiles_t = b.lex_tile0[d + 1] - b.lex_tile0[d];
      in_base = a.in + b.in_off[d];
      n = (long long)b.n[d];
      st = b.status + d;
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
          for (int k = 0; k < 16; ++k) {
            const long long p = g + k;
            dst[16 * v + k] = (p >= 0 && p < n) ? in[p] : 0;
          }
        }
      }
    }
    const long long g0 = load0 + (long long)t * kLexChunk;
    int nb = 0;
    if (g0 >= 0 && g0 < n) nb = (int)min((long long)kLexChunk, n - g0);
    sm->nbytes[t] = (uint8_t)nb;
    __syncthreads();

    // ---- pass 1: the set of live states until it is a single state, then
    // one lane recording boundaries ----
    // The set walk (machines of at most 64 states) costs one lookup per live
    // state per byte and merges equal states for free; it gives no per-start
    // mapping, so a chunk whose set never shrinks to one state is walked again
    // with lanes tracked per start state (slots in lst/lrm).
    uint8_t *tb8 = reinterpret_cast<uint8_t *>(sm->bytes) + t * kLexChunk;
    uint32_t active = 0;
    unsigned long long bmask = 0;
    int jconv = kNotConverged;
    {
      int c0 = 0;
      bool exact = a.M > 64;
      if (nb > 0) {
        c0 = sm->cls_id[tb8[0]];
        const int cnt = __ldg(a.img_cnt + c0);
        int lconv = -1;
        uint32_t s = 0;
        int j = 1;
        if (!exact) {
          const unsigned long long live = dead >= 0 ? ~(1ull << dead) : ~0ull;
          unsigned long long set = 0;
          if (a.img2 && nb >= 2) {  // the first two bytes at once
            set = __ldg(a.img2 + c0 * a.C + sm->cls_id[tb8[1]]);
            j = 2;
          } else {
            for (int l = 0; l < cnt; l++) set |= 1ull << __ldg(a.img + c0 * kMaxLanes + l);
          }
          while (j < nb && __popcll(set) > 1) {
            const uint32_t cp = cls_pre(tb, tb8[j]);
            unsigned long long ns = 0;
            for (unsigned long long m = set; m; m &= m - 1)
              ns |= 1ull << (entry(tb, cp, (uint32_t)(__ffsll((long long)m) - 1)) & 0x7f);
            set = ns & live;
            ++j;
          }
          if (__popcll(set) > 1) {
            exact = true;
          } else if (set) {
            lconv = 0;
            s = (uint32_t)(__ffsll((long long)set) - 1);
            active = 1;
          }  // else every lane died: active = 0, not converged
        }
        if (exact) {
          active = cnt ? ((1u << cnt) - 1u) : 0u;
          for (int l = 0; l < cnt; l++) {
            sm->lst[l * kLexThreads + t] = __ldg(a.img + c0 * kMaxLanes + l);
            sm->lrm[l * kLexThreads + t] = (uint8_t)l;
          }
          j = 1;
          while (j < nb && __popc(active) > 1) {
            const uint32_t cp = cls_pre(tb, tb8[j]);
            for (uint32_t m = active; m; m &= m - 1) {
              const int l = __ffs(m) - 1;
              const int s2 = (int)(entry(tb, cp, sm->lst[l * kLexThreads + t]) & 0x7f);
              if (s2 == dead) active &= ~(1u << l);
              else sm->lst[l * kLexThreads + t] = (uint8_t)s2;
            }
            if (__popc(active) > 1) {
              for (uint32_t m1 = active; m1; m1 &= m1 - 1) {
                const int l1 = __ffs(m1) - 1;
                if (!((active >> l1) & 1)) continue;
                const int s1 = sm->lst[l1 * kLexThreads + t];
                for (uint32_t m2 = active & ~((2u << l1) - 1u); m2; m2 &= m2 - 1) {
                  const int l2 = __ffs(m2) - 1;
                  if (sm->lst[l2 * kLexThreads + t] == s1) {
                    active &= ~(1u << l2);
                    for (int k = 0; k < cnt; k++)
                      if (sm->lrm[k * kLexThreads + t] == l2) sm->lrm[k * kLexThreads + t] = (uint8_t)l1;
                  }
                }
              }
            }
            ++j;
          }
          if (__popc(active) == 1) {
            lconv = __ffs(active) - 1;
            s = sm->lst[lconv * kLexThreads + t];
          }
        }
        if (lconv >= 0) {
          jconv = j;
          sm->cstate[t] = (uint8_t)s;
          // the hot loop: one class lookup and one transition per byte. The
          // dead state is absorbing and never produces, so a lane that dies
          // records nothing further and needs no test inside the loop.
#pragma unroll 4
          for (; j < nb; ++j) {
            const uint32_t e = entry(tb, cls_pre(tb, tb8[j]), s);
            if (e & 0x80) {
              bmask |= 1ull << j;
              tb8[j] = (uint8_t)s;  // state of the token ending before byte j
            }
            s = e & 0x7f;
          }
          if ((int)s == dead) active = 0;
          else sm->lst[lconv * kLexThreads + t] = (uint8_t)s;
        }
      }
      sm->active[t] = (uint16_t)active;
      sm->c0[t] = (uint8_t)c0;
      sm->exact[t] = exact ? 1 : 0;
      if (a.diag) {
        const unsigned w = __reduce_add_sync(0xffffffffu, (unsigned)(jconv == kNotConverged ? nb : jconv));
        if (lane == 0) atomicAdd(&st->scratch[3], (unsigned long long)w);
      }
    }
    __syncthreads();

    // ---- resolution: nearest constant chunk before each chunk ----
    const bool is_const = nb > 0 && __popc(active) <= 1;
    long long ktot;
    const long long kex = block_exclusive_scan<long long>(is_const ? (long long)t : -1ll, MaxI64(), -1ll,
                                                          sm->scan_tmp, &ktot);
    sm->kconst[t] = (int)kex;
    if (t == kLexHalo) sm->need_lookback = kex < 0 ? 1 : 0;
    if (t == 0) sm->out_published = 0;
    if (a.diag) {
      const int nconst = __syncthreads_count(is_const);
      if (t == 0) atomicAdd(&st->scratch[1], (unsigned long long)nconst);
    }
    __syncthreads();
    if (ktot >= 0) {
      // the outgoing state does not depend on the incoming one: publish now
      if (t == 0) {
        int x = const_value(a, sm, (int)ktot);
        for (int jj = (int)ktot + 1; jj < kLexThreads; ++jj) x = eval_chunk(a, sm, jj, x);
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
        x = const_value(a, sm, k);
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
    if (t == 0 && !sm->out_published) {
      const int x = eval_chunk(a, sm, kLexThreads - 1, sm->start[kLexThreads - 1]);
      a.st1_state[tile] = (uint8_t)(x < 0 ? 0 : x);
      __threadfence();
      st_release_u32(a.st1_flag + tile, 2u);
    }

    // ---- pass 2a: re-walk the pre-merge bytes from the true start ----
    long long cnt = 0, lastb = 0;
    bool final_tok = false, final_kept = false;
    int final_term = 0;
    if (t >= kLexHalo && nb > 0) {
      int x = sm->start[t];
      bool died = (x == dead);
      const int jc = jconv == kNotConverged ? nb : jconv;
      for (int j = 0; j < jc && !died; ++j) {
        const uint32_t e = entry(tb, cls_pre(tb, tb8[j]), (uint32_t)x);
        if (g0 + j >= 1 && (e & 0x80)) {
          bmask |= 1ull << j;
          tb8[j] = (uint8_t)x;
        }
        x = (int)(e & 0x7f);
        if (x == dead) died = true;
      }
      if (!died && jconv != kNotConverged) {
        if (x != sm->cstate[t]) atomicCAS(&st->error, 0, -1 /* lanes disagree: internal error */);
        if (!active) died = true;  // the merged lane died further on
        else x = sm->lst[(__ffs(active) - 1) * kLexThreads + t];
      }
      if (died) record_reject(st, &st->lex_reject_reason, 1);
      for (unsigned long long m = bmask; m; m &= m - 1) {
        const int j = __ffsll((long long)m) - 1;
        if (sm->sflags[tb8[j]] & 4) ++cnt;
      }
      if (bmask) lastb = g0 + 63 - __clzll((long long)bmask);
      if (g0 + nb == n && !a.open_end) {  // this chunk holds the last byte of the input
        final_tok = true;
        final_term = sm->sterm[x];
        final_kept = (sm->sflags[x] & 4) != 0;
        if (final_kept) ++cnt;
        if (!(sm->sflags[x] & 2) || died) record_reject(st, &st->lex_reject_reason, 2);
      }
    }
    // ---- (count, last boundary) carry ----
    Pair64 cp_tot;
    const Pair64 cp_ex = block_exclusive_scan_pair(Pair64{cnt, lastb}, CntPosOp(), Pair64{0, 0}, sm->pair_tmp, &cp_tot);
    const long long cnt_ex = cp_ex.a, pos_ex = cp_ex.b;
    const long long cnt_tot = cp_tot.a, pos_tot = cp_tot.b;
    if (a.stage_ids) {
      // ---- staged: tile-local offsets, no wait on other tiles ----
      if (t == 0) {
        a.tile_cnt[tile] = (uint32_t)cnt_tot;
        a.tile_pos[tile] = (uint32_t)pos_tot;
      }
      if (t >= kLexHalo && nb > 0) {
        unsigned long long out = tile * (unsigned long long)kLexData + (unsigned long long)cnt_ex;
        long long tok_start = pos_ex;  // 0: the token starts before this tile
        for (unsigned long long m = bmask; m; m &= m - 1) {
          const int j = __ffsll((long long)m) - 1;
          const long long p = g0 + j;
          const int s = tb8[j];
          if (sm->sflags[s] & 4) {
            a.stage_ids[out] = sm->sterm[s];
            a.stage_starts[out] = (uint32_t)tok_start;
            a.stage_ends[out] = (uint32_t)p;
            ++out;
          }
          tok_start = p;
        }
        if (final_tok && final_kept) {
          a.stage_ids[out] = (uint8_t)final_term;
          a.stage_starts[out] = (uint32_t)tok_start;
          a.stage_ends[out] = (uint32_t)n;
        }
      }
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
        if (lt + 1 == tiles_t) st->num_tokens = (unsigned long long)inc.a;
      }
    }
    __syncthreads();

    // ---- pass 2b: write this chunk's kept tokens ----
    if (t >= kLexHalo && nb > 0) {
      unsigned long long out = (unsigned long long)(sm->cnt_prefix + cnt_ex);
      long long tok_start = sm->pos_prefix > pos_ex ? sm->pos_prefix : pos_ex;
      const unsigned long long len_max = a.len_max;
      bool too_long = false;
      for (unsigned long long m = bmask; m; m &= m - 1) {
        const int j = __ffsll((long long)m) - 1;
        const long long p = g0 + j;
        const int s = tb8[j];
        if (sm->sflags[s] & 4) {
          const unsigned long long len = (unsigned long long)(p - tok_start);
          if (len > len_max) too_long = true;
          store_uint(a.tok_ids, out, a.term_w, (unsigned long long)sm->sterm[s]);
          store_uint(a.tok_starts, out, a.idx_w, (unsigned long long)tok_start);
          store_uint(a.tok_lens, out, a.len_w, len);
          ++out;
        }
        tok_start = p;
      }
      if (final_tok && final_kept) {
        const unsigned long long len = (unsigned long long)(n - tok_start);
        if (len > len_max) too_long = true;
        store_uint(a.tok_ids, out, a.term_w, (unsigned long long)final_term);
        store_uint(a.tok_starts, out, a.idx_w, (unsigned long long)tok_start);
        store_uint(a.tok_lens, out, a.len_w, len);
      }
      if (too_long) record_reject(st, &st->lex_reject_reason, 3);
    }
  }
}

// ---------------------------------------------------------------------------
// Placement of staged tokens
// ---------------------------------------------------------------------------

// Exclusive (count, last boundary) prefix over the tiles, by one CTA; also the
// total token count. In a batch the prefix restarts at each document's first
// tile (a segmented scan: the flag bit kSeg marks a segment start) and the
// offsets are placed in the document's token region.
constexpr long long kSeg = 1ll << 62;

struct SegCntPosOp {
  __device__ Pair64 operator()(Pair64 l, Pair64 r) const {
    if (r.b & kSeg) return r;
    const long long lp = l.b & ~kSeg;
    return Pair64{l.a + r.a, (lp > r.b ? lp : r.b) | (l.b & kSeg)};
  }
};

__global__ void __launch_bounds__(kLexScanThreads) lex_scan_kernel(LexPlaceArgs a) {
  __shared__ Pair64 tmp[kLexScanThreads / 32];
  const int t = threadIdx.x;
  constexpr int kPer = 16;
  const BatchDesc *bd = a.batch;
  // segment start of tile i (a batch document's first tile) and its document
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
      run = Pair64{run.a + (long long)a.tile_cnt[i0 + k],
                   ((run.b & ~kSeg) > (long long)a.tile_pos[i0 + k] ? (run.b & ~kSeg) : (long long)a.tile_pos[i0 + k])};
      // the document's token count, at its last tile
      if (bd && i0 + k + 1 == bd->lex_tile0[d + 1]) bd->status[d].num_tokens = (unsigned long long)run.a;
    }
    carry = SegCntPosOp()(carry, tot);
  }
  if (t == 0 && !bd) {
    a.status->num_tokens = (unsigned long long)(carry.a);
    a.status->last_boundary = (unsigned long long)(carry.b & ~kSeg);
  }
}

// Each CTA copies whole tiles' staged tokens to their final places; a token
// whose start lies before its tile takes the last boundary before the tile.
__global__ void __launch_bounds__(256) lex_place_kernel(LexPlaceArgs a) {
  bool too_long = false;
  DeviceStatus *st = a.status;
  for (unsigned long long tile = blockIdx.x; tile < a.num_tiles; tile += gridDim.x) {
    DeviceStatus *sd = a.batch ? a.batch->status + batch_doc(a.batch->lex_tile0, a.batch->docs, tile) : a.status;
    if (sd != st) {
      if (too_long) record_reject(st, &st->lex_reject_reason, 3);
      too_long = false;
      st = sd;
    }
    const unsigned c = a.tile_cnt[tile];
    const unsigned long long off = a.tile_off[tile];
    const uint32_t prev = a.tile_prev[tile];
    const unsigned long long base = tile * (unsigned long long)a.tile_data;
    for (unsigned i = threadIdx.x; i < c; i += blockDim.x) {
      const uint32_t s0 = a.stage_starts[base + i];
      const uint32_t start = s0 > prev ? s0 : prev;
      const uint32_t end = a.stage_ends[base + i];
      const unsigned long long len = end - start;
      if (len > a.len_max) too_long = true;
      store_uint(a.tok_ids, off + i, a.term_w, a.stage_ids[base + i]);
      store_uint(a.tok_starts, off + i, a.idx_w, a.index_base + start);
      store_uint(a.tok_lens, off + i, a.len_w, len);
    }
  }
  if (too_long) record_reject(st, &st->lex_reject_reason, 3);
}

}  // namespace alpacc
