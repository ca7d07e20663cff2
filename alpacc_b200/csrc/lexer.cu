// Data-parallel lexer for sm_100a: the sequential semantics of lex_string
// (backends/c/lexer.c:39-97) computed tile-parallel.
//
// The lexer is a Moore machine over byte classes (device_tables.cpp derives
// it from TO_STATE / COMPOSE / ACCEPT). A tile is 256 threads x 60 bytes,
// loaded with 16-byte vector loads into shared memory; 60 bytes = 15 words
// per thread, an odd stride, so the per-thread walks are bank-conflict free.
//
// Pass 1: each thread computes its chunk's transition function without knowing
//   its start state by running the machine from every live state the first
//   byte can lead to ("lanes") and merging lanes that meet; after a few bytes
//   one lane is left, so the walk costs one table lookup per byte. A chunk
//   whose lanes merged into one has a constant function (up to death).
// Tile resolution: thread t's start state follows from the nearest constant
//   chunk before it (or the tile's incoming state), so a tile that contains
//   any constant chunk knows its outgoing state before it knows its incoming
//   state and publishes it at once; look-back therefore rarely waits.
// Pass 2: every thread re-walks its chunk from its true start, marks token
//   boundaries (produce flag of the next state) and counts kept tokens; a
//   (count, last boundary) carry is scanned across the tile and across tiles
//   by decoupled look-back; tokens are written as structure-of-arrays.
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

struct LexSmem {
  uint32_t bytes[kLexThreads * kLexWords];      // the tile, linear
  uint32_t cls[64 * 32];                        // byte -> class, one copy per bank
  uint8_t lst[kMaxLanes * kLexThreads];         // lane states, slot-major
  uint8_t lrm[kMaxLanes * kLexThreads];         // original slot -> merged slot
  uint16_t active[kLexThreads];
  uint8_t c0[kLexThreads];
  uint8_t nbytes[kLexThreads];
  uint8_t start[kLexThreads];
  long long scan_tmp[kLexThreads / 32 * 2];
  int kconst[kLexThreads];
  int s_in;
  int out_published;
  long long tile_cnt_prefix;
  long long tile_pos_prefix;
};

struct LexCtx {
  const LexArgs *a;
  LexSmem *sm;
  const uint32_t *trans;  // smem, replicated `rep` times
  int rep;
  int lane;
};

__device__ __forceinline__ int cls_of(const LexCtx &c, uint32_t b) {
  return (c.sm->cls[(b >> 2) * 32 + c.lane] >> ((b & 3) * 8)) & 0xff;
}

__device__ __forceinline__ int step(const LexCtx &c, int s, int cl) {
  const uint32_t i = (uint32_t)s * (uint32_t)c.a->C + (uint32_t)cl;
  const uint32_t w = c.trans[(i >> 2) * c.rep + (c.rep == 32 ? c.lane : 0)];
  return (w >> ((i & 3) * 8)) & 0xff;
}

__device__ __forceinline__ uint32_t chunk_byte(const LexSmem *sm, int t, int j) {
  const uint32_t w = sm->bytes[t * kLexWords + (j >> 2)];
  return (w >> ((j & 3) * 8)) & 0xff;
}

// f_t(x): the state after thread t's chunk when it starts in state x.
__device__ __forceinline__ int eval_chunk(const LexCtx &c, int t, int x) {
  const LexSmem *sm = c.sm;
  if (sm->nbytes[t] == 0) return x;
  const int dead = c.a->dead;
  if (x == dead) return dead;
  const int c0 = sm->c0[t];
  const int slot = __ldg(c.a->lane_of + (size_t)c0 * c.a->M + x);
  if (slot == 0xff) return dead;
  const int r = sm->lrm[slot * kLexThreads + t];
  if (!((sm->active[t] >> r) & 1)) return dead;
  return sm->lst[r * kLexThreads + t];
}

}  // namespace

__global__ void __launch_bounds__(kLexThreads) lex_kernel(LexArgs args) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  __shared__ __align__(16) LexSmem sm_static;
  LexSmem *sm = &sm_static;
  const LexArgs *a = &args;
  const int t = threadIdx.x;
  const int lane = t & 31;
  uint32_t *s_trans = reinterpret_cast<uint32_t *>(dyn_smem);
  LexCtx c{a, sm, s_trans, a->trans_rep, lane};
  DeviceStatus *st = a->status;

  // ---- tile ticket (tiles are processed in ticket order) ----
  __shared__ unsigned s_tile;
  if (t == 0) s_tile = atomicAdd(a->ticket, 1u);
  // ---- replicated tables into shared memory ----
  for (int i = t; i < 64 * 32; i += kLexThreads) sm->cls[i] = __ldg(a->cls_words + (i >> 5));
  {
    const int words = a->trans_words * a->trans_rep;
    for (int i = t; i < words; i += kLexThreads) s_trans[i] = __ldg(a->trans_words_ptr + i / a->trans_rep);
  }
  __syncthreads();
  const unsigned long long tile = s_tile;
  const unsigned long long n = a->n;
  const unsigned long long base = tile * (unsigned long long)kLexTile;

  // ---- load the tile ----
  {
    const unsigned long long avail = n > base ? n - base : 0;
    const int tile_bytes = avail >= (unsigned long long)kLexTile ? kLexTile : (int)avail;
    const uint8_t *src = a->in + base;
    uint8_t *dst = reinterpret_cast<uint8_t *>(sm->bytes);
    const bool aligned = ((reinterpret_cast<uintptr_t>(src) & 15) == 0);
    if (aligned && tile_bytes == kLexTile) {
      const uint4 *s4 = reinterpret_cast<const uint4 *>(src);
      uint4 *d4 = reinterpret_cast<uint4 *>(dst);
      for (int i = t; i < kLexTile / 16; i += kLexThreads) d4[i] = __ldg(s4 + i);
    } else {
      for (int i = t; i < kLexTile; i += kLexThreads) dst[i] = i < tile_bytes ? src[i] : 0;
    }
  }
  // ---- per-thread chunk geometry ----
  const unsigned long long g0 = base + (unsigned long long)t * kLexChunk;
  const int nb = g0 < n ? (int)((n - g0) < (unsigned long long)kLexChunk ? (n - g0) : kLexChunk) : 0;
  sm->nbytes[t] = (uint8_t)nb;
  __syncthreads();

  const int dead = a->dead;
  // ---- pass 1: chunk function by converging lanes ----
  {
    uint32_t active = 0;
    int c0 = 0;
    int multi_bytes = 0;
    if (nb > 0) {
      c0 = cls_of(c, chunk_byte(sm, t, 0));
      const int cnt = __ldg(a->img_cnt + c0);
      active = cnt ? ((1u << cnt) - 1u) : 0u;
      for (int l = 0; l < cnt; l++) {
        sm->lst[l * kLexThreads + t] = __ldg(a->img + c0 * kMaxLanes + l);
        sm->lrm[l * kLexThreads + t] = (uint8_t)l;
      }
      const int nl = cnt;
      int j = 1;
      // several lanes: step each, drop dead ones, merge equal ones
      while (j < nb && __popc(active) > 1) {
        const int cl = cls_of(c, chunk_byte(sm, t, j));
        for (uint32_t m = active; m; m &= m - 1) {
          const int l = __ffs(m) - 1;
          const int s2 = step(c, sm->lst[l * kLexThreads + t], cl);
          if (s2 == dead) active &= ~(1u << l);
          else sm->lst[l * kLexThreads + t] = (uint8_t)s2;
        }
        for (int l1 = 0; l1 < nl; l1++) {
          if (!((active >> l1) & 1)) continue;
          const int s1 = sm->lst[l1 * kLexThreads + t];
          for (int l2 = l1 + 1; l2 < nl; l2++) {
            if (((active >> l2) & 1) && sm->lst[l2 * kLexThreads + t] == s1) {
              active &= ~(1u << l2);
              for (int k = 0; k < nl; k++)
                if (sm->lrm[k * kLexThreads + t] == l2) sm->lrm[k * kLexThreads + t] = (uint8_t)l1;
            }
          }
        }
        ++j;
        ++multi_bytes;
      }
      // one lane: the hot loop, one lookup per byte
      if (active && __popc(active) == 1 && j < nb) {
        const int l = __ffs(active) - 1;
        int s = sm->lst[l * kLexThreads + t];
        for (; j < nb; ++j) {
          s = step(c, s, cls_of(c, chunk_byte(sm, t, j)));
          if (s == dead) break;
        }
        if (s == dead) active = 0;
        else sm->lst[l * kLexThreads + t] = (uint8_t)s;
      }
    }
    sm->active[t] = (uint16_t)active;
    sm->c0[t] = (uint8_t)c0;
    if (a->diag) {
      const unsigned w = __reduce_add_sync(0xffffffffu, (unsigned)multi_bytes);
      if ((t & 31) == 0) atomicAdd(&st->scratch[3], (unsigned long long)w);
    }
  }
  __syncthreads();

  // ---- tile resolution: nearest constant chunk before each thread ----
  const bool is_const = nb > 0 && __popc((uint32_t)sm->active[t]) <= 1;
  long long ktot;
  long long kex = block_exclusive_scan<long long>(is_const ? (long long)t : -1ll, MaxI64(), -1ll, sm->scan_tmp, &ktot);
  sm->kconst[t] = (int)kex;
  if (t == 0) sm->out_published = 0;
  if (a->diag) {
    const int nconst = __syncthreads_count(is_const);
    if (t == 0) {
      atomicAdd(&st->scratch[1], (unsigned long long)nconst);
      if (ktot < 0) atomicAdd(&st->scratch[0], 1ull);
    }
    const unsigned chain = (unsigned)(kex >= 0 ? t - 1 - kex : t);
    const unsigned w = __reduce_add_sync(0xffffffffu, chain);
    if ((t & 31) == 0) atomicAdd(&st->scratch[2], (unsigned long long)w);
  }
  __syncthreads();

  // value of a constant chunk (its single live lane, or dead)
  auto const_value = [&](int k) -> int {
    const uint32_t act = sm->active[k];
    if (!act) return dead;
    return sm->lst[(__ffs(act) - 1) * kLexThreads + k];
  };
  const unsigned long long num_tiles = a->num_tiles;
  if (ktot >= 0) {
    // outgoing state is independent of the incoming one: publish now
    if (t == 0) {
      int x = const_value((int)ktot);
      for (int jj = (int)ktot + 1; jj < kLexThreads; ++jj) x = eval_chunk(c, jj, x);
      a->st1_state[tile] = (uint8_t)(x < 0 ? 0 : x);
      __threadfence();
      st_release_u32(a->st1_flag + tile, 2u);
      sm->out_published = 1;
    }
  } else if (tile + 1 < num_tiles) {
    // no constant chunk: publish the tile's full transition vector
    for (int s = t; s < a->M; s += kLexThreads) {
      int x = s;
      for (int jj = 0; jj < kLexThreads; ++jj) x = eval_chunk(c, jj, x);
      a->st1_vec[tile * (unsigned long long)a->M + s] = (uint8_t)(x < 0 ? 0 : x);
    }
    __syncthreads();
    if (t == 0) {
      __threadfence();
      st_release_u32(a->st1_flag + tile, 1u);
    }
  }
  // ---- incoming state by look-back ----
  if (t == 0) {
    int s_in = a->m0;
    if (tile > 0) {
      long long j = (long long)tile - 1;
      int base_state = a->m0;
      bool have = false;
      while (j >= 0) {
        const unsigned f = wait_flag(a->st1_flag + j, 1u, st, kSiteLexState);
        if (f == 0) break;  // timed out (recorded)
        if (f >= 2) {
          base_state = *reinterpret_cast<volatile uint8_t *>(a->st1_state + j);
          have = true;
          break;
        }
        --j;
      }
      if (!have) { j = -1; base_state = a->m0; }
      // tiles j+1 .. tile-1 published transition vectors
      int x = base_state;
      for (long long jj = j + 1; jj < (long long)tile; ++jj) {
        if (x == dead || x < 0) break;
        x = *reinterpret_cast<volatile uint8_t *>(a->st1_vec + jj * (unsigned long long)a->M + x);
      }
      s_in = x;
    }
    sm->s_in = s_in;
  }
  __syncthreads();
  // ---- each thread's start state ----
  {
    const int k = sm->kconst[t];
    int x = k < 0 ? sm->s_in : const_value(k);
    for (int jj = k + 1; jj < t; ++jj) x = eval_chunk(c, jj, x);
    sm->start[t] = (uint8_t)(x < 0 ? 0 : x);
  }
  __syncthreads();
  if (t == 0 && !sm->out_published) {
    int x = eval_chunk(c, kLexThreads - 1, sm->start[kLexThreads - 1]);
    a->st1_state[tile] = (uint8_t)(x < 0 ? 0 : x);
    __threadfence();
    st_release_u32(a->st1_flag + tile, 2u);
  }

  // ---- pass 2a: boundaries and kept-token count from the true start ----
  const uint8_t *sflags = a->sflags;
  const uint8_t *sterm = a->sterm;
  unsigned long long bmask = 0;
  long long cnt = 0, lastb = 0;
  int x = sm->start[t];
  bool final_tok = false;
  int final_term = 0;
  {
    uint8_t *tbytes = reinterpret_cast<uint8_t *>(sm->bytes) + t * kLexChunk;
    bool died = false;
    for (int j = 0; j < nb; ++j) {
      const unsigned long long p = g0 + j;
      const int y = step(c, x, cls_of(c, tbytes[j]));
      if (p >= 1 && (__ldg(sflags + y) & 1)) {
        bmask |= 1ull << j;
        const int tm = __ldg(sterm + x);
        tbytes[j] = (uint8_t)tm;  // terminal of the token ending at p-1
        if (__ldg(sflags + x) & 4) ++cnt;
        lastb = (long long)p;
      }
      if (y == dead) died = true;
      x = y;
    }
    if (died) record_reject(st, &st->lex_reject_reason, 1);
    if (nb > 0 && g0 + nb == n) {  // this thread holds the last byte
      final_tok = true;
      final_term = __ldg(sterm + x);
      if (__ldg(sflags + x) & 4) ++cnt;
      if (!(__ldg(sflags + x) & 2)) record_reject(st, &st->lex_reject_reason, 2);
    }
  }
  // ---- (count, last boundary) carry: block scan then look-back ----
  long long cnt_tot, pos_tot;
  const long long cnt_ex = block_exclusive_scan<long long>(cnt, AddI64(), 0ll, sm->scan_tmp, &cnt_tot);
  const long long pos_ex = block_exclusive_scan<long long>(lastb, MaxI64(), 0ll, sm->scan_tmp, &pos_tot);
  if (t == 0) {
    struct PairOp {
      __device__ Pair64 operator()(Pair64 e, Pair64 l) const { return Pair64{e.a + l.a, e.b > l.b ? e.b : l.b}; }
    };
    Pair64 agg{cnt_tot, pos_tot};
    Pair64 prefix{0, 0};
    if (tile > 0) {
      publish_pair(a->st2, (long long)tile, agg, false);
      prefix = lookback_pair(a->st2, (long long)tile, Pair64{0, 0}, PairOp(), st, kSiteLexCount);
    }
    const Pair64 inc = PairOp()(prefix, agg);
    publish_pair(a->st2, (long long)tile, inc, true);
    sm->tile_cnt_prefix = prefix.a;
    sm->tile_pos_prefix = prefix.b;
    if (tile + 1 == num_tiles) st->num_tokens = (unsigned long long)inc.a;
  }
  __syncthreads();

  // ---- pass 2b: write this chunk's kept tokens ----
  {
    unsigned long long out = (unsigned long long)(sm->tile_cnt_prefix + cnt_ex);
    long long tok_start = sm->tile_pos_prefix > pos_ex ? sm->tile_pos_prefix : pos_ex;
    const uint8_t *tbytes = reinterpret_cast<const uint8_t *>(sm->bytes) + t * kLexChunk;
    const int ignore = a->ignore;
    const unsigned long long len_max = a->len_max;
    bool too_long = false;
    for (unsigned long long m = bmask; m; m &= m - 1) {
      const int j = __ffsll((long long)m) - 1;
      const long long p = (long long)(g0 + j);
      const int tm = tbytes[j];
      if (tm != ignore) {
        const unsigned long long len = (unsigned long long)(p - tok_start);
        if (len > len_max) too_long = true;
        store_uint(a->tok_ids, out, a->term_w, (unsigned long long)tm);
        store_uint(a->tok_starts, out, a->idx_w, (unsigned long long)tok_start);
        store_uint(a->tok_lens, out, a->len_w, len);
        ++out;
      }
      tok_start = p;
    }
    if (final_tok && final_term != ignore) {
      const unsigned long long len = n - (unsigned long long)tok_start;
      if (len > len_max) too_long = true;
      store_uint(a->tok_ids, out, a->term_w, (unsigned long long)final_term);
      store_uint(a->tok_starts, out, a->idx_w, (unsigned long long)tok_start);
      store_uint(a->tok_lens, out, a->len_w, len);
    }
    if (too_long) record_reject(st, &st->lex_reject_reason, 3);
  }
}

}  // namespace alpacc
