// Data-parallel LLP parser for sm_100a: the semantics of parse_test,
// compute_parents and compact_tree (backends/c/parser.c:49-153).
//
// pair_kernel     per token position: the (q, k) key around it, a dense-table
//                 lookup of its stack actions and productions, and the scatter
//                 of both into flat arrays at offsets from a decoupled
//                 look-back scan (parser.c:60-84; parser.cu:378-449 phases A-C).
// pse_tile_kernel depth walk over brackets (+1 left, -1 right) or productions
//                 (+arity-1), with the match of each right bracket / the parent
//                 of each production found as the previous element whose depth
//                 is <= a query value: inside a thread's 8 elements, then in
//                 earlier chunks of the tile via a sparse table of chunk
//                 minima; the rest is queued (parser.c:74-87,103-118).
// pse_resolve     queued queries walk back over tile minima, then chunk
//                 minima, then elements of the tile that holds the answer.
// compact_kernel  drops terminal productions, remaps parents and writes
//                 token_parents (parser.c:126-153).
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

__global__ void __launch_bounds__(kPairThreads) pair_kernel(PairArgs a) {
  __shared__ unsigned s_tile;
  __shared__ long long s_tmp[kPairThreads / 32];
  __shared__ long long s_prefix_b, s_prefix_p;
  const int t = threadIdx.x;
  DeviceStatus *st = a.status;
  if (t == 0) s_tile = atomicAdd(a.ticket, 1u);
  __syncthreads();
  const unsigned long long tile = s_tile;
  const long long T = (long long)*a.num_tokens;
  const long long m = T + 2;
  const long long tile0 = (long long)tile * kPairTile;
  if (tile0 >= m) return;  // beyond the data: nobody waits on this tile
  const int L = a.q + a.k;

  uint32_t rec[kPairItems];
  long long sb = 0, sp = 0;
  bool missing = false;
#pragma unroll
  for (int j = 0; j < kPairItems; ++j) {
    const long long i = tile0 + (long long)t * kPairItems + j;
    rec[j] = 0xffffffffu;
    if (i >= m) continue;
    unsigned long long d = 0;
    for (int x = 0; x < L; ++x) {
      const long long pos = i - a.q + x;
      int term;
      if (pos < 0 || pos >= m) term = a.empty_t;
      else if (pos == 0) term = a.start_t;
      else if (pos == m - 1) term = a.end_t;
      else term = (int)load_uint(a.tok_ids, (unsigned long long)(pos - 1), a.term_w);
      d = d * (unsigned long long)a.nt + (unsigned long long)term;
    }
    const uint32_t r = __ldg(a.dense + d);
    rec[j] = r;
    if (r == 0xffffffffu) {
      missing = true;
      continue;
    }
    sb += __ldg(a.rec_nb + r);
    sp += __ldg(a.rec_np + r);
  }
  if (missing) record_reject(st, &st->parse_reject_reason, 1);
  long long tb, tp;
  const long long eb = block_exclusive_scan<long long>(sb, AddI64(), 0ll, s_tmp, &tb);
  const long long ep = block_exclusive_scan<long long>(sp, AddI64(), 0ll, s_tmp, &tp);
  if (t < kWarp) {
    const Pair64 agg{tb, tp};
    Pair64 prefix{0, 0};
    if (tile > 0) {
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
  unsigned long long ob = (unsigned long long)(s_prefix_b + eb);
  unsigned long long op = (unsigned long long)(s_prefix_p + ep);
  bool overflow = false;
#pragma unroll
  for (int j = 0; j < kPairItems; ++j) {
    const uint32_t r = rec[j];
    if (r == 0xffffffffu) continue;
    const int nb = __ldg(a.rec_nb + r), np = __ldg(a.rec_np + r);
    const uint32_t ss = __ldg(a.rec_ss + r), ps = __ldg(a.rec_ps + r);
    if (ob + nb > a.br_cap || op + np > a.pr_cap) {
      overflow = true;
      break;
    }
    for (int x = 0; x < nb; ++x) a.br_out[ob + x] = __ldg(a.stacks + ss + x);
    for (int x = 0; x < np; ++x) a.pr_out[op + x] = __ldg(a.prods + ps + x);
    ob += nb;
    op += np;
  }
  if (overflow) atomicCAS(&st->error, 0, -4 /* ALPACC_E_CAPACITY */);
}

// ---------------------------------------------------------------------------
// Previous-smaller search over depth walks
// ---------------------------------------------------------------------------

namespace {

constexpr int kPseStride = kPseItems + 1;  // odd word stride: conflict-free per-thread rows

struct PseSmem {
  int32_t h[kPseThreads * kPseStride];
  uint32_t v[kPseThreads * kPseStride];
  int32_t lv[8][kPseThreads];   // lv[l][i] = min of chunk minima (i-2^l, i]
  int32_t pm[kPseThreads];      // prefix minimum of chunk minima
  long long tmp[kPseThreads / 32];
  long long prefix_a, prefix_b;
  unsigned long long qbase;
};

// step of an element and whether it carries a query
__device__ __forceinline__ int pse_step(const PseArgs &a, uint32_t v) {
  if (a.mode == kPseBrackets) return (v >> 31) ? 1 : -1;
  return __ldg(a.arity + v) - 1;
}

}  // namespace

__global__ void __launch_bounds__(kPseThreads, 4) pse_tile_kernel(PseArgs a) {
  __shared__ unsigned s_tile;
  __shared__ PseSmem sm;
  const int t = threadIdx.x;
  DeviceStatus *st = a.status;
  if (t == 0) s_tile = atomicAdd(a.ticket, 1u);
  __syncthreads();
  const unsigned long long tile = s_tile;
  const long long E = (long long)*a.count;
  const long long tile0 = (long long)tile * kPseTile;
  if (tile0 >= E) return;
  const bool parents = a.mode == kPseParents;

  // ---- load, local steps ----
  int rel[kPseItems];
  int loc_term[kPseItems];
  long long ssum = 0, tsum = 0;
#pragma unroll
  for (int j = 0; j < kPseItems; ++j) {
    const long long e = tile0 + (long long)t * kPseItems + j;
    uint32_t v = 0;
    int stp = 0, tm = 0;
    if (e < E) {
      v = a.elems[e];
      stp = pse_step(a, v);
      if (parents) tm = __ldg(a.is_term + v) ? 1 : 0;
    }
    sm.v[t * kPseStride + j] = v;
    rel[j] = (int)ssum;
    ssum += stp;
    tsum += tm;
    loc_term[j] = (int)tsum;
  }
  long long tot_s, tot_t;
  const long long ex_s = block_exclusive_scan<long long>(ssum, AddI64(), 0ll, sm.tmp, &tot_s);
  const long long ex_t = block_exclusive_scan<long long>(tsum, AddI64(), 0ll, sm.tmp, &tot_t);
  // Publish the aggregate at once, so that later tiles' look-back can pass
  // this tile while it is still searching; tile 0's aggregate is its
  // inclusive prefix.
  if (t == 0) publish_pair(a.st, (long long)tile, Pair64{tot_s, tot_t}, tile == 0);

  // ---- depths relative to the tile start, chunk minima ----
  // The search compares depths only with each other, so it runs on relative
  // depths; the tile's offset is added when the results are written.
  int cmin = INT_MAX;
#pragma unroll
  for (int j = 0; j < kPseItems; ++j) {
    const long long e = tile0 + (long long)t * kPseItems + j;
    const int32_t h = (int32_t)(ex_s + rel[j]);
    sm.h[t * kPseStride + j] = h;
    if (e < E && h < cmin) cmin = h;
  }
  sm.lv[0][t] = cmin;
  __syncthreads();
  for (int l = 1; l < 8; ++l) {
    const int w = 1 << (l - 1);
    int v = sm.lv[l - 1][t];
    if (t >= w) {
      const int o = sm.lv[l - 1][t - w];
      v = o < v ? o : v;
    }
    sm.lv[l][t] = v;
    __syncthreads();
  }
  sm.pm[t] = sm.lv[7][t];  // covers (t-128, t]; complete with a second window below
  __syncthreads();
  if (t >= 128) {
    const int o = sm.lv[7][t - 128];
    if (o < sm.pm[t]) sm.pm[t] = o;
  }
  __syncthreads();

  // ---- queries inside the tile ----
  int pending = 0;
  int32_t ans[kPseItems];
#pragma unroll
  for (int j = 0; j < kPseItems; ++j) {
    ans[j] = INT_MIN;  // INT_MIN: no query
    const long long e = tile0 + (long long)t * kPseItems + j;
    if (e >= E) continue;
    const uint32_t v = sm.v[t * kPseStride + j];
    const int32_t h = sm.h[t * kPseStride + j];
    int32_t qv;
    if (parents) {
      if (e == 0) {
        ans[j] = 0;
        continue;
      }
      qv = h;
    } else {
      if (v >> 31) continue;  // left bracket: no query
      qv = h - 1;
    }
    int32_t found = -1;
    for (int jj = j - 1; jj >= 0; --jj)
      if (sm.h[t * kPseStride + jj] <= qv) {
        found = t * kPseItems + jj;
        break;
      }
    if (found < 0 && t > 0 && sm.pm[t - 1] <= qv) {
      int pos = t - 1;
      for (int l = 7; l >= 0; --l)
        if (pos - (1 << l) + 1 >= 0 && sm.lv[l][pos] > qv) pos -= 1 << l;
      for (int jj = kPseItems - 1; jj >= 0; --jj)
        if (sm.h[pos * kPseStride + jj] <= qv) {
          found = pos * kPseItems + jj;
          break;
        }
    }
    if (found >= 0) {
      if (!parents) {
        const uint32_t pv = sm.v[(found / kPseItems) * kPseStride + found % kPseItems];
        if ((pv & 0x7fffffffu) != (v & 0x7fffffffu)) record_reject(st, &st->parse_reject_reason, 2);
      }
      ans[j] = (int32_t)(tile0 + found);
    } else {
      ans[j] = -1;
      ++pending;
    }
  }
  long long tot_p;
  const long long ex_p = block_exclusive_scan<long long>(pending, AddI64(), 0ll, sm.tmp, &tot_p);

  // ---- the tile's prefix: look-back by warp 0, now that predecessors had time ----
  if (t < kWarp) {
    Pair64 prefix{0, 0};
    if (tile > 0) prefix = warp_lookback_pair(a.st, (long long)tile, Pair64{0, 0}, AddPair(), st, kSitePse);
    if (t == 0) {
      const Pair64 inc{prefix.a + tot_s, prefix.b + tot_t};
      if (tile > 0) publish_pair(a.st, (long long)tile, inc, true);
      sm.prefix_a = prefix.a;
      sm.prefix_b = prefix.b;
      if (tot_p > 0) sm.qbase = atomicAdd(a.queue_len, (unsigned long long)tot_p);
      if (tile0 + kPseTile >= E) {  // last tile: global checks
        if (!parents) {
          if (inc.a != 0) record_reject(st, &st->parse_reject_reason, 3);
        } else {
          const long long T = (long long)st->num_tokens;
          if (inc.b != T) record_reject(st, &st->parse_reject_reason, 4);
          st->num_nodes = (unsigned long long)(E - inc.b);
        }
      }
    }
  }
  __syncthreads();

  // ---- absolute depths, minima, terminal counts, answers, queue ----
  const int32_t off = (int32_t)((parents ? 1 : 0) + sm.prefix_a);
#pragma unroll
  for (int j = 0; j < kPseItems; ++j) {
    const long long e = tile0 + (long long)t * kPseItems + j;
    if (e < E) {
      a.h[e] = sm.h[t * kPseStride + j] + off;
      if (parents) a.tinc[e] = (int32_t)(sm.prefix_b + ex_t + loc_term[j]);
    }
  }
  a.chunk_min[tile * kPseThreads + t] = cmin == INT_MAX ? INT_MAX : cmin + off;
  if (t == 0) {
    const int32_t r = sm.lv[7][kPseThreads - 1] < sm.lv[7][127] ? sm.lv[7][kPseThreads - 1] : sm.lv[7][127];
    const int32_t tm = r + off;  // the tile holds at least one element
    a.tile_min[tile] = tm;
    atomicMin(a.super_min + (tile >> kPseSuperShift), tm);
  }
  unsigned long long qi = sm.qbase + (unsigned long long)ex_p;
#pragma unroll
  for (int j = 0; j < kPseItems; ++j) {
    const long long e = tile0 + (long long)t * kPseItems + j;
    if (e >= E || ans[j] == INT_MIN) continue;
    if (parents) a.answer[e] = ans[j];
    if (ans[j] == -1) {
      if (qi < a.queue_cap) a.queue[qi] = (unsigned long long)e;
      else atomicCAS(&st->error, 0, -4 /* ALPACC_E_CAPACITY */);
      ++qi;
    }
  }
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

}  // namespace

// One warp per queued query: latest tile whose minimum is <= the query
// (within the query's super-tile of 256 tiles, else via super-tile minima),
// then the latest chunk of that tile, then the latest element of that chunk.
__global__ void pse_resolve_kernel(PseArgs a) {
  DeviceStatus *st = a.status;
  const unsigned long long qn = *a.queue_len;
  const long long E = (long long)*a.count;
  const bool parents = a.mode == kPseParents;
  const int lane = threadIdx.x & 31;
  const unsigned long long warp = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) >> 5;
  const unsigned long long warps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long qi = warp; qi < qn && qi < a.queue_cap; qi += warps) {
    const long long e = (long long)a.queue[qi];
    const uint32_t v = a.elems[e];
    const int32_t h = a.h[e];
    const int32_t qv = parents ? h : h - 1;
    const long long tile = e / kPseTile;
    const long long sup0 = (tile >> kPseSuperShift) << kPseSuperShift;
    long long tt = warp_latest_le(a.tile_min, tile - 1, sup0, qv, lane);
    if (tt < 0 && sup0 > 0) {
      const long long sp = warp_latest_le(a.super_min, (sup0 >> kPseSuperShift) - 1, 0, qv, lane);
      if (sp >= 0) tt = warp_latest_le(a.tile_min, ((sp + 1) << kPseSuperShift) - 1, sp << kPseSuperShift, qv, lane);
    }
    long long found = -1;
    if (tt >= 0) {
      const long long c = warp_latest_le(a.chunk_min + tt * kPseThreads, kPseThreads - 1, 0, qv, lane);
      if (c >= 0) {
        const long long base = tt * kPseTile + c * kPseItems;
        const long long hi = base + kPseItems - 1 < E - 1 ? base + kPseItems - 1 : E - 1;
        found = warp_latest_le(a.h, hi, base, qv, lane);
      }
    }
    if (lane == 0) {
      if (parents) {
        // compute_parents takes 0 when its stack is empty
        a.answer[e] = found >= 0 ? (int32_t)found : 0;
      } else {
        if (found < 0) record_reject(st, &st->parse_reject_reason, 3);
        else if ((a.elems[found] & 0x7fffffffu) != (v & 0x7fffffffu)) record_reject(st, &st->parse_reject_reason, 2);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Compaction (compact_tree)
// ---------------------------------------------------------------------------

__global__ void compact_kernel(CompactArgs a) {
  const unsigned long long P = *a.count;
  const long long T = (long long)*a.num_tokens;
  for (unsigned long long e = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; e < P;
       e += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t prod = a.prods[e];
    long long p = e == 0 ? 0 : a.parent[e];
    if (p < 0 || (unsigned long long)p >= P) p = 0;  // only after a recorded reject or error
    const long long p_new = p - (long long)a.tinc[p];
    const long long ti = a.tinc[e];
    if (__ldg(a.is_term + prod)) {
      if (ti >= 1 && ti <= T)
        store_uint(a.token_parents, (unsigned long long)(ti - 1), a.idx_w, (unsigned long long)p_new);
    } else {
      const long long o = (long long)e - ti;
      if (o >= 0) {
        store_uint(a.node_prods, (unsigned long long)o, a.prod_w, prod);
        store_uint(a.node_parents, (unsigned long long)o, a.idx_w, (unsigned long long)p_new);
      }
    }
  }
}

}  // namespace alpacc
