// Shared device utilities for the sm_100a lex + parse kernels.
//
// * Status words: every kernel reports into a DeviceStatus in device memory
//   (reject / error / timeout) instead of trapping, so a bad input or an
//   exhausted wait never faults or hangs the GPU.
// * Tile publication for single-pass scans: payload words are written first,
//   then a flag with release semantics; readers spin on the flag with acquire
//   semantics and a bounded number of iterations (decoupled look-back,
//   Merrill & Garland 2016). A wait that runs out records ALPACC_E_TIMEOUT and
//   the kernel proceeds with a neutral value, so every CTA still finishes.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace alpacc {

constexpr int kWarp = 32;

// Where a bounded wait gave up (recorded in DeviceStatus::timeout_site).
enum TimeoutSite : int {
  kSiteNone = 0,
  kSiteLexState = 1,
  kSiteLexCount = 2,
  kSitePairs = 3,
  kSitePse = 4,
  kSiteLexLanes = 5,   // a loop bound below was exceeded (internal error)
  kSitePseQuery = 6,
  kSiteLexTiles = 7,
};

struct DeviceStatus {
  int reject;        // 1 when the input is rejected
  int error;         // ALPACC_E_* (negative) on an internal failure
  int timeout_site;  // TimeoutSite of the first wait that ran out
  int overflow;      // 1 when a scratch array was too small (the host grows it and runs again)
  unsigned long long num_tokens;
  unsigned long long num_brackets;
  unsigned long long num_productions;
  unsigned long long num_nodes;
  int lex_reject_reason;    // 1 dead state, 2 not accepting, 3 length overflow
  int parse_reject_reason;  // 1 missing pair, 2 bracket mismatch, 3 unbalanced, 4 terminal count
  unsigned long long scratch[4];
  unsigned long long last_boundary;  // last token boundary of the input (single-document lexer)
  int final_kept;    // the input's last token (ending at byte n) is kept: its terminal in final_term
  int final_term;
};

// Upper bound on spin iterations of one wait; with the back-off below this is
// several seconds, far beyond any legitimate wait on a healthy device.
constexpr unsigned kSpinLimit = 1u << 22;

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void record_timeout(DeviceStatus *st, int site) {
  atomicCAS(&st->timeout_site, 0, site);
  atomicCAS(&st->error, 0, -5 /* ALPACC_E_TIMEOUT */);
}

// A scratch array of the call is too small. Unlike an error, this does not
// stop the look-backs, so the counts the kernels publish stay exact and the
// host can size the retry from them.
__device__ __forceinline__ void record_overflow(DeviceStatus *st) {
  if (*reinterpret_cast<volatile int *>(&st->overflow) == 0) atomicExch(&st->overflow, 1);
}

__device__ __forceinline__ void record_reject(DeviceStatus *st, int *reason, int why) {
  if (st->reject == 0) atomicExch(&st->reject, 1);
  if (reason) atomicCAS(reason, 0, why);
}

// Spin until *flag >= want (acquire). Returns the flag value, or 0 after the
// iteration limit (and records a timeout).
__device__ __forceinline__ unsigned wait_flag(const unsigned *flag, unsigned want, DeviceStatus *st, int site) {
  unsigned ns = 32;
  for (unsigned it = 0; it < kSpinLimit; ++it) {
    unsigned v = ld_acquire_u32(flag);
    if (v >= want) return v;
    if (*reinterpret_cast<volatile int *>(&st->error) != 0) return 0;  // a CTA already failed
    __nanosleep(ns);
    if (ns < 1024) ns <<= 1;
  }
  record_timeout(st, site);
  return 0;
}

// ---------------------------------------------------------------------------
// Block-wide scans (warp shuffles + one shared-memory pass).
// ---------------------------------------------------------------------------

template <typename T, typename Op>
__device__ __forceinline__ T warp_inclusive_scan(T v, Op op) {
  const int lane = threadIdx.x & (kWarp - 1);
#pragma unroll
  for (int d = 1; d < kWarp; d <<= 1) {
    T o = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v = op(o, v);
  }
  return v;
}

// Exclusive scan over the block; `identity` is the neutral element. Returns
// this thread's exclusive prefix and writes the block total to *total.
// `smem` needs (blockDim.x / 32) elements.
template <typename T, typename Op>
__device__ __forceinline__ T block_exclusive_scan(T v, Op op, T identity, T *smem, T *total) {
  const int lane = threadIdx.x & (kWarp - 1);
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  T inc = warp_inclusive_scan(v, op);
  if (lane == kWarp - 1) smem[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < nwarps ? smem[lane] : identity;
    T wi = warp_inclusive_scan(w, op);
    if (lane < nwarps) smem[lane] = wi;  // inclusive prefix of warp totals
  }
  __syncthreads();
  T warp_prefix = warp == 0 ? identity : smem[warp - 1];
  T excl_in_warp = __shfl_up_sync(0xffffffffu, inc, 1);
  if (lane == 0) excl_in_warp = identity;
  T res = op(warp_prefix, excl_in_warp);
  *total = smem[nwarps - 1];
  __syncthreads();
  return res;
}

// 16-byte asynchronous global-to-shared copies (cp.async, cache-global):
// issued now, waited for with cp_async_wait<n> (at most n groups left in
// flight); both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// L2 prefetch of the 16-byte-aligned interior of [p, p + bytes) with one
// bulk prefetch (nothing outside the range is touched).
__device__ __forceinline__ void prefetch_l2(const void *p, unsigned long long bytes) {
  const unsigned long long a = ((unsigned long long)p + 15) & ~15ull;
  const unsigned long long e = ((unsigned long long)p + bytes) & ~15ull;
  if (e > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(a), "r"((unsigned)(e - a)) : "memory");
}

struct AddU64 {
  __device__ __forceinline__ unsigned long long operator()(unsigned long long a, unsigned long long b) const {
    return a + b;
  }
};
struct AddI64 {
  __device__ __forceinline__ long long operator()(long long a, long long b) const { return a + b; }
};
struct AddI32 {
  __device__ __forceinline__ int operator()(int a, int b) const { return a + b; }
};
struct MaxI32 {
  __device__ __forceinline__ int operator()(int a, int b) const { return a > b ? a : b; }
};
struct MaxI64 {
  __device__ __forceinline__ long long operator()(long long a, long long b) const { return a > b ? a : b; }
};
struct MinI64 {
  __device__ __forceinline__ long long operator()(long long a, long long b) const { return a < b ? a : b; }
};

// Two 32-bit exclusive scans over the block at once: a sum of `c` and a
// maximum of `p` (identity 0 for both). `sa` and `sb` need (blockDim.x / 32)
// elements each.
__device__ __forceinline__ void block_exclusive_scan2(int *sa, int *sb, int c, int p, int *c_ex, int *p_ex,
                                                      int *c_tot, int *p_tot) {
  const int lane = threadIdx.x & (kWarp - 1);
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  int ci = c, pi = p;
#pragma unroll
  for (int d = 1; d < kWarp; d <<= 1) {
    const int oc = __shfl_up_sync(0xffffffffu, ci, d);
    const int op = __shfl_up_sync(0xffffffffu, pi, d);
    if (lane >= d) {
      ci += oc;
      pi = op > pi ? op : pi;
    }
  }
  if (lane == kWarp - 1) {
    sa[warp] = ci;
    sb[warp] = pi;
  }
  __syncthreads();
  if (warp == 0) {
    int wc = lane < nwarps ? sa[lane] : 0, wp = lane < nwarps ? sb[lane] : 0;
#pragma unroll
    for (int d = 1; d < kWarp; d <<= 1) {
      const int oc = __shfl_up_sync(0xffffffffu, wc, d);
      const int op = __shfl_up_sync(0xffffffffu, wp, d);
      if (lane >= d) {
        wc += oc;
        wp = op > wp ? op : wp;
      }
    }
    if (lane < nwarps) {
      sa[lane] = wc;  // inclusive prefix of warp totals
      sb[lane] = wp;
    }
  }
  __syncthreads();
  int ec = __shfl_up_sync(0xffffffffu, ci, 1), ep = __shfl_up_sync(0xffffffffu, pi, 1);
  if (lane == 0) ec = ep = 0;
  if (warp > 0) {
    ec += sa[warp - 1];
    ep = sb[warp - 1] > ep ? sb[warp - 1] : ep;
  }
  *c_ex = ec;
  *p_ex = ep;
  *c_tot = sa[nwarps - 1];
  *p_tot = sb[nwarps - 1];
  __syncthreads();
}

// A pair scanned component-wise (used for (count, position) and (brackets,
// productions) carries).
struct Pair64 {
  long long a, b;
};

// ---------------------------------------------------------------------------
// Decoupled look-back over tiles for an associative pair carry.
//
// Tile i publishes its aggregate (flag 1) as soon as it is known and its
// inclusive prefix (flag 2) once the look-back resolved. A tile walks back
// from i-1, combining aggregates until it meets an inclusive prefix; one warp
// examines 32 predecessors per step.
// `tiles` holds per tile: flag (u32) in flags[i], aggregate in agg[i], inclusive
// in inc[i] (two u64 each).
// ---------------------------------------------------------------------------

struct PairTileState {
  unsigned *flags;            // [num_tiles]
  unsigned long long *agg;    // [num_tiles * 2]
  unsigned long long *inc;    // [num_tiles * 2]
};

template <typename Op>
__device__ __forceinline__ Pair64 combine(Pair64 x, Pair64 y, Op op) {
  return op(x, y);
}

// Exclusive block-wide scan of a pair carry (one pass instead of one per
// component); `smem` needs (blockDim.x / 32) elements.
template <typename Op>
__device__ __forceinline__ Pair64 block_exclusive_scan_pair(Pair64 v, Op op, Pair64 identity, Pair64 *smem,
                                                            Pair64 *total) {
  const int lane = threadIdx.x & (kWarp - 1);
  const int warp = threadIdx.x >> 5;
  const int nwarps = blockDim.x >> 5;
  Pair64 inc = v;
#pragma unroll
  for (int d = 1; d < kWarp; d <<= 1) {
    const Pair64 o{__shfl_up_sync(0xffffffffu, inc.a, d), __shfl_up_sync(0xffffffffu, inc.b, d)};
    if (lane >= d) inc = op(o, inc);
  }
  if (lane == kWarp - 1) smem[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    Pair64 w = lane < nwarps ? smem[lane] : identity;
#pragma unroll
    for (int d = 1; d < kWarp; d <<= 1) {
      const Pair64 o{__shfl_up_sync(0xffffffffu, w.a, d), __shfl_up_sync(0xffffffffu, w.b, d)};
      if (lane >= d) w = op(o, w);
    }
    if (lane < nwarps) smem[lane] = w;
  }
  __syncthreads();
  const Pair64 warp_prefix = warp == 0 ? identity : smem[warp - 1];
  Pair64 ex{__shfl_up_sync(0xffffffffu, inc.a, 1), __shfl_up_sync(0xffffffffu, inc.b, 1)};
  if (lane == 0) ex = identity;
  *total = smem[nwarps - 1];
  __syncthreads();
  return op(warp_prefix, ex);
}

__device__ __forceinline__ void publish_pair(PairTileState ts, long long tile, Pair64 v, bool inclusive) {
  unsigned long long *dst = inclusive ? ts.inc : ts.agg;
  st_relaxed_u64(dst + 2 * tile, (unsigned long long)v.a);
  st_relaxed_u64(dst + 2 * tile + 1, (unsigned long long)v.b);
  st_release_u32(ts.flags + tile, inclusive ? 2u : 1u);  // orders the payload stores before the flag
}

// Exclusive prefix of tile `tile`, computed by all 32 lanes of one warp (the
// result is returned to every lane). Each round reads the flags of the 32
// nearest unexamined predecessors at once (lane l: tile - 1 - l - 32*round),
// waits (bounded) until all of them have published, combines the aggregates
// up to the nearest inclusive prefix and stops there. `op` must be
// associative and commutative (sums and maxima here), so the lanes' values can
// be combined in any order.
template <typename Op>
__device__ Pair64 warp_lookback_pair(PairTileState ts, long long tile, Pair64 identity, Op op, DeviceStatus *st,
                                     int site) {
  const int lane = threadIdx.x & (kWarp - 1);
  Pair64 acc = identity;
  for (long long hi = tile - 1; hi >= 0; hi -= kWarp) {
    const long long j = hi - lane;
    unsigned f = j >= 0 ? ld_acquire_u32(ts.flags + j) : 2u;  // before tile 0: an inclusive identity
    unsigned ns = 32;
    unsigned it = 0;
    while (__any_sync(0xffffffffu, f == 0u)) {
      const bool failed = __any_sync(0xffffffffu, *reinterpret_cast<volatile int *>(&st->error) != 0);
      if (failed || ++it >= kSpinLimit) {
        if (!failed && lane == 0) record_timeout(st, site);
        return acc;  // neutral continuation; the status word carries the failure
      }
      __nanosleep(ns);
      if (ns < 1024) ns <<= 1;
      if (f == 0u) f = ld_acquire_u32(ts.flags + j);
    }
    const unsigned incl = __ballot_sync(0xffffffffu, f >= 2u);
    const int stop = incl ? __ffs(incl) - 1 : kWarp;  // nearest predecessor holding an inclusive prefix
    Pair64 v = identity;
    if (j >= 0 && lane < stop) {
      v = Pair64{(long long)ld_relaxed_u64(ts.agg + 2 * j), (long long)ld_relaxed_u64(ts.agg + 2 * j + 1)};
    } else if (j >= 0 && lane == stop) {
      v = Pair64{(long long)ld_relaxed_u64(ts.inc + 2 * j), (long long)ld_relaxed_u64(ts.inc + 2 * j + 1)};
    }
#pragma unroll
    for (int d = kWarp / 2; d; d >>= 1) {
      const Pair64 o{__shfl_xor_sync(0xffffffffu, v.a, d), __shfl_xor_sync(0xffffffffu, v.b, d)};
      v = op(v, o);
    }
    acc = op(v, acc);
    if (incl) break;
  }
  return acc;
}

}  // namespace alpacc
