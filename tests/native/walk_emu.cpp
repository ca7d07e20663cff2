// Test harness (tests only): a sequential CPU emulation of the depth-walk
// algorithm of alpacc_b200/csrc/parser.cu (pse_tile_kernel and
// pse_resolve_kernel) - tiles of 2048 elements, chunks of 8 per thread, the
// near queries (own chunk, previous chunk), the warps' queued queries with the
// binary descent over window minima and the earlier warps, each tile's
// staircase and unanswered queries, and the resolve's walk back over tile and
// super-tile minima with a binary search of the answering tile's staircase.
// Its answers are compared with the definition they implement, walked
// directly: the latest earlier element whose depth is <= the query value (a
// right bracket's h - 1, a production's h), the bracket type check, and the
// parent / compaction formulas. The parallel mechanics (barriers, look-back,
// tickets) are not emulated.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

namespace {

constexpr int kThreads = 256, kItems = 8, kTile = kThreads * kItems, kWarp = 32, kWarps = kThreads / kWarp;
constexpr int kSuperShift = 8;

}  // namespace

// mode 0: brackets (elems: bit 31 = left, low bits type); mode 1: parents
// (elems: production ids, arity / is_term per production). Fills parent[e]
// (parents) with the answer index, or -1 for the root; returns the reject
// reason (0 when none), or -1 when the emulation and the direct walk disagree
// (details in mismatch[0..1]: element or tile, kind).
extern "C" int walk_emu(int mode, const uint32_t *elems, long long E, const int32_t *arity, const uint8_t *is_term,
                        long long *parent, long long *mismatch) {
  const bool parents = mode == 1;
  auto step = [&](uint32_t v) { return parents ? arity[v] - 1 : ((v >> 31) ? 1 : -1); };
  auto term = [&](uint32_t v) { return parents ? (is_term[v] ? 1 : 0) : 0; };
  const long long tiles = (E + kTile - 1) / kTile;
  // ---- direct definition ----
  std::vector<long long> h(E), tinc(E);
  {
    long long d = parents ? 1 : 0, tc = 0;
    for (long long e = 0; e < E; ++e) {
      h[e] = d;
      d += step(elems[e]);
      tc += term(elems[e]);
      tinc[e] = tc;
    }
  }
  std::vector<long long> want(E, -2);  // -2: no query
  int want_reject = 0;
  {
    std::vector<long long> stack;  // indices with strictly increasing depths, latest last
    for (long long e = 0; e < E; ++e) {
      bool query = parents ? e > 0 : !(elems[e] >> 31);
      if (query) {
        const long long qv = parents ? h[e] : h[e] - 1;
        long long f = -1;
        for (long long k = (long long)stack.size() - 1; k >= 0; --k)
          if (h[stack[k]] <= qv) {
            f = stack[k];
            break;
          }
        want[e] = f;
        if (!parents) {
          if (f < 0) want_reject = want_reject ? want_reject : 3;
          else if ((elems[f] ^ elems[e]) & 0x7fffffffu) want_reject = want_reject ? want_reject : 2;
        }
      }
      while (!stack.empty() && h[stack.back()] >= h[e]) stack.pop_back();
      stack.push_back(e);
    }
  }
  // ---- the tile algorithm ----
  std::vector<long long> got(E, -2);
  int reject = 0;
  auto rej = [&](int r) {
    if (!reject) reject = r;
  };
  std::vector<long long> tile_min(tiles, LLONG_MAX);
  std::vector<std::vector<long long>> stair_off(tiles), stair_val(tiles), q_off(tiles), q_val(tiles);
  long long prefix_s = 0;
  for (long long tile = 0; tile < tiles; ++tile) {
    const long long tile0 = tile * kTile;
    std::vector<long long> hr(kTile, 0);
    std::vector<int> valid(kTile, 0);
    long long run = 0;
    for (int i = 0; i < kTile; ++i) {
      hr[i] = run;
      if (tile0 + i < E) {
        valid[i] = 1;
        run += step(elems[tile0 + i]);
      }
    }
    std::vector<long long> cmin(kThreads, LLONG_MAX);
    for (int t = 0; t < kThreads; ++t)
      for (int j = 0; j < kItems; ++j)
        if (valid[t * kItems + j]) cmin[t] = std::min(cmin[t], hr[t * kItems + j]);
    // lv[k][i]: min of chunk minima over (i - 2^k, i] within i's warp
    std::vector<std::vector<long long>> lv(6, std::vector<long long>(kThreads));
    for (int i = 0; i < kThreads; ++i) {
      const int lane = i % kWarp;
      for (int k = 0; k < 6; ++k) {
        long long m = LLONG_MAX;
        for (int x = std::max(0, lane - (1 << k) + 1); x <= lane; ++x) m = std::min(m, cmin[i - lane + x]);
        lv[k][i] = m;
      }
    }
    std::vector<long long> wmin(kWarps);
    for (int w = 0; w < kWarps; ++w) wmin[w] = lv[5][w * kWarp + kWarp - 1];
    std::vector<int> ans(kTile, -2);  // local answer index; -1 pending; -2 no query; -3 root
    auto latest_le = [&](int chunk, long long qv) {
      for (int jj = kItems - 1; jj >= 0; --jj)
        if (hr[chunk * kItems + jj] <= qv) return chunk * kItems + jj;
      return -1;
    };
    for (int t = 0; t < kThreads; ++t)
      for (int j = 0; j < kItems; ++j) {
        const int i = t * kItems + j;
        const long long e = tile0 + i;
        if (!valid[i]) continue;
        long long qv;
        if (parents) {
          if (e == 0) {
            ans[i] = -3;
            continue;
          }
          qv = hr[i];
        } else {
          if (elems[e] >> 31) continue;
          qv = hr[i] - 1;
        }
        int f = -1;
        for (int jj = 0; jj < j; ++jj)
          if (hr[t * kItems + jj] <= qv) f = t * kItems + jj;
        if (f < 0 && t > 0 && cmin[t - 1] <= qv) f = latest_le(t - 1, qv);
        ans[i] = f >= 0 ? f : -1;
      }
    // the warps' queued queries
    for (int i = 0; i < kTile; ++i) {
      if (ans[i] != -1) continue;
      const int ct = i / kItems, warp = ct / kWarp;
      const long long qv = hr[i] - (parents ? 0 : 1);
      int found = -1;
      int pos = ct - warp * kWarp - 2;
      if (pos >= 0 && lv[5][warp * kWarp + pos] <= qv) {
        for (int k = 4; k >= 0; --k)
          if (pos >= (1 << k) && lv[k][warp * kWarp + pos] > qv) pos -= 1 << k;
        found = latest_le(warp * kWarp + pos, qv);
      }
      for (int w = warp - 1; w >= 0 && found < 0; --w) {
        if (wmin[w] > qv) continue;
        int p = w * kWarp + kWarp - 1;
        for (int k = 4; k >= 0; --k)
          if (lv[k][p] > qv && p - (1 << k) >= w * kWarp) p -= 1 << k;
        found = latest_le(p, qv);
      }
      ans[i] = found;
    }
    for (int i = 0; i < kTile; ++i) {
      if (!valid[i]) continue;
      const long long e = tile0 + i;
      if (ans[i] >= 0) {
        got[e] = tile0 + ans[i];
        if (!parents && ((elems[tile0 + ans[i]] ^ elems[e]) & 0x7fffffffu)) rej(2);
      } else if (ans[i] == -3) {
        got[e] = -1;
      }
    }
    // staircase and unanswered queries (global depths)
    const long long off = (parents ? 1 : 0) + prefix_s;
    long long later = LLONG_MAX;
    std::vector<long long> so, sv;
    for (int i = kTile - 1; i >= 0; --i) {
      if (!valid[i]) continue;
      if (hr[i] < later) {
        so.push_back(i);
        sv.push_back(hr[i] + off);
        later = hr[i];
      }
    }
    std::reverse(so.begin(), so.end());
    std::reverse(sv.begin(), sv.end());
    for (size_t k = 1; k < sv.size(); ++k)
      if (sv[k] <= sv[k - 1]) return mismatch[0] = tile, mismatch[1] = 10, -1;  // the staircase must increase
    stair_off[tile] = so;
    stair_val[tile] = sv;
    for (int i = 0; i < kTile; ++i)
      if (valid[i] && ans[i] == -1) {
        q_off[tile].push_back(i);
        q_val[tile].push_back(hr[i] + off - (parents ? 0 : 1));
      }
    for (size_t k = 1; k < q_val[tile].size(); ++k)
      if (q_val[tile][k] >= q_val[tile][k - 1]) return mismatch[0] = tile, mismatch[1] = 11, -1;  // must decrease
    long long m = LLONG_MAX;
    for (int w = 0; w < kWarps; ++w) m = std::min(m, wmin[w]);
    tile_min[tile] = m + off;
    prefix_s += run;
    if (tile == tiles - 1 && !parents && prefix_s != 0) rej(3);
  }
  // ---- resolve ----
  const long long supers = (tiles >> kSuperShift) + 1;
  std::vector<long long> super_min(supers, LLONG_MAX);
  for (long long tl = 0; tl < tiles; ++tl) super_min[tl >> kSuperShift] = std::min(super_min[tl >> kSuperShift], tile_min[tl]);
  auto latest_tile_le = [&](long long hi, long long qv) -> long long {
    const long long sup0 = (hi >> kSuperShift) << kSuperShift;
    for (long long x = hi; x >= sup0; --x)
      if (tile_min[x] <= qv) return x;
    for (long long sp = (sup0 >> kSuperShift) - 1; sp >= 0; --sp) {
      if (super_min[sp] > qv) continue;
      for (long long x = ((sp + 1) << kSuperShift) - 1; x >= (sp << kSuperShift); --x)
        if (x < tiles && tile_min[x] <= qv) return x;
      return -1;  // the super-tile's minimum comes from a tile above (cannot happen in one document)
    }
    return -1;
  };
  for (long long tile = 0; tile < tiles; ++tile) {
    const size_t nq = q_off[tile].size();
    long long j = tile - 1;
    size_t q = 0;
    while (q < nq) {
      j = j >= 0 ? latest_tile_le(j, q_val[tile][q]) : -1;
      if (j < 0) break;
      size_t ok = 0;
      for (size_t l = 0; l < 32 && q + l < nq; ++l) {
        const long long qv = q_val[tile][q + l];
        if (qv < tile_min[j]) break;  // the answered lanes are a prefix (values decrease)
        const std::vector<long long> &sv = stair_val[j];
        int lo = 0, hi = (int)sv.size() - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (sv[mid] <= qv) lo = mid;
          else hi = mid - 1;
        }
        const long long e = tile * kTile + q_off[tile][q + l];
        const long long p = j * kTile + stair_off[j][lo];
        got[e] = p;
        if (!parents && ((elems[p] ^ elems[e]) & 0x7fffffffu)) rej(2);
        ++ok;
      }
      q += ok;
    }
    for (; q < nq; ++q) {  // no earlier tile answers the rest
      const long long e = tile * kTile + q_off[tile][q];
      if (!parents) rej(3);
      got[e] = -1;  // compute_parents' parent 0 of an empty stack
    }
  }
  // ---- compare ----
  for (long long e = 0; e < E; ++e) {
    const long long w = want[e] == -2 ? -2 : want[e];
    const long long g = got[e];
    if (parents) {
      const long long ws = e == 0 ? -1 : w;  // the root has no query
      if (g != ws) return mismatch[0] = e, mismatch[1] = 1, -1;
      parent[e] = g;
    } else if (w != -2 && w >= 0 && g != w) {
      return mismatch[0] = e, mismatch[1] = 2, -1;
    }
  }
  // (which reason a rejected walk records first depends on the order tiles
  // finish on the GPU; the record of a rejected parse does not carry it)
  if ((reject != 0) != (want_reject != 0)) return mismatch[0] = reject, mismatch[1] = want_reject, -1;
  (void)tinc;
  return reject;
}
