// Shared-memory subtree phase of the left-balanced builders (build.cu and
// inplace.cu): scalar keys, the per-dimension presort and the level loop.
#pragma once

#include "common.cuh"

namespace ckb {
namespace build {

constexpr int ilog2_floor(int x) { return x <= 1 ? 0 : 1 + ilog2_floor(x >> 1); }
// Max subtree size a single tree's subtree phase finishes in shared memory:
// 1024 points (54 KB, 4 CTAs of 256 threads per SM) measured faster than
// 2048 (108 KB, 2 per SM; one global level fewer) -- 10M points 5.60 against
// 5.71 ms.  The forest keeps three tile classes (kForestTiles).
constexpr int kTile = 1024;
// threads of a subtree CTA, every tile class (for 2048-point tiles 256
// measured faster than 512 with the ballot partitions: batched build 15.0
// against 15.5 ms)
constexpr int kSubThreads = 256;

// ---------------------------------------------------------------------------
// scalar helpers
// ---------------------------------------------------------------------------
template <int SC> struct Scalar;
template <> struct Scalar<0> {
  __device__ static uint32_t key(uint32_t bits) { return float_key(__uint_as_float(bits)); }
  __device__ static uint32_t bits(uint32_t key) { return __float_as_uint(key_float(key)); }
  // box.h:112-125 widestDimension (ties to the higher dim) on a key box
  __device__ static int widest(const uint32_t *lo, const uint32_t *hi, int D)
  {
    int best = 0;
    float wbest = 0.f;
    for (int d = 0; d < D; d++) {
      float w = __fsub_rn(key_float(hi[d]), key_float(lo[d]));
      if (w < wbest) continue;
      wbest = w;
      best = d;
    }
    return best;
  }
};
template <> struct Scalar<1> {
  __device__ static uint32_t key(uint32_t bits) { return int_key(int32_t(bits)); }
  __device__ static uint32_t bits(uint32_t key) { return uint32_t(key_int(key)); }
  __device__ static int widest(const uint32_t *lo, const uint32_t *hi, int D)
  {
    int best = 0;
    int32_t wbest = 0;
    for (int d = 0; d < D; d++) {
      int32_t w = int32_t(uint32_t(key_int(hi[d])) - uint32_t(key_int(lo[d])));
      if (w < wbest) continue;
      wbest = w;
      best = d;
    }
    return best;
  }
};

__device__ inline int rr_dim(int64_t g, int D) { return level_of(g) % D; }

// ---------------------------------------------------------------------------
// subtree phase: one CTA per subtree of <= kTile points
// ---------------------------------------------------------------------------
template <int D, int TILE, int NT>
struct SubSmem {
  uint32_t key[D][TILE];
  uint32_t idx[TILE];
  uint16_t list[2][D][TILE];
  uint16_t segOf[2][TILE];
  union {
    struct {
      uint32_t scan[TILE];  // level partitions: per-subtree offsets
      struct {
        uint16_t t0[TILE], t1[TILE], b[TILE], r[TILE];
      } u_sub;
    } lv;                            // the levels
    uint16_t rh[D][NT / 32][256];    // presort: per dim, per-warp digit counts
  };
  uint32_t red[D * 2 * (NT / 32)];
  uint16_t locPivot[2 * TILE];
  uint8_t locDim[2 * TILE];
  uint8_t flag[TILE];
  uint8_t subDim[TILE];
  uint16_t queue[TILE];
  uint32_t warpSums[TILE / 32];  // partitions: per (round, warp) side counts
  uint32_t qcount[2];  // run queue length, by level parity
  uint32_t rootLo[D], rootHi[D];
};

// Presort (subtree phase): one stable LSD radix sort per dimension of the
// indices 0..m-1 by key[d][i], the D sorts sharing each pass's barriers.
// Keys are sorted over their span (key - min), so 0 to 4 passes of 8-bit
// digits.  Warp w owns a contiguous run of positions; match_any ranks equal
// digits inside a round of 32, per-warp digit counts are scanned digit-major
// over the warps.
// S.list[0][d] receives the sorted indices of dim d, S.list[1][d] is
// scratch.  (Sharing the barriers: batched build 15.2 -> 14.3 ms at
// 1024-point tiles; ranks kept from the histogram rounds: batched build
// 14.4 -> 13.2 ms, the 10M-point build 4.90 -> 4.85 ms.)
template <int D, int TILE, int NT>
__device__ void sub_radix_sort_all(SubSmem<D, TILE, NT> &S, int m)
{
  constexpr int W = NT / 32;
  static_assert(NT >= 256 && NT % 256 == 0, "a thread per digit in the scan");
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  uint32_t lo[D], hi[D];
#pragma unroll
  for (int d = 0; d < D; d++) {
    lo[d] = 0xffffffffu;
    hi[d] = 0u;
  }
  for (int i = tid; i < m; i += NT) {
#pragma unroll
    for (int d = 0; d < D; d++) {
      const uint32_t k = S.key[d][i];
      lo[d] = min(lo[d], k);
      hi[d] = max(hi[d], k);
      S.list[0][d][i] = uint16_t(i);
    }
  }
#pragma unroll
  for (int d = 0; d < D; d++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = min(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = max(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
    if (lane == 0) {
      S.red[d * 2 * W + wid] = lo[d];
      S.red[d * 2 * W + W + wid] = hi[d];
    }
  }
  __syncthreads();
  uint32_t kmin[D];
  int passes[D];
  int maxPasses = 0;
#pragma unroll
  for (int d = 0; d < D; d++) {
    uint32_t a = 0xffffffffu, z = 0u;
    for (int w = 0; w < W; w++) {
      a = min(a, S.red[d * 2 * W + w]);
      z = max(z, S.red[d * 2 * W + W + w]);
    }
    kmin[d] = a;
    const uint32_t span = z >= a ? z - a : 0u;
    passes[d] = ((span ? 32 - __clz(span) : 0) + 7) >> 3;
    maxPasses = max(maxPasses, passes[d]);
  }
  __syncthreads();  // red is reused by the scans below
  const int per = (m + W - 1) / W;
  const int w0 = min(m, wid * per), w1 = min(m, w0 + per);
  const uint32_t ltMask = (1u << lane) - 1u;
  uint32_t inTmp = 0;  // bit d: dim d's current order sits in S.list[1][d]
  // Where D x R words fit in registers, the histogram rounds keep each
  // item's index, digit and rank among its warp's items of that digit
  // (match_any plus the count before the round), so the scatter rounds only
  // add the warp's offset: no second match_any, key gather or warp syncs.
  constexpr int R = TILE / NT;  // rounds of 32 positions per warp (per <= 32 R)
  constexpr bool kKeep = D * R <= 16;
  static_assert(!kKeep || 32 * R <= 256, "ranks below 256 (8 bits)");
  uint32_t rec[kKeep ? D : 1][kKeep ? R : 1];
  for (int ps = 0; ps < maxPasses; ps++) {
    const int shift = ps * 8;
    for (int i = tid; i < D * W * 256; i += NT) (&S.rh[0][0][0])[i] = 0;
    __syncthreads();
#pragma unroll
    for (int d = 0; d < D; d++) {
      if (ps >= passes[d]) continue;
      const uint16_t *src = S.list[(inTmp >> d) & 1u][d];
      if constexpr (kKeep) {
#pragma unroll
        for (int rr = 0; rr < R; rr++) {
          const int i = w0 + rr * 32 + lane;
          const bool valid = i < w1;
          const uint32_t v = valid ? uint32_t(src[i]) : 0u;
          const uint32_t dg = valid ? ((S.key[d][v] - kmin[d]) >> shift) & 255u : 256u + lane;
          const uint32_t peers = __match_any_sync(0xffffffffu, dg);
          const uint32_t below = __popc(peers & ltMask);
          const uint32_t before = valid ? uint32_t(S.rh[d][wid][dg]) : 0u;
          __syncwarp();  // every lane has read the count before its leader adds
          if (valid && below == 0) S.rh[d][wid][dg] = uint16_t(before + __popc(peers));
          __syncwarp();
          rec[d][rr] = valid ? (v << 16) | (dg << 8) | (before + below) : 0xffffffffu;
        }
      } else {
        for (int base = w0; base < w1; base += 32) {
          const int i = base + lane;
          const bool valid = i < w1;
          const uint32_t dg = valid ? ((S.key[d][src[i]] - kmin[d]) >> shift) & 255u : 256u + lane;
          const uint32_t peers = __match_any_sync(0xffffffffu, dg);
          if (valid && (peers & ltMask) == 0) S.rh[d][wid][dg] += uint16_t(__popc(peers));
          __syncwarp();  // the next round's leaders read these counts
        }
      }
    }
    __syncthreads();
    {
      // digit-major exclusive offsets: threads 0..255 own one digit of each dim
      uint32_t run[D], incl[D];
#pragma unroll
      for (int d = 0; d < D; d++) {
        run[d] = 0;
        incl[d] = 0;
        if (tid < 256 && ps < passes[d]) {
#pragma unroll
          for (int w = 0; w < W; w++) {
            const uint32_t c = S.rh[d][w][tid];
            S.rh[d][w][tid] = uint16_t(run[d]);
            run[d] += c;
          }
          incl[d] = run[d];
          for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, incl[d], o);
            if (lane >= o) incl[d] += t;
          }
          if (lane == 31) S.red[d * W + wid] = incl[d];
        }
      }
      __syncthreads();
      if (tid < 256) {
#pragma unroll
        for (int d = 0; d < D; d++) {
          if (ps >= passes[d]) continue;
          uint32_t wbase = 0;
          for (int w = 0; w < wid; w++) wbase += S.red[d * W + w];
          const uint32_t dbase = wbase + incl[d] - run[d];
#pragma unroll
          for (int w = 0; w < W; w++) S.rh[d][w][tid] = uint16_t(S.rh[d][w][tid] + dbase);
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < D; d++) {
      if (ps >= passes[d]) continue;
      const uint16_t *src = S.list[(inTmp >> d) & 1u][d];
      uint16_t *dst = S.list[((inTmp >> d) & 1u) ^ 1u][d];
      if constexpr (kKeep) {
        // position = the warp's offset for the digit + the rank kept above
#pragma unroll
        for (int rr = 0; rr < R; rr++) {
          const uint32_t x = rec[d][rr];
          if (x != 0xffffffffu)
            dst[S.rh[d][wid][(x >> 8) & 255u] + (x & 255u)] = uint16_t(x >> 16);
        }
        continue;
      }
      for (int base = w0; base < w1; base += 32) {
        const int i = base + lane;
        const bool valid = i < w1;
        const uint16_t v = valid ? src[i] : uint16_t(0);
        const uint32_t dg = valid ? ((S.key[d][v] - kmin[d]) >> shift) & 255u : 256u + lane;
        const uint32_t peers = __match_any_sync(0xffffffffu, dg);
        const uint32_t pos = valid ? uint32_t(S.rh[d][wid][dg]) + __popc(peers & ltMask) : 0u;
        __syncwarp();
        if (valid) {
          dst[pos] = v;
          if ((peers & ltMask) == 0) S.rh[d][wid][dg] = uint16_t(S.rh[d][wid][dg] + __popc(peers));
        }
        __syncwarp();
      }
    }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < D; d++)
      if (ps < passes[d]) inTmp ^= 1u << d;
  }
  if (inTmp) {
#pragma unroll
    for (int d = 0; d < D; d++)
      if ((inTmp >> d) & 1u)
        for (int i = tid; i < m; i += NT) S.list[0][d][i] = S.list[1][d][i];
    __syncthreads();
  }
}

// Finishes the subtree under node s (level L0) of a tree of n records.
// Src supplies the data and takes the result:
//   src.load(S, m)             fills S.key[d][i] and S.idx[i] (the composite
//                              key's last word, unique) for the m points, in
//                              any order, and S.rootLo / S.rootHi (the
//                              subtree's domain box as keys) when the split
//                              dims are explicit; every thread calls it
//   src.anc_dim(a)             split dim of ancestor a of s (explicit dims)
//   src.settle(g, u, piv, dim, S)  node g (local index u) is the point in
//                              slot piv, split along dim
template <int SC, int D, int TILE, int NT, class Src>
__device__ void subtree_body(Src &src, int64_t n, int L0, int64_t s, bool explicitDims,
                             SubSmem<D, TILE, NT> &S)
{
  const int tid = threadIdx.x;
  const int m = int(subtree_size(s, n));
  if (m == 0) return;

  for (int i = tid; i < m; i += NT) S.segOf[0][i] = 0;
  src.load(S, m);
  if (tid < 2) S.qcount[tid] = 0;
  __syncthreads();

  // one coordinate-sorted index list per dimension (equal keys in any
  // order; runs of equal keys are ranked by the composite key below)
  sub_radix_sort_all<D, TILE, NT>(S, m);

  int cur = 0;
  int mact = m;
  const int lane = tid & 31, wid = tid >> 5;
  for (int j = 0; mact > 0; j++) {
    const int lvl = L0 + j;
    const int64_t g0 = ((s + 1) << j) - 1;
    const int64_t base0 = seg_begin(g0, lvl, n);
    const int nsub = 1 << j;
    int nexist = int(min(int64_t(nsub), max(int64_t(0), n - g0)));
    uint32_t &qcount = S.qcount[j & 1];
    if (tid == 0) S.qcount[(j + 1) & 1] = 0;  // the next level's; read last a level ago
    // A: per subtree, its dim, pivot rank position and equal-key run
    for (int t = tid; t < nexist; t += NT) {
      const int64_t g = g0 + t;
      const int sz = int(subtree_size(g, n));
      const int bt = int(seg_begin(g, lvl, n) - base0);
      const int r = int(left_size(g, n));
      const int u = (1 << j) - 1 + t;
      int dim;
      if (explicitDims) {
        uint32_t lo[D], hi[D];
#pragma unroll
        for (int d = 0; d < D; d++) {
          lo[d] = S.rootLo[d];
          hi[d] = S.rootHi[d];
        }
        // the a-th ancestor of local node u is ((u + 1) >> a) - 1; its loads
        // do not depend on the nearer ancestors', so they issue together
        constexpr int kMaxDepth = ilog2_floor(TILE);
#pragma unroll
        for (int a = 1; a <= kMaxDepth; a++) {
          const bool on = a <= j;
          const int c = on ? ((u + 1) >> (a - 1)) - 1 : 0;
          const int p = on ? ((u + 1) >> a) - 1 : 0;
          const int pd = on ? int(S.locDim[p]) : 0;
          const uint32_t pc = S.key[pd][on ? int(S.locPivot[p]) : 0];
          if (on) {
            if (c & 1)
              hi[pd] = min(hi[pd], pc);
            else
              lo[pd] = max(lo[pd], pc);
          }
        }
        dim = Scalar<SC>::widest(lo, hi, D);
      } else {
        dim = lvl % D;
      }
      S.locDim[u] = uint8_t(dim);
      const uint16_t *Ld = S.list[cur][dim];
      const uint32_t *Kd = S.key[dim];
      const int pp = bt + r;
      const uint32_t v = Kd[Ld[pp]];
      // neighbours first: a run of one (distinct keys) needs no search
      const bool lone0 = pp == bt || Kd[Ld[pp - 1]] < v;
      const bool lone1 = pp + 1 == bt + sz || Kd[Ld[pp + 1]] > v;
      int lo = bt, hi = pp;  // first q in [bt,pp] with key >= v
      if (lone0) lo = pp;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (Kd[Ld[mid]] < v)
          lo = mid + 1;
        else
          hi = mid;
      }
      const int t0 = lo;
      lo = pp + 1;
      hi = bt + sz;  // first q in [pp+1, bt+sz) with key > v
      if (lone1) hi = lo;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (Kd[Ld[mid]] <= v)
          lo = mid + 1;
        else
          hi = mid;
      }
      const int t1 = lo;
      S.lv.u_sub.t0[t] = uint16_t(t0);
      S.lv.u_sub.t1[t] = uint16_t(t1);
      S.lv.u_sub.b[t] = uint16_t(bt);
      S.lv.u_sub.r[t] = uint16_t(r);
      S.subDim[t] = uint8_t(dim);
      if (t1 - t0 == 1) {
        const int piv = Ld[pp];
        S.flag[piv] = 2;
        S.locPivot[u] = uint16_t(piv);
        src.settle(g, u, piv, dim, S);
      } else {
        S.queue[atomicAdd(&qcount, 1u)] = uint16_t(t);
      }
    }
    __syncthreads();
    // Thread tid owns the positions q*NT + tid (round q < PER) of the level;
    // each position's subtree and whether it is its subtree's first position
    // stay in registers for B and C.
    constexpr int PER = TILE / NT;
    constexpr int NW = NT / 32;
    constexpr int NE = PER * NW;  // (round, warp) pairs, in position order
    static_assert(PER >= 1 && NE <= 64, "one to two (round, warp) pairs per lane");
    uint16_t tq[PER];
    uint32_t startMask = 0;
#pragma unroll
    for (int q = 0; q < PER; q++) {
      const int p = q * NT + tid;
      tq[q] = 0;
      if (p < mact) {
        tq[q] = S.segOf[cur][p];
        if (p == 0 || S.segOf[cur][p - 1] != tq[q]) startMask |= 1u << q;
      }
    }
    // B: sides of all points outside the runs
#pragma unroll
    for (int q = 0; q < PER; q++) {
      const int p = q * NT + tid;
      if (p < mact) {
        const int t = tq[q];
        const int e = S.list[cur][S.subDim[t]][p];
        if (p < S.lv.u_sub.t0[t])
          S.flag[e] = 0;
        else if (p >= S.lv.u_sub.t1[t])
          S.flag[e] = 1;
      }
    }
    // A2: rank equal-coordinate runs by the composite key (one warp each;
    // the points of runs and those B flags are disjoint)
    for (int qi = wid; qi < int(qcount); qi += NT / 32) {
      const int t = S.queue[qi];
      const int64_t g = g0 + t;
      const int u = (1 << j) - 1 + t;
      const int dim = S.subDim[t];
      const int t0 = S.lv.u_sub.t0[t], t1 = S.lv.u_sub.t1[t];
      const int pp = S.lv.u_sub.b[t] + S.lv.u_sub.r[t];
      int cd[D];
      int ncd = 0;
      cd[ncd++] = dim;
      {
        int c = u;
        int64_t ga = g;
        while (ga > 0 && ncd < D) {
          int da;
          if (c > 0) {
            c = (c - 1) >> 1;
            da = S.locDim[c];
          } else {
            da = explicitDims ? src.anc_dim((ga - 1) >> 1) : rr_dim((ga - 1) >> 1, D);
          }
          ga = (ga - 1) >> 1;
          bool seen = false;
          for (int i = 0; i < ncd; i++) seen |= (cd[i] == da);
          if (!seen) cd[ncd++] = da;
        }
      }
      const uint16_t *Ld = S.list[cur][dim];
      const int len = t1 - t0;
      for (int x = lane; x < len; x += 32) {
        const int ex = Ld[t0 + x];
        int rk = 0;
        for (int y = 0; y < len; y++) {
          const int ey = Ld[t0 + y];
          bool less = false, decided = false;
          for (int w = 1; w < ncd && !decided; w++) {
            const uint32_t ky = S.key[cd[w]][ey], kx = S.key[cd[w]][ex];
            if (ky != kx) {
              less = ky < kx;
              decided = true;
            }
          }
          if (!decided) less = S.idx[ey] < S.idx[ex];
          rk += less;
        }
        const int want = pp - t0;
        if (rk < want)
          S.flag[ex] = 0;
        else if (rk > want)
          S.flag[ex] = 1;
        else {
          S.flag[ex] = 2;
          S.locPivot[u] = uint16_t(ex);
          src.settle(g, u, ex, dim, S);
        }
      }
    }
    __syncthreads();
    // C: stable partition of every list (pivots dropped).  Sides are warp
    // ballots, so a count of left / right points before a position is a
    // popc plus the exclusive scan of the per-(round, warp) counts; the low /
    // high 16 bits of a count word hold the two sides.  Each subtree's first
    // position stores in pack[t] the offsets that turn those counts into new
    // positions (pack aliases `scan`, free here).  List d+1 is counted in
    // the phase that scatters list d.
    const uint32_t ltMask = (1u << lane) - 1u;
    uint32_t *pack = S.lv.scan;
    uint16_t eq[PER];
    uint32_t bl[PER], br[PER];
    auto count_sides = [&](int d) {
      const uint16_t *Lc = S.list[cur][d];
#pragma unroll
      for (int q = 0; q < PER; q++) {
        const int p = q * NT + tid;
        int f = 2;
        eq[q] = 0;
        if (p < mact) {
          eq[q] = Lc[p];
          f = S.flag[eq[q]];
        }
        bl[q] = __ballot_sync(0xffffffffu, f == 0);
        br[q] = __ballot_sync(0xffffffffu, f == 1);
        if (lane == 0) S.warpSums[q * NW + wid] = uint32_t(__popc(bl[q])) | (uint32_t(__popc(br[q])) << 16);
      }
    };
    count_sides(0);
    for (int d = 0; d < D; d++) {
      __syncthreads();
      // exclusive scan of the NE pair counts, two per lane
      const uint32_t a0 = 2 * lane < NE ? S.warpSums[2 * lane] : 0u;
      const uint32_t a1 = 2 * lane + 1 < NE ? S.warpSums[2 * lane + 1] : 0u;
      uint32_t incl = a0 + a1;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const uint32_t excl = incl - a0 - a1;
      uint32_t bef[PER];
#pragma unroll
      for (int q = 0; q < PER; q++) {
        const int ei = q * NW + wid;
        const uint32_t x = __shfl_sync(0xffffffffu, excl, ei >> 1);
        const uint32_t y = __shfl_sync(0xffffffffu, a0, ei >> 1);
        bef[q] = x + ((ei & 1) ? y : 0u) +
                 (uint32_t(__popc(bl[q] & ltMask)) | (uint32_t(__popc(br[q] & ltMask)) << 16));
        if ((startMask >> q) & 1u) {
          const int t = tq[q];
          const int nb = q * NT + tid - t;  // first new position of subtree t
          const int lb = nb - int(bef[q] & 0xffffu);
          const int rb = nb + S.lv.u_sub.r[t] - int(bef[q] >> 16);
          pack[t] = uint32_t(uint16_t(lb)) | (uint32_t(uint16_t(rb)) << 16);
        }
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < PER; q++) {
        const bool left = (bl[q] >> lane) & 1u, right = (br[q] >> lane) & 1u;
        if (left || right) {
          const int t = tq[q];
          const uint32_t pk = pack[t];
          const int np = left ? int(int16_t(pk & 0xffffu)) + int(bef[q] & 0xffffu)
                              : int(int16_t(pk >> 16)) + int(bef[q] >> 16);
          if (unsigned(np) < unsigned(TILE)) {
            S.list[cur ^ 1][d][np] = eq[q];
            if (d == 0) S.segOf[cur ^ 1][np] = uint16_t(2 * t + (right ? 1 : 0));
          }
        }
      }
      if (d + 1 < D) count_sides(d + 1);
    }
    __syncthreads();
    mact -= nexist;
    cur ^= 1;
  }
}

}  // namespace build
}  // namespace ckb
