// The fast exact kNN / FCP traversal of one query (float coordinates,
// D = 2..4, k <= 32): the body of fast.cu's knn_fast_kernel and of the
// learned path's fused kernel (learned.cu).  The exactness argument is in
// fast.cu's header.
#pragma once

#include "common.cuh"
#include "fast.cuh"

namespace ckb {
namespace fast {

// Far-child stack entries hold the node and, per dimension, the squared
// offset from the query to the closest point of the node's box, truncated
// to bf16 (the top 16 bits of the float): 12 bytes for D = 3 or 4, 8 for
// D = 2, instead of the closest point plus its distance (20 bytes).
// Truncation rounds toward zero, so a popped box's distance -- the sum of
// its truncated offsets -- never exceeds the exact corner distance: culling
// only becomes more permissive, and the answer cannot change.
template <int D> struct PackedOffsets {
  static constexpr int W = (D + 1) / 2;
  uint32_t w[W];
};
template <int D>
__device__ __forceinline__ PackedOffsets<D> pack_offsets(const float (&o)[D])
{
  PackedOffsets<D> p;
#pragma unroll
  for (int j = 0; j < PackedOffsets<D>::W; j++) {
    const uint32_t lo = __float_as_uint(o[2 * j]) >> 16;
    const uint32_t hi = 2 * j + 1 < D ? (__float_as_uint(o[2 * j + 1]) & 0xffff0000u) : 0u;
    p.w[j] = hi | lo;
  }
  return p;
}
template <int D>
__device__ __forceinline__ void unpack_offsets(const uint32_t *w, float (&o)[D])
{
#pragma unroll
  for (int d = 0; d < D; d++)
    o[d] = __uint_as_float((d & 1) ? (w[d >> 1] & 0xffff0000u) : (w[d >> 1] << 16));
}

// One thread per query (queries in Morton order).  Culling uses the
// closest-corner distance of each subtree's domain box, the bound of
// traverse_cct (traverse-cct.h:25-99): the far child's box differs from its
// parent's only in the split dim, so its closest point to the query is the
// parent's with that coordinate set to the split value.  The traversal keeps
// the squared offsets of that closest point per dimension, off[d]; the box
// distance is their sum in dimension order.  Corner distances never exceed
// the distance of any point inside (every term is a rounded difference of a
// smaller magnitude), so "<=" culling sees every point with d2 <= the final
// (k+1)-th distance.
//
// i: the query's position in the visiting order; myq: its index;
// hasSeed / seedR: a per-query initial cull radius (learned proposal,
// before fa.radius_scale) or none.
template <int D, bool EXPL, bool VEC16, int KC>
__device__ __forceinline__ void knn_fast_one(const FastArgs &fa, int64_t i, int64_t myq,
                                             bool hasSeed, float seedR)
{
  const query::QArgs &a = fa.q;
  const query::TreeView tv = query::tree_of<D, 4>(a, myq);
  const int N = int(tv.n);
  const int k = fa.kk;  // live slots: k+1, right-aligned
  const uint8_t *tree = tv.tree;

  float q[D];
  {
    const float *qp = (const float *)a.queries + myq * D;
#pragma unroll
    for (int d = 0; d < D; d++) q[d] = __ldg(qp + d);
  }
  float r2 = __fmul_rn(a.cutoff, a.cutoff);
  if (hasSeed) {
    const float rr = __fmul_rn(seedR, fa.radius_scale);
    const float rb = __fmul_rn(rr, rr);
    r2 = rb < r2 ? rb : r2;
  }
  const float r2init = r2;
  float e[KC];
  int id[KC];
#pragma unroll
  for (int j = 0; j < KC; j++) {
    e[j] = j < KC - (k + 1) ? -1.f : r2;
    id[j] = -1;
  }
  float cull = r2;
  bool sawInit = false;
  int visits = 0;

  auto sq = [](float x) { return __fmul_rn(x, x); };
  auto dist2 = [&](const float *c) {
    float s = sq(__fsub_rn(c[0], q[0]));
#pragma unroll
    for (int d = 1; d < D; d++) s = __fadd_rn(s, sq(__fsub_rn(c[d], q[d])));
    return s;
  };
  auto sum = [](const float (&o)[D]) {
    float s = o[0];
#pragma unroll
    for (int d = 1; d < D; d++) s = __fadd_rn(s, o[d]);
    return s;
  };

  // squared offsets of the root box's closest point (the world bounds, or
  // all of space)
  float off[D];
  const float *bnd = (const float *)tv.bounds;
#pragma unroll
  for (int d = 0; d < D; d++) {
    float v = q[d];
    if (bnd) {
      const float lo = __ldg(bnd + d), hi = __ldg(bnd + D + d);
      v = v < lo ? lo : v;
      v = hi < v ? hi : v;
    }
    off[d] = sq(__fsub_rn(v, q[d]));
  }

  int nodeSt[32];
  uint32_t offSt[32][PackedOffsets<D>::W];
  int sp = 0;
  int curr = (N > 0 && sum(off) <= cull) ? 0 : N;
  for (;;) {
    if (curr >= N) {
      bool found = false;
      while (sp > 0) {
        --sp;
        float o[D];
        unpack_offsets<D>(offSt[sp], o);
        if (sum(o) <= cull) {
#pragma unroll
          for (int d = 0; d < D; d++) off[d] = o[d];
          curr = nodeSt[sp];
          found = true;
          break;
        }
      }
      if (!found) break;
    }
    float p[D];
    int dim;
    if (VEC16) {
      const uint4 v = __ldg((const uint4 *)(tree + int64_t(curr) * 16));
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int d = 0; d < D; d++) p[d] = __uint_as_float(w[d]);
      dim = EXPL ? int((w[3] >> a.dshift) & a.dmask) : (level_of(curr) % D);
    } else {
      const float *c = (const float *)(tree + int64_t(curr) * a.stride + a.poff);
#pragma unroll
      for (int d = 0; d < D; d++) p[d] = __ldg(c + d);
      dim = EXPL ? int((__ldg((const uint32_t *)(tree + int64_t(curr) * a.stride + a.doff)) >>
                        a.dshift) & a.dmask)
                 : (level_of(curr) % D);
    }
    const float d2 = dist2(p);
    ++visits;
    sawInit |= (d2 == r2init);
    if (d2 < e[KC - 1]) {
      // insert d2 into the ascending list, dropping the largest: each slot
      // is computed from its two old neighbours, with no dependency chain
      // through the list
#pragma unroll
      for (int j = KC - 1; j >= 0; j--) {
        const bool lt = d2 < e[j];
        const bool ltBelow = j > 0 ? (d2 < e[j - 1]) : false;
        const float below = j > 0 ? e[j - 1] : 0.f;
        const int belowId = j > 0 ? id[j - 1] : 0;
        e[j] = ltBelow ? below : (lt ? d2 : e[j]);
        id[j] = ltBelow ? belowId : (lt ? curr : id[j]);
      }
      cull = e[KC - 1];
    }
    float nodeC = p[0], queryC = q[0];
#pragma unroll
    for (int d = 1; d < D; d++)
      if (d == dim) {
        nodeC = p[d];
        queryC = q[d];
      }
    const bool leftIsClose = queryC < nodeC;
    const int lChild = 2 * curr + 1;
    const int farChild = leftIsClose ? lChild + 1 : lChild;
    if (farChild < N) {
      float fo[D];
      const float split = sq(__fsub_rn(nodeC, queryC));
#pragma unroll
      for (int d = 0; d < D; d++) fo[d] = d == dim ? split : off[d];
      if (sum(fo) <= cull) {
        const PackedOffsets<D> pk = pack_offsets<D>(fo);
#pragma unroll
        for (int j = 0; j < PackedOffsets<D>::W; j++) offSt[sp][j] = pk.w[j];
        nodeSt[sp] = farChild;
        sp++;
      }
    }
    curr = leftIsClose ? lChild : lChild + 1;
  }

  // ---- decide: answer now, or queue for the reference-order traversal
  const float X = e[KC - 2];  // k-th smallest d2
  const float Y = e[KC - 1];  // (k+1)-th smallest d2
  const int idX = id[KC - 2];
  bool ok;
  if (fa.fcp) {
    // unique minimum, or nothing below the cut-off (strict '<' in FCPResult)
    ok = idX < 0 ? !hasSeed : (Y > X);
  } else if (idX >= 0) {
    ok = Y > X;  // strict gap at the k-th boundary
  } else {
    ok = !hasSeed && !sawInit;  // fewer than k inside the cut-off
  }
  if (!(X == X)) ok = false;  // NaN coordinates
  if (a.visits) a.visits[myq] += visits;  // accumulated over chained passes
  if (!ok) {
    const int slot = atomicAdd(fa.fb_count, 1);
    fa.fb_list[slot] = int32_t(myq);
    if (fa.status) fa.status[myq] = 1;
    return;
  }
  if (fa.status) fa.status[myq] = 0;
  if (fa.fcp) {
    if (a.out_ids) a.out_ids[myq] = idX >= 0 ? idX : -1;
    if (a.out_d2) ((float *)a.out_d2)[myq] = idX >= 0 ? X : r2init;
    return;
  }
  // the list is sorted by d2; equal-d2 entries must be ordered by id like
  // the reference's (d2, id) keys -- rare, sorted only when present
  unsigned long long key[KC];
  bool anyEq = false;
#pragma unroll
  for (int j = 0; j < KC; j++) {
    const bool live = j >= KC - 1 - k && j < KC - 1;
    key[j] = live ? ((unsigned long long)__float_as_uint(e[j]) << 32) | uint32_t(id[j]) : ~0ull;
    if (live && j + 1 < KC - 1) anyEq |= (e[j] == e[j + 1]);
  }
  if (anyEq) {
#pragma unroll
    for (int pass = 0; pass < KC; pass++) {
#pragma unroll
      for (int j = (pass & 1); j + 1 < KC; j += 2) {
        const unsigned long long x = key[j], y = key[j + 1];
        key[j] = x < y ? x : y;
        key[j + 1] = x < y ? y : x;
      }
    }
  }
  const int off0 = anyEq ? 0 : KC - 1 - k;
  int32_t *oid = a.out_ids ? a.out_ids + myq * k : nullptr;
  float *od = a.out_d2 ? (float *)a.out_d2 + myq * k : nullptr;
#pragma unroll
  for (int j = 0; j < KC; j++) {
    const int o = j - off0;
    if (o >= 0 && o < k) {
      if (oid) oid[o] = int32_t(uint32_t(key[j]));
      if (od) od[o] = __uint_as_float(uint32_t(key[j] >> 32));
    }
  }
  if (a.out_max) ((float *)a.out_max)[myq] = X;
}

}  // namespace fast
}  // namespace ckb
