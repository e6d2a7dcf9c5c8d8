// Warp-cooperative kNN over a left-balanced tree (float coordinates, D = 2..4,
// k = 2..32), selected with CUKD_QUERY_WARP_PACKET: the 32 lanes of a warp
// take 32 consecutive queries of the visiting order (Morton order) and walk
// ONE node stream together.  Every node is loaded once per warp (all lanes
// read the same address); each lane tests its own query against it and keeps
// its own candidate list; a subtree is entered when ANY lane's box distance
// is within that lane's cull bound (a warp ballot), and the two children are
// visited in the order most lanes prefer.  The culling is the fast kernel's
// (closest-corner squared offsets per dimension, fast_one.cuh), so the
// exactness argument and the fallback of undecided queries are the same
// (fast.cu's header): answers are bit-identical to cukd_knn's.
//
// The per-lane part of a stack entry (the lane's box offsets for the pushed
// child) sits in local memory at the warp-uniform stack depth, so its loads
// and stores are coalesced; the node index is warp-uniform.
#include <algorithm>

#include "common.cuh"
#include "fast.cuh"
#include "fast_one.cuh"

namespace ckb {
namespace fast {

using query::QArgs;

template <int D, bool EXPL, bool VEC16, int KC>
__global__ void __launch_bounds__(128, 4) knn_packet_kernel(FastArgs fa)
{
  const QArgs &a = fa.q;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int k = fa.kk;
  const int64_t nq = a.nq;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t w = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); w * 32 < nq;
       w += warps) {
    const int64_t i = w * 32 + lane;
    const bool live = i < nq;
    const int64_t myq = live ? (a.order ? int64_t(a.order[i]) : i) : 0;
    const query::TreeView tv = query::tree_of<D, 4>(a, myq);
    const int N = int(tv.n);  // the same tree for every lane (no forest)
    const uint8_t *tree = tv.tree;
    float q[D];
    {
      const float *qp = (const float *)a.queries + myq * D;
#pragma unroll
      for (int d = 0; d < D; d++) q[d] = __ldg(qp + d);
    }
    float r2 = __fmul_rn(a.cutoff, a.cutoff);
    const bool seeded = fa.radius != nullptr;
    if (seeded) {
      const float rr = __fmul_rn(__ldg(fa.radius + myq), fa.radius_scale);
      const float rb = __fmul_rn(rr, rr);
      r2 = rb < r2 ? rb : r2;
    }
    // lanes past the end take part in the walk with an empty ball
    if (!live) r2 = -1.f;
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
    auto sum = [](const float (&o)[D]) {
      float s = o[0];
#pragma unroll
      for (int d = 1; d < D; d++) s = __fadd_rn(s, o[d]);
      return s;
    };
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
    int curr = (N > 0 && __any_sync(full, sum(off) <= cull)) ? 0 : N;
    for (;;) {
      if (curr >= N) {
        bool found = false;
        while (sp > 0) {
          --sp;
          float o[D];
          unpack_offsets<D>(offSt[sp], o);
          if (__any_sync(full, sum(o) <= cull)) {
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
        const uint32_t wd[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int d = 0; d < D; d++) p[d] = __uint_as_float(wd[d]);
        dim = EXPL ? int((wd[3] >> a.dshift) & a.dmask) : (level_of(curr) % D);
      } else {
        const float *c = (const float *)(tree + int64_t(curr) * a.stride + a.poff);
#pragma unroll
        for (int d = 0; d < D; d++) p[d] = __ldg(c + d);
        dim = EXPL ? int((__ldg((const uint32_t *)(tree + int64_t(curr) * a.stride + a.doff)) >>
                          a.dshift) & a.dmask)
                   : (level_of(curr) % D);
      }
      // this lane's own box test: does the node's box reach its ball?
      const bool mine = sum(off) <= cull;
      float d2 = 0.f;
      if (mine) {
        d2 = 0.f;
        d2 = sq(__fsub_rn(p[0], q[0]));
#pragma unroll
        for (int d = 1; d < D; d++) d2 = __fadd_rn(d2, sq(__fsub_rn(p[d], q[d])));
        ++visits;
        sawInit |= (d2 == r2init);
        if (d2 < e[KC - 1]) {
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
      }
      float nodeC = p[0], queryC = q[0];
#pragma unroll
      for (int d = 1; d < D; d++)
        if (d == dim) {
          nodeC = p[d];
          queryC = q[d];
        }
      const int lChild = 2 * curr + 1;
      if (lChild >= N) {
        curr = N;
        continue;
      }
      // each lane's box offsets for both children: the child on the query's
      // side keeps the parent's offset in `dim`, the other gets the plane's
      const float plane = sq(__fsub_rn(nodeC, queryC));
      const bool leftNear = queryC < nodeC;
      float ol[D], orr[D];
#pragma unroll
      for (int d = 0; d < D; d++) {
        ol[d] = (d == dim && !leftNear) ? plane : off[d];
        orr[d] = (d == dim && leftNear) ? plane : off[d];
      }
      const bool needL = __any_sync(full, sum(ol) <= cull);
      const bool needR = lChild + 1 < N && __any_sync(full, sum(orr) <= cull);
      // visit first the child most lanes are on the side of
      const bool leftFirst = __popc(__ballot_sync(full, leftNear)) >= 16;
      const int first = leftFirst ? lChild : lChild + 1;
      const bool needFirst = leftFirst ? needL : needR;
      const bool needSecond = leftFirst ? needR : needL;
      if (needSecond) {
        const PackedOffsets<D> pk = pack_offsets<D>(leftFirst ? orr : ol);
#pragma unroll
        for (int j = 0; j < PackedOffsets<D>::W; j++) offSt[sp][j] = pk.w[j];
        nodeSt[sp] = leftFirst ? lChild + 1 : lChild;
        sp++;
      }
      if (needFirst) {
#pragma unroll
        for (int d = 0; d < D; d++) off[d] = leftFirst ? ol[d] : orr[d];
        curr = first;
      } else {
        curr = N;
      }
    }
    if (!live) continue;

    // ---- decide and write, as the fast kernel does
    const float X = e[KC - 2];
    const float Y = e[KC - 1];
    const int idX = id[KC - 2];
    bool ok;
    if (idX >= 0)
      ok = Y > X;
    else
      ok = !seeded && !sawInit;
    if (!(X == X)) ok = false;
    if (a.visits) a.visits[myq] += visits;
    if (!ok) {
      const int slot = atomicAdd(fa.fb_count, 1);
      fa.fb_list[slot] = int32_t(myq);
      if (fa.status) fa.status[myq] = 1;
      continue;
    }
    if (fa.status) fa.status[myq] = 0;
    unsigned long long key[KC];
    bool anyEq = false;
#pragma unroll
    for (int j = 0; j < KC; j++) {
      const bool lv = j >= KC - 1 - k && j < KC - 1;
      key[j] = lv ? ((unsigned long long)__float_as_uint(e[j]) << 32) | uint32_t(id[j]) : ~0ull;
      if (lv && j + 1 < KC - 1) anyEq |= (e[j] == e[j + 1]);
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
}

template <int D, bool EXPL, bool VEC16, int KC>
int launch_packet(const FastArgs &fa, cudaStream_t st)
{
  const int bs = 128;
  const int64_t grid = std::max<int64_t>(1, div_up(fa.q.nq, int64_t(bs)));
  knn_packet_kernel<D, EXPL, VEC16, KC><<<unsigned(grid), bs, 0, st>>>(fa);
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

template <int D, bool EXPL, bool VEC16>
int packet_kc(const FastArgs &fa, cudaStream_t st)
{
  const int slots = fa.kk + 1;
  if (slots <= 5) return launch_packet<D, EXPL, VEC16, 5>(fa, st);
  if (slots <= 9) return launch_packet<D, EXPL, VEC16, 9>(fa, st);
  if (slots <= 17) return launch_packet<D, EXPL, VEC16, 17>(fa, st);
  if (slots <= 33) return launch_packet<D, EXPL, VEC16, 33>(fa, st);
  return CUKD_ERR_UNSUPPORTED;
}

template <int D>
int packet_layout(const FastArgs &fa, cudaStream_t st)
{
  const QArgs &a = fa.q;
  const bool expl = a.doff >= 0;
  const bool vec16 = a.stride == 16 && a.poff == 0 && (!expl || a.doff == 12) && D <= 3;
  if (expl) return vec16 ? packet_kc<D, true, true>(fa, st) : packet_kc<D, true, false>(fa, st);
  return vec16 ? packet_kc<D, false, true>(fa, st) : packet_kc<D, false, false>(fa, st);
}

}  // namespace fast

int run_packet(const fast::FastArgs &fa, int D, cudaStream_t st)
{
  if (fa.fcp || fa.kk < 2 || fa.kk > 32 || fa.q.count_ptr || fa.q.q_cloud)
    return CUKD_ERR_UNSUPPORTED;
  if (fa.q.nq == 0) return CUKD_OK;
  if (D == 2) return fast::packet_layout<2>(fa, st);
  if (D == 3) return fast::packet_layout<3>(fa, st);
  if (D == 4) return fast::packet_layout<4>(fa, st);
  return CUKD_ERR_UNSUPPORTED;
}

}  // namespace ckb
