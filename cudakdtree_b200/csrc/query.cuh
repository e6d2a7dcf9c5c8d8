// Device-side traversal cores and result objects shared by the query,
// batched and learned-radius kernels.  Each traversal restates the
// reference routine named in its comment statement for statement.
#pragma once

#include "common.cuh"

namespace ckb {
namespace query {

struct QArgs {
  const uint8_t *tree;
  int64_t n;
  int stride, poff, doff, dshift;
  uint32_t dmask;
  const void *bounds;   // box_t: lower[D], upper[D]
  const void *queries;  // point_t[nq]
  int64_t nq;
  const int32_t *order;  // optional visiting order of the queries
  int k;
  float cutoff;
  int64_t cutoff_d2;
  float eps;
  bool heap_order;
  int32_t *out_ids;
  void *out_d2;
  void *out_max;
  int64_t *visits;
  const float *radius;  // optional per-query initial cull radius (learned path)
  int32_t *flags_out;   // optional per-query status (learned path)
  int block_size;
  const int *count_ptr;  // optional device-side number of queries in `order`
  // forest (batched clouds): when q_cloud is set, query i searches the tree
  // of cloud q_cloud[i], records [cloud_base[c], cloud_base[c + 1]) of
  // `tree`, whose box is cloud_bounds[c] (lower[D], upper[D]; optional);
  // the ids are local to that cloud
  const int32_t *q_cloud;
  const int64_t *cloud_base;
  const void *cloud_bounds;
  int queries_per_thread;  // fast kernel: queries a thread runs in turn
};

// the tree a query searches: the whole tree, or its cloud's (forest)
struct TreeView {
  const uint8_t *tree;
  int64_t n;
  const void *bounds;
};
template <int D, int BYTES>
__device__ __forceinline__ TreeView tree_of(const QArgs &a, int64_t qi)
{
  TreeView t{a.tree, a.n, a.bounds};
  if (a.q_cloud) {
    const int c = __ldg(a.q_cloud + qi);
    const int64_t b0 = __ldg((const long long *)a.cloud_base + c);
    t.n = __ldg((const long long *)a.cloud_base + c + 1) - b0;
    t.tree = a.tree + b0 * a.stride;
    t.bounds = a.cloud_bounds ? (const uint8_t *)a.cloud_bounds + int64_t(c) * 2 * D * BYTES
                              : nullptr;
  }
  return t;
}

enum { RES_FCP = 0, RES_FIX4, RES_FIX8, RES_FIX16, RES_FIX32, RES_HEAP128, RES_HEAP1024 };

template <int SC> struct Traits;
template <> struct Traits<0> {
  using T = float;
  using DT = float;  // squared distances
  __device__ static DT sub(T a, T b) { return __fsub_rn(a, b); }
  __device__ static DT sqr(DT a) { return __fmul_rn(a, a); }
  __device__ static DT add(DT a, DT b) { return __fadd_rn(a, b); }
  // candidate key: (float bits of d2) << 32 | uint32(id)  (knn.h:343-353)
  using Key = unsigned long long;
  __device__ static Key encode(DT d2, int32_t id)
  {
    return ((unsigned long long)__float_as_uint(d2) << 32) | uint32_t(id);
  }
  __device__ static DT key_d2(Key k) { return __uint_as_float(uint32_t(k >> 32)); }
  __device__ static int32_t key_id(Key k) { return int32_t(uint32_t(k)); }
  __device__ static bool less(Key a, Key b) { return a < b; }
  __device__ static Key min_key() { return 0ull; }  // <= every (d2 >= +0, id) key
  __device__ static DT init_cull(const QArgs &a) { return __fmul_rn(a.cutoff, a.cutoff); }
};
// int coordinates: exact int64 squared distances, key = (d2, id) compared
// lexicographically (no reference counterpart; the reference's int vector
// types lack operator-/dot, cukd-math.h:100-112)
struct IKey {
  long long d;
  uint32_t id;
};
template <> struct Traits<1> {
  using T = int32_t;
  using DT = long long;
  __device__ static DT sub(T a, T b) { return (long long)a - (long long)b; }
  __device__ static DT sqr(DT a) { return a * a; }
  __device__ static DT add(DT a, DT b) { return a + b; }
  using Key = IKey;
  __device__ static Key encode(DT d2, int32_t id) { return IKey{d2, uint32_t(id)}; }
  __device__ static DT key_d2(Key k) { return k.d; }
  __device__ static int32_t key_id(Key k) { return int32_t(k.id); }
  __device__ static bool less(Key a, Key b) { return a.d < b.d || (a.d == b.d && a.id < b.id); }
  __device__ static Key min_key() { return IKey{-1ll, 0u}; }  // below every d2 >= 0
  __device__ static DT init_cull(const QArgs &a) { return a.cutoff_d2; }
};

template <int SC, int D>
__device__ inline typename Traits<SC>::DT sqr_dist(const typename Traits<SC>::T *a,
                                                   const typename Traits<SC>::T *b)
{
  using Tr = Traits<SC>;
  typename Tr::DT s = Tr::sqr(Tr::sub(a[0], b[0]));
#pragma unroll
  for (int d = 1; d < D; d++) s = Tr::add(s, Tr::sqr(Tr::sub(a[d], b[d])));
  return s;
}

// node record reader (data_traits::get_point / get_dim of the caller's
// record layout)
template <int SC, int D, bool EXPL, bool VEC16>
struct NodeReader {
  using T = typename Traits<SC>::T;
  const uint8_t *tree;
  int stride, poff, doff, dshift;
  uint32_t dmask;
  __device__ NodeReader(const QArgs &a)
      : tree(a.tree), stride(a.stride), poff(a.poff), doff(a.doff), dshift(a.dshift),
        dmask(a.dmask)
  {
  }
  // loads the point of `node` into p, returns its split dim
  __device__ __forceinline__ int load(int64_t node, T *p) const
  {
    if (VEC16) {
      const uint4 v = __ldg((const uint4 *)(tree + node * 16));
      const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
      for (int d = 0; d < D; d++) p[d] = reinterpret_cast<const T &>(w[d]);
      if (EXPL) return int((w[3] >> dshift) & dmask);
      return level_of(node) % D;
    } else {
      const T *c = (const T *)(tree + node * stride + poff);
#pragma unroll
      for (int d = 0; d < D; d++) p[d] = __ldg(c + d);
      if (EXPL) return int((__ldg((const uint32_t *)(tree + node * stride + doff)) >> dshift) & dmask);
      return level_of(node) % D;
    }
  }
};

// ---------------------------------------------------------------------------
// result objects
// ---------------------------------------------------------------------------
// FCPResult (fcp.h:179-207): strict '<', first visited wins a tie
template <int SC>
struct FcpRes {
  using Tr = Traits<SC>;
  using DT = typename Tr::DT;
  DT best;
  int32_t id;
  long long visits;
  __device__ FcpRes(const QArgs &a) : best(Tr::init_cull(a)), id(-1), visits(0) {}
  __device__ DT init() const { return best; }
  __device__ __forceinline__ DT process(int32_t cand, DT d2)
  {
    visits++;
    if (d2 < best) {
      best = d2;
      id = cand;
    }
    return best;
  }
  __device__ void write(const QArgs &a, int64_t qi) const
  {
    if (a.out_ids) a.out_ids[qi] = id;
    if (a.out_d2) ((DT *)a.out_d2)[qi] = best;
    if (a.visits) a.visits[qi] = visits;
  }
};

// FixedCandidateList<k> (knn.h:503-548) in KC >= k registers.  The k live
// slots are right-aligned: slots [0, KC-k) hold the smallest possible key,
// so after every insertion the list's last register is the reference
// list's slot k-1 (its maxRadius2) and every index stays compile-time
// (a runtime-indexed register array would be demoted to local memory).
template <int SC, int KC>
struct FixedRes {
  using Tr = Traits<SC>;
  using DT = typename Tr::DT;
  using Key = typename Tr::Key;
  Key e[KC];
  int k;
  DT cull;
  long long visits;
  __device__ FixedRes(const QArgs &a) : k(a.k), visits(0)
  {
    const Key init = Tr::encode(Tr::init_cull(a), -1);
    const Key pad = Tr::min_key();
#pragma unroll
    for (int i = 0; i < KC; i++) e[i] = i < KC - k ? pad : init;
    cull = Tr::key_d2(init);
  }
  __device__ DT init() const { return cull; }
  __device__ __forceinline__ DT process(int32_t cand, DT d2)
  {
    visits++;
    Key v = Tr::encode(d2, cand);
    if (Tr::less(v, e[KC - 1])) {
#pragma unroll
      for (int i = 0; i < KC; i++) {
        const bool lt = Tr::less(v, e[i]);
        const Key lo = lt ? v : e[i];
        const Key hi = lt ? e[i] : v;
        e[i] = lo;
        v = hi;
      }
      cull = Tr::key_d2(e[KC - 1]);
    }
    return cull;
  }
  __device__ void write(const QArgs &a, int64_t qi) const
  {
    const int off = KC - k;
    if (a.out_ids) {
#pragma unroll
      for (int i = 0; i < KC; i++)
        if (i >= off) a.out_ids[qi * k + (i - off)] = Tr::key_id(e[i]);
    }
    if (a.out_d2) {
#pragma unroll
      for (int i = 0; i < KC; i++)
        if (i >= off) ((DT *)a.out_d2)[qi * k + (i - off)] = Tr::key_d2(e[i]);
    }
    if (a.out_max) ((DT *)a.out_max)[qi] = cull;
    if (a.visits) a.visits[qi] = visits;
  }
};

// HeapCandidateList / FlexHeapCandidateList (knn.h:360-493): max-heap of
// the k smallest keys, runtime k <= KC, in local memory.
template <int SC, int KC>
struct HeapRes {
  using Tr = Traits<SC>;
  using DT = typename Tr::DT;
  using Key = typename Tr::Key;
  Key e[KC];
  int k;
  long long visits;
  __device__ HeapRes(const QArgs &a) : k(a.k), visits(0)
  {
    const Key init = Tr::encode(Tr::init_cull(a), -1);
    for (int i = 0; i < k; i++) e[i] = init;
  }
  __device__ DT init() const { return Tr::key_d2(e[0]); }
  __device__ __forceinline__ DT process(int32_t cand, DT d2)
  {
    visits++;
    const Key v = Tr::encode(d2, cand);
    if (!Tr::less(v, e[0])) return Tr::key_d2(e[0]);
    int pos = 0;
    for (;;) {
      const int c1 = 2 * pos + 1, c2 = c1 + 1;
      int largest = k;
      Key lv = v;
      if (c1 < k) {
        largest = c1;
        lv = e[c1];
      }
      if (c2 < k && Tr::less(lv, e[c2])) {
        largest = c2;
        lv = e[c2];
      }
      if (largest == k || Tr::less(lv, v)) {
        e[pos] = v;
        break;
      }
      e[pos] = lv;
      pos = largest;
    }
    return Tr::key_d2(e[0]);
  }
  __device__ void write(const QArgs &a, int64_t qi)
  {
    const DT maxd = Tr::key_d2(e[0]);
    if (!a.heap_order) {
      // heap sort in place: ascending (d2, id), like FixedCandidateList
      for (int end = k - 1; end > 0; end--) {
        const Key top = e[0];
        const Key x = e[end];
        int pos = 0;
        for (;;) {
          const int c1 = 2 * pos + 1, c2 = c1 + 1;
          int largest = -1;
          Key lv = x;
          if (c1 < end && Tr::less(lv, e[c1])) {
            largest = c1;
            lv = e[c1];
          }
          if (c2 < end && Tr::less(lv, e[c2])) {
            largest = c2;
            lv = e[c2];
          }
          if (largest < 0) break;
          e[pos] = lv;
          pos = largest;
        }
        e[pos] = x;
        e[end] = top;
      }
    }
    if (a.out_ids)
      for (int i = 0; i < k; i++) a.out_ids[qi * k + i] = Tr::key_id(e[i]);
    if (a.out_d2)
      for (int i = 0; i < k; i++) ((DT *)a.out_d2)[qi * k + i] = Tr::key_d2(e[i]);
    if (a.out_max) ((DT *)a.out_max)[qi] = maxd;
    if (a.visits) a.visits[qi] = visits;
  }
};

// ---------------------------------------------------------------------------
// traversals
// ---------------------------------------------------------------------------
// traverse_default (traverse-default-stack-based.h:24-108)
template <int SC, int D, class Res, class RD>
__device__ __forceinline__ void trav_stack_based(Res &res, const typename Traits<SC>::T *q,
                                                 const RD &rd, int64_t n)
{
  using Tr = Traits<SC>;
  using T = typename Tr::T;
  using DT = typename Tr::DT;
  DT cullDist = res.init();
  int nodeStack[32];
  DT distStack[32];
  int sp = 0;
  int curr = 0;
  const int N = int(n);
  for (;;) {
    while (curr < N) {
      T p[D];
      const int dim = rd.load(curr, p);
      const DT d2 = sqr_dist<SC, D>(p, q);
      cullDist = res.process(curr, d2);
      T nodeCoord = p[0], queryCoord = q[0];
#pragma unroll
      for (int d = 1; d < D; d++)
        if (d == dim) {
          nodeCoord = p[d];
          queryCoord = q[d];
        }
      const bool leftIsClose = queryCoord < nodeCoord;
      const int lChild = 2 * curr + 1;
      const int rChild = lChild + 1;
      const int closeChild = leftIsClose ? lChild : rChild;
      const int farChild = leftIsClose ? rChild : lChild;
      const DT planeDiff = Tr::sub(queryCoord, nodeCoord);
      const DT sqrDistToPlane = Tr::sqr(planeDiff);
      if (sqrDistToPlane < cullDist && farChild < N) {
        nodeStack[sp] = farChild;
        distStack[sp] = sqrDistToPlane;
        sp++;
      }
      curr = closeChild;
    }
    for (;;) {
      if (sp == 0) return;
      --sp;
      if (distStack[sp] >= cullDist) continue;
      curr = nodeStack[sp];
      break;
    }
  }
}

// traverse_stack_free (traverse-stack-free.h:24-117)
template <int SC, int D, class Res, class RD>
__device__ __forceinline__ void trav_stack_free(Res &res, const typename Traits<SC>::T *q,
                                                const RD &rd, int64_t n, float eps)
{
  using Tr = Traits<SC>;
  using T = typename Tr::T;
  using DT = typename Tr::DT;
  const int N = int(n);
  if (N <= 0) return;  // the reference reads node -1 for an empty tree
  const float epsErr = __fadd_rn(1.f, eps);
  DT cullDist = res.init();
  int prev = -1, curr = 0;
  for (;;) {
    const int parent = (curr + 1) / 2 - 1;
    if (curr >= N) {
      prev = curr;
      curr = parent;
      continue;
    }
    T p[D];
    const int dim = rd.load(curr, p);
    const int child = 2 * curr + 1;
    const bool fromChild = prev >= child;
    if (!fromChild) {
      const DT d2 = sqr_dist<SC, D>(q, p);
      cullDist = res.process(curr, d2);
    }
    T nodeCoord = p[0], queryCoord = q[0];
#pragma unroll
    for (int d = 1; d < D; d++)
      if (d == dim) {
        nodeCoord = p[d];
        queryCoord = q[d];
      }
    const DT dimDist = Tr::sub(queryCoord, nodeCoord);
    const int side = dimDist > DT(0);
    const int closeChild = 2 * curr + 1 + side;
    const int farChild = 2 * curr + 2 - side;
    int next;
    if (prev == closeChild) {
      bool farOk;
      if (SC == 0)
        farOk = __fmul_rn(__fmul_rn(float(dimDist), float(dimDist)), epsErr) < float(cullDist);
      else
        farOk = Tr::sqr(dimDist) < cullDist;
      next = (farChild < N && farOk) ? farChild : parent;
    } else if (prev == farChild) {
      next = parent;
    } else {
      next = child < N ? closeChild : parent;
    }
    if (next == -1) return;
    prev = curr;
    curr = next;
  }
}

// traverse_cct (traverse-cct.h:25-99)
template <int SC, int D, class Res, class RD>
__device__ __forceinline__ void trav_cct(Res &res, const typename Traits<SC>::T *q,
                                         const RD &rd, int64_t n,
                                         const typename Traits<SC>::T *bounds)
{
  using Tr = Traits<SC>;
  using T = typename Tr::T;
  using DT = typename Tr::DT;
  const int N = int(n);
  DT cullDist = res.init();
  int nodeStack[32];
  T cornerStack[32][D];
  int sp = 0;
  T closest[D];
#pragma unroll
  for (int d = 0; d < D; d++) {
    const T lo = __ldg(bounds + d), hi = __ldg(bounds + D + d);
    T v = q[d];
    v = (v < lo) ? lo : v;  // max(point, lower)
    v = (hi < v) ? hi : v;  // min(., upper)   (box.h:98-102)
    closest[d] = v;
  }
  if (sqr_dist<SC, D>(q, closest) > cullDist) return;
  int nodeID = 0;
  for (;;) {
    if (nodeID >= N) {
      for (;;) {
        if (sp == 0) return;
        --sp;
#pragma unroll
        for (int d = 0; d < D; d++) closest[d] = cornerStack[sp][d];
        if (sqr_dist<SC, D>(closest, q) >= cullDist) continue;
        nodeID = nodeStack[sp];
        break;
      }
    }
    T p[D];
    const int dim = rd.load(nodeID, p);
    {
      const DT d2 = sqr_dist<SC, D>(p, q);
      cullDist = res.process(nodeID, d2);
    }
    T nodeDim = p[0], queryDim = q[0];
#pragma unroll
    for (int d = 1; d < D; d++)
      if (d == dim) {
        nodeDim = p[d];
        queryDim = q[d];
      }
    const bool leftIsClose = queryDim < nodeDim;
    const int lChild = 2 * nodeID + 1;
    const int rChild = lChild + 1;
    T farCorner[D];
#pragma unroll
    for (int d = 0; d < D; d++) farCorner[d] = (d == dim) ? nodeDim : closest[d];
    const int farChild = leftIsClose ? rChild : lChild;
    if (farChild < N && sqr_dist<SC, D>(farCorner, q) < cullDist) {
#pragma unroll
      for (int d = 0; d < D; d++) cornerStack[sp][d] = farCorner[d];
      nodeStack[sp] = farChild;
      sp++;
    }
    nodeID = leftIsClose ? lChild : rChild;
  }
}

int run_query(const QArgs &a, int scalar, int D, int method, int kind, cudaStream_t st);

}  // namespace query
}  // namespace ckb
