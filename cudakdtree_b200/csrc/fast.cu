// Fast exact kNN / FCP over a left-balanced tree, with reference-order
// fallback.  (float coordinates, D = 2..4, k <= 32)
//
// Why the answer can be computed in any visiting order.  The reference's
// traversals (traverse-default-stack-based.h, traverse-stack-free.h,
// traverse-cct.h) keep the k smallest (d2, id) keys among the nodes they
// visit, and skip a subtree only when its plane/corner distance is not below
// the current cull distance (the k-th key's d2, which never drops below the
// final k-th d2 X).  A point with d2 < X is therefore always visited, and a
// point with d2 == X can only be skipped once k keys with d2 <= X are
// already in the list.  So whenever exactly k points have d2 <= X (the
// (k+1)-th smallest d2 is strictly greater than X) the reference returns
// exactly those k points, whatever its visiting order.  The same holds for
// FCP (FCPResult, fcp.h:179-207) when the smallest d2 is unique.
//
// This kernel keeps the k+1 smallest d2 (ties in any order), culls with
// "<=" so every point with d2 <= its final (k+1)-th distance is seen, and at
// the end checks that the (k+1)-th d2 is strictly above the k-th.  Queries
// that fail the check (distance ties at the boundary, or a point at exactly
// the cut-off radius) are queued and re-run by the reference-order kernel of
// the requested method, so every answer is bit-identical to the reference.
//
// Throughput features (none changes an answer):
//   - whichever traversal the caller names, subtrees are culled with the
//     closest-corner bound of traverse_cct, which is far tighter than the
//     split-plane bound on clustered data (the named traversal still
//     answers every queued query, in its own order);
//   - the candidate list is d2-only floats + ids in registers (right-aligned
//     k+1 live slots in KC registers), no 64-bit compares;
//   - far-child stack entries of 12 bytes (node + bf16-truncated squared
//     offsets of the box's closest point, fast_one.cuh);
//   - optional per-query initial cull radius (learned radius proposal).
#include <algorithm>

#include "common.cuh"
#include "fast.cuh"
#include "fast_one.cuh"

namespace ckb {
namespace fast {

using query::QArgs;
using query::TreeView;

// Register cap: at most 64 registers (1024 resident threads per SM) for
// lists of up to 17 slots in 2-D / 3-D (9 in 4-D), 128 otherwise.  The
// kernel is latency-bound: the extra resident warps outweigh the few spilled
// registers (measured 12% faster at k = 16 on the 10M-point benchmark).
// Blocks of up to 512 threads (the batched path's autotuner tries 512).
template <int D, bool EXPL, bool VEC16, int KC>
__global__ void __launch_bounds__(512, ((KC <= 9 || (KC <= 17 && D <= 3)) ? 2 : 1))
    knn_fast_kernel(FastArgs fa)
{
  const int64_t limit = fa.q.count_ptr ? int64_t(*fa.q.count_ptr) : fa.q.nq;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < limit;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t myq = fa.q.order ? int64_t(fa.q.order[i]) : i;
    const bool seeded = fa.radius != nullptr;
    const float r = seeded ? __ldg(fa.radius + myq) : 0.f;
    knn_fast_one<D, EXPL, VEC16, KC>(fa, i, myq, seeded, r);
  }
}

// Large k (k + 1 > 33): the same corner-culled traversal keeping the k+1
// smallest (d2, id) keys in a max-heap of u64 keys (d2 bits << 32 | id) in
// local memory, initialised with (r2, -1).  A candidate enters when its key
// is below the root; culling is "<=" against the root's d2.  At the end a
// heapsort leaves the keys in the reference's (d2, id) order.
template <int D, bool EXPL, bool VEC16, int KH>
__global__ void __launch_bounds__(256) knn_fast_heap_kernel(FastArgs fa)
{
  const QArgs &a = fa.q;
  const int64_t limit = a.count_ptr ? int64_t(*a.count_ptr) : a.nq;
  const int k = fa.kk;
  const int K1 = k + 1;  // <= KH
  unsigned long long heap[KH];
  int nodeSt[32];
  float cornerSt[32][D];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < limit;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t myq = a.order ? int64_t(a.order[i]) : i;
    const TreeView tv = query::tree_of<D, 4>(a, myq);
    const int N = int(tv.n);
    const uint8_t *tree = tv.tree;
    float q[D];
    const float *qp = (const float *)a.queries + myq * D;
#pragma unroll
    for (int d = 0; d < D; d++) q[d] = __ldg(qp + d);
    float r2 = __fmul_rn(a.cutoff, a.cutoff);
    if (fa.radius) {
      const float rr = __fmul_rn(__ldg(fa.radius + myq), fa.radius_scale);
      const float rb = __fmul_rn(rr, rr);
      r2 = rb < r2 ? rb : r2;
    }
    const float r2init = r2;
    const unsigned long long initKey = ((unsigned long long)__float_as_uint(r2) << 32) | 0xffffffffull;
    for (int j = 0; j < K1; j++) heap[j] = initKey;
    float cull = r2;
    bool sawInit = false;
    int visits = 0;
    auto dist2 = [&](const float *c) {
      float s = __fmul_rn(__fsub_rn(c[0], q[0]), __fsub_rn(c[0], q[0]));
#pragma unroll
      for (int d = 1; d < D; d++)
        s = __fadd_rn(s, __fmul_rn(__fsub_rn(c[d], q[d]), __fsub_rn(c[d], q[d])));
      return s;
    };
    float closest[D];
    const float *bnd = (const float *)tv.bounds;
#pragma unroll
    for (int d = 0; d < D; d++) {
      float v = q[d];
      if (bnd) {
        const float lo = __ldg(bnd + d), hi = __ldg(bnd + D + d);
        v = v < lo ? lo : v;
        v = hi < v ? hi : v;
      }
      closest[d] = v;
    }
    int sp = 0;
    int curr = (N > 0 && dist2(closest) <= cull) ? 0 : N;
    for (;;) {
      if (curr >= N) {
        bool found = false;
        while (sp > 0) {
          --sp;
#pragma unroll
          for (int d = 0; d < D; d++) closest[d] = cornerSt[sp][d];
          if (dist2(closest) <= cull) {
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
      const unsigned long long key = ((unsigned long long)__float_as_uint(d2) << 32) | uint32_t(curr);
      if (key < heap[0]) {
        // replace the root, sift down
        int x = 0;
        for (;;) {
          const int l = 2 * x + 1;
          if (l >= K1) break;
          int c = l;
          unsigned long long hc = heap[l];
          if (l + 1 < K1 && heap[l + 1] > hc) {
            c = l + 1;
            hc = heap[c];
          }
          if (hc <= key) break;
          heap[x] = hc;
          x = c;
        }
        heap[x] = key;
        cull = __uint_as_float(uint32_t(heap[0] >> 32));
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
        float fc[D];
#pragma unroll
        for (int d = 0; d < D; d++) fc[d] = d == dim ? nodeC : closest[d];
        if (dist2(fc) <= cull) {
#pragma unroll
          for (int d = 0; d < D; d++) cornerSt[sp][d] = fc[d];
          nodeSt[sp] = farChild;
          sp++;
        }
      }
      curr = leftIsClose ? lChild : lChild + 1;
    }
    // heapsort: ascending keys in heap[0..K1)
    for (int end = K1 - 1; end > 0; end--) {
      const unsigned long long top = heap[0];
      const unsigned long long key = heap[end];
      heap[end] = top;
      int x = 0;
      for (;;) {
        const int l = 2 * x + 1;
        if (l >= end) break;
        int c = l;
        unsigned long long hc = heap[l];
        if (l + 1 < end && heap[l + 1] > hc) {
          c = l + 1;
          hc = heap[c];
        }
        if (hc <= key) break;
        heap[x] = hc;
        x = c;
      }
      heap[x] = key;
    }
    const float X = __uint_as_float(uint32_t(heap[k - 1] >> 32));
    const float Y = __uint_as_float(uint32_t(heap[k] >> 32));
    const int idX = int32_t(uint32_t(heap[k - 1]));
    bool ok = idX >= 0 ? (Y > X) : (!fa.radius && !sawInit);
    if (!(X == X)) ok = false;
    if (a.visits) a.visits[myq] += visits;
    if (!ok) {
      const int slot = atomicAdd(fa.fb_count, 1);
      fa.fb_list[slot] = int32_t(myq);
      if (fa.status) fa.status[myq] = 1;
      continue;
    }
    if (fa.status) fa.status[myq] = 0;
    int32_t *oid = a.out_ids ? a.out_ids + myq * k : nullptr;
    float *od = a.out_d2 ? (float *)a.out_d2 + myq * k : nullptr;
    for (int j = 0; j < k; j++) {
      if (oid) oid[j] = int32_t(uint32_t(heap[j]));
      if (od) od[j] = __uint_as_float(uint32_t(heap[j] >> 32));
    }
    if (a.out_max) ((float *)a.out_max)[myq] = X;
  }
}

template <int D, bool EXPL, bool VEC16, int KH>
int launch_fast_heap(const FastArgs &fa, cudaStream_t st)
{
  // the heap kernel takes blocks of at most 256 threads
  const int bs = fa.q.block_size > 0 ? std::min(fa.q.block_size, 256) : 128;
  const int64_t grid = std::max<int64_t>(1, div_up(fa.q.nq, int64_t(bs)));
  knn_fast_heap_kernel<D, EXPL, VEC16, KH><<<unsigned(grid), bs, 0, st>>>(fa);
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

template <int D, bool EXPL, bool VEC16, int KC>
int launch_fast(const FastArgs &fa, cudaStream_t st)
{
  const int bs = fa.q.block_size > 0 ? fa.q.block_size : 128;
  const int qpt = fa.q.queries_per_thread > 1 ? fa.q.queries_per_thread : 1;
  const int64_t grid = std::max<int64_t>(1, div_up(fa.q.nq, int64_t(bs) * qpt));
  knn_fast_kernel<D, EXPL, VEC16, KC><<<unsigned(grid), bs, 0, st>>>(fa);
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

template <int D, bool EXPL, bool VEC16>
int dispatch_kc(const FastArgs &fa, cudaStream_t st)
{
  const int slots = fa.kk + 1;
  if (slots <= 2) return launch_fast<D, EXPL, VEC16, 2>(fa, st);
  if (slots <= 5) return launch_fast<D, EXPL, VEC16, 5>(fa, st);
  if (slots <= 9) return launch_fast<D, EXPL, VEC16, 9>(fa, st);
  if (slots <= 17) return launch_fast<D, EXPL, VEC16, 17>(fa, st);
  if (slots <= 33) return launch_fast<D, EXPL, VEC16, 33>(fa, st);
  if (fa.fcp) return CUKD_ERR_UNSUPPORTED;
  if (slots <= 65) return launch_fast_heap<D, EXPL, VEC16, 65>(fa, st);
  if (slots <= 129) return launch_fast_heap<D, EXPL, VEC16, 129>(fa, st);
  return CUKD_ERR_UNSUPPORTED;
}

template <int D>
int dispatch_layout(const FastArgs &fa, cudaStream_t st)
{
  const QArgs &a = fa.q;
  const bool expl = a.doff >= 0;
  const bool vec16 = a.stride == 16 && a.poff == 0 && (!expl || a.doff == 12) && D <= 3;
  if (expl) {
    if (vec16) return dispatch_kc<D, true, true>(fa, st);
    return dispatch_kc<D, true, false>(fa, st);
  }
  if (vec16) return dispatch_kc<D, false, true>(fa, st);
  return dispatch_kc<D, false, false>(fa, st);
}

}  // namespace fast

int run_fast(const fast::FastArgs &fa, int D, cudaStream_t st)
{
  if (D == 2) return fast::dispatch_layout<2>(fa, st);
  if (D == 3) return fast::dispatch_layout<3>(fa, st);
  if (D == 4) return fast::dispatch_layout<4>(fa, st);
  return CUKD_ERR_UNSUPPORTED;
}

}  // namespace ckb
