// Fast exact kNN over int32 trees (k = 2..128), the integer counterpart of
// the float fast path (fast.cu; its header gives the argument why any
// visiting order is exact once the (k+1)-th distance is strictly above the
// k-th).  The reference has no integer traversal (its int vector types lack
// operator- / dot, cukd-math.h:100-112); this library's reference-order
// integer kernels (query.cuh, Traits<1>: exact int64 squared distances,
// (d2, id) keys) define the answer, and every query this kernel cannot
// settle is re-run by them.
//
// Per query: closest-corner culling ("<=") with integer corners (exact), the
// k+1 smallest (d2, id) keys in a local-memory max-heap (d2 and ids in two
// arrays), a heapsort at the end, the strict-gap check at the k-th boundary.
#include <algorithm>

#include "common.cuh"
#include "fast.cuh"

namespace ckb {
namespace fast {

using query::QArgs;
using query::TreeView;

__device__ __forceinline__ bool key_gt(long long ad, uint32_t ai, long long bd, uint32_t bi)
{
  return ad > bd || (ad == bd && ai > bi);
}

template <int D, bool EXPL, bool VEC16, int KH>
__global__ void __launch_bounds__(256) knn_fast_int_kernel(FastArgs fa)
{
  const QArgs &a = fa.q;
  const int64_t limit = a.count_ptr ? int64_t(*a.count_ptr) : a.nq;
  const int k = fa.kk;
  const int K1 = k + 1;  // <= KH
  long long hd[KH];
  uint32_t hid[KH];
  int nodeSt[32];
  int32_t cornerSt[32][D];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < limit;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t myq = a.order ? int64_t(a.order[i]) : i;
    const TreeView tv = query::tree_of<D, 4>(a, myq);
    const int N = int(tv.n);
    const uint8_t *tree = tv.tree;
    int32_t q[D];
    const int32_t *qp = (const int32_t *)a.queries + myq * D;
#pragma unroll
    for (int d = 0; d < D; d++) q[d] = __ldg(qp + d);
    long long r2 = a.cutoff_d2;
    if (fa.radius) {
      // learned initial radius (any bound is exact: the answer is checked
      // below; only the number of fallbacks depends on it)
      const double rr = double(__ldg(fa.radius + myq)) * double(fa.radius_scale);
      const double rb = ceil(rr * rr);
      const long long seed = rb >= 9.0e18 ? 0x7fffffffffffffffll : (long long)rb;
      r2 = seed < r2 ? seed : r2;
    }
    for (int j = 0; j < K1; j++) {
      hd[j] = r2;
      hid[j] = 0xffffffffu;
    }
    long long cull = r2;
    bool sawInit = false;
    auto dist2 = [&](const int32_t *c) {
      long long s = 0;
#pragma unroll
      for (int d = 0; d < D; d++) {
        const long long df = (long long)c[d] - (long long)q[d];
        s += df * df;
      }
      return s;
    };
    int32_t closest[D];
    const int32_t *bnd = (const int32_t *)tv.bounds;
#pragma unroll
    for (int d = 0; d < D; d++) {
      int32_t v = q[d];
      if (bnd) {
        const int32_t lo = __ldg(bnd + d), hi = __ldg(bnd + D + d);
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
      int32_t p[D];
      int dim;
      if (VEC16) {
        const uint4 v = __ldg((const uint4 *)(tree + int64_t(curr) * 16));
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int d = 0; d < D; d++) p[d] = int32_t(w[d]);
        dim = EXPL ? int((w[3] >> a.dshift) & a.dmask) : (level_of(curr) % D);
      } else {
        const int32_t *c = (const int32_t *)(tree + int64_t(curr) * a.stride + a.poff);
#pragma unroll
        for (int d = 0; d < D; d++) p[d] = __ldg(c + d);
        dim = EXPL ? int((__ldg((const uint32_t *)(tree + int64_t(curr) * a.stride + a.doff)) >>
                          a.dshift) & a.dmask)
                   : (level_of(curr) % D);
      }
      const long long d2 = dist2(p);
      sawInit |= (d2 == r2);
      const uint32_t id = uint32_t(curr);
      if (key_gt(hd[0], hid[0], d2, id)) {
        int x = 0;
        for (;;) {
          const int l = 2 * x + 1;
          if (l >= K1) break;
          int c = l;
          if (l + 1 < K1 && key_gt(hd[l + 1], hid[l + 1], hd[l], hid[l])) c = l + 1;
          if (!key_gt(hd[c], hid[c], d2, id)) break;
          hd[x] = hd[c];
          hid[x] = hid[c];
          x = c;
        }
        hd[x] = d2;
        hid[x] = id;
        cull = hd[0];
      }
      int32_t nodeC = p[0], queryC = q[0];
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
        int32_t fc[D];
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
    // heapsort: ascending (d2, id)
    for (int end = K1 - 1; end > 0; end--) {
      const long long td = hd[0];
      const uint32_t ti = hid[0];
      const long long kd = hd[end];
      const uint32_t ki = hid[end];
      hd[end] = td;
      hid[end] = ti;
      int x = 0;
      for (;;) {
        const int l = 2 * x + 1;
        if (l >= end) break;
        int c = l;
        if (l + 1 < end && key_gt(hd[l + 1], hid[l + 1], hd[l], hid[l])) c = l + 1;
        if (!key_gt(hd[c], hid[c], kd, ki)) break;
        hd[x] = hd[c];
        hid[x] = hid[c];
        x = c;
      }
      hd[x] = kd;
      hid[x] = ki;
    }
    const long long X = hd[k - 1];
    const long long Y = hd[k];
    const bool filled = hid[k - 1] != 0xffffffffu;
    const bool ok = filled ? (Y > X) : (!fa.radius && !sawInit);
    if (!ok) {
      const int slot = atomicAdd(fa.fb_count, 1);
      fa.fb_list[slot] = int32_t(myq);
      if (fa.status) fa.status[myq] = 1;
      continue;
    }
    if (fa.status) fa.status[myq] = 0;
    int32_t *oid = a.out_ids ? a.out_ids + myq * k : nullptr;
    long long *od = a.out_d2 ? (long long *)a.out_d2 + myq * k : nullptr;
    for (int j = 0; j < k; j++) {
      if (oid) oid[j] = hid[j] == 0xffffffffu ? -1 : int32_t(hid[j]);
      if (od) od[j] = hd[j];
    }
    if (a.out_max) ((long long *)a.out_max)[myq] = X;
  }
}

template <int D, bool EXPL, bool VEC16, int KH>
int launch_fast_int(const FastArgs &fa, cudaStream_t st)
{
  const int bs = fa.q.block_size > 0 ? fa.q.block_size : 128;
  const int64_t grid = std::max<int64_t>(1, div_up(fa.q.nq, int64_t(bs)));
  knn_fast_int_kernel<D, EXPL, VEC16, KH><<<unsigned(grid), bs, 0, st>>>(fa);
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

template <int D, bool EXPL, bool VEC16>
int dispatch_int_kh(const FastArgs &fa, cudaStream_t st)
{
  const int slots = fa.kk + 1;
  if (slots <= 9) return launch_fast_int<D, EXPL, VEC16, 9>(fa, st);
  if (slots <= 17) return launch_fast_int<D, EXPL, VEC16, 17>(fa, st);
  if (slots <= 33) return launch_fast_int<D, EXPL, VEC16, 33>(fa, st);
  if (slots <= 65) return launch_fast_int<D, EXPL, VEC16, 65>(fa, st);
  if (slots <= 129) return launch_fast_int<D, EXPL, VEC16, 129>(fa, st);
  return CUKD_ERR_UNSUPPORTED;
}

template <int D>
int dispatch_int_layout(const FastArgs &fa, cudaStream_t st)
{
  const QArgs &a = fa.q;
  const bool expl = a.doff >= 0;
  const bool vec16 = a.stride == 16 && a.poff == 0 && (!expl || a.doff == 12) && D <= 3;
  if (expl) {
    if (vec16) return dispatch_int_kh<D, true, true>(fa, st);
    return dispatch_int_kh<D, true, false>(fa, st);
  }
  if (vec16) return dispatch_int_kh<D, false, true>(fa, st);
  return dispatch_int_kh<D, false, false>(fa, st);
}

}  // namespace fast

int run_fast_int(const fast::FastArgs &fa, int D, cudaStream_t st)
{
  if (fa.fcp || fa.kk < 2) return CUKD_ERR_UNSUPPORTED;
  if (D == 2) return fast::dispatch_int_layout<2>(fa, st);
  if (D == 3) return fast::dispatch_int_layout<3>(fa, st);
  if (D == 4) return fast::dispatch_int_layout<4>(fa, st);
  return CUKD_ERR_UNSUPPORTED;
}

}  // namespace ckb
