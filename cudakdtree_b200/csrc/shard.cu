// Sharded kNN: per-query candidate lists that persist across calls, each
// call folding one more tree shard into them.  This is the device step of
// the reference's ring over shards (samples/mpiHugeQuery.cu:173-205, whose
// FlexHeapCandidateList resumes from the previous round's list,
// knn.h:360-371); the ring itself -- shards passed from rank to rank -- is
// host code (cudakdtree_b200/shard.py).
//
// List format (device uint64[nq][k], ascending): key = float bits of d2 << 32
// | global id, where global id = shard-local node index + the shard's
// id_offset (the reference keeps shard-local ids, mpiHugeQuery.cu:84-86,
// which cannot tell shards apart; the offset makes ids global).  Unfilled
// slots hold (max_radius^2, 0xffffffff).  After any set of calls a list
// holds exactly the k smallest (d2, global id) keys over every point of
// every shard folded in, whatever the order of the shards -- so the k-th
// distance equals the reference's result bit for bit.
//
// Per query: the list is loaded reversed (a descending array is a valid
// max-heap), the shard is traversed with closest-corner culling at "<="
// against the heap's root, better keys replace the root, and a heapsort
// writes the list back ascending.
#include <algorithm>

#include "common.cuh"
#include "query.cuh"

namespace ckb {
namespace shard {

using query::QArgs;

template <int D, bool EXPL, bool VEC16, int KH>
__global__ void __launch_bounds__(256) knn_accumulate_kernel(QArgs a, int k, int init,
                                                             unsigned long long *lists,
                                                             uint32_t idOffset)
{
  unsigned long long heap[KH];
  int nodeSt[32];
  float cornerSt[32][D];
  const int N = int(a.n);
  const uint8_t *tree = a.tree;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < a.nq;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t myq = a.order ? int64_t(a.order[i]) : i;
    unsigned long long *L = lists + myq * k;
    float q[D];
    const float *qp = (const float *)a.queries + myq * D;
#pragma unroll
    for (int d = 0; d < D; d++) q[d] = __ldg(qp + d);
    if (init) {
      const float r2 = __fmul_rn(a.cutoff, a.cutoff);
      const unsigned long long initKey =
          ((unsigned long long)__float_as_uint(r2) << 32) | 0xffffffffull;
      for (int j = 0; j < k; j++) heap[j] = initKey;
    } else {
      for (int j = 0; j < k; j++) heap[j] = L[k - 1 - j];
    }
    float cull = __uint_as_float(uint32_t(heap[0] >> 32));
    auto dist2 = [&](const float *c) {
      float s = __fmul_rn(__fsub_rn(c[0], q[0]), __fsub_rn(c[0], q[0]));
#pragma unroll
      for (int d = 1; d < D; d++)
        s = __fadd_rn(s, __fmul_rn(__fsub_rn(c[d], q[d]), __fsub_rn(c[d], q[d])));
      return s;
    };
    float closest[D];
    const float *bnd = (const float *)a.bounds;
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
      const unsigned long long key =
          ((unsigned long long)__float_as_uint(d2) << 32) | uint32_t(uint32_t(curr) + idOffset);
      if (key < heap[0]) {
        int x = 0;
        for (;;) {
          const int l = 2 * x + 1;
          if (l >= k) break;
          int c = l;
          unsigned long long hc = heap[l];
          if (l + 1 < k && heap[l + 1] > hc) {
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
    // heapsort to ascending, write back
    for (int end = k - 1; end > 0; end--) {
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
    for (int j = 0; j < k; j++) L[j] = heap[j];
  }
}

// ids (-1 for unfilled), d2, and the k-th distance: sqrt of the k-th d2
// unless infinite, as mpiHugeQuery.cu's extractFinalResult writes it
__global__ void lists_extract_kernel(const unsigned long long *__restrict__ lists, int64_t nq,
                                     int k, int32_t *ids, float *d2, float *kth)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nq * k;
       i += int64_t(gridDim.x) * blockDim.x) {
    const unsigned long long key = lists[i];
    const uint32_t id = uint32_t(key);
    const float v = __uint_as_float(uint32_t(key >> 32));
    if (ids) ids[i] = id == 0xffffffffu ? -1 : int32_t(id);
    if (d2) d2[i] = v;
    if (kth && (i % k) == k - 1) kth[i / k] = isinf(v) ? v : __fsqrt_rn(v);
  }
}

template <int D, bool EXPL, bool VEC16>
int launch(const QArgs &a, int k, int init, unsigned long long *lists, uint32_t off,
           cudaStream_t st)
{
  const int bs = a.block_size > 0 ? a.block_size : 128;
  const int64_t grid = std::max<int64_t>(1, std::min<int64_t>(div_up(a.nq, bs), int64_t(kNumSMs) * 64));
  if (k <= 32)
    knn_accumulate_kernel<D, EXPL, VEC16, 32><<<unsigned(grid), bs, 0, st>>>(a, k, init, lists, off);
  else
    knn_accumulate_kernel<D, EXPL, VEC16, 128><<<unsigned(grid), bs, 0, st>>>(a, k, init, lists, off);
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

template <int D>
int dispatch(const QArgs &a, int k, int init, unsigned long long *lists, uint32_t off,
             cudaStream_t st)
{
  const bool expl = a.doff >= 0;
  const bool vec16 = a.stride == 16 && a.poff == 0 && (!expl || a.doff == 12) && D <= 3;
  if (expl) {
    if (vec16) return launch<D, true, true>(a, k, init, lists, off, st);
    return launch<D, true, false>(a, k, init, lists, off, st);
  }
  if (vec16) return launch<D, false, true>(a, k, init, lists, off, st);
  return launch<D, false, false>(a, k, init, lists, off, st);
}

}  // namespace shard
}  // namespace ckb

extern "C" {

int cukd_knn_accumulate(const void *d_tree, int64_t n, const cukd_layout *layout,
                        const void *d_world_bounds, int64_t id_offset, const void *d_queries,
                        int64_t nq, const int32_t *d_order, int k, float max_radius, int init,
                        uint64_t *d_lists, cudaStream_t stream)
{
  using namespace ckb;
  Layout L;
  if (!make_layout(layout, &L) || L.scalar != CUKD_FLOAT32) return CUKD_ERR_INVALID_ARGUMENT;
  if (n < 0 || nq < 0 || k < 1 || k > 128) return CUKD_ERR_INVALID_ARGUMENT;
  if (id_offset < 0 || id_offset + n > int64_t(0xffffffffll)) return CUKD_ERR_INVALID_ARGUMENT;
  if (n > kMaxQueryTree) return CUKD_ERR_UNSUPPORTED;
  if (nq == 0) return CUKD_OK;
  if (!d_queries || !d_lists || (n > 0 && !d_tree) || !(max_radius >= 0.f))
    return CUKD_ERR_INVALID_ARGUMENT;
  query::QArgs a = {};
  a.tree = (const uint8_t *)d_tree;
  a.n = n;
  a.stride = L.stride;
  a.poff = L.poff;
  a.doff = L.doff;
  a.dshift = L.dshift;
  a.dmask = L.dmask;
  a.bounds = d_world_bounds;
  a.queries = d_queries;
  a.nq = nq;
  a.order = d_order;
  a.cutoff = max_radius;
  a.k = k;
  unsigned long long *lists = (unsigned long long *)d_lists;
  const uint32_t off = uint32_t(id_offset);
  switch (L.D) {
    case 2: return shard::dispatch<2>(a, k, init != 0, lists, off, stream);
    case 3: return shard::dispatch<3>(a, k, init != 0, lists, off, stream);
    case 4: return shard::dispatch<4>(a, k, init != 0, lists, off, stream);
  }
  return CUKD_ERR_UNSUPPORTED;
}

int cukd_knn_lists_extract(const uint64_t *d_lists, int64_t nq, int k, int32_t *d_out_ids,
                           float *d_out_d2, float *d_out_kth_dist, cudaStream_t stream)
{
  using namespace ckb;
  if (nq < 0 || k < 1 || k > 128 || (nq > 0 && !d_lists)) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq == 0) return CUKD_OK;
  const int64_t total = nq * k;
  const int blocks = int(std::max<int64_t>(1, std::min<int64_t>(div_up(total, 256), kNumSMs * 16)));
  shard::lists_extract_kernel<<<blocks, 256, 0, stream>>>((const unsigned long long *)d_lists, nq,
                                                          k, d_out_ids, d_out_d2, d_out_kth_dist);
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

}  // extern "C"
