// Whole-batch FCP / kNN queries over a left-balanced k-d tree (sm_100a).
//
// One thread runs one query with exactly the reference's control flow --
// traverse_default (traverse-default-stack-based.h:24-108),
// traverse_stack_free (traverse-stack-free.h:24-117) and traverse_cct
// (traverse-cct.h:25-99) -- so candidates reach the result object in the
// same order and the answers are bit-identical, ties included.  What is
// B200-specific is around that core:
//   - queries are visited in 30-bit Morton order (morton.cu) so a warp's
//     32 traversals walk nearby paths, and results are scattered back;
//   - node records are read through the read-only path (__ldg), 16-byte
//     vector loads for 16-byte records;
//   - fixed-size candidate lists live in registers with an early-out
//     before the insertion network (same result: a key not below the
//     current k-th key leaves the list unchanged);
//   - distances use __fmul_rn/__fadd_rn so no FMA contraction can change
//     a bit, matching the reference's ((dx*dx+dy*dy)+dz*dz) evaluation.
#include <algorithm>

#include "common.cuh"
#include "fast.cuh"
#include "query.cuh"
#include "sort.cuh"

namespace ckb {
namespace query {

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
template <int SC, int D, bool EXPL, bool VEC16, int METHOD, class Res>
__global__ void __launch_bounds__(256) query_kernel(QArgs a)
{
  using Tr = Traits<SC>;
  using T = typename Tr::T;
  const int64_t limit = a.count_ptr ? int64_t(*a.count_ptr) : a.nq;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < limit;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int64_t qi = a.order ? int64_t(a.order[i]) : i;
    T q[D];
    const T *qp = (const T *)a.queries + qi * D;
#pragma unroll
    for (int d = 0; d < D; d++) q[d] = __ldg(qp + d);
    const TreeView tv = tree_of<D, sizeof(T)>(a, qi);
    NodeReader<SC, D, EXPL, VEC16> rd(a);
    rd.tree = tv.tree;
    Res res(a);
    if (METHOD == CUKD_STACK_BASED)
      trav_stack_based<SC, D>(res, q, rd, tv.n);
    else if (METHOD == CUKD_STACK_FREE)
      trav_stack_free<SC, D>(res, q, rd, tv.n, a.eps);
    else
      trav_cct<SC, D>(res, q, rd, tv.n, (const T *)tv.bounds);
    res.write(a, qi);
  }
}

// Tree-path key of each query: the bits of the left / right choices of a
// closest-side descent from the root to a leaf, left-aligned to the tree's
// depth, so that sorting by it groups queries by the subtrees they enter
// (an order adapted to this tree's splits; results are unchanged).
template <int SC, int D, bool EXPL, bool VEC16>
__global__ void __launch_bounds__(256) tree_path_kernel(QArgs a, int levels, uint32_t *codes,
                                                        uint32_t *vals)
{
  using T = typename Traits<SC>::T;
  const NodeReader<SC, D, EXPL, VEC16> rd(a);
  const int N = int(a.n);
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < a.nq;
       i += int64_t(gridDim.x) * blockDim.x) {
    T q[D];
    const T *qp = (const T *)a.queries + i * D;
#pragma unroll
    for (int d = 0; d < D; d++) q[d] = __ldg(qp + d);
    uint32_t code = 0;
    int depth = 0, curr = 0;
    while (curr < N) {
      T p[D];
      const int dim = rd.load(curr, p);
      T nodeC = p[0], queryC = q[0];
#pragma unroll
      for (int d = 1; d < D; d++)
        if (d == dim) {
          nodeC = p[d];
          queryC = q[d];
        }
      const uint32_t right = queryC < nodeC ? 0u : 1u;
      code = (code << 1) | right;
      depth++;
      curr = 2 * curr + 1 + int(right);
    }
    codes[i] = levels > depth ? code << (levels - depth) : code;
    vals[i] = uint32_t(i);
  }
}

template <int SC, int D, bool EXPL, bool VEC16>
int launch_tree_path(const QArgs &a, int levels, uint32_t *codes, uint32_t *vals,
                     cudaStream_t st)
{
  const int blocks = int(std::max<int64_t>(1, std::min<int64_t>(div_up(a.nq, 256), kNumSMs * 16)));
  tree_path_kernel<SC, D, EXPL, VEC16><<<blocks, 256, 0, st>>>(a, levels, codes, vals);
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

int run_tree_path(const QArgs &a, int scalar, int D, int levels, uint32_t *codes, uint32_t *vals,
                  cudaStream_t st)
{
  const bool expl = a.doff >= 0;
  const bool vec16 = a.stride == 16 && a.poff == 0 && (!expl || a.doff == 12) && D <= 3;
#define CKB_TP(SC_, D_)                                                                   \
  if (scalar == SC_ && D == D_) {                                                         \
    if (expl) return vec16 ? launch_tree_path<SC_, D_, true, true>(a, levels, codes, vals, st) \
                           : launch_tree_path<SC_, D_, true, false>(a, levels, codes, vals, st); \
    return vec16 ? launch_tree_path<SC_, D_, false, true>(a, levels, codes, vals, st)      \
                 : launch_tree_path<SC_, D_, false, false>(a, levels, codes, vals, st);    \
  }
  CKB_TP(0, 2) CKB_TP(0, 3) CKB_TP(0, 4)
  CKB_TP(1, 2) CKB_TP(1, 3) CKB_TP(1, 4)
#undef CKB_TP
  return CUKD_ERR_UNSUPPORTED;
}

template <int SC, int D, bool EXPL, bool VEC16, int METHOD, class Res>
int launch(const QArgs &a, cudaStream_t st)
{
  const int bs = a.block_size > 0 ? a.block_size : 128;
  int64_t grid = div_up(a.nq, bs);
  if (a.count_ptr) grid = std::min<int64_t>(grid, int64_t(kNumSMs) * 16);
  query_kernel<SC, D, EXPL, VEC16, METHOD, Res><<<unsigned(grid), bs, 0, st>>>(a);
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

template <int SC, int D, bool EXPL, bool VEC16, int METHOD>
int dispatch_res(const QArgs &a, int kind, cudaStream_t st)
{
  switch (kind) {
    case RES_FCP: return launch<SC, D, EXPL, VEC16, METHOD, FcpRes<SC>>(a, st);
    case RES_FIX4: return launch<SC, D, EXPL, VEC16, METHOD, FixedRes<SC, 4>>(a, st);
    case RES_FIX8: return launch<SC, D, EXPL, VEC16, METHOD, FixedRes<SC, 8>>(a, st);
    case RES_FIX16: return launch<SC, D, EXPL, VEC16, METHOD, FixedRes<SC, 16>>(a, st);
    case RES_FIX32: return launch<SC, D, EXPL, VEC16, METHOD, FixedRes<SC, 32>>(a, st);
    case RES_HEAP128: return launch<SC, D, EXPL, VEC16, METHOD, HeapRes<SC, 128>>(a, st);
    case RES_HEAP1024: return launch<SC, D, EXPL, VEC16, METHOD, HeapRes<SC, 1024>>(a, st);
  }
  return CUKD_ERR_UNSUPPORTED;
}

template <int SC, int D, bool EXPL, bool VEC16>
int dispatch_method(const QArgs &a, int method, int kind, cudaStream_t st)
{
  switch (method) {
    case CUKD_STACK_BASED: return dispatch_res<SC, D, EXPL, VEC16, CUKD_STACK_BASED>(a, kind, st);
    case CUKD_STACK_FREE: return dispatch_res<SC, D, EXPL, VEC16, CUKD_STACK_FREE>(a, kind, st);
    case CUKD_CCT: return dispatch_res<SC, D, EXPL, VEC16, CUKD_CCT>(a, kind, st);
  }
  return CUKD_ERR_INVALID_ARGUMENT;
}

template <int SC, int D>
int dispatch_layout(const QArgs &a, int method, int kind, cudaStream_t st)
{
  const bool expl = a.doff >= 0;
  const bool vec16 = a.stride == 16 && a.poff == 0 && (!expl || a.doff == 12) && D <= 3;
  if (expl) {
    if (vec16) return dispatch_method<SC, D, true, true>(a, method, kind, st);
    return dispatch_method<SC, D, true, false>(a, method, kind, st);
  }
  if (vec16) return dispatch_method<SC, D, false, true>(a, method, kind, st);
  return dispatch_method<SC, D, false, false>(a, method, kind, st);
}

int run_query(const QArgs &a, int scalar, int D, int method, int kind, cudaStream_t st)
{
#define CKB_CASE(SC_, D_) \
  if (scalar == SC_ && D == D_) return dispatch_layout<SC_, D_>(a, method, kind, st);
  CKB_CASE(0, 2) CKB_CASE(0, 3) CKB_CASE(0, 4) CKB_CASE(0, 5) CKB_CASE(0, 6) CKB_CASE(0, 7)
  CKB_CASE(0, 8) CKB_CASE(1, 2) CKB_CASE(1, 3) CKB_CASE(1, 4) CKB_CASE(1, 5) CKB_CASE(1, 6)
  CKB_CASE(1, 7) CKB_CASE(1, 8)
#undef CKB_CASE
  return CUKD_ERR_UNSUPPORTED;
}

}  // namespace query

int morton_order_impl(const float *pts, int64_t n, int D, const float *bounds, int32_t *perm,
                      cudaStream_t st, const cukd_mem_resource *mem);


static int common_query(const void *d_tree, int64_t n, const cukd_layout *layout,
                        const void *d_world_bounds, const void *d_queries, int64_t nq,
                        const cukd_query_params *p, bool knn, int32_t *ids, void *d2,
                        void *maxd2, int64_t *visits, cudaStream_t st,
                        const cukd_mem_resource *mem)
{
  using namespace query;
  Layout L;
  if (!make_layout(layout, &L) || !p) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq < 0 || n < 0) return CUKD_ERR_INVALID_ARGUMENT;
  if (n > kMaxQueryTree) return CUKD_ERR_UNSUPPORTED;
  if (nq == 0) return CUKD_OK;
  if (!d_queries || (!ids && !visits) || (n > 0 && !d_tree)) return CUKD_ERR_INVALID_ARGUMENT;
  if (p->method < CUKD_STACK_BASED || p->method > CUKD_CCT) return CUKD_ERR_INVALID_ARGUMENT;
  if (p->method == CUKD_CCT && !d_world_bounds) return CUKD_ERR_INVALID_ARGUMENT;
  if (p->block_size != 0 && (p->block_size < 32 || p->block_size > 256 || p->block_size % 32))
    return CUKD_ERR_INVALID_ARGUMENT;
  int kind = RES_FCP;
  if (knn) {
    const int k = p->k;
    if (k < 1 || k > 1024) return CUKD_ERR_INVALID_ARGUMENT;
    const bool heap = (p->flags & (CUKD_QUERY_FORCE_HEAP | CUKD_QUERY_HEAP_ORDER)) || k > 32;
    if (heap)
      kind = k <= 128 ? RES_HEAP128 : RES_HEAP1024;
    else
      kind = k <= 4 ? RES_FIX4 : (k <= 8 ? RES_FIX8 : (k <= 16 ? RES_FIX16 : RES_FIX32));
  }
  QArgs a = {};
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
  a.k = knn ? p->k : 1;
  a.cutoff = p->cutoff_radius;
  a.cutoff_d2 = p->cutoff_d2;
  a.eps = p->eps;
  a.heap_order = (p->flags & CUKD_QUERY_HEAP_ORDER) != 0;
  a.out_ids = ids;
  a.out_d2 = d2;
  a.out_max = maxd2;
  a.visits = visits;
  a.block_size = p->block_size;
  TempArena arena(st, mem);
  // query orders (tree path, Morton) and the fast path: up to 4 dims
  const bool narrow = L.D <= kMaxFastDims;
  if ((p->flags & CUKD_QUERY_TREE_ORDER) && nq > 1 && n > 0 && narrow) {
    uint32_t *codes = nullptr, *codes2 = nullptr, *vals = nullptr, *vals2 = nullptr;
    CKB_TRY(arena.alloc(&codes, nq));
    CKB_TRY(arena.alloc(&codes2, nq));
    CKB_TRY(arena.alloc(&vals, nq));
    CKB_TRY(arena.alloc(&vals2, nq));
    const int levels = num_levels(n);
    CKB_TRY(run_tree_path(a, L.scalar, L.D, levels, codes, vals, st));
    CKB_TRY(radix_sort_pairs(codes, vals, codes2, vals2, nq, levels, st, &arena));
    a.order = (const int32_t *)vals;
  } else if ((p->flags & CUKD_QUERY_MORTON) && nq > 1 && L.scalar == CUKD_FLOAT32 && narrow) {
    int32_t *perm = nullptr;
    CKB_TRY(arena.alloc(&perm, nq));
    // the Morton grid spans the tree's world bounds when the caller passes
    // them (no bounds pass over the queries; queries outside are clamped to
    // the box faces, which only coarsens their order), else the queries' own
    CKB_TRY(morton_order_impl((const float *)d_queries, nq, L.D, (const float *)d_world_bounds,
                              perm, st, mem));
    a.order = perm;
  }
  // fast exact path (see fast.cu): any visiting order, boundary-tie check,
  // reference-order re-run of the queued queries
  const bool fastOk = !visits && !a.heap_order && !(p->flags & CUKD_QUERY_REFERENCE_ORDER) &&
                      knn && p->k >= 2 && p->k <= 128 && n < (int64_t(1) << 31) - 1 && narrow;
  // (FCP and k = 1 stay on the reference traversals: with a single
  // candidate the split-plane bound is already cheap and the corner
  // bookkeeping does not pay for itself)
  if (fastOk) {
    fast::FastArgs fa = {};
    fa.q = a;
    fa.kk = knn ? p->k : 1;
    fa.fcp = !knn;
    int *ctr = nullptr;
    CKB_TRY(arena.alloc(&ctr, 2));
    CKB_CUDA(cudaMemsetAsync(ctr, 0, 2 * sizeof(int), st));
    fa.work = ctr;
    fa.fb_count = ctr + 1;
    CKB_TRY(arena.alloc(&fa.fb_list, nq));
    const bool packet = (p->flags & CUKD_QUERY_WARP_PACKET) && L.scalar == CUKD_FLOAT32 &&
                        knn && p->k <= 32;
    CKB_TRY(packet ? run_packet(fa, L.D, st)
                   : (L.scalar == CUKD_FLOAT32 ? run_fast(fa, L.D, st) : run_fast_int(fa, L.D, st)));
    if (p->d_reordered_count)
      CKB_CUDA(cudaMemcpyAsync(p->d_reordered_count, fa.fb_count, sizeof(int),
                               cudaMemcpyDeviceToDevice, st));
    QArgs b = a;
    b.order = fa.fb_list;
    b.count_ptr = fa.fb_count;
    return run_query(b, L.scalar, L.D, p->method, kind, st);
  }
  return run_query(a, L.scalar, L.D, p->method, kind, st);
}

}  // namespace ckb

extern "C" {

void cukd_query_params_init(cukd_query_params *p)
{
  if (!p) return;
  p->method = CUKD_STACK_BASED;
  p->k = 8;
  p->cutoff_radius = __builtin_huge_valf();
  p->eps = 0.f;
  p->cutoff_d2 = INT64_MAX;
  p->flags = CUKD_QUERY_MORTON;
  p->block_size = 0;
  p->d_reordered_count = nullptr;
}

int cukd_fcp(const void *d_tree, int64_t n, const cukd_layout *layout,
             const void *d_world_bounds, const void *d_queries, int64_t nq,
             const cukd_query_params *params, int32_t *d_out_ids, void *d_out_d2,
             cudaStream_t stream, const cukd_mem_resource *mem)
{
  return ckb::common_query(d_tree, n, layout, d_world_bounds, d_queries, nq, params, false,
                           d_out_ids, d_out_d2, nullptr, nullptr, stream, mem);
}

int cukd_knn(const void *d_tree, int64_t n, const cukd_layout *layout,
             const void *d_world_bounds, const void *d_queries, int64_t nq,
             const cukd_query_params *params, int32_t *d_out_ids, void *d_out_d2,
             void *d_out_max_d2, cudaStream_t stream, const cukd_mem_resource *mem)
{
  if (!d_out_ids && nq > 0) return CUKD_ERR_INVALID_ARGUMENT;
  return ckb::common_query(d_tree, n, layout, d_world_bounds, d_queries, nq, params, true,
                           d_out_ids, d_out_d2, d_out_max_d2, nullptr, stream, mem);
}

int cukd_knn_visits(const void *d_tree, int64_t n, const cukd_layout *layout,
                    const void *d_world_bounds, const void *d_queries, int64_t nq,
                    const cukd_query_params *params, int64_t *d_out_visits,
                    cudaStream_t stream, const cukd_mem_resource *mem)
{
  if (!d_out_visits && nq > 0) return CUKD_ERR_INVALID_ARGUMENT;
  return ckb::common_query(d_tree, n, layout, d_world_bounds, d_queries, nq, params,
                           params && params->k > 0, nullptr, nullptr, nullptr, d_out_visits,
                           stream, mem);
}

}  // extern "C"
