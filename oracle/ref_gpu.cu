// GPU entry points into the UNMODIFIED reference library, compiled with
// -fmad=false so that its distance sums round like the CPU oracle.  Test
// infrastructure only (oracle/_ref/); used by the GPU parity tests to check
// that the product library reproduces the reference's own GPU builders and
// traversals bit for bit.
//
//   builders : cukd::buildTree_thrust   (cukd/builder_thrust.h:414-512)
//              cukd::buildTree_bitonic  (cukd/builder_bitonic.h:346-379)
//              cukd::buildTree_inPlace  (cukd/builder_inplace.h:444-471)
//              cukd::buildTree(SpatialKDTree&,...) (cukd/spatial-kdtree.h:632-645)
//   queries  : one thread per query calling the reference's fcp/knn, the
//              pattern of testing/floatN-knn-and-fcp.cu:146-220.
#include "ref_types.h"
#include <stdexcept>

using namespace refo;

namespace {

template <typename data_t, typename traits>
int build_gpu(int builder, void *d_pts, int n, void *d_bounds)
{
  using point_t = typename traits::point_t;
  try {
    if (builder == 0)
      cukd::buildTree_thrust<data_t, traits>((data_t *)d_pts, n, (cukd::box_t<point_t> *)d_bounds);
    else if (builder == 1)
      cukd::buildTree_bitonic<data_t, traits>((data_t *)d_pts, n, (cukd::box_t<point_t> *)d_bounds);
    else
      cukd::buildTree_inPlace<data_t, traits>((data_t *)d_pts, n, (cukd::box_t<point_t> *)d_bounds);
  } catch (const std::exception &) {
    return 1;
  }
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

template <typename data_t, typename traits>
__global__ void fcp_kernel(int method, const data_t *nodes, int n,
                           cukd::box_t<typename traits::point_t> box,
                           const typename traits::point_t *q, int nq, float cutoff, float eps,
                           int *out_ids)
{
  int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= nq) return;
  cukd::FcpSearchParams params;
  params.cutOffRadius = cutoff;
  params.eps = eps;
  int id;
  if (method == 0)
    id = cukd::stackBased::fcp<data_t, traits>(q[i], box, nodes, n, params);
  else if (method == 1)
    id = cukd::stackFree::fcp<data_t, traits>(q[i], box, nodes, n, params);
  else
    id = cukd::cct::fcp<data_t, traits>(q[i], box, nodes, n, params);
  out_ids[i] = id;
}

template <typename data_t, typename traits, typename list_t>
__global__ void knn_kernel(int method, const data_t *nodes, int n,
                           cukd::box_t<typename traits::point_t> box,
                           const typename traits::point_t *q, int nq, float cutoff,
                           int *out_ids, float *out_d2)
{
  enum { k = list_t::num_k };
  int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= nq) return;
  list_t result(cutoff);
  if (method == 0)
    cukd::stackBased::knn<list_t, data_t, traits>(result, q[i], box, nodes, n);
  else if (method == 1)
    cukd::stackFree::knn<list_t, data_t, traits>(result, q[i], box, nodes, n);
  else
    cukd::cct::knn<list_t, data_t, traits>(result, q[i], box, nodes, n);
  for (int j = 0; j < k; j++) {
    out_ids[(long)i * k + j] = result.get_pointID(j);
    out_d2[(long)i * k + j] = result.get_dist2(j);
  }
}

}  // namespace

// The GPU arm instantiates a narrower matrix than the host arm to keep its
// compile time bounded: the float3 types and the lists the configs use.
#define REFG_TYPES(X)                                                 \
  X(0, float2, cukd::default_data_traits<float2>, float2)             \
  X(1, float3, cukd::default_data_traits<float3>, float3)             \
  X(2, float4, cukd::default_data_traits<float4>, float4)             \
  X(4, refo::PointDim<float3>, refo::PointDim_traits<float3>, float3) \
  X(6, refo::PointPayload, refo::PointPayload_traits, float3)         \
  X(7, refo::PointPacked, refo::PointPacked_traits, float3)
#define REFG_LISTS(X) X(0, 1) X(0, 8) X(0, 16) X(1, 20) X(1, 32) X(1, 64)

extern "C" {

int refg_build(int type, int builder, void *d_pts, int n, void *d_bounds)
{
#define X(code, D, T, P) \
  if (type == code) return build_gpu<D, T>(builder, d_pts, n, d_bounds);
  REFG_TYPES(X)
#undef X
  return -1;
}

int refg_fcp(int type, int method, const void *d_tree, int n, const void *h_bounds,
             const void *d_queries, int nq, float cutoff, float eps, int *d_out_ids)
{
#define X(code, D, T, P)                                                                 \
  if (type == code) {                                                                    \
    fcp_kernel<D, T><<<(nq + 127) / 128, 128>>>(method, (const D *)d_tree, n,            \
                                                *(const cukd::box_t<P> *)h_bounds,       \
                                                (const P *)d_queries, nq, cutoff, eps,   \
                                                d_out_ids);                              \
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;                               \
  }
  REFG_TYPES(X)
#undef X
  return -1;
}

int refg_knn(int type, int method, int list_kind, int k, const void *d_tree, int n,
             const void *h_bounds, const void *d_queries, int nq, float cutoff, int *d_out_ids,
             float *d_out_d2)
{
#define L(kind, kk)                                                                     \
  if (list_kind == kind && k == kk) {                                                   \
    knn_kernel<DT, TT, typename ListOf<kind, kk>::type><<<(nq + 127) / 128, 128>>>(      \
        method, (const DT *)d_tree, n, *(const cukd::box_t<PT> *)h_bounds,              \
        (const PT *)d_queries, nq, cutoff, d_out_ids, d_out_d2);                        \
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;                              \
  }
#define X(code, D, T, P) \
  if (type == code) {    \
    using DT = D;        \
    using TT = T;        \
    using PT = P;        \
    REFG_LISTS(L)        \
    return -2;           \
  }
  REFG_TYPES(X)
#undef X
#undef L
  return -1;
}

// Spatial k-d tree built by the reference's GPU builder; the arrays it
// allocates are copied out to caller-provided host buffers of sufficient
// size (nodes: 2*n entries of 12 bytes, primIDs: n entries) and freed.
int refg_spatial_build_float3(const void *d_pts, int n, int leaf_threshold, void *h_nodes,
                              void *h_primIDs, int *h_numNodes, void *h_bounds)
{
  cukd::SpatialKDTree<float3> tree;
  cukd::BuildConfig cfg;
  cfg.makeLeafThreshold = leaf_threshold;
  cukd::buildTree(tree, (float3 *)d_pts, n, cfg);
  if (cudaDeviceSynchronize() != cudaSuccess) return 2;
  cudaMemcpy(h_nodes, tree.nodes, tree.numNodes * sizeof(*tree.nodes), cudaMemcpyDeviceToHost);
  cudaMemcpy(h_primIDs, tree.primIDs, tree.numPrims * sizeof(uint32_t), cudaMemcpyDeviceToHost);
  *h_numNodes = tree.numNodes;
  *(cukd::box_t<float3> *)h_bounds = tree.bounds;
  cukd::free(tree);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

// The same build timed alone (CUDA events around the reference's buildTree
// call, its own allocations included), the tree freed afterwards.
int refg_spatial_build_ms_float3(const void *d_pts, int n, int leaf_threshold, float *ms)
{
  cukd::SpatialKDTree<float3> tree;
  cukd::BuildConfig cfg;
  cfg.makeLeafThreshold = leaf_threshold;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, 0);
  cukd::buildTree(tree, (float3 *)d_pts, n, cfg);
  cudaEventRecord(b, 0);
  const bool ok = cudaEventSynchronize(b) == cudaSuccess;
  cudaEventElapsedTime(ms, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cukd::free(tree);
  return ok && cudaDeviceSynchronize() == cudaSuccess ? 0 : 2;
}

}  // extern "C"
