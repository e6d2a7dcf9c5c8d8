// cukd/spatial-kdtree.h -- drop-in shim of the reference's spatial k-d tree
// (cukd/spatial-kdtree.h:69-126, traversals cukd/fcp.h:256-427 and
// cukd/knn.h:566-752).  The tree is built on the GPU by cukd_spatial_build
// (children numbered in parent order; otherwise the reference's tree), its
// arrays come from the memory resource and go back with cukd::free().  The
// records are not reordered: leaves list indices into `data`.
#pragma once

#include "cukd/builder.h"
#include "cukd/knn.h"

namespace cukd {

template <typename data_t, typename data_traits = default_data_traits<data_t>>
struct SpatialKDTree {
  using point_t = typename data_traits::point_t;
  using scalar_t = typename point_traits<point_t>::scalar_t;
  using box_t = cukd::box_t<point_t>;
  struct Node {
    float pos;        // split position (inner nodes)
    uint32_t offset;  // first child (inner) or first prim id (leaf)
    uint16_t count;   // prims in the leaf, 0 for inner nodes
    int16_t dim;      // split dimension (inner nodes)
  };
  box_t bounds;
  Node *nodes = nullptr;
  uint32_t *primIDs = nullptr;
  const data_t *data = nullptr;
  int numPrims = 0;
  int numNodes = 0;
};

struct BuildConfig {
  int makeLeafThreshold = 0;  // 0: the builder's default (8)
};

namespace detail {
template <typename data_t, typename traits>
__global__ void shim_points(const data_t *in, int n, typename traits::point_t *out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = traits::get_point(in[i]);
}
}  // namespace detail

template <typename data_t, typename data_traits = default_data_traits<data_t>>
void buildTree(SpatialKDTree<data_t, data_traits> &tree, data_t *d_points, int numPrims,
               BuildConfig buildConfig = {}, cudaStream_t stream = 0,
               GpuMemoryResource &memResource = defaultGpuMemResource())
{
  using point_t = typename data_traits::point_t;
  static_assert(std::is_same<typename point_traits<point_t>::scalar_t, float>::value,
                "spatial k-d trees are built over float points");
  cukd_mem_resource c = detail::as_c(memResource);
  point_t *pts = nullptr;
  const bool plain = std::is_same<data_t, point_t>::value;
  if (!plain && numPrims > 0) {
    if (memResource.malloc((void **)&pts, sizeof(point_t) * size_t(numPrims), stream) !=
        cudaSuccess)
      throw std::runtime_error("cukd::buildTree(SpatialKDTree): out of device memory");
    detail::shim_points<data_t, data_traits>
        <<<divRoundUp(numPrims, 256), 256, 0, stream>>>(d_points, numPrims, pts);
    CUKD_CUDA_CHECK(cudaGetLastError());
  }
  const cukd_layout l = detail::layout_of<point_t>(int(sizeof(point_t)), -1);
  cukd_spatial_tree t;
  const int rc = cukd_spatial_build(plain ? (const void *)d_points : (const void *)pts, numPrims,
                                    &l, buildConfig.makeLeafThreshold, &t, stream, &c);
  if (pts) memResource.free(pts, stream);
  detail::check(rc, "buildTree(SpatialKDTree)");
  CUKD_CUDA_CHECK(cudaStreamSynchronize(stream));
  tree.nodes = (typename SpatialKDTree<data_t, data_traits>::Node *)t.nodes;
  tree.primIDs = t.prim_ids;
  tree.data = d_points;
  tree.numPrims = t.num_prims;
  tree.numNodes = t.num_nodes;
  for (int d = 0; d < point_traits<point_t>::num_dims; d++) {
    set_coord(tree.bounds.lower, d, t.bounds[d]);
    set_coord(tree.bounds.upper, d, t.bounds[4 + d]);
  }
}

template <typename data_t, typename data_traits = default_data_traits<data_t>>
void free(SpatialKDTree<data_t, data_traits> &tree, cudaStream_t stream = 0,
          GpuMemoryResource &memResource = defaultGpuMemResource())
{
  if (tree.nodes) memResource.free(tree.nodes, stream);
  if (tree.primIDs) memResource.free(tree.primIDs, stream);
  tree.nodes = nullptr;
  tree.primIDs = nullptr;
  tree.numNodes = 0;
  tree.numPrims = 0;
}

namespace detail {
// The reference's spatial traversals (stack of 50; "STACK OVERFLOW" ends the
// query with -1 for FCP and the list as it is for kNN).  CCT tracks the
// closest corner of each subtree's box, stackBased the split-plane distance.
template <bool CCT, typename result_t, typename data_t, typename traits>
inline __both__ bool spatial_traverse(result_t &result, const SpatialKDTree<data_t, traits> &tree,
                                      typename traits::point_t q)
{
  using point_t = typename traits::point_t;
  float cullDist = result.initialCullDist2();
  int stackNode[50];
  float stackDist[50];
  point_t stackCorner[CCT ? 50 : 1];
  int sp = 0;
  point_t closest = q;
  if (CCT) {
    closest = project(tree.bounds, q);
    if (sqrDistance(q, closest) > cullDist) return true;
  }
  int nodeID = 0;
  for (;;) {
    typename SpatialKDTree<data_t, traits>::Node node;
    for (;;) {
      node = tree.nodes[nodeID];
      if (node.count) break;
      const float qc = get_coord(q, node.dim);
      const bool leftIsClose = qc < node.pos;
      const int lChild = int(node.offset), rChild = lChild + 1;
      const int farChild = leftIsClose ? rChild : lChild;
      bool push;
      if (CCT) {
        point_t fc = closest;
        set_coord(fc, node.dim, node.pos);
        push = sqrDistance(fc, q) < cullDist;
        if (push) stackCorner[sp] = fc;
      } else {
        const float diff = qc - node.pos;
        const float d2 = diff * diff;
        push = d2 < cullDist;
        if (push) stackDist[sp] = d2;
      }
      if (push) {
        stackNode[sp] = farChild;
        if (++sp >= 50) return false;
      }
      nodeID = leftIsClose ? lChild : rChild;
    }
    for (int i = 0; i < node.count; i++) {
      const int primID = int(tree.primIDs[node.offset + i]);
      cullDist = result.processCandidate(primID,
                                         sqrDistance(traits::get_point(tree.data[primID]), q));
    }
    for (;;) {
      if (sp == 0) return true;
      --sp;
      if (CCT) {
        closest = stackCorner[sp];
        if (sqrDistance(closest, q) >= cullDist) continue;
      } else {
        if (stackDist[sp] >= cullDist) continue;
      }
      nodeID = stackNode[sp];
      break;
    }
  }
}
}  // namespace detail

#define CUKD_SHIM_SPATIAL(NS, CCT)                                                           \
  namespace NS {                                                                            \
  template <typename data_t, typename data_traits = default_data_traits<data_t>>            \
  inline __both__ int fcp(const SpatialKDTree<data_t, data_traits> &tree,                   \
                          typename data_traits::point_t queryPoint,                          \
                          FcpSearchParams params = FcpSearchParams{})                        \
  {                                                                                         \
    FCPResult r;                                                                            \
    r.clear(params.cutOffRadius * params.cutOffRadius);                                     \
    if (!detail::spatial_traverse<CCT>(r, tree, queryPoint)) return -1;                     \
    return r.returnValue();                                                                 \
  }                                                                                         \
  template <typename CandidateList, typename data_t,                                        \
            typename data_traits = default_data_traits<data_t>>                             \
  inline __both__ float knn(CandidateList &result,                                          \
                            const SpatialKDTree<data_t, data_traits> &tree,                 \
                            typename data_traits::point_t queryPoint)                        \
  {                                                                                         \
    if (!detail::spatial_traverse<CCT>(result, tree, queryPoint)) return -1.f;              \
    return result.returnValue();                                                            \
  }                                                                                         \
  }
CUKD_SHIM_SPATIAL(stackBased, false)
CUKD_SHIM_SPATIAL(cct, true)
#undef CUKD_SHIM_SPATIAL

}  // namespace cukd
