// cukd/traverse.h -- the three balanced-tree traversals of the reference,
// restated for user kernels of the drop-in shim (device/host inline):
//   traverse_default     traverse-default-stack-based.h:24-108
//   traverse_stack_free  traverse-stack-free.h:24-117
//   traverse_cct         traverse-cct.h:25-99
// Each offers candidates to `result` (processCandidate(id, d2) -> cull
// distance) in the reference's visiting order, so answers match it bit for
// bit.
#pragma once

#include "cukd/data.h"
#include "cukd/helpers.h"

namespace cukd {
namespace detail {

template <typename data_t, typename traits>
inline __both__ int split_dim(const data_t *nodes, int i)
{
  enum { D = point_traits<typename traits::point_t>::num_dims };
  // get_dim is only required of traits with explicit dims
  if constexpr (bool(traits::has_explicit_dim))
    return traits::get_dim(nodes[i]);
  else
    return BinaryTree::levelOf(i) % D;
}

}  // namespace detail

template <typename result_t, typename data_t, typename data_traits = default_data_traits<data_t>>
inline __both__ void traverse_default(result_t &result,
                                      typename data_traits::point_t queryPoint,
                                      const data_t *d_nodes, int numPoints)
{
  using point_t = typename data_traits::point_t;
  using scalar_t = typename point_traits<point_t>::scalar_t;
  scalar_t cullDist = result.initialCullDist2();
  int stackNode[32];
  float stackDist[32];
  int sp = 0;
  int curr = 0;
  for (;;) {
    while (curr < numPoints) {
      const int dim = detail::split_dim<data_t, data_traits>(d_nodes, curr);
      const data_t &node = d_nodes[curr];
      cullDist = result.processCandidate(curr, sqrDistance(data_traits::get_point(node),
                                                           queryPoint));
      const auto nodeCoord = data_traits::get_coord(node, dim);
      const auto queryCoord = get_coord(queryPoint, dim);
      const bool leftIsClose = queryCoord < nodeCoord;
      const int lChild = 2 * curr + 1, rChild = lChild + 1;
      const int farChild = leftIsClose ? rChild : lChild;
      const auto diff = queryCoord - nodeCoord;
#ifdef __CUDA_ARCH__
      const float planeD2 = __fmul_rn(diff, diff);
#else
      const float planeD2 = float(diff * diff);
#endif
      if (planeD2 < cullDist && farChild < numPoints) {
        stackNode[sp] = farChild;
        stackDist[sp] = planeD2;
        sp++;
      }
      curr = leftIsClose ? lChild : rChild;
    }
    for (;;) {
      if (sp == 0) return;
      --sp;
      if (stackDist[sp] >= cullDist) continue;
      curr = stackNode[sp];
      break;
    }
  }
}

template <typename result_t, typename data_t, typename data_traits = default_data_traits<data_t>>
inline __both__ void traverse_stack_free(result_t &result,
                                         typename data_traits::point_t queryPoint,
                                         const data_t *d_nodes, int N, float eps = 0.f)
{
  using point_t = typename data_traits::point_t;
  using scalar_t = typename point_traits<point_t>::scalar_t;
  if (N <= 0) return;
  const float epsErr = 1.f + eps;
  scalar_t cullDist = result.initialCullDist2();
  int prev = -1, curr = 0;
  for (;;) {
    const int parent = (curr + 1) / 2 - 1;
    if (curr >= N) {
      prev = curr;
      curr = parent;
      continue;
    }
    const data_t &node = d_nodes[curr];
    const int child = 2 * curr + 1;
    if (!(prev >= child))
      cullDist = result.processCandidate(curr, sqrDistance(queryPoint,
                                                           data_traits::get_point(node)));
    const int dim = detail::split_dim<data_t, data_traits>(d_nodes, curr);
    const float dimDist = get_coord(queryPoint, dim) - data_traits::get_coord(node, dim);
    const int side = dimDist > 0.f;
    const int closeChild = 2 * curr + 1 + side, farChild = 2 * curr + 2 - side;
    int next;
    if (prev == closeChild) {
#ifdef __CUDA_ARCH__
      const bool farOk = __fmul_rn(__fmul_rn(dimDist, dimDist), epsErr) < cullDist;
#else
      const bool farOk = dimDist * dimDist * epsErr < cullDist;
#endif
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

template <typename result_t, typename data_t, typename data_traits = default_data_traits<data_t>>
inline __both__ void traverse_cct(result_t &result, typename data_traits::point_t queryPoint,
                                  const box_t<typename data_traits::point_t> d_bounds,
                                  const data_t *d_nodes, int numPoints)
{
  using point_t = typename data_traits::point_t;
  using scalar_t = typename point_traits<point_t>::scalar_t;
  scalar_t cullDist = result.initialCullDist2();
  int stackNode[32];
  point_t stackCorner[32];
  int sp = 0;
  point_t closest = project(d_bounds, queryPoint);
  if (sqrDistance(queryPoint, closest) > cullDist) return;
  int nodeID = 0;
  for (;;) {
    if (nodeID >= numPoints) {
      for (;;) {
        if (sp == 0) return;
        --sp;
        closest = stackCorner[sp];
        if (sqrDistance(closest, queryPoint) >= cullDist) continue;
        nodeID = stackNode[sp];
        break;
      }
    }
    const data_t &node = d_nodes[nodeID];
    const point_t nodePoint = data_traits::get_point(node);
    cullDist = result.processCandidate(nodeID, sqrDistance(nodePoint, queryPoint));
    const int dim = detail::split_dim<data_t, data_traits>(d_nodes, nodeID);
    const auto nodeDim = get_coord(nodePoint, dim);
    const bool leftIsClose = get_coord(queryPoint, dim) < nodeDim;
    const int lChild = 2 * nodeID + 1, rChild = lChild + 1;
    point_t farCorner = closest;
    set_coord(farCorner, dim, nodeDim);
    const int farChild = leftIsClose ? rChild : lChild;
    if (farChild < numPoints && sqrDistance(farCorner, queryPoint) < cullDist) {
      stackCorner[sp] = farCorner;
      stackNode[sp] = farChild;
      sp++;
    }
    nodeID = leftIsClose ? lChild : rChild;
  }
}

}  // namespace cukd
