// cukd/fcp.h -- drop-in shim: find-closest-point queries for user kernels
// (reference cukd/fcp.h:35-254).  Same names, parameters and semantics:
// FcpSearchParams, FCPResult (strict '<': the first visited of equally close
// points wins), stackBased / stackFree / cct ::fcp returning the node index or
// -1 when nothing lies within the cut-off radius.
#pragma once

#include "cukd/traverse.h"

namespace cukd {

struct FcpSearchParams {
  int far_node_inspect_budget = INT_MAX;  // accepted, not used (like the reference)
  float cutOffRadius = INFINITY;
  float eps = 0.f;                        // honoured by stackFree only
};

struct FCPResult {
  inline __both__ float initialCullDist2() const { return closestDist2; }
  inline __both__ float clear(float initialDist2)
  {
    closestDist2 = initialDist2;
    closestPrimID = -1;
    return closestDist2;
  }
  inline __both__ float processCandidate(int candPrimID, float candDist2)
  {
    if (candDist2 < closestDist2) {
      closestDist2 = candDist2;
      closestPrimID = candPrimID;
    }
    return closestDist2;
  }
  inline __both__ int returnValue() const { return closestPrimID; }
  int closestPrimID;
  float closestDist2;
};

namespace stackBased {
template <typename data_t, typename data_traits = default_data_traits<data_t>>
inline __both__ int fcp(typename data_traits::point_t queryPoint, const data_t *dataPoints,
                        int numDataPoints, FcpSearchParams params = FcpSearchParams{})
{
  FCPResult r;
  r.clear(params.cutOffRadius * params.cutOffRadius);
  traverse_default<FCPResult, data_t, data_traits>(r, queryPoint, dataPoints, numDataPoints);
  return r.returnValue();
}
template <typename data_t, typename data_traits = default_data_traits<data_t>>
inline __both__ int fcp(typename data_traits::point_t queryPoint,
                        const box_t<typename data_traits::point_t> worldBounds,
                        const data_t *dataPoints, int numDataPoints,
                        FcpSearchParams params = FcpSearchParams{})
{
  return fcp<data_t, data_traits>(queryPoint, dataPoints, numDataPoints, params);
}
}  // namespace stackBased

namespace stackFree {
template <typename data_t, typename data_traits = default_data_traits<data_t>>
inline __both__ int fcp(typename data_traits::point_t queryPoint, const data_t *dataPoints,
                        int numDataPoints, FcpSearchParams params = FcpSearchParams{})
{
  FCPResult r;
  r.clear(params.cutOffRadius * params.cutOffRadius);
  traverse_stack_free<FCPResult, data_t, data_traits>(r, queryPoint, dataPoints, numDataPoints,
                                                      params.eps);
  return r.returnValue();
}
template <typename data_t, typename data_traits = default_data_traits<data_t>>
inline __both__ int fcp(typename data_traits::point_t queryPoint,
                        const box_t<typename data_traits::point_t> worldBounds,
                        const data_t *dataPoints, int numDataPoints,
                        FcpSearchParams params = FcpSearchParams{})
{
  return fcp<data_t, data_traits>(queryPoint, dataPoints, numDataPoints, params);
}
}  // namespace stackFree

namespace cct {
template <typename data_t, typename data_traits = default_data_traits<data_t>>
inline __both__ int fcp(typename data_traits::point_t queryPoint,
                        const box_t<typename data_traits::point_t> worldBounds,
                        const data_t *dataPoints, int numDataPoints,
                        FcpSearchParams params = FcpSearchParams{})
{
  FCPResult r;
  r.clear(params.cutOffRadius * params.cutOffRadius);
  traverse_cct<FCPResult, data_t, data_traits>(r, queryPoint, worldBounds, dataPoints,
                                               numDataPoints);
  return r.returnValue();
}
}  // namespace cct

}  // namespace cukd
