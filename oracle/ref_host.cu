// Host-side (CPU) entry points into the UNMODIFIED reference library, for
// use as the test oracle and as the timed CPU baseline.  Test
// infrastructure only; built by oracle/Makefile into oracle/_ref/.
//
// What runs here is the reference's own code:
//   build   : cukd::buildTree_host            (cukd/builder_thrust.h:514-601)
//   fcp     : cukd::{stackBased,stackFree,cct}::fcp   (cukd/fcp.h:210-254)
//   knn     : cukd::{stackBased,stackFree,cct}::knn   (cukd/knn.h:551-678)
//   spatial : cukd::{stackBased,cct}::{fcp,knn} over a SpatialKDTree whose
//             arrays live in host memory (cukd/fcp.h:256-427, knn.h:566-752)
// called from OpenMP loops over queries, the pattern of sampleHost.cu:58-73.
#include "ref_types.h"
#include <omp.h>
#include <stdexcept>

using namespace refo;

namespace {

template <typename data_t, typename traits>
int build_host(void *pts, int n, void *bounds)
{
  using point_t = typename traits::point_t;
  try {
    cukd::buildTree_host<data_t, traits>((data_t *)pts, n, (cukd::box_t<point_t> *)bounds);
  } catch (const std::exception &) {
    return 1;
  }
  return 0;
}

template <typename data_t, typename traits>
void fcp_host(int method, const void *tree, int n, const void *bounds, const void *queries,
              long nq, float cutoff, float eps, int *out_ids, int nthreads)
{
  using point_t = typename traits::point_t;
  const data_t *nodes = (const data_t *)tree;
  const cukd::box_t<point_t> box = *(const cukd::box_t<point_t> *)bounds;
  const point_t *q = (const point_t *)queries;
  cukd::FcpSearchParams params;
  params.cutOffRadius = cutoff;
  params.eps = eps;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1024)
  for (long i = 0; i < nq; i++) {
    int id;
    if (method == 0)
      id = cukd::stackBased::fcp<data_t, traits>(q[i], box, nodes, n, params);
    else if (method == 1)
      id = cukd::stackFree::fcp<data_t, traits>(q[i], box, nodes, n, params);
    else
      id = cukd::cct::fcp<data_t, traits>(q[i], box, nodes, n, params);
    out_ids[i] = id;
  }
}

template <typename data_t, typename traits, typename list_t>
void knn_host(int method, const void *tree, int n, const void *bounds, const void *queries,
              long nq, float cutoff, int *out_ids, float *out_d2, float *out_ret, int nthreads)
{
  using point_t = typename traits::point_t;
  enum { k = list_t::num_k };
  const data_t *nodes = (const data_t *)tree;
  const cukd::box_t<point_t> box = *(const cukd::box_t<point_t> *)bounds;
  const point_t *q = (const point_t *)queries;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 256)
  for (long i = 0; i < nq; i++) {
    list_t result(cutoff);
    float r;
    if (method == 0)
      r = cukd::stackBased::knn<list_t, data_t, traits>(result, q[i], box, nodes, n);
    else if (method == 1)
      r = cukd::stackFree::knn<list_t, data_t, traits>(result, q[i], box, nodes, n);
    else
      r = cukd::cct::knn<list_t, data_t, traits>(result, q[i], box, nodes, n);
    if (out_ret) out_ret[i] = r;
    for (int j = 0; j < k; j++) {
      out_ids[i * k + j] = result.get_pointID(j);
      out_d2[i * k + j] = result.get_dist2(j);
    }
  }
}

template <typename data_t, typename traits>
void spatial_fcp_host(int method, const void *nodes, const void *primIDs, const void *data,
                      int numPrims, int numNodes, const void *bounds, const void *queries,
                      long nq, float cutoff, int *out_ids, int nthreads)
{
  using point_t = typename traits::point_t;
  cukd::SpatialKDTree<data_t, traits> tree;
  tree.bounds = *(const cukd::box_t<point_t> *)bounds;
  tree.nodes = (typename cukd::SpatialKDTree<data_t, traits>::Node *)nodes;
  tree.primIDs = (uint32_t *)primIDs;
  tree.data = (const data_t *)data;
  tree.numPrims = numPrims;
  tree.numNodes = numNodes;
  const point_t *q = (const point_t *)queries;
  cukd::FcpSearchParams params;
  params.cutOffRadius = cutoff;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 1024)
  for (long i = 0; i < nq; i++) {
    int id;
    if (method == 0)
      id = cukd::stackBased::fcp<data_t, traits>(tree, q[i], params);
    else
      id = cukd::cct::fcp<data_t, traits>(tree, q[i], params);
    out_ids[i] = id;
  }
}

template <typename data_t, typename traits, typename list_t>
void spatial_knn_host(int method, const void *nodes, const void *primIDs, const void *data,
                      int numPrims, int numNodes, const void *bounds, const void *queries,
                      long nq, float cutoff, int *out_ids, float *out_d2, int nthreads)
{
  using point_t = typename traits::point_t;
  enum { k = list_t::num_k };
  cukd::SpatialKDTree<data_t, traits> tree;
  tree.bounds = *(const cukd::box_t<point_t> *)bounds;
  tree.nodes = (typename cukd::SpatialKDTree<data_t, traits>::Node *)nodes;
  tree.primIDs = (uint32_t *)primIDs;
  tree.data = (const data_t *)data;
  tree.numPrims = numPrims;
  tree.numNodes = numNodes;
  const point_t *q = (const point_t *)queries;
#pragma omp parallel for num_threads(nthreads) schedule(dynamic, 256)
  for (long i = 0; i < nq; i++) {
    list_t result(cutoff);
    if (method == 0)
      cukd::stackBased::knn<list_t, data_t, traits>(result, tree, q[i]);
    else
      cukd::cct::knn<list_t, data_t, traits>(result, tree, q[i]);
    for (int j = 0; j < k; j++) {
      out_ids[i * k + j] = result.get_pointID(j);
      out_d2[i * k + j] = result.get_dist2(j);
    }
  }
}

}  // namespace

extern "C" {

int refh_max_threads() { return omp_get_max_threads(); }

int refh_build(int type, void *pts, int n, void *bounds)
{
#define X(code, D, T, P) \
  if (type == code) return build_host<D, T>(pts, n, bounds);
  REFO_TYPES(X)
#undef X
  return -1;
}

int refh_fcp(int type, int method, const void *tree, int n, const void *bounds,
             const void *queries, long nq, float cutoff, float eps, int *out_ids, int nthreads)
{
#define X(code, D, T, P)                                                              \
  if (type == code) {                                                                 \
    fcp_host<D, T>(method, tree, n, bounds, queries, nq, cutoff, eps, out_ids, nthreads); \
    return 0;                                                                         \
  }
  REFO_TYPES(X)
#undef X
  return -1;
}

int refh_knn(int type, int method, int list_kind, int k, const void *tree, int n,
             const void *bounds, const void *queries, long nq, float cutoff, int *out_ids,
             float *out_d2, float *out_ret, int nthreads)
{
#define L(kind, kk)                                                                     \
  if (list_kind == kind && k == kk) {                                                   \
    knn_host<DT, TT, typename ListOf<kind, kk>::type>(method, tree, n, bounds, queries, \
                                                      nq, cutoff, out_ids, out_d2,      \
                                                      out_ret, nthreads);               \
    return 0;                                                                           \
  }
#define X(code, D, T, P)  \
  if (type == code) {     \
    using DT = D;         \
    using TT = T;         \
    REFO_LISTS(L)         \
    return -2;            \
  }
  REFO_TYPES(X)
#undef X
#undef L
  return -1;
}

int refh_spatial_fcp(int type, int method, const void *nodes, const void *primIDs,
                     const void *data, int numPrims, int numNodes, const void *bounds,
                     const void *queries, long nq, float cutoff, int *out_ids, int nthreads)
{
#define X(code, D, T, P)                                                                \
  if (type == code) {                                                                   \
    spatial_fcp_host<D, T>(method, nodes, primIDs, data, numPrims, numNodes, bounds,    \
                           queries, nq, cutoff, out_ids, nthreads);                     \
    return 0;                                                                           \
  }
  REFO_TYPES(X)
#undef X
  return -1;
}

int refh_spatial_knn(int type, int method, int list_kind, int k, const void *nodes,
                     const void *primIDs, const void *data, int numPrims, int numNodes,
                     const void *bounds, const void *queries, long nq, float cutoff,
                     int *out_ids, float *out_d2, int nthreads)
{
#define L(kind, kk)                                                                        \
  if (list_kind == kind && k == kk) {                                                      \
    spatial_knn_host<DT, TT, typename ListOf<kind, kk>::type>(                             \
        method, nodes, primIDs, data, numPrims, numNodes, bounds, queries, nq, cutoff,     \
        out_ids, out_d2, nthreads);                                                        \
    return 0;                                                                              \
  }
#define X(code, D, T, P)  \
  if (type == code) {     \
    using DT = D;         \
    using TT = T;         \
    REFO_LISTS(L)         \
    return -2;            \
  }
  REFO_TYPES(X)
#undef X
#undef L
  return -1;
}

}  // extern "C"
