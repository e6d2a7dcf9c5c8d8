// cukd/builder.h -- drop-in shim of the reference's builders
// (cukd/builder.h:108-152, builder_thrust.h:90-118, builder_bitonic.h:83-94,
// builder_inplace.h:82-102) on top of libcukd_b200.so.
//
// Same template signatures and defaults; the tree is built on the GPU by
// cukd_build_tree.  Plain point arrays (float2/3/4, int2/3/4 with default
// traits) are passed straight to the C ABI.  Any other data_traits is served
// generically: the points are packed with the traits into a record the ABI
// can describe ({point; input index; dim}), the tree is built over those
// records, and the caller's structs are gathered into node order (and their
// dims written through data_traits::set_dim) by kernels instantiated in the
// caller's translation unit.  Errors throw std::runtime_error like the
// reference.
#pragma once

#include <stddef.h>

#include <type_traits>
#include <vector>

#include "cukd/data.h"
#include "cukd/helpers.h"

namespace cukd {
namespace detail {

template <typename point_t> struct ShimRecord {
  point_t p;
  uint32_t idx;
  int32_t dim;
};

template <typename point_t> inline cukd_layout layout_of(int stride, int dim_offset)
{
  using S = typename point_traits<point_t>::scalar_t;
  static_assert(point_traits<point_t>::num_dims >= 2 && point_traits<point_t>::num_dims <= 8,
                "cukd-b200 builds trees over 2 to 8 dimensions");
  static_assert(std::is_same<S, float>::value || std::is_same<S, int>::value,
                "cukd-b200 builds trees over float or int coordinates");
  cukd_layout l;
  l.scalar_type = std::is_same<S, float>::value ? CUKD_FLOAT32 : CUKD_INT32;
  l.num_dims = point_traits<point_t>::num_dims;
  l.stride = stride;
  l.point_offset = 0;
  l.dim_offset = dim_offset;
  l.dim_shift = 0;
  l.dim_bits = 32;
  return l;
}

template <typename data_t, typename traits>
__global__ void shim_pack(const data_t *in, int n, ShimRecord<typename traits::point_t> *rec,
                          data_t *copy)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const data_t d = in[i];
  copy[i] = d;
  rec[i].p = traits::get_point(d);
  rec[i].idx = uint32_t(i);
  rec[i].dim = 0;
}

template <typename data_t, typename traits>
__global__ void shim_unpack(const data_t *copy, const ShimRecord<typename traits::point_t> *rec,
                            int n, data_t *out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  data_t d = copy[rec[i].idx];
  if constexpr (bool(traits::has_explicit_dim)) traits::set_dim(d, rec[i].dim);
  out[i] = d;
}

template <typename data_t, typename traits>
void build(data_t *d_points, int numPoints, box_t<typename traits::point_t> *worldBounds,
           cudaStream_t stream, GpuMemoryResource &mr, int builder, const char *name)
{
  using point_t = typename traits::point_t;
  if (numPoints < 1) return;
  if (traits::has_explicit_dim && !worldBounds)
    throw std::runtime_error(std::string("cukd::") + name +
                             ": asked to build k-d tree over nodes with explicit dims, but no "
                             "memory for world bounds provided");
  cukd_mem_resource c = as_c(mr);
  const bool plain = std::is_same<data_t, point_t>::value && !traits::has_explicit_dim &&
                     std::is_same<traits, default_data_traits<data_t>>::value;
  if (plain) {
    const cukd_layout l = layout_of<point_t>(int(sizeof(data_t)), -1);
    check(cukd_build_tree(d_points, numPoints, &l, worldBounds, builder, stream, &c), name);
    // like the reference's builders, return after the work is done and
    // throw if it failed (a bounded device-side wait that gave up)
    check(cukd_build_check(stream), name);
    return;
  }
  ShimRecord<point_t> *rec = nullptr;
  data_t *copy = nullptr;
  if (mr.malloc((void **)&rec, sizeof(*rec) * size_t(numPoints), stream) != cudaSuccess ||
      mr.malloc((void **)&copy, sizeof(data_t) * size_t(numPoints), stream) != cudaSuccess)
    throw std::runtime_error(std::string("cukd::") + name + ": out of device memory");
  const int bs = 256, nb = divRoundUp(numPoints, bs);
  shim_pack<data_t, traits><<<nb, bs, 0, stream>>>(d_points, numPoints, rec, copy);
  CUKD_CUDA_CHECK(cudaGetLastError());
  const cukd_layout l =
      layout_of<point_t>(int(sizeof(*rec)),
                         traits::has_explicit_dim ? int(offsetof(ShimRecord<point_t>, dim)) : -1);
  const int rc = cukd_build_tree(rec, numPoints, &l, worldBounds, builder, stream, &c);
  if (rc == CUKD_OK) {
    shim_unpack<data_t, traits><<<nb, bs, 0, stream>>>(copy, rec, numPoints, d_points);
    CUKD_CUDA_CHECK(cudaGetLastError());
  }
  mr.free(rec, stream);
  mr.free(copy, stream);
  check(rc, name);
  check(cukd_build_check(stream), name);
}

}  // namespace detail

template <typename data_t, typename data_traits = default_data_traits<data_t>>
void buildTree(data_t *d_points, int numPoints,
               box_t<typename data_traits::point_t> *worldBounds = 0, cudaStream_t stream = 0,
               GpuMemoryResource &memResource = defaultGpuMemResource())
{
  detail::build<data_t, data_traits>(d_points, numPoints, worldBounds, stream, memResource,
                                     CUKD_BUILDER_DEFAULT, "buildTree");
}

template <typename data_t, typename data_traits = default_data_traits<data_t>>
void buildTree_thrust(data_t *d_points, int numPoints,
                      box_t<typename data_traits::point_t> *worldBounds = 0,
                      cudaStream_t stream = 0,
                      GpuMemoryResource &memResource = defaultGpuMemResource())
{
  detail::build<data_t, data_traits>(d_points, numPoints, worldBounds, stream, memResource,
                                     CUKD_BUILDER_THRUST, "buildTree_thrust");
}

template <typename data_t, typename data_traits = default_data_traits<data_t>>
void buildTree_bitonic(data_t *d_points, int numPoints,
                       box_t<typename data_traits::point_t> *worldBounds = 0,
                       cudaStream_t stream = 0,
                       GpuMemoryResource &memResource = defaultGpuMemResource())
{
  detail::build<data_t, data_traits>(d_points, numPoints, worldBounds, stream, memResource,
                                     CUKD_BUILDER_BITONIC, "buildTree_bitonic");
}

template <typename data_t, typename data_traits = default_data_traits<data_t>>
void buildTree_inPlace(data_t *d_points, int numPoints,
                       box_t<typename data_traits::point_t> *worldBounds = 0,
                       cudaStream_t stream = 0,
                       GpuMemoryResource &memResource = defaultGpuMemResource())
{
  detail::build<data_t, data_traits>(d_points, numPoints, worldBounds, stream, memResource,
                                     CUKD_BUILDER_INPLACE, "buildTree_inPlace");
}

// Builds over host memory (the reference's buildTree_host runs on the CPU;
// here the points are copied to the GPU, built there, and copied back --
// the result is the same array).
template <typename data_t, typename data_traits = default_data_traits<data_t>>
void buildTree_host(data_t *points, int numPoints,
                    box_t<typename data_traits::point_t> *worldBounds = 0)
{
  using box = box_t<typename data_traits::point_t>;
  if (numPoints < 1) return;
  data_t *d = nullptr;
  box *db = nullptr;
  CUKD_CUDA_CHECK(cudaMalloc(&d, sizeof(data_t) * size_t(numPoints)));
  CUKD_CUDA_CHECK(cudaMalloc(&db, sizeof(box)));
  CUKD_CUDA_CHECK(cudaMemcpy(d, points, sizeof(data_t) * size_t(numPoints),
                             cudaMemcpyHostToDevice));
  buildTree<data_t, data_traits>(d, numPoints, db);
  CUKD_CUDA_CHECK(cudaMemcpy(points, d, sizeof(data_t) * size_t(numPoints),
                             cudaMemcpyDeviceToHost));
  if (worldBounds) CUKD_CUDA_CHECK(cudaMemcpy(worldBounds, db, sizeof(box), cudaMemcpyDeviceToHost));
  cudaFree(d);
  cudaFree(db);
}

// World bounds of the records (their point must be the record's first member).
template <typename data_t, typename data_traits = default_data_traits<data_t>>
void computeBounds(box_t<typename data_traits::point_t> *d_bounds, const data_t *d_points,
                   int numPoints, cudaStream_t stream = 0)
{
  using point_t = typename data_traits::point_t;
  const cukd_layout l = detail::layout_of<point_t>(int(sizeof(data_t)), -1);
  detail::check(cukd_compute_bounds(d_points, numPoints, &l, d_bounds, stream), "computeBounds");
}

}  // namespace cukd
