// Data types and traits used to drive the UNMODIFIED reference library
// (ingowald/cudaKDTree headers, included from where they lie) as the
// test oracle.  This file is test infrastructure: it is compiled only into
// oracle/_ref/*.so, never into the product library.
//
// The layouts here are the same byte layouts that the product library's
// C-ABI describes with `cukd_layout` (include/cukd_b200.h):
//   type code 0..2   float2/3/4, round-robin split dims
//                    (reference: cukd/data.h:56-112 default_data_traits)
//   type code 3..5   {floatN p; int dim;} explicit split dim
//                    (reference pattern: testing/floatN-knn-and-fcp.cu:42-60)
//   type code 6      {float3 p; int payload;}  round-robin, payload carried
//                    (reference pattern: testing/testPayloadSampleFromReadme.cu)
//   type code 7      {float3 p; uint32 payload;} dim packed in payload bits
//                    30..31, index in bits 0..29 (16-byte record)
#pragma once

#include "cukd/builder.h"
#include "cukd/spatial-kdtree.h"
#include "cukd/fcp.h"
#include "cukd/knn.h"

namespace refo {

template <typename P>
struct PointDim {
  P p;
  int dim;
};

template <typename P>
struct PointDim_traits : public cukd::default_data_traits<P> {
  using point_t = P;
  using data_t = PointDim<P>;
  enum { has_explicit_dim = true };
  static inline __host__ __device__ const P &get_point(const data_t &n) { return n.p; }
  static inline __host__ __device__ float get_coord(const data_t &n, int d)
  { return cukd::get_coord(n.p, d); }
  static inline __host__ __device__ int get_dim(const data_t &n) { return n.dim; }
  static inline __host__ __device__ void set_dim(data_t &n, int d) { n.dim = d; }
};

struct PointPayload {
  float3 p;
  int payload;
};

struct PointPayload_traits : public cukd::default_data_traits<float3> {
  using point_t = float3;
  using data_t = PointPayload;
  static inline __host__ __device__ const float3 &get_point(const data_t &n) { return n.p; }
  static inline __host__ __device__ float get_coord(const data_t &n, int d)
  { return cukd::get_coord(n.p, d); }
  // never called (has_explicit_dim is false) but the traversals name them
  static inline __host__ __device__ int get_dim(const data_t &) { return -1; }
  static inline __host__ __device__ void set_dim(data_t &, int) {}
};

struct PointPacked {
  float3 p;
  uint32_t payload;
};

struct PointPacked_traits : public cukd::default_data_traits<float3> {
  using point_t = float3;
  using data_t = PointPacked;
  enum { has_explicit_dim = true };
  static inline __host__ __device__ const float3 &get_point(const data_t &n) { return n.p; }
  static inline __host__ __device__ float get_coord(const data_t &n, int d)
  { return cukd::get_coord(n.p, d); }
  static inline __host__ __device__ int get_dim(const data_t &n) { return int(n.payload >> 30); }
  static inline __host__ __device__ void set_dim(data_t &n, int d)
  { n.payload = (n.payload & 0x3fffffffu) | (uint32_t(d) << 30); }
};

}  // namespace refo

// X-macro over the type matrix: (code, data_t, traits, point_t)
#define REFO_TYPES(X)                                                        \
  X(0, float2, cukd::default_data_traits<float2>, float2)                    \
  X(1, float3, cukd::default_data_traits<float3>, float3)                    \
  X(2, float4, cukd::default_data_traits<float4>, float4)                    \
  X(3, refo::PointDim<float2>, refo::PointDim_traits<float2>, float2)        \
  X(4, refo::PointDim<float3>, refo::PointDim_traits<float3>, float3)        \
  X(5, refo::PointDim<float4>, refo::PointDim_traits<float4>, float4)        \
  X(6, refo::PointPayload, refo::PointPayload_traits, float3)                \
  X(7, refo::PointPacked, refo::PointPacked_traits, float3)

// candidate lists: (list kind 0 = FixedCandidateList, 1 = HeapCandidateList, k)
#define REFO_LISTS(X)                                                        \
  X(0, 1) X(0, 4) X(0, 8) X(0, 16) X(0, 32) X(0, 64)                         \
  X(1, 4) X(1, 8) X(1, 16) X(1, 20) X(1, 32) X(1, 50) X(1, 64)

namespace refo {
template <int kind, int k> struct ListOf;
template <int k> struct ListOf<0, k> { using type = cukd::FixedCandidateList<k>; };
template <int k> struct ListOf<1, k> { using type = cukd::HeapCandidateList<k>; };
}  // namespace refo
