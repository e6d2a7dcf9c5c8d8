// cukd/cukd-math.h -- drop-in shim (point types and their traits).
// Same names and semantics as the reference's cukd/cukd-math.h:
// scalar_type_of / num_dims_of / get_coord / set_coord for float2/3/4 and
// int2/3/4, vec_float<N>, point_traits<T>, and float vector operators with
// sqrDistance = dot(a-b, a-b) summed left to right.
#pragma once

#include "cukd/common.h"

namespace cukd {

#ifdef __CUDA_ARCH__
using ::max;
using ::min;
#else
using std::max;
using std::min;
#endif

template <typename T> struct scalar_type_of;
template <> struct scalar_type_of<float2> { using type = float; };
template <> struct scalar_type_of<float3> { using type = float; };
template <> struct scalar_type_of<float4> { using type = float; };
template <> struct scalar_type_of<int2> { using type = int; };
template <> struct scalar_type_of<int3> { using type = int; };
template <> struct scalar_type_of<int4> { using type = int; };

template <typename T> struct num_dims_of;
template <> struct num_dims_of<float2> { enum { value = 2 }; };
template <> struct num_dims_of<float3> { enum { value = 3 }; };
template <> struct num_dims_of<float4> { enum { value = 4 }; };
template <> struct num_dims_of<int2> { enum { value = 2 }; };
template <> struct num_dims_of<int3> { enum { value = 3 }; };
template <> struct num_dims_of<int4> { enum { value = 4 }; };

// coordinate d of a CUDA vector type
#define CUKD_SHIM_COORDS(V, S)                                                          \
  inline __both__ S get_coord(const V &v, int d) { return d == 0 ? v.x : v.y; }        \
  inline __both__ S &get_coord(V &v, int d) { return d == 0 ? v.x : v.y; }             \
  inline __both__ void set_coord(V &v, int d, S s) { (d == 0 ? v.x : v.y) = s; }
#define CUKD_SHIM_COORDS3(V, S)                                                         \
  inline __both__ S get_coord(const V &v, int d) { return d == 0 ? v.x : (d == 1 ? v.y : v.z); } \
  inline __both__ S &get_coord(V &v, int d) { return d == 0 ? v.x : (d == 1 ? v.y : v.z); }      \
  inline __both__ void set_coord(V &v, int d, S s) { (d == 0 ? v.x : (d == 1 ? v.y : v.z)) = s; }
#define CUKD_SHIM_COORDS4(V, S)                                                         \
  inline __both__ S get_coord(const V &v, int d)                                       \
  { return d == 0 ? v.x : (d == 1 ? v.y : (d == 2 ? v.z : v.w)); }                     \
  inline __both__ S &get_coord(V &v, int d)                                            \
  { return d == 0 ? v.x : (d == 1 ? v.y : (d == 2 ? v.z : v.w)); }                     \
  inline __both__ void set_coord(V &v, int d, S s)                                     \
  { (d == 0 ? v.x : (d == 1 ? v.y : (d == 2 ? v.z : v.w))) = s; }
CUKD_SHIM_COORDS(float2, float)
CUKD_SHIM_COORDS3(float3, float)
CUKD_SHIM_COORDS4(float4, float)
CUKD_SHIM_COORDS(int2, int)
CUKD_SHIM_COORDS3(int3, int)
CUKD_SHIM_COORDS4(int4, int)
#undef CUKD_SHIM_COORDS
#undef CUKD_SHIM_COORDS3
#undef CUKD_SHIM_COORDS4

template <int N> struct vec_float { float v[N]; };
template <int N> struct scalar_type_of<vec_float<N>> { using type = float; };
template <int N> struct num_dims_of<vec_float<N>> { enum { value = N }; };
template <int N> inline __both__ float get_coord(const vec_float<N> &v, int d) { return v.v[d]; }
template <int N> inline __both__ float &get_coord(vec_float<N> &v, int d) { return v.v[d]; }
template <int N> inline __both__ void set_coord(vec_float<N> &v, int d, float s) { v.v[d] = s; }

// traits of a point type: scalar type, dimension, coordinate access
template <typename point_t> struct point_traits {
  enum { num_dims = num_dims_of<point_t>::value };
  using scalar_t = typename scalar_type_of<point_t>::type;
  static inline __both__ scalar_t get_coord(const point_t &p, int d) { return cukd::get_coord(p, d); }
  static inline __both__ void set_coord(point_t &p, int d, scalar_t s) { cukd::set_coord(p, d, s); }
};

template <typename S> inline __host__ __device__ auto sqr(S s) { return s * s; }

// squared distance, ((d0*d0 + d1*d1) + d2*d2) + ..., no FMA contraction
template <typename point_t>
inline __both__ typename scalar_type_of<point_t>::type sqrDistance(const point_t &a,
                                                                   const point_t &b)
{
  using S = typename scalar_type_of<point_t>::type;
  enum { D = num_dims_of<point_t>::value };
#ifdef __CUDA_ARCH__
  S s = 0;
  for (int d = 0; d < D; d++) {
    const S diff = get_coord(a, d) - get_coord(b, d);
    s = __fadd_rn(s, __fmul_rn(diff, diff));
  }
  return s;
#else
  volatile S s = 0;
  for (int d = 0; d < D; d++) {
    volatile S diff = get_coord(a, d) - get_coord(b, d);
    volatile S sq = diff * diff;
    s = s + sq;
  }
  return s;
#endif
}

template <typename point_t> inline __both__ auto distance(const point_t &a, const point_t &b)
{
  return sqrtf(sqrDistance(a, b));
}

}  // namespace cukd
