// cukd/box.h -- drop-in shim: box_t<point_t> (reference cukd/box.h:35-125).
#pragma once

#include <float.h>

#include "cukd/cukd-math.h"

namespace cukd {

template <typename T> inline __both__ T empty_box_lower();
template <typename T> inline __both__ T empty_box_upper();
template <> inline __both__ float empty_box_lower<float>() { return +INFINITY; }
template <> inline __both__ float empty_box_upper<float>() { return -INFINITY; }
template <> inline __both__ int empty_box_lower<int>() { return INT_MAX; }
template <> inline __both__ int empty_box_upper<int>() { return INT_MIN; }

template <typename point_t> struct box_t {
  using traits = point_traits<point_t>;
  using scalar_t = typename traits::scalar_t;
  enum { num_dims = traits::num_dims };
  point_t lower, upper;

  // widest extent; equal extents resolve to the higher dimension
  inline __both__ int widestDimension() const
  {
    int best = 0;
    scalar_t wbest = scalar_t(0);
    for (int d = 0; d < num_dims; d++) {
      const scalar_t w = traits::get_coord(upper, d) - traits::get_coord(lower, d);
      if (w < wbest) continue;
      wbest = w;
      best = d;
    }
    return best;
  }
  inline __both__ bool contains(const point_t &p) const
  {
    for (int d = 0; d < num_dims; d++) {
      if (traits::get_coord(p, d) < traits::get_coord(lower, d)) return false;
      if (traits::get_coord(p, d) > traits::get_coord(upper, d)) return false;
    }
    return true;
  }
  inline __both__ void grow(const point_t &p)
  {
    for (int d = 0; d < num_dims; d++) {
      const scalar_t v = traits::get_coord(p, d);
      if (v < traits::get_coord(lower, d)) traits::set_coord(lower, d, v);
      if (traits::get_coord(upper, d) < v) traits::set_coord(upper, d, v);
    }
  }
  inline __both__ void setEmpty()
  {
    for (int d = 0; d < num_dims; d++) {
      traits::set_coord(lower, d, empty_box_lower<scalar_t>());
      traits::set_coord(upper, d, empty_box_upper<scalar_t>());
    }
  }
  inline __both__ void setInfinite()
  {
    for (int d = 0; d < num_dims; d++) {
      traits::set_coord(lower, d, empty_box_upper<scalar_t>());
      traits::set_coord(upper, d, empty_box_lower<scalar_t>());
    }
  }
};

// closest point of the box to `point` (min(max(point, lower), upper))
template <typename point_t>
inline __both__ point_t project(const box_t<point_t> &box, const point_t &point)
{
  using traits = point_traits<point_t>;
  point_t r = point;
  for (int d = 0; d < traits::num_dims; d++) {
    auto v = traits::get_coord(point, d);
    const auto lo = traits::get_coord(box.lower, d), hi = traits::get_coord(box.upper, d);
    v = v < lo ? lo : v;
    v = hi < v ? hi : v;
    traits::set_coord(r, d, v);
  }
  return r;
}

template <typename point_t>
inline __both__ auto sqrDistance(const box_t<point_t> &box, const point_t &point)
{
  return sqrDistance(project(box, point), point);
}

}  // namespace cukd
