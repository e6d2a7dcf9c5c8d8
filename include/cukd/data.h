// cukd/data.h -- drop-in shim: default_data_traits (reference cukd/data.h:56-112).
// A data_traits describes a record type to the library: its point type, how
// to read the point and a coordinate, and -- with has_explicit_dim -- how to
// read and write a per-node split dimension.
#pragma once

#include "cukd/box.h"

namespace cukd {

template <typename _point_t, typename _point_traits = point_traits<_point_t>>
struct default_data_traits {
  using point_t = _point_t;
  using point_traits = _point_traits;
  using data_t = _point_t;
  using scalar_t = typename _point_traits::scalar_t;
  static inline __both__ const point_t &get_point(const data_t &n) { return n; }
  static inline __both__ scalar_t get_coord(const data_t &n, int d)
  {
    return point_traits::get_coord(get_point(n), d);
  }
  enum { has_explicit_dim = false };
  static inline __both__ int get_dim(const data_t &) { return -1; }
  static inline __both__ void set_dim(data_t &, int) {}
};

}  // namespace cukd
