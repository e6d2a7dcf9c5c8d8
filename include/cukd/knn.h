// cukd/knn.h -- drop-in shim: k-nearest-neighbour queries for user kernels
// (reference cukd/knn.h:27-755).  Candidate lists keep keys
// (float bits of d2) << 32 | id, so equal distances order by lower id;
// unfilled slots hold (cutOffRadius^2, -1).  FixedCandidateList<k> is a sorted
// register list, HeapCandidateList<k> a max-heap, FlexHeapCandidateList a
// runtime-k heap over caller memory that can resume from a stored heap
// (radius < 0).  knn() returns maxRadius2().
#pragma once

#include <string.h>

#include "cukd/fcp.h"

namespace cukd {

struct BaseCandidateList {
 protected:
  static inline __both__ uint32_t f2u(float f)
  {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    memcpy(&u, &f, 4);
    return u;
#endif
  }
  static inline __both__ float u2f(uint32_t u)
  {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    memcpy(&f, &u, 4);
    return f;
#endif
  }
  static inline __both__ uint64_t encode(float d2, int id)
  {
    return (uint64_t(f2u(d2)) << 32) | uint32_t(id);
  }
  static inline __both__ float decode_dist2(uint64_t v) { return u2f(uint32_t(v >> 32)); }
  static inline __both__ int decode_pointID(uint64_t v) { return int(uint32_t(v)); }
};

template <int k> struct CandidateList : public BaseCandidateList {
  inline __both__ float get_dist2(int i) const { return decode_dist2(entry[i]); }
  inline __both__ int get_pointID(int i) const { return decode_pointID(entry[i]); }
  uint64_t entry[k];
  enum { num_k = k };
};

template <int k> struct FixedCandidateList : public CandidateList<k> {
  using CandidateList<k>::entry;
  inline __both__ FixedCandidateList(float cutOffRadius)
  {
    for (int i = 0; i < k; i++) entry[i] = this->encode(cutOffRadius * cutOffRadius, -1);
  }
  inline __both__ float maxRadius2() const { return this->decode_dist2(entry[k - 1]); }
  inline __both__ float returnValue() const { return maxRadius2(); }
  inline __both__ float initialCullDist2() const { return maxRadius2(); }
  inline __both__ void push(float dist, int pointID)
  {
    uint64_t v = this->encode(dist, pointID);
    for (int i = 0; i < k; i++) {
      const uint64_t lo = entry[i] < v ? entry[i] : v;
      const uint64_t hi = entry[i] < v ? v : entry[i];
      entry[i] = lo;
      v = hi;
    }
  }
  inline __both__ float processCandidate(int candPrimID, float candDist2)
  {
    push(candDist2, candPrimID);
    return maxRadius2();
  }
};

namespace detail {
// sift-down insert of `e` into a max-heap of k keys (root = largest)
inline __both__ void heap_insert(uint64_t *entry, int k, uint64_t e)
{
  if (e >= entry[0]) return;
  int pos = 0;
  for (;;) {
    const int c1 = 2 * pos + 1, c2 = c1 + 1;
    int largest = k;
    uint64_t lv = e;
    if (c1 < k) {
      largest = c1;
      lv = entry[c1];
    }
    if (c2 < k && entry[c2] > lv) {
      largest = c2;
      lv = entry[c2];
    }
    if (largest == k || lv < e) {
      entry[pos] = e;
      return;
    }
    entry[pos] = lv;
    pos = largest;
  }
}
}  // namespace detail

template <int k> struct HeapCandidateList : public CandidateList<k> {
  using CandidateList<k>::entry;
  inline __both__ HeapCandidateList(float cutOffRadius)
  {
    for (int i = 0; i < k; i++) entry[i] = this->encode(cutOffRadius * cutOffRadius, -1);
  }
  inline __both__ float maxRadius2() const { return this->decode_dist2(entry[0]); }
  inline __both__ float returnValue() const { return maxRadius2(); }
  inline __both__ float initialCullDist2() const { return maxRadius2(); }
  inline __both__ void push(float dist, int pointID)
  {
    detail::heap_insert(entry, k, this->encode(dist, pointID));
  }
  inline __both__ float processCandidate(int candPrimID, float candDist2)
  {
    push(candDist2, candPrimID);
    return maxRadius2();
  }
};

struct FlexHeapCandidateList : public BaseCandidateList {
  inline __both__ FlexHeapCandidateList(uint64_t *entryMem, int k, float cutOffRadius)
      : entry(entryMem), k(k)
  {
    if (cutOffRadius >= 0.f)
      for (int i = 0; i < k; i++) entry[i] = encode(cutOffRadius * cutOffRadius, -1);
  }
  inline __both__ float maxRadius2() const { return decode_dist2(entry[0]); }
  inline __both__ float returnValue() const { return maxRadius2(); }
  inline __both__ float initialCullDist2() const { return maxRadius2(); }
  inline __both__ void push(float dist, int pointID)
  {
    detail::heap_insert(entry, k, encode(dist, pointID));
  }
  inline __both__ float processCandidate(int candPrimID, float candDist2)
  {
    push(candDist2, candPrimID);
    return maxRadius2();
  }
  inline __both__ float get_dist2(int i) const { return decode_dist2(entry[i]); }
  inline __both__ int get_pointID(int i) const { return decode_pointID(entry[i]); }
  uint64_t *const entry;
  int const k;
};

#define CUKD_SHIM_KNN(NS, TRAVERSE_CALL)                                                     \
  namespace NS {                                                                            \
  template <typename CandidateList, typename data_t,                                        \
            typename data_traits = default_data_traits<data_t>>                             \
  inline __both__ float knn(CandidateList &result, typename data_traits::point_t queryPoint, \
                            const box_t<typename data_traits::point_t> worldBounds,         \
                            const data_t *d_nodes, int N)                                   \
  {                                                                                         \
    TRAVERSE_CALL;                                                                          \
    return result.returnValue();                                                            \
  }                                                                                         \
  }

CUKD_SHIM_KNN(stackBased, (traverse_default<CandidateList, data_t, data_traits>(result, queryPoint, d_nodes, N)))
CUKD_SHIM_KNN(stackFree, (traverse_stack_free<CandidateList, data_t, data_traits>(result, queryPoint, d_nodes, N)))
CUKD_SHIM_KNN(cct, (traverse_cct<CandidateList, data_t, data_traits>(result, queryPoint, worldBounds, d_nodes, N)))
#undef CUKD_SHIM_KNN

namespace stackBased {
template <typename CandidateList, typename data_t,
          typename data_traits = default_data_traits<data_t>>
inline __both__ float knn(CandidateList &result, typename data_traits::point_t queryPoint,
                          const data_t *d_nodes, int N)
{
  traverse_default<CandidateList, data_t, data_traits>(result, queryPoint, d_nodes, N);
  return result.returnValue();
}
}  // namespace stackBased
namespace stackFree {
template <typename CandidateList, typename data_t,
          typename data_traits = default_data_traits<data_t>>
inline __both__ float knn(CandidateList &result, typename data_traits::point_t queryPoint,
                          const data_t *d_nodes, int N)
{
  traverse_stack_free<CandidateList, data_t, data_traits>(result, queryPoint, d_nodes, N);
  return result.returnValue();
}
}  // namespace stackFree

}  // namespace cukd
