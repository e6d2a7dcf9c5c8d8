// cukd/common.h -- drop-in shim of ingowald/cudaKDTree's cukd/common.h for
// the cukd-b200 library (libcukd_b200.so, C ABI in cukd_b200.h).
// Only what user code of the reference relies on is provided: the __both__
// qualifier, divRoundUp, the CUDA error macros (common.h:276-342 of the
// reference throw std::runtime_error / exit on a CUDA error) and the point
// file loader loadPoints (common.h:245-267).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <limits.h>

#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>

#ifndef __both__
#define __both__ __host__ __device__
#endif

#define CUKD_CUDA_CHECK(call)                                                      \
  do {                                                                             \
    cudaError_t rc_ = call;                                                        \
    if (rc_ != cudaSuccess) {                                                      \
      std::stringstream ss_;                                                       \
      ss_ << "CUDA call (" << #call << ") failed: " << cudaGetErrorString(rc_);    \
      throw std::runtime_error(ss_.str());                                         \
    }                                                                              \
  } while (0)
#define CUKD_CUDA_CALL(call) CUKD_CUDA_CHECK(cuda##call)
#define CUKD_CUDA_SYNC_CHECK() CUKD_CUDA_CHECK(cudaDeviceSynchronize())

namespace cukd {

inline __both__ int32_t divRoundUp(int32_t a, int32_t b) { return (a + b - 1) / b; }
inline __both__ uint32_t divRoundUp(uint32_t a, uint32_t b) { return (a + b - 1) / b; }
inline __both__ int64_t divRoundUp(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline __both__ uint64_t divRoundUp(uint64_t a, uint64_t b) { return (a + b - 1) / b; }

// Reads a point file -- a uint64 record count followed by the raw records --
// into CUDA managed memory (release with cudaFree), as the reference's
// loader does; throws std::runtime_error when the file is missing or short.
template <typename T>
inline T *loadPoints(std::string fileName, size_t &count)
{
  std::ifstream in(fileName, std::ios::binary);
  uint64_t n = 0;
  if (!in.read(reinterpret_cast<char *>(&n), sizeof(n)))
    throw std::runtime_error("loadPoints: cannot read the record count of " + fileName);
  T *points = nullptr;
  CUKD_CUDA_CHECK(cudaMallocManaged(reinterpret_cast<void **>(&points), (n ? n : 1) * sizeof(T)));
  if (!in.read(reinterpret_cast<char *>(points), std::streamsize(n * sizeof(T)))) {
    cudaFree(points);
    throw std::runtime_error("loadPoints: " + fileName + " holds fewer records than its count");
  }
  count = size_t(n);
  return points;
}

template <typename T>
inline T *loadPoints(std::string fileName, int &count)
{
  size_t n = 0;
  T *points = loadPoints<T>(fileName, n);
  count = int(n);
  return points;
}

}  // namespace cukd
