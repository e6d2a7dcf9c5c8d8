// cukd/helpers.h -- drop-in shim: memory resources and implicit-tree helpers
// (reference cukd/helpers.h:30-100).
#pragma once

#include "cukd/common.h"
#include "cukd_b200.h"

namespace cukd {

// Where builders take temporary (and spatial trees their persistent) device
// memory from; the library calls back into it through cukd_mem_resource.
struct GpuMemoryResource {
  virtual cudaError_t malloc(void **ptr, size_t size, cudaStream_t s) = 0;
  virtual cudaError_t free(void *ptr, cudaStream_t s) = 0;
  virtual ~GpuMemoryResource() {}
};

struct ManagedMemMemoryResource : public GpuMemoryResource {
  cudaError_t malloc(void **ptr, size_t size, cudaStream_t s) override
  {
    cudaStreamSynchronize(s);
    return cudaMallocManaged(ptr, size);
  }
  cudaError_t free(void *ptr, cudaStream_t s) override
  {
    cudaStreamSynchronize(s);
    return cudaFree(ptr);
  }
};

struct AsyncGpuMemoryResource final : GpuMemoryResource {
  cudaError_t malloc(void **ptr, size_t size, cudaStream_t s) override
  {
    return cudaMallocAsync(ptr, size, s);
  }
  cudaError_t free(void *ptr, cudaStream_t s) override { return cudaFreeAsync(ptr, s); }
};

inline GpuMemoryResource &defaultGpuMemResource()
{
  static AsyncGpuMemoryResource memResource;
  return memResource;
}

namespace detail {
inline int mr_alloc(void *ctx, void **ptr, size_t bytes, cudaStream_t s)
{
  return ((GpuMemoryResource *)ctx)->malloc(ptr, bytes, s) == cudaSuccess ? 0 : 1;
}
inline int mr_release(void *ctx, void *ptr, cudaStream_t s)
{
  return ((GpuMemoryResource *)ctx)->free(ptr, s) == cudaSuccess ? 0 : 1;
}
// C-ABI view of a GpuMemoryResource
inline cukd_mem_resource as_c(GpuMemoryResource &mr)
{
  cukd_mem_resource c;
  c.ctx = &mr;
  c.alloc = mr_alloc;
  c.release = mr_release;
  return c;
}
// status -> exception, like the reference's error paths
inline void check(int status, const char *what)
{
  if (status == CUKD_OK) return;
  std::string msg = std::string(what) + ": " + cukd_status_string(status);
  if (status == CUKD_ERR_CUDA) msg += std::string(" (") + cukd_last_cuda_error() + ")";
  throw std::runtime_error(msg);
}
}  // namespace detail

// implicit binary tree of nodes 0..N-1, children of i at 2i+1 and 2i+2
struct BinaryTree {
  static inline __both__ int rootNode() { return 0; }
  static inline __both__ int parentOf(int node) { return (node - 1) / 2; }
  static inline __both__ int isLeftSibling(int node) { return node & 1; }
  static inline __both__ int leftChildOf(int node) { return 2 * node + 1; }
  static inline __both__ int rightChildOf(int node) { return 2 * node + 2; }
  static inline __both__ int firstNodeInLevel(int L) { return (1 << L) - 1; }
  static inline __both__ int levelOf(int node)
  {
#ifdef __CUDA_ARCH__
    return 63 - __clzll((long long)node + 1);
#else
    return 63 - __builtin_clzll((unsigned long long)node + 1);
#endif
  }
  static inline __both__ int numLevelsFor(int numPoints) { return levelOf(numPoints - 1) + 1; }
};

}  // namespace cukd
