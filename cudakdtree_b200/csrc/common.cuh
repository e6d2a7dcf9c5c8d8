// Shared device/host helpers of the B200 k-d tree library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <vector>

#include "cukd_b200.h"

namespace ckb {

// ---------------------------------------------------------------------------
// status plumbing
// ---------------------------------------------------------------------------
void set_cuda_error(cudaError_t e);
// number of kernels this library has launched (reported by the benchmark)
void count_launch();
// adjusts the count: + kernels a replayed CUDA graph launched, - kernels
// that were only recorded into a graph
void add_launches(long long d);
unsigned long long launch_count();

#define CKB_CHECK_LAUNCH()                           \
  do {                                               \
    ::ckb::count_launch();                           \
    cudaError_t _e = cudaGetLastError();             \
    if (_e != cudaSuccess) {                         \
      ::ckb::set_cuda_error(_e);                     \
      return CUKD_ERR_CUDA;                          \
    }                                                \
  } while (0)

#define CKB_CUDA(call)                               \
  do {                                               \
    cudaError_t _e = (call);                         \
    if (_e != cudaSuccess) {                         \
      ::ckb::set_cuda_error(_e);                     \
      return CUKD_ERR_CUDA;                          \
    }                                                \
  } while (0)

#define CKB_TRY(expr)                                \
  do {                                               \
    int _s = (expr);                                 \
    if (_s != CUKD_OK) return _s;                    \
  } while (0)

// ---------------------------------------------------------------------------
// stream-ordered temporaries through the caller's memory resource
// (reference: GpuMemoryResource, cukd/helpers.h:30-70)
// ---------------------------------------------------------------------------
// Keeps memory freed by cudaFreeAsync in the current device's default pool
// (by default the pool returns it to the driver at every synchronisation,
// and the next build would map it again).  Per process and device.
void keep_default_pool_memory();

struct TempArena {
  cudaStream_t stream;
  const cukd_mem_resource *mem;
  cudaMemPool_t pool;  // without a caller's resource: this pool, else the device's default
  std::vector<void *> ptrs;
  TempArena(cudaStream_t s, const cukd_mem_resource *m, cudaMemPool_t p = nullptr)
      : stream(s), mem(m), pool(p)
  {
    if (!mem || !mem->alloc) keep_default_pool_memory();
  }
  ~TempArena() { release_all(); }
  template <typename T>
  int alloc(T **out, size_t count)
  {
    void *p = nullptr;
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    bytes = (bytes + 255) & ~size_t(255);
    void *use = nullptr;
    if (mem && mem->alloc) {
      // the builder's bulk copies need 16-byte-aligned arrays, and a caller's
      // pool may hand out less: ask for 16 bytes more and align up (the
      // block's own pointer is what goes back to the pool)
      if (mem->alloc(mem->ctx, &p, bytes + 16, stream) != 0 || !p) return CUKD_ERR_OUT_OF_MEMORY;
      use = reinterpret_cast<void *>((reinterpret_cast<uintptr_t>(p) + 15u) & ~uintptr_t(15));
    } else {
      cudaError_t e =
          pool ? cudaMallocFromPoolAsync(&p, bytes, pool, stream) : cudaMallocAsync(&p, bytes, stream);
      if (e != cudaSuccess) {
        cudaGetLastError();
        return e == cudaErrorMemoryAllocation ? CUKD_ERR_OUT_OF_MEMORY : CUKD_ERR_CUDA;
      }
      use = p;
    }
    ptrs.push_back(p);
    *out = (T *)use;
    return CUKD_OK;
  }
  void release_all()
  {
    for (void *p : ptrs) {
      if (mem && mem->release)
        mem->release(mem->ctx, p, stream);
      else
        cudaFreeAsync(p, stream);
    }
    ptrs.clear();
  }
};

// ---------------------------------------------------------------------------
// order-preserving 32-bit keys of coordinates
// ---------------------------------------------------------------------------
// float: IEEE total order on non-NaN values with -0.0 folded onto +0.0, so
// that keys compare exactly like the reference's `coord_a < coord_b`.
__host__ __device__ inline uint32_t float_key(float f)
{
#ifdef __CUDA_ARCH__
  uint32_t u = __float_as_uint(f);
#else
  uint32_t u;
  memcpy(&u, &f, 4);
#endif
  if ((u << 1) == 0) u = 0;
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ inline float key_float(uint32_t k)
{
  uint32_t u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
#ifdef __CUDA_ARCH__
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}
__host__ __device__ inline uint32_t int_key(int32_t i) { return uint32_t(i) ^ 0x80000000u; }
__host__ __device__ inline int32_t key_int(uint32_t k) { return int32_t(k ^ 0x80000000u); }

// ---------------------------------------------------------------------------
// implicit left-balanced tree geometry (same quantities as the reference's
// BinaryTree / ArbitraryBinaryTree / ArrayLayoutInStep, helpers.h:75-257,
// computed in closed form with 64-bit arithmetic)
// ---------------------------------------------------------------------------
__host__ __device__ inline int level_of(int64_t node)
{
#ifdef __CUDA_ARCH__
  return 63 - __clzll((long long)(node + 1));
#else
  return 63 - __builtin_clzll((unsigned long long)(node + 1));
#endif
}
__host__ __device__ inline int num_levels(int64_t n) { return n < 1 ? 0 : level_of(n - 1) + 1; }

// nodes in the subtree under `g` (0 if g >= n)
__host__ __device__ inline int64_t subtree_size(int64_t g, int64_t n)
{
  if (g >= n) return 0;
  const int L = num_levels(n);
  const int h = L - level_of(g);  // levels of the full subtree under g
  const int64_t lastCap = int64_t(1) << (h - 1);
  const int64_t firstLast = ((g + 1) << (h - 1)) - 1;
  int64_t onLast = n - firstLast;
  onLast = onLast < 0 ? 0 : (onLast > lastCap ? lastCap : onLast);
  return (lastCap - 1) + onLast;
}
__host__ __device__ inline int64_t left_size(int64_t g, int64_t n)
{
  return subtree_size(2 * g + 1, n);
}
// Offset of level-`lvl` subtree `g` when the not-yet-settled points are
// stored subtree after subtree in node order (this library's working
// layout: pivots of levels < lvl removed).
__host__ __device__ inline int64_t seg_begin(int64_t g, int lvl, int64_t n)
{
  const int L = num_levels(n);
  const int h = L - lvl;
  const int64_t t = g - ((int64_t(1) << lvl) - 1);
  const int64_t lastCap = int64_t(1) << (h - 1);
  const int64_t M = n - ((int64_t(1) << (L - 1)) - 1);  // nodes on the last level
  int64_t onLastBefore = t * lastCap;
  if (onLastBefore > M) onLastBefore = M;
  return t * (lastCap - 1) + onLastBefore;
}

// ---------------------------------------------------------------------------
// record access
// ---------------------------------------------------------------------------
// points of up to 8 dims (the reference's vec_float<N>, cukd-math.h:133-181,
// tested up to N = 8 in testing/testBuildersSameResult.cu:404-428) build with
// every builder and answer through the reference-order traversals; the fast
// kNN, learned, spatial, batched, Morton and allocation-free paths take up
// to 4
constexpr int kMaxDims = 8;
constexpr int kMaxFastDims = 4;

struct Layout {
  int scalar, D, stride, poff, doff, dshift;
  uint32_t dmask;
};
inline bool make_layout(const cukd_layout *l, Layout *out)
{
  if (!l) return false;
  if (l->scalar_type != CUKD_FLOAT32 && l->scalar_type != CUKD_INT32) return false;
  if (l->num_dims < 2 || l->num_dims > kMaxDims) return false;
  if (l->stride <= 0 || (l->stride & 3) || (l->point_offset & 3) || l->point_offset < 0) return false;
  if (l->point_offset + 4 * l->num_dims > l->stride) return false;
  out->scalar = l->scalar_type;
  out->D = l->num_dims;
  out->stride = l->stride;
  out->poff = l->point_offset;
  out->doff = l->dim_offset;
  out->dshift = 0;
  out->dmask = 0;
  if (l->dim_offset >= 0) {
    if ((l->dim_offset & 3) || l->dim_offset + 4 > l->stride) return false;
    if (l->dim_bits < 1 || l->dim_bits > 32 || l->dim_shift < 0 ||
        l->dim_shift + l->dim_bits > 32)
      return false;
    if (l->dim_bits < 32 && (1u << l->dim_bits) < (uint32_t)l->num_dims) return false;
    out->dshift = l->dim_shift;
    out->dmask = l->dim_bits == 32 ? 0xffffffffu : ((1u << l->dim_bits) - 1u);
  }
  return true;
}

inline int64_t div_up(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Largest tree the traversals accept: their node indices are 32-bit ints (as
// the reference's are), and a node's children 2i+1, 2i+2 must fit one.
constexpr int64_t kMaxQueryTree = (int64_t(1) << 30) - 1;

constexpr int kNumSMs = 148;

}  // namespace ckb
