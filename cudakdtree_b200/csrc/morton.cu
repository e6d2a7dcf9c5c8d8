// Morton (Z-order) query reordering and the stable LSD radix sort it uses.
//
// The reference has no query reordering: callers launch one thread per
// query in input order (sample.cu:49-74).  Sorting queries along a Morton
// curve makes the 32 traversals of a warp walk nearly the same tree path,
// which cuts divergence and raises L1/L2 hit rates.  It never changes a
// result: every query is still answered by its own traversal, and the
// answers are scattered back to the caller's order.
#include <algorithm>

#include "common.cuh"
#include "sort.cuh"

namespace ckb {

namespace {

__device__ inline uint32_t expand_bits(uint32_t v, int D)
{
  // spread the low bits of v so that consecutive bits land D apart
  uint32_t r = 0;
  const int bits = 30 / D;
  for (int b = 0; b < bits; b++) r |= ((v >> b) & 1u) << (b * D);
  return r;
}

__global__ void query_bounds_kernel(const float *__restrict__ pts, int64_t n, int D,
                                    uint32_t *kmin, uint32_t *kmax)
{
  uint32_t lo[4] = {~0u, ~0u, ~0u, ~0u}, hi[4] = {0, 0, 0, 0};
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    for (int d = 0; d < D; d++) {
      const uint32_t k = float_key(pts[i * D + d]);
      lo[d] = min(lo[d], k);
      hi[d] = max(hi[d], k);
    }
  }
  for (int d = 0; d < D; d++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = min(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = max(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
    if ((threadIdx.x & 31) == 0 && lo[d] <= hi[d]) {
      atomicMin(&kmin[d], lo[d]);
      atomicMax(&kmax[d], hi[d]);
    }
  }
}

__global__ void morton_code_kernel(const float *__restrict__ pts, int64_t n, int D,
                                   const uint32_t *kmin, const uint32_t *kmax,
                                   const float *bounds, uint32_t *codes, uint32_t *vals)
{
  const int bits = 30 / D;
  const float cells = float(1u << bits);
  float lo[4], scale[4];
  for (int d = 0; d < D; d++) {
    const float l = bounds ? bounds[d] : key_float(kmin[d]);
    const float h = bounds ? bounds[D + d] : key_float(kmax[d]);
    lo[d] = l;
    scale[d] = h > l ? cells / (h - l) : 0.f;
  }
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    uint32_t code = 0;
    for (int d = 0; d < D; d++) {
      const float x = (pts[i * D + d] - lo[d]) * scale[d];
      const uint32_t c = x >= 0.f ? (x < cells ? uint32_t(x) : (1u << bits) - 1u) : 0u;
      code |= expand_bits(c, D) << (D - 1 - d);
    }
    codes[i] = code;
    vals[i] = uint32_t(i);
  }
}

}  // namespace

int morton_order_impl(const float *pts, int64_t n, int D, const float *bounds, int32_t *perm,
                      cudaStream_t st, const cukd_mem_resource *mem)
{
  if (n <= 0) return CUKD_OK;
  if (D < 1 || D > 4) return CUKD_ERR_INVALID_ARGUMENT;
  TempArena arena(st, mem);
  uint32_t *codes = nullptr, *codes2 = nullptr, *vals2 = nullptr, *kb = nullptr;
  CKB_TRY(arena.alloc(&codes, n));
  CKB_TRY(arena.alloc(&codes2, n));
  CKB_TRY(arena.alloc(&vals2, n));
  CKB_TRY(arena.alloc(&kb, 8));
  const int blocks = int(std::max<int64_t>(1, std::min<int64_t>(div_up(n, 256), kNumSMs * 8)));
  if (!bounds) {
    CKB_CUDA(cudaMemsetAsync(kb, 0xff, 16, st));
    CKB_CUDA(cudaMemsetAsync(kb + 4, 0, 16, st));
    query_bounds_kernel<<<blocks, 256, 0, st>>>(pts, n, D, kb, kb + 4);
    CKB_CHECK_LAUNCH();
  }
  morton_code_kernel<<<blocks, 256, 0, st>>>(pts, n, D, kb, kb + 4, bounds, codes,
                                             (uint32_t *)perm);
  CKB_CHECK_LAUNCH();
  const int bits = (30 / D) * D;
  return radix_sort_pairs(codes, (uint32_t *)perm, codes2, vals2, n, bits, st, &arena);
}

}  // namespace ckb

extern "C" int cukd_morton_order(const float *d_points, int64_t n, int num_dims,
                                 const float *d_bounds, int32_t *d_out_perm,
                                 cudaStream_t stream, const cukd_mem_resource *mem)
{
  if (n < 0 || (n > 0 && (!d_points || !d_out_perm))) return CUKD_ERR_INVALID_ARGUMENT;
  return ckb::morton_order_impl(d_points, n, num_dims, d_bounds, d_out_perm, stream, mem);
}
