// Stable LSD radix sort, 8 bits per pass: per-tile digit histograms, one
// exclusive scan over (digit, tile), and a scatter that ranks equal digits
// in index order with warp match/ballot so every pass is stable.
#include <algorithm>

#include "sort.cuh"

namespace ckb {
namespace {

constexpr int kThreads = 256;
constexpr int kItems = 16;
constexpr int kTileItems = kThreads * kItems;

__global__ void __launch_bounds__(kThreads) upsweep_kernel(const uint32_t *__restrict__ keys,
                                                           int64_t n, int shift, int numTiles,
                                                           uint32_t *counts)
{
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = int64_t(blockIdx.x) * kTileItems;
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const int64_t i = base + j * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  counts[int64_t(threadIdx.x) * numTiles + blockIdx.x] = h[threadIdx.x];
}

// single-CTA exclusive scan of `len` counts
__global__ void __launch_bounds__(1024) scan_kernel(uint32_t *counts, int64_t len)
{
  __shared__ uint32_t warpSums[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int64_t off = 0; off < len; off += 1024) {
    const int64_t i = off + threadIdx.x;
    const uint32_t v = i < len ? counts[i] : 0u;
    uint32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warpSums[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      const uint32_t s = warpSums[lane];
      uint32_t si = s;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, si, o);
        if (lane >= o) si += t;
      }
      warpSums[lane] = si - s;
    }
    __syncthreads();
    const uint32_t c = carry;
    if (i < len) counts[i] = c + warpSums[wid] + incl - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry = c + warpSums[wid] + incl;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kThreads) scatter_kernel(
    const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, int64_t n, int shift,
    int numTiles, const uint32_t *__restrict__ offsets, uint32_t *__restrict__ keysOut,
    uint32_t *__restrict__ valsOut)
{
  constexpr int W = kThreads / 32;
  __shared__ uint32_t running[256];
  __shared__ uint32_t wcnt[W][256];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  running[threadIdx.x] = offsets[int64_t(threadIdx.x) * numTiles + blockIdx.x];
  for (int w = 0; w < W; w++) wcnt[w][threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = int64_t(blockIdx.x) * kTileItems;
  const uint32_t ltMask = (1u << lane) - 1u;
  for (int j = 0; j < kItems; j++) {
    const int64_t i = base + j * kThreads + threadIdx.x;
    const bool valid = i < n;
    const uint32_t k = valid ? keys[i] : 0u;
    const uint32_t v = valid ? vals[i] : 0u;
    const uint32_t digit = valid ? ((k >> shift) & 255u) : 256u + lane;
    const uint32_t peers = __match_any_sync(0xffffffffu, digit);
    const uint32_t rank = __popc(peers & ltMask);
    if (valid && rank == 0) wcnt[wid][digit] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t pre = 0;
      for (int w = 0; w < wid; w++) pre += wcnt[w][digit];
      const uint32_t pos = running[digit] + pre + rank;
      keysOut[pos] = k;
      valsOut[pos] = v;
    }
    __syncthreads();
    {
      uint32_t tot = 0;
      for (int w = 0; w < W; w++) {
        tot += wcnt[w][threadIdx.x];
        wcnt[w][threadIdx.x] = 0;
      }
      running[threadIdx.x] += tot;
    }
    __syncthreads();
  }
}

}  // namespace

int64_t radix_sort_counts(int64_t n) { return std::max<int64_t>(1, div_up(n, kTileItems)) * 256; }

int radix_sort_pairs(uint32_t *keys, uint32_t *vals, uint32_t *keys2, uint32_t *vals2,
                     int64_t n, int bits, cudaStream_t st, TempArena *arena)
{
  if (n <= 1 || bits <= 0) return CUKD_OK;
  uint32_t *counts = nullptr;
  CKB_TRY(arena->alloc(&counts, size_t(radix_sort_counts(n))));
  return radix_sort_pairs_ws(keys, vals, keys2, vals2, n, bits, counts, st);
}

int radix_sort_pairs_ws(uint32_t *keys, uint32_t *vals, uint32_t *keys2, uint32_t *vals2,
                        int64_t n, int bits, uint32_t *counts, cudaStream_t st)
{
  if (n <= 1 || bits <= 0) return CUKD_OK;
  const int numTiles = int(div_up(n, kTileItems));
  uint32_t *ka = keys, *va = vals, *kb = keys2, *vb = vals2;
  int passes = 0;
  for (int shift = 0; shift < bits; shift += 8, passes++) {
    upsweep_kernel<<<numTiles, kThreads, 0, st>>>(ka, n, shift, numTiles, counts);
    CKB_CHECK_LAUNCH();
    scan_kernel<<<1, 1024, 0, st>>>(counts, int64_t(numTiles) * 256);
    CKB_CHECK_LAUNCH();
    scatter_kernel<<<numTiles, kThreads, 0, st>>>(ka, va, n, shift, numTiles, counts, kb, vb);
    CKB_CHECK_LAUNCH();
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    CKB_CUDA(cudaMemcpyAsync(keys, ka, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
    CKB_CUDA(cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st));
  }
  return CUKD_OK;
}

}  // namespace ckb
