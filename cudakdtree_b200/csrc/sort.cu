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

// exclusive scan of one digit's column of per-tile counts (one CTA per
// digit, counts stored digit-major); the column total goes to digitTotals
__global__ void __launch_bounds__(kThreads) column_scan_kernel(uint32_t *counts, int numTiles,
                                                               uint32_t *digitTotals)
{
  __shared__ uint32_t warpSums[kThreads / 32];
  __shared__ uint32_t carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t *col = counts + int64_t(blockIdx.x) * numTiles;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  constexpr int PER = 4;
  for (int off = 0; off < numTiles; off += kThreads * PER) {
    uint32_t v[PER], s = 0;
    const int b = off + threadIdx.x * PER;
#pragma unroll
    for (int j = 0; j < PER; j++) {
      v[j] = b + j < numTiles ? col[b + j] : 0u;
      s += v[j];
    }
    uint32_t incl = s;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) warpSums[wid] = incl;
    __syncthreads();
    uint32_t wbase = 0, tot = 0;
    for (int w = 0; w < kThreads / 32; w++) {
      const uint32_t x = warpSums[w];
      wbase += w < wid ? x : 0u;
      tot += x;
    }
    uint32_t run = carry + wbase + incl - s;
#pragma unroll
    for (int j = 0; j < PER; j++) {
      if (b + j < numTiles) col[b + j] = run;
      run += v[j];
    }
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) digitTotals[blockIdx.x] = carry;
}

__global__ void __launch_bounds__(kThreads) scatter_kernel(
    const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, int64_t n, int shift,
    int numTiles, const uint32_t *__restrict__ offsets, const uint32_t *__restrict__ digitTotals,
    uint32_t *__restrict__ keysOut, uint32_t *__restrict__ valsOut)
{
  constexpr int W = kThreads / 32;
  __shared__ uint32_t running[256];
  __shared__ uint32_t wcnt[W][256];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  {
    // exclusive prefix of the 256 digit totals (computed by every CTA)
    const uint32_t t = digitTotals[threadIdx.x];
    uint32_t incl = t;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t u = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += u;
    }
    if (lane == 31) wcnt[0][wid] = incl;
    __syncthreads();
    uint32_t wbase = 0;
    for (int w = 0; w < wid; w++) wbase += wcnt[0][w];
    running[threadIdx.x] = offsets[int64_t(threadIdx.x) * numTiles + blockIdx.x] + wbase + incl - t;
    __syncthreads();
  }
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

int64_t radix_sort_counts(int64_t n) { return (std::max<int64_t>(1, div_up(n, kTileItems)) + 1) * 256; }

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
  uint32_t *totals = counts + int64_t(numTiles) * 256;  // 256 digit totals
  uint32_t *ka = keys, *va = vals, *kb = keys2, *vb = vals2;
  int passes = 0;
  for (int shift = 0; shift < bits; shift += 8, passes++) {
    upsweep_kernel<<<numTiles, kThreads, 0, st>>>(ka, n, shift, numTiles, counts);
    CKB_CHECK_LAUNCH();
    column_scan_kernel<<<256, kThreads, 0, st>>>(counts, numTiles, totals);
    CKB_CHECK_LAUNCH();
    scatter_kernel<<<numTiles, kThreads, 0, st>>>(ka, va, n, shift, numTiles, counts, totals, kb,
                                                  vb);
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
