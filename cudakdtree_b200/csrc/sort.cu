// Stable LSD radix sort, 8 bits per pass: per-tile digit histograms, one
// exclusive scan over (digit, tile), and a scatter that ranks equal digits
// in index order with warp match so every pass is stable.
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

// One tile of kTileItems keys per CTA.  Warp w owns the tile's positions
// [w * 512, (w + 1) * 512), lane l its items w * 512 + 32 j + l (j < 16), so
// ranking the items of a digit in (warp, j, lane) order is index order: the
// pass is stable.  Each item's rank among its warp's items of that digit
// comes from match_any over the rounds; digit-major offsets over the warps
// and over the digits place it in the tile; the tile is staged in shared
// memory in digit order and written out in that order, so the writes of a
// digit's run from this tile are consecutive addresses.  (The earlier form
// ranked 256 items at a time with three barriers each and wrote straight
// to global memory: 180 us a pass over 10M keys in a cold ncu replay.)
__global__ void __launch_bounds__(kThreads, 3) scatter_kernel(
    const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, int64_t n, int shift,
    int numTiles, const uint32_t *__restrict__ offsets, const uint32_t *__restrict__ digitTotals,
    uint32_t *__restrict__ keysOut, uint32_t *__restrict__ valsOut)
{
  constexpr int W = kThreads / 32;
  constexpr int kWarpItems = kTileItems / W;
  static_assert(kWarpItems == 32 * kItems, "a warp's items: kItems rounds of 32");
  static_assert(kThreads == 256, "a thread per digit");
  __shared__ uint32_t sk[kTileItems], sv[kTileItems];
  __shared__ uint16_t wh[W][256];     // per warp and digit: count, then exclusive offset
  __shared__ uint32_t tileStart[256];  // a digit's first position in the tile
  __shared__ uint32_t outBase[256];    // a digit's first output position from this tile
  __shared__ uint32_t red[2][W];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int64_t base = int64_t(blockIdx.x) * kTileItems;
  const int64_t wbase = base + int64_t(wid) * kWarpItems;
  for (int i = tid; i < W * 256; i += kThreads) (&wh[0][0])[i] = 0;
  // this warp's items in the tile: positions below lim are in the input
  const int64_t rem = n - wbase;
  const int lim = rem <= 0 ? 0 : (rem < kWarpItems ? int(rem) : kWarpItems);
  const uint32_t *kw = keys + wbase, *vw = vals + wbase;
  uint32_t k[kItems], v[kItems];
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const int i = j * 32 + lane;
    k[j] = i < lim ? kw[i] : 0u;
    v[j] = i < lim ? vw[i] : 0u;
  }
  __syncthreads();
  const uint32_t ltMask = (1u << lane) - 1u;
  uint32_t r[kItems / 2];  // ranks (< 512), two per word
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    const bool valid = j * 32 + lane < lim;
    const uint32_t d = valid ? (k[j] >> shift) & 255u : 256u + lane;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t below = __popc(peers & ltMask);
    const uint32_t cnt = valid ? uint32_t(wh[wid][d]) : 0u;
    __syncwarp();  // every lane has read the count before its leader adds
    if (valid && below == 0) wh[wid][d] = uint16_t(cnt + __popc(peers));
    __syncwarp();
    if (j & 1)
      r[j >> 1] |= (cnt + below) << 16;
    else
      r[j >> 1] = cnt + below;
  }
  __syncthreads();
  {
    // thread tid owns digit tid: the warps' exclusive offsets (digit-major),
    // then exclusive scans over the digits of the tile's counts and of the
    // digit totals of the whole pass
    const int d = tid;
    uint32_t run = 0;
#pragma unroll
    for (int w = 0; w < W; w++) {
      const uint32_t c = wh[w][d];
      wh[w][d] = uint16_t(run);
      run += c;
    }
    const uint32_t tot = digitTotals[d];
    uint32_t a = run, b = tot;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t ta = __shfl_up_sync(0xffffffffu, a, o);
      const uint32_t tb = __shfl_up_sync(0xffffffffu, b, o);
      if (lane >= o) {
        a += ta;
        b += tb;
      }
    }
    if (lane == 31) {
      red[0][wid] = a;
      red[1][wid] = b;
    }
    __syncthreads();
    uint32_t pa = 0, pb = 0;
    for (int w = 0; w < wid; w++) {
      pa += red[0][w];
      pb += red[1][w];
    }
    tileStart[d] = pa + a - run;
    outBase[d] = offsets[int64_t(d) * numTiles + blockIdx.x] + pb + b - tot;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kItems; j++) {
    if (j * 32 + lane < lim) {
      const uint32_t d = (k[j] >> shift) & 255u;
      const uint32_t p = tileStart[d] + wh[wid][d] + ((r[j >> 1] >> (16 * (j & 1))) & 0xffffu);
      sk[p] = k[j];
      sv[p] = v[j];
    }
  }
  __syncthreads();
  const int m = n - base < kTileItems ? int(n - base) : kTileItems;
  for (int p = tid; p < m; p += kThreads) {
    const uint32_t key = sk[p];
    const uint32_t d = (key >> shift) & 255u;
    const uint32_t g = outBase[d] + uint32_t(p) - tileStart[d];
    keysOut[g] = key;
    valsOut[g] = sv[p];
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
