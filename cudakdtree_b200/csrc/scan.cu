#include <algorithm>

#include "scan.cuh"

namespace ckb {
namespace {

constexpr int kT = 256;
constexpr int kPer = 16;
constexpr int kTile = kT * kPer;

__device__ inline uint32_t block_excl_scan(uint32_t v, uint32_t *warpSums, uint32_t *total)
{
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warpSums[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    const uint32_t s = lane < kT / 32 ? warpSums[lane] : 0u;
    uint32_t si = s;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += t;
    }
    if (lane < kT / 32) warpSums[lane] = si - s;
    if (lane == kT / 32 - 1) *total = si;
  }
  __syncthreads();
  return warpSums[wid] + incl - v;
}

__global__ void __launch_bounds__(kT) tile_sums(const uint32_t *__restrict__ in, int64_t n,
                                                uint32_t *sums)
{
  __shared__ uint32_t ws[kT / 32];
  __shared__ uint32_t tot;
  const int64_t base = int64_t(blockIdx.x) * kTile + int64_t(threadIdx.x) * kPer;
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kPer; j++)
    if (base + j < n) s += in[base + j];
  block_excl_scan(s, ws, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// single block scans the tile sums (count <= 65536 * kTile elements total)
__global__ void __launch_bounds__(1024) scan_sums(uint32_t *sums, int64_t m, uint32_t *total)
{
  __shared__ uint32_t ws[32];
  __shared__ uint32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int64_t off = 0; off < m; off += 1024) {
    const int64_t i = off + threadIdx.x;
    const uint32_t v = i < m ? sums[i] : 0u;
    uint32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) ws[wid] = incl;
    __syncthreads();
    if (wid == 0) {
      const uint32_t s = ws[lane];
      uint32_t si = s;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, si, o);
        if (lane >= o) si += t;
      }
      ws[lane] = si - s;
    }
    __syncthreads();
    const uint32_t c = carry;
    if (i < m) sums[i] = c + ws[wid] + incl - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry = c + ws[wid] + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void __launch_bounds__(kT) tile_scan(const uint32_t *in, uint32_t *out, int64_t n,
                                                const uint32_t *__restrict__ sums)
{
  __shared__ uint32_t ws[kT / 32];
  __shared__ uint32_t tot;
  const int64_t base = int64_t(blockIdx.x) * kTile + int64_t(threadIdx.x) * kPer;
  uint32_t v[kPer];
  uint32_t s = 0;
#pragma unroll
  for (int j = 0; j < kPer; j++) {
    v[j] = base + j < n ? in[base + j] : 0u;
    s += v[j];
  }
  uint32_t run = block_excl_scan(s, ws, &tot) + sums[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kPer; j++) {
    if (base + j < n) out[base + j] = run;
    run += v[j];
  }
}

}  // namespace

int exclusive_scan_u32(const uint32_t *in, uint32_t *out, int64_t n, uint32_t *total,
                       cudaStream_t st, TempArena *arena)
{
  if (n <= 0) {
    if (total) CKB_CUDA(cudaMemsetAsync(total, 0, sizeof(uint32_t), st));
    return CUKD_OK;
  }
  const int64_t tiles = div_up(n, kTile);
  uint32_t *sums = nullptr;
  CKB_TRY(arena->alloc(&sums, tiles));
  tile_sums<<<unsigned(tiles), kT, 0, st>>>(in, n, sums);
  CKB_CHECK_LAUNCH();
  scan_sums<<<1, 1024, 0, st>>>(sums, tiles, total);
  CKB_CHECK_LAUNCH();
  tile_scan<<<unsigned(tiles), kT, 0, st>>>(in, out, n, sums);
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

}  // namespace ckb
