// Left-balanced k-d tree builder for sm_100a.
//
// The reference (cukd/builder_thrust.h:414-512) runs, for every tree level,
// a full stable sort of (subtree tag, split coordinate) over all N points
// and then retags (:222-235, :321-345).  Because every sort is stable, the
// points of the subtree under node g (level l) are ordered by the
// composite key
//     (c[dim(g)], c[dim(parent)], c[dim(grandparent)], ..., input index)
// (a dim already listed is skipped), and the point of rank leftSize(g)
// (helpers.h:237-252) becomes node g.  This builder computes the same tree
// by SELECTION on that composite key instead of L full sorts:
//
//  global phase -- levels whose subtrees hold more than kTile points; all
//  subtrees of a level are processed by the same launches:
//    hist_kernel      histogram of the split coordinate into equal-width
//                     bins over the subtree's data range
//    select_kernel    the bin holding rank leftSize(g) (a warp or a CTA per
//                     subtree)
//    partition_kernel points of lower bins -> left child's segment, higher
//                     bins -> right child's segment, the pivot bin's points
//                     -> candidate buffer; grows the children's data bounds
//    resolve_kernel   MSD radix select over the composite key among the
//                     candidates; settles the pivot, appends the other
//                     candidates to the children, derives the children's
//                     domain boxes and split dims (widest extent of the
//                     domain box, box.h:112-125, builder_thrust.h:238-306)
//    Once a level's subtrees fit one staged chunk (kFusedMax points),
//    level_fused_kernel does all four steps with one CTA per subtree.
//  subtree phase -- one CTA per subtree of <= kTile points, all remaining
//    levels in shared memory: one index list per dimension is sorted once
//    by coordinate; per level the pivot is read from the list of the
//    level's dim at rank leftSize (an equal-coordinate run around it is
//    ranked by the composite key), and all lists are stably partitioned
//    with warp ballots and a block-wide scan of their counts.
//  finalize_kernel -- gathers the caller's records into node order and
//    writes the explicit split dims.
//
// Working data are SoA: one uint32 order-preserving key array per
// dimension plus the input index, ping-ponged between two buffers.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <mutex>
#include <type_traits>
#include <vector>

#include "async.cuh"
#include "common.cuh"
#include "forest.cuh"
#include "subtree.cuh"

namespace ckb {

unsigned long long launch_count();
static thread_local cudaError_t g_last_cuda = cudaSuccess;
void set_cuda_error(cudaError_t e) { g_last_cuda = e; }
static std::atomic<unsigned long long> g_launches{0};
void keep_default_pool_memory()
{
  static thread_local int doneMask[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return;
  }
  const int slot = dev & 7, bit = 1 << ((dev >> 3) & 31);
  if (doneMask[slot] & bit) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  cudaGetLastError();
  doneMask[slot] |= bit;
}
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void add_launches(long long d) { g_launches.fetch_add((unsigned long long)d, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(); }
const char *last_cuda_error_string() { return cudaGetErrorString(g_last_cuda); }

namespace build {

constexpr int kChunk = kLevelChunk;  // points per CTA in hist / partition
constexpr int kGThreads = 256;
constexpr int kMaxBins = 4096;
// partition staging: elements per array (a chunk plus 16-byte alignment slack)
constexpr int kStageSpan = kChunk + 8;
// partition chunks per hist_kernel CTA: fewer CTAs merge fewer bin counts
// into the global histogram with atomics (10M-point build: 1 -> 5.27 ms,
// 4 -> 5.14 ms, 8 -> 5.23 ms)
constexpr int kHistGroup = 4;
// levels with at most this many subtrees resolve with 1024-thread CTAs
// (10M-point build 5.13 -> 5.06 ms)
constexpr int kWideResolveSegs = 16;
// global levels whose largest subtree holds at most this many points run
// level_fused_kernel (10M-point build: 5.61 -> 5.43 ms)
constexpr int64_t kFusedMax = kChunk;
constexpr uint32_t kWaitPolls = 1u << 22;  // bound of a bulk-copy barrier wait
static_assert(kWaitPolls == CUKD_ASYNC_WAIT_POLLS_DEFAULT, "documented default");
// bulk-copy barrier waits that gave up: never expected (the copies read
// memory the build owns), but a wait that does not complete must end the
// kernel rather than hang it.  The build's status word is then set: every
// later kernel of that build returns at once and the caller's records are
// left as they were; cukd_async_wait_timeouts() reports the count and
// cukd_build_check() turns it into CUKD_ERR_TIMEOUT.
__device__ unsigned int g_wait_timeouts = 0;
// consistency checks of the bounded-memory builders (inplace.cu) that
// failed; cukd_build_check turns a change into CUKD_ERR_INTERNAL
__device__ unsigned int g_build_faults = 0;
// polls of the first (staging) wait; cukd_set_async_wait_polls changes it
// so that a test can make the wait run out (the second wait, which lets the
// copies in flight land before the CTA exits, always uses kWaitPolls)
__device__ uint32_t g_wait_polls = kWaitPolls;
constexpr int kBinPoints = 32;  // target points per histogram bin (global levels)

struct Bufs {
  uint32_t *key[2][kMaxDims];
  uint32_t *idx[2];
  uint32_t *ckey[kMaxDims];
  uint32_t *cidx;
  uint32_t *perm;  // node -> input index
  uint8_t *ndim;   // node -> split dim
  // per-segment arrays: [0] current level, [1] next level
  uint8_t *sdim[2];
  uint32_t *sbmin[2], *sbmax[2];  // data bounds as keys, [seg][D]
  uint32_t *sbox[2];              // domain box as keys, [seg][2D] (lo then hi)
  uint32_t *hist;                 // [seg][nb]
  uint32_t *sel;                  // [seg][3]: pivot bin, count below, pivot-bin count
  uint32_t *cur;                  // [seg][3]: left / right / candidate cursors
  uint32_t *wbmin, *wbmax;        // world bounds as keys, [D]
  uint32_t *status;               // this build's failure flags (0 = fine)
};

// A bulk-copy wait of this build gave up: the CTA-uniform answer (the flag
// can be set by another CTA of the same launch while this one starts).
// Every thread of the block must call it.
__device__ __forceinline__ bool build_failed(const Bufs &b)
{
  __shared__ uint32_t failed;
  if (threadIdx.x == 0) failed = b.status ? *(volatile const uint32_t *)b.status : 0u;
  __syncthreads();
  return failed != 0;
}

// Equal-width binning over a subtree's data range.  Monotone
// non-decreasing in the key, so composite-key order implies bin order.
template <int SC> struct Binner;
template <> struct Binner<0> {
  float lo, scale;
  int nb;
  __device__ Binner(uint32_t klo, uint32_t khi, int nbins) : nb(nbins)
  {
    lo = key_float(klo);
    float span = __fsub_rn(key_float(khi), lo);
    scale = span > 0.f ? __fdiv_rn(float(nbins), span) : 0.f;
  }
  __device__ int operator()(uint32_t k) const
  {
    float x = __fmul_rn(__fsub_rn(key_float(k), lo), scale);
    return x >= 0.f ? (x < float(nb) ? int(x) : nb - 1) : 0;
  }
};
template <> struct Binner<1> {
  uint32_t klo;
  uint64_t span;
  int nb;
  __device__ Binner(uint32_t lo, uint32_t hi, int nbins) : klo(lo), nb(nbins)
  {
    span = hi >= lo ? uint64_t(hi - lo) + 1 : 1;
  }
  __device__ int operator()(uint32_t k) const
  {
    uint32_t off = k >= klo ? k - klo : 0;
    uint64_t b = (uint64_t(off) * uint64_t(nb)) / span;
    return b < uint64_t(nb) ? int(b) : nb - 1;
  }
};


// ---------------------------------------------------------------------------
// extract: records -> SoA keys + input index, copy of the records, bounds
// ---------------------------------------------------------------------------
template <int SC, int D>
__global__ void __launch_bounds__(256) extract_kernel(const uint8_t *__restrict__ pts, int64_t n,
                                                      int stride, int poff,
                                                      uint8_t *__restrict__ orig, Bufs b)
{
  uint32_t lo[D], hi[D];
#pragma unroll
  for (int d = 0; d < D; d++) {
    lo[d] = 0xffffffffu;
    hi[d] = 0u;
  }
  const int words = stride >> 2;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const uint32_t *src = (const uint32_t *)(pts + i * stride);
    uint32_t *dst = (uint32_t *)(orig + i * stride);
    for (int w = 0; w < words; w++) dst[w] = src[w];
    const uint32_t *c = (const uint32_t *)(pts + i * stride + poff);
#pragma unroll
    for (int d = 0; d < D; d++) {
      uint32_t k = Scalar<SC>::key(c[d]);
      b.key[0][d][i] = k;
      lo[d] = min(lo[d], k);
      hi[d] = max(hi[d], k);
    }
    b.idx[0][i] = uint32_t(i);
  }
#pragma unroll
  for (int d = 0; d < D; d++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = min(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = max(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
    if ((threadIdx.x & 31) == 0 && lo[d] <= hi[d]) {
      atomicMin(&b.wbmin[d], lo[d]);
      atomicMax(&b.wbmax[d], hi[d]);
    }
  }
}

// root subtree info and the optional world-bounds output (box_t layout)
template <int SC, int D>
__global__ void root_kernel(Bufs b, void *worldBounds, bool explicitDims)
{
  if (threadIdx.x != 0) return;
  uint32_t *wb = (uint32_t *)worldBounds;
  for (int d = 0; d < D; d++) {
    if (wb) {
      wb[d] = Scalar<SC>::bits(b.wbmin[d]);
      wb[D + d] = Scalar<SC>::bits(b.wbmax[d]);
    }
    b.sbmin[0][d] = b.wbmin[d];
    b.sbmax[0][d] = b.wbmax[d];
    b.sbox[0][d] = b.wbmin[d];
    b.sbox[0][D + d] = b.wbmax[d];
  }
  b.sdim[0][0] = explicitDims ? uint8_t(Scalar<SC>::widest(b.wbmin, b.wbmax, D)) : 0;
}

// ---------------------------------------------------------------------------
// global phase kernels
// ---------------------------------------------------------------------------
struct LevelArgs {
  int64_t n;
  int level;
  int nb;
  int chunksPerSeg;
  int nseg;
  int cb;  // current key buffer
  // forest builds (many trees in one array): per work item its cloud, its
  // subtree's index on the level and its first child's work item in the next
  // level (-1: the children are finished by the subtree phase); per cloud its
  // first record and record count.  Null for a single tree.
  const int32_t *wCloud, *wLocal, *wChild;
  const int64_t *cBase, *cN;
};

// subtree handled by work item w: tree size, node id, the tree's first
// record in the working arrays, and the children's work item
struct SegGeo {
  int64_t n, g, base, child;
};
__device__ inline SegGeo seg_geo(const LevelArgs &a, int w)
{
  SegGeo s;
  if (a.wCloud) {
    const int c = a.wCloud[w];
    s.n = a.cN[c];
    s.base = a.cBase[c];
    s.g = ((int64_t(1) << a.level) - 1) + a.wLocal[w];
    s.child = a.wChild[w];
  } else {
    s.n = a.n;
    s.base = 0;
    s.g = ((int64_t(1) << a.level) - 1) + w;
    s.child = 2 * int64_t(w);
  }
  return s;
}

template <int SC, int D>
__global__ void __launch_bounds__(kGThreads) hist_kernel(Bufs b, LevelArgs a)
{
  if (build_failed(b)) return;
  __shared__ uint32_t sh[kMaxBins];
  const int groups = (a.chunksPerSeg + kHistGroup - 1) / kHistGroup;
  const int seg = blockIdx.x / groups;
  const int grp = blockIdx.x % groups;
  const SegGeo sg = seg_geo(a, seg);
  const int64_t sb = sg.base + seg_begin(sg.g, a.level, sg.n);
  const int64_t sz = subtree_size(sg.g, sg.n);
  const int64_t c0 = int64_t(grp) * kHistGroup * kChunk;
  if (c0 >= sz) return;
  const int64_t c1 = min(sz, c0 + int64_t(kHistGroup) * kChunk);
  for (int i = threadIdx.x; i < a.nb; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const int dim = b.sdim[0][seg];
  const Binner<SC> bin(b.sbmin[0][seg * D + dim], b.sbmax[0][seg * D + dim], a.nb);
  const uint32_t *__restrict__ kd = b.key[a.cb][dim] + sb;
  for (int64_t i = c0 + threadIdx.x; i < c1; i += blockDim.x) atomicAdd(&sh[bin(kd[i])], 1u);
  __syncthreads();
  uint32_t *gh = b.hist + int64_t(seg) * a.nb;
  for (int i = threadIdx.x; i < a.nb; i += blockDim.x)
    if (sh[i]) atomicAdd(&gh[i], sh[i]);
}

// one warp per subtree: the bin that holds rank leftSize(g)
__global__ void select_kernel(Bufs b, LevelArgs a)
{
  if (build_failed(b)) return;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= a.nseg) return;
  const SegGeo sg = seg_geo(a, warp);
  const uint32_t r = uint32_t(left_size(sg.g, sg.n));
  const uint32_t *h = b.hist + int64_t(warp) * a.nb;
  const int per = a.nb / 32;
  uint32_t s = 0;
  for (int i = 0; i < per; i++) s += h[lane * per + i];
  uint32_t incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  const uint32_t excl = incl - s;
  if (r >= excl && r < incl) {
    uint32_t cum = excl;
    for (int i = 0; i < per; i++) {
      uint32_t c = h[lane * per + i];
      if (r < cum + c) {
        b.sel[warp * 3 + 0] = uint32_t(lane * per + i);
        b.sel[warp * 3 + 1] = cum;
        b.sel[warp * 3 + 2] = c;
        break;
      }
      cum += c;
    }
  }
  if (lane < 3) b.cur[warp * 3 + lane] = 0;
}

// the same with one 256-thread CTA per subtree, for levels with >= 512 bins
// (a warp summing 128 bins per lane was latency bound there)
__global__ void __launch_bounds__(256) select_block_kernel(Bufs b, LevelArgs a)
{
  if (build_failed(b)) return;
  __shared__ uint32_t warpSum[8];
  const int seg = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const SegGeo sg = seg_geo(a, seg);
  const uint32_t r = uint32_t(left_size(sg.g, sg.n));
  const uint32_t *h = b.hist + int64_t(seg) * a.nb;
  const int per = a.nb / 256;
  uint32_t s = 0;
  for (int i = 0; i < per; i++) s += h[tid * per + i];
  uint32_t incl = s;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) warpSum[wid] = incl;
  __syncthreads();
  uint32_t wbase = 0;
  for (int w = 0; w < wid; w++) wbase += warpSum[w];
  const uint32_t excl = wbase + incl - s;
  if (r >= excl && r < excl + s) {
    uint32_t cum = excl;
    for (int i = 0; i < per; i++) {
      const uint32_t c = h[tid * per + i];
      if (r < cum + c) {
        b.sel[seg * 3 + 0] = uint32_t(tid * per + i);
        b.sel[seg * 3 + 1] = cum;
        b.sel[seg * 3 + 2] = c;
        break;
      }
      cum += c;
    }
  }
  if (tid < 3) b.cur[seg * 3 + tid] = 0;
}

// warp-reduce per-child bounds and merge them into the next level's arrays
template <int D>
__device__ inline void merge_child_bounds(uint32_t (&lo)[2][D], uint32_t (&hi)[2][D],
                                          uint32_t *bmin, uint32_t *bmax, int64_t childIdx)
{
  if (childIdx < 0) return;  // children finished by the subtree phase
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int d = 0; d < D; d++) {
      uint32_t l = lo[s][d], h = hi[s][d];
      for (int o = 16; o > 0; o >>= 1) {
        l = min(l, __shfl_xor_sync(0xffffffffu, l, o));
        h = max(h, __shfl_xor_sync(0xffffffffu, h, o));
      }
      if ((threadIdx.x & 31) == 0 && l <= h) {
        atomicMin(&bmin[(childIdx + s) * D + d], l);
        atomicMax(&bmax[(childIdx + s) * D + d], h);
      }
    }
}

// The CTA's chunk of keys and indices is staged in shared memory by one bulk
// copy per array (TMA engine, all in flight at once; the partition was
// load-latency bound with per-thread loads).  Each warp owns a contiguous
// run of kChunk / 8 points and walks it 32 at a time; per class (left /
// right / pivot-bin candidate) a ballot ranks the lanes, so every store
// instruction writes one contiguous run per class (the order inside a
// child's segment is irrelevant to the algorithm).
template <int D>
constexpr size_t partition_smem()
{
  return size_t(D + 1) * kStageSpan * sizeof(uint32_t);
}

template <int SC, int D>
__global__ void __launch_bounds__(kGThreads) partition_kernel(Bufs b, LevelArgs a)
{
  if (build_failed(b)) return;
  constexpr int W = kGThreads / 32;
  constexpr int PER_WARP = kChunk / W;
  constexpr int ROUNDS = PER_WARP / 32;
  static_assert(ROUNDS <= 16, "2-bit class codes packed in one uint32");
  extern __shared__ __align__(128) uint32_t stage[];  // [D + 1][kStageSpan]
  __shared__ uint32_t warpTot[W][3];
  __shared__ uint32_t warpBase[W][3];
  __shared__ __align__(8) uint64_t bar;
  const int seg = blockIdx.x / a.chunksPerSeg;
  const int chunk = blockIdx.x % a.chunksPerSeg;
  const SegGeo sg = seg_geo(a, seg);
  const int64_t g = sg.g;
  const int64_t sb = sg.base + seg_begin(g, a.level, sg.n);
  const int64_t sz = subtree_size(g, sg.n);
  const int64_t c0 = int64_t(chunk) * kChunk;
  if (c0 >= sz) return;
  const int64_t c1 = min(sz, c0 + kChunk);
  const int dim = b.sdim[0][seg];
  const Binner<SC> bin(b.sbmin[0][seg * D + dim], b.sbmax[0][seg * D + dim], a.nb);
  const uint32_t pb = b.sel[seg * 3 + 0];
  const int cb = a.cb, nbuf = cb ^ 1;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const uint32_t ltMask = (1u << lane) - 1u;
  const int64_t w0 = c0 + int64_t(wid) * PER_WARP;

  // stage [a0, a1): the chunk with its start rounded down and its end up to
  // 16 bytes (at most 3 extra elements a side, inside the arrays: their
  // allocations are rounded up to 256 bytes)
  const int64_t e0 = sb + c0, e1 = sb + c1;
  const int64_t a0 = e0 & ~int64_t(3), a1 = (e1 + 3) & ~int64_t(3);
  const uint32_t bytes = uint32_t(a1 - a0) * uint32_t(sizeof(uint32_t));
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_arrive_expect_tx(&bar, bytes * uint32_t(D + 1));
#pragma unroll
    for (int d = 0; d < D; d++) bulk_copy_g2s(stage + d * kStageSpan, b.key[cb][d] + a0, bytes, &bar);
    bulk_copy_g2s(stage + D * kStageSpan, b.idx[cb] + a0, bytes, &bar);
  }
  if (!mbar_wait_bounded(&bar, 0, g_wait_polls)) {
    if (threadIdx.x == 0) {
      atomicAdd(&g_wait_timeouts, 1u);
      atomicOr(b.status, 1u);
    }
    mbar_wait_bounded(&bar, 0, kWaitPolls);  // let copies in flight land first
    return;
  }
  // chunk position i (c0 <= i < c1) is staged element i - c0 + so
  const int so = int(e0 - a0);
  const uint32_t *kd = stage + dim * kStageSpan + so;

  // pass 1: class 0 = left, 1 = right, 2 = candidate; per-warp counts
  uint32_t cls = 0;
  uint32_t cnt[3] = {0, 0, 0};
#pragma unroll
  for (int r = 0; r < ROUNDS; r++) {
    const int64_t i = w0 + r * 32 + lane;
    uint32_t c = 3;
    if (i < c1) {
      const uint32_t bb = uint32_t(bin(kd[int(i - c0)]));
      c = bb < pb ? 0u : (bb > pb ? 1u : 2u);
    }
    cls |= (c & 3u) << (2 * r);
#pragma unroll
    for (int x = 0; x < 3; x++) cnt[x] += __popc(__ballot_sync(0xffffffffu, c == uint32_t(x)));
  }
  if (lane < 3) warpTot[wid][lane] = lane == 0 ? cnt[0] : (lane == 1 ? cnt[1] : cnt[2]);
  __syncthreads();
  if (threadIdx.x < 3) {
    const int c = threadIdx.x;
    uint32_t tot = 0;
    for (int w = 0; w < W; w++) {
      warpBase[w][c] = tot;
      tot += warpTot[w][c];
    }
    const uint32_t base = tot ? atomicAdd(&b.cur[seg * 3 + c], tot) : 0u;
    for (int w = 0; w < W; w++) warpBase[w][c] += base;
  }
  __syncthreads();
  uint32_t pos[3];
#pragma unroll
  for (int c = 0; c < 3; c++) pos[c] = warpBase[wid][c];

  const int64_t lchild = 2 * g + 1;
  const int lvlNext = a.level + 1;
  const int64_t lBeg = sg.base + seg_begin(lchild, lvlNext, sg.n);
  const int64_t rBeg = sg.base + seg_begin(lchild + 1, lvlNext, sg.n);
  uint32_t lo[2][D], hi[2][D];
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int d = 0; d < D; d++) {
      lo[s][d] = 0xffffffffu;
      hi[s][d] = 0u;
    }
  // pass 2: reads from the staged chunk, one contiguous write run per class
  // per round.  Class-indexed values are picked with selects so that
  // nothing lands in local memory.
  constexpr int RB = 4;
  static_assert(ROUNDS % RB == 0, "rounds in batches");
  for (int r0 = 0; r0 < ROUNDS; r0 += RB) {
    uint32_t kk[RB][D], idv[RB];
#pragma unroll
    for (int u = 0; u < RB; u++) {
      const int64_t i = w0 + (r0 + u) * 32 + lane;
      const uint32_t c = (cls >> (2 * (r0 + u))) & 3u;
      if (c < 3u) {
#pragma unroll
        for (int d = 0; d < D; d++) kk[u][d] = stage[d * kStageSpan + so + int(i - c0)];
        idv[u] = stage[D * kStageSpan + so + int(i - c0)];
      }
    }
#pragma unroll
    for (int u = 0; u < RB; u++) {
      const uint32_t c = (cls >> (2 * (r0 + u))) & 3u;
      const uint32_t m0 = __ballot_sync(0xffffffffu, c == 0u);
      const uint32_t m1 = __ballot_sync(0xffffffffu, c == 1u);
      const uint32_t m2 = __ballot_sync(0xffffffffu, c == 2u);
      if (c < 3u) {
        const uint32_t mc = c == 0u ? m0 : (c == 1u ? m1 : m2);
        const uint32_t pc = c == 0u ? pos[0] : (c == 1u ? pos[1] : pos[2]);
        const uint32_t rank = pc + __popc(mc & ltMask);
        if (c == 2u) {
          const int64_t dst = sb + rank;
#pragma unroll
          for (int d = 0; d < D; d++) b.ckey[d][dst] = kk[u][d];
          b.cidx[dst] = idv[u];
        } else {
          const int64_t dst = (c == 0u ? lBeg : rBeg) + rank;
#pragma unroll
          for (int d = 0; d < D; d++) b.key[nbuf][d][dst] = kk[u][d];
          b.idx[nbuf][dst] = idv[u];
          if (c == 0u) {
#pragma unroll
            for (int d = 0; d < D; d++) {
              lo[0][d] = min(lo[0][d], kk[u][d]);
              hi[0][d] = max(hi[0][d], kk[u][d]);
            }
          } else {
#pragma unroll
            for (int d = 0; d < D; d++) {
              lo[1][d] = min(lo[1][d], kk[u][d]);
              hi[1][d] = max(hi[1][d], kk[u][d]);
            }
          }
        }
      }
      pos[0] += __popc(m0);
      pos[1] += __popc(m1);
      pos[2] += __popc(m2);
    }
  }
  merge_child_bounds<D>(lo, hi, b.sbmin[1], b.sbmax[1], sg.child);
}

// MSD radix select on the composite key among a subtree's candidates, then
// the candidates' final placement.  One CTA of NT threads per subtree: 1024
// on the top levels, whose few subtrees have thousands of candidates each
// (each pass is a latency-bound loop over them), 256 below.
template <int SC, int D, int NT>
__global__ void __launch_bounds__(NT) resolve_kernel(Bufs b, LevelArgs a, bool explicitDims)
{
  if (build_failed(b)) return;
  __shared__ uint32_t hist[256];
  __shared__ uint32_t sDigit, sCount, sRank, sPivot, sNl, sNr, sLo, sHi;
  __shared__ uint32_t pw[D + 1];
  const int seg = blockIdx.x;
  if (threadIdx.x == 0) {
    sLo = 0xffffffffu;
    sHi = 0u;
  }
  const SegGeo sg = seg_geo(a, seg);
  const int64_t g = sg.g;
  const int64_t sb = sg.base + seg_begin(g, a.level, sg.n);
  const int64_t sz = subtree_size(g, sg.n);
  const uint32_t below = b.sel[seg * 3 + 1];
  const uint32_t m = b.sel[seg * 3 + 2];
  const uint32_t r = uint32_t(left_size(g, sg.n));
  const int dim = b.sdim[0][seg];

  // composite order: own dim, then ancestors' dims nearest first, then index
  int cd[D];
  int ncd = 0;
  cd[ncd++] = dim;
  for (int64_t an = g; an > 0 && ncd < D;) {
    an = (an - 1) >> 1;
    const int da = explicitDims ? int(b.ndim[sg.base + an]) : rr_dim(an, D);
    bool seen = false;
    for (int i = 0; i < ncd; i++) seen |= (cd[i] == da);
    if (!seen) cd[ncd++] = da;
  }
  const int nwords = ncd + 1;
  auto word = [&](uint32_t i, int w) -> uint32_t {
    return w < ncd ? b.ckey[cd[w]][sb + i] : b.cidx[sb + i];
  };

  // the split-dim keys of the candidates share one bin: their digits are
  // taken relative to the smallest over the bits of their span
  uint32_t kmin = 0xffffffffu, kmax = 0u;
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
    const uint32_t v = word(i, 0);
    kmin = min(kmin, v);
    kmax = max(kmax, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
    kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
  }
  __syncthreads();  // sLo / sHi initialised
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&sLo, kmin);
    atomicMax(&sHi, kmax);
  }
  __syncthreads();
  const uint32_t klo = sLo, khi = sHi;
  uint32_t rank = r - below;
  bool unique = false;
  int w = 0;
  uint32_t cp = 0, cm = 0, base = 0;
  for (w = 0; w < nwords && !unique; w++) {
    cp = 0;
    cm = 0;
    base = w == 0 ? klo : 0u;
    const uint32_t span = w == 0 ? (khi >= klo ? khi - klo : 0u) : 0xffffffffu;
    const int top = span ? ((31 - __clz(span)) & ~7) : -8;  // no digit: one value
    for (int shift = top; shift >= 0; shift -= 8) {
      for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0;
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
        bool ok = true;
        for (int pw_i = 0; pw_i < w && ok; pw_i++) ok = word(i, pw_i) == pw[pw_i];
        if (!ok) continue;
        const uint32_t v = word(i, w) - base;
        if ((v & cm) != cp) continue;
        atomicAdd(&hist[(v >> shift) & 255u], 1u);
      }
      __syncthreads();
      if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        uint32_t s = 0;
        for (int k = 0; k < 8; k++) s += hist[lane * 8 + k];
        uint32_t incl = s;
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        const uint32_t excl = incl - s;
        if (rank >= excl && rank < incl) {
          uint32_t cum = excl;
          for (int k = 0; k < 8; k++) {
            const uint32_t c = hist[lane * 8 + k];
            if (rank < cum + c) {
              sDigit = uint32_t(lane * 8 + k);
              sCount = c;
              sRank = rank - cum;
              break;
            }
            cum += c;
          }
        }
      }
      __syncthreads();
      rank = sRank;
      cp |= sDigit << shift;
      cm |= 0xffu << shift;
      if (sCount == 1) {
        unique = true;
        break;
      }
    }
    if (!unique && threadIdx.x == 0) pw[w] = cp + base;
    __syncthreads();
  }
  // w now indexes the word being matched when the pivot became unique
  // (or nwords when every word was fully resolved; the index is unique).
  const int wl = unique ? w - 1 : nwords - 1;
  if (!unique) {
    cp = pw[nwords - 1];
    cm = 0xffffffffu;
    base = 0;
  }
  if (threadIdx.x == 0) sPivot = 0xffffffffu;
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
    bool ok = true;
    for (int pw_i = 0; pw_i < wl && ok; pw_i++) ok = word(i, pw_i) == pw[pw_i];
    if (ok && ((word(i, wl) - base) & cm) == cp) sPivot = i;
  }
  if (threadIdx.x == 0) {
    sNl = 0;
    sNr = 0;
  }
  __syncthreads();
  // exactly one candidate matches; the clamp only guards memory safety
  const uint32_t piv = sPivot < m ? sPivot : 0u;
  uint32_t pk[D + 1];
  for (int x = 0; x < nwords; x++) pk[x] = word(piv, x);
  uint32_t pkey[D];
#pragma unroll
  for (int d = 0; d < D; d++) pkey[d] = b.ckey[d][sb + piv];

  const int64_t lchild = 2 * g + 1;
  const int lvlNext = a.level + 1;
  const int64_t lBeg = sg.base + seg_begin(lchild, lvlNext, sg.n) + below;
  const int64_t rBeg = sg.base + seg_begin(lchild + 1, lvlNext, sg.n) + (uint32_t(sz) - m - below);
  const int nbuf = a.cb ^ 1;
  uint32_t lo[2][D], hi[2][D];
#pragma unroll
  for (int s = 0; s < 2; s++)
#pragma unroll
    for (int d = 0; d < D; d++) {
      lo[s][d] = 0xffffffffu;
      hi[s][d] = 0u;
    }
  for (uint32_t i0 = 0; i0 < m; i0 += blockDim.x) {
    const uint32_t i = i0 + threadIdx.x;
    if (i < m && i != piv) {
      int side = 0;  // 0 left, 1 right
      for (int x = 0; x < nwords; x++) {
        const uint32_t v = word(i, x);
        if (v != pk[x]) {
          side = v > pk[x];
          break;
        }
      }
      const int64_t dst = side ? rBeg + atomicAdd(&sNr, 1u) : lBeg + atomicAdd(&sNl, 1u);
#pragma unroll
      for (int d = 0; d < D; d++) {
        const uint32_t k = b.ckey[d][sb + i];
        b.key[nbuf][d][dst] = k;
        lo[side][d] = min(lo[side][d], k);
        hi[side][d] = max(hi[side][d], k);
      }
      b.idx[nbuf][dst] = b.cidx[sb + i];
    }
  }
  merge_child_bounds<D>(lo, hi, b.sbmin[1], b.sbmax[1], sg.child);
  if (threadIdx.x == 0) {
    b.perm[sg.base + g] = b.cidx[sb + piv];
    b.ndim[sg.base + g] = uint8_t(dim);
  }
  if (threadIdx.x == 0 && sg.child >= 0) {
    uint32_t bl[D], bh[D];
    for (int d = 0; d < D; d++) {
      bl[d] = b.sbox[0][int64_t(seg) * 2 * D + d];
      bh[d] = b.sbox[0][int64_t(seg) * 2 * D + D + d];
    }
    for (int s = 0; s < 2; s++) {
      uint32_t cl[D], ch[D];
      for (int d = 0; d < D; d++) {
        cl[d] = bl[d];
        ch[d] = bh[d];
      }
      if (s == 0)
        ch[dim] = pkey[dim];
      else
        cl[dim] = pkey[dim];
      const int64_t ci = sg.child + s;
      for (int d = 0; d < D; d++) {
        b.sbox[1][ci * 2 * D + d] = cl[d];
        b.sbox[1][ci * 2 * D + D + d] = ch[d];
      }
      b.sdim[1][ci] = explicitDims ? uint8_t(Scalar<SC>::widest(cl, ch, D))
                                   : uint8_t((a.level + 1) % D);
    }
  }
}

// One whole global level for subtrees of at most kChunk points, one CTA per
// subtree, in place of hist / select / partition / resolve (at the deepest
// global levels those launches were bound by per-CTA latency, not by
// bandwidth).  The subtree is staged in shared memory by bulk copies; the
// point of rank leftSize(g) under the composite key is found by an MSD radix
// select over the staged words (the split-dim key's digits taken over its
// data span, so 2-3 passes instead of 4); the other points go to the
// children's segments.  Same pivot, same children's sets and bounds as the
// four-kernel path (the order inside a child's segment is irrelevant).
template <int SC, int D>
__global__ void __launch_bounds__(kGThreads) level_fused_kernel(Bufs b, LevelArgs a,
                                                                bool explicitDims)
{
  if (build_failed(b)) return;
  extern __shared__ __align__(128) uint32_t stage[];  // [D + 1][kStageSpan]
  __shared__ uint32_t hist[256];
  __shared__ uint32_t sDigit, sCount, sRank, sPivot, sNl, sNr;
  __shared__ uint32_t pw[D + 1];
  __shared__ __align__(8) uint64_t bar;
  const int tid = threadIdx.x, lane = tid & 31;
  const int seg = blockIdx.x;
  const SegGeo sg = seg_geo(a, seg);
  const int64_t g = sg.g;
  const int64_t sb = sg.base + seg_begin(g, a.level, sg.n);
  const int64_t sz = subtree_size(g, sg.n);
  if (sz < 1 || sz > kChunk) return;  // the host launches this for sz <= kChunk only
  const uint32_t m = uint32_t(sz);
  const uint32_t r = uint32_t(left_size(g, sg.n));
  const int dim = b.sdim[0][seg];

  // composite order: own dim, then ancestors' dims nearest first, then index
  int cd[D];
  int ncd = 0;
  cd[ncd++] = dim;
  for (int64_t an = g; an > 0 && ncd < D;) {
    an = (an - 1) >> 1;
    const int da = explicitDims ? int(b.ndim[sg.base + an]) : rr_dim(an, D);
    bool seen = false;
    for (int i = 0; i < ncd; i++) seen |= (cd[i] == da);
    if (!seen) cd[ncd++] = da;
  }
  const int nwords = ncd + 1;

  // stage the subtree (16-byte-aligned span, as in partition_kernel)
  const int64_t a0 = sb & ~int64_t(3), a1 = (sb + sz + 3) & ~int64_t(3);
  const uint32_t bytes = uint32_t(a1 - a0) * uint32_t(sizeof(uint32_t));
  const int cb = a.cb, nbuf = cb ^ 1;
  if (tid == 0) mbar_init(&bar, 1);
  __syncthreads();
  if (tid == 0) {
    mbar_arrive_expect_tx(&bar, bytes * uint32_t(D + 1));
#pragma unroll
    for (int d = 0; d < D; d++) bulk_copy_g2s(stage + d * kStageSpan, b.key[cb][d] + a0, bytes, &bar);
    bulk_copy_g2s(stage + D * kStageSpan, b.idx[cb] + a0, bytes, &bar);
  }
  if (!mbar_wait_bounded(&bar, 0, g_wait_polls)) {
    if (tid == 0) {
      atomicAdd(&g_wait_timeouts, 1u);
      atomicOr(b.status, 1u);
    }
    mbar_wait_bounded(&bar, 0, kWaitPolls);  // let copies in flight land first
    return;
  }
  const uint32_t *sw = stage + int(sb - a0);  // staged element i: sw[x * kStageSpan + i]
  auto word = [&](uint32_t i, int w) -> uint32_t {
    return sw[(w < ncd ? cd[w] : D) * kStageSpan + int(i)];
  };

  // MSD radix select of rank r
  const uint32_t klo = b.sbmin[0][seg * D + dim], khi = b.sbmax[0][seg * D + dim];
  uint32_t rank = r;
  bool unique = false;
  int w = 0;
  uint32_t cp = 0, cm = 0, base = 0;
  for (w = 0; w < nwords && !unique; w++) {
    cp = 0;
    cm = 0;
    base = w == 0 ? klo : 0u;
    const uint32_t span = w == 0 ? (khi >= klo ? khi - klo : 0u) : 0xffffffffu;
    const int top = span ? ((31 - __clz(span)) & ~7) : -8;  // no digit: one value
    for (int shift = top; shift >= 0; shift -= 8) {
      for (int i = tid; i < 256; i += blockDim.x) hist[i] = 0;
      __syncthreads();
      for (uint32_t i = tid; i < m; i += blockDim.x) {
        bool ok = true;
        for (int q = 0; q < w && ok; q++) ok = word(i, q) == pw[q];
        if (!ok) continue;
        const uint32_t v = word(i, w) - base;
        if ((v & cm) != cp) continue;
        atomicAdd(&hist[(v >> shift) & 255u], 1u);
      }
      __syncthreads();
      if (tid < 32) {
        uint32_t s8 = 0;
        for (int k = 0; k < 8; k++) s8 += hist[lane * 8 + k];
        uint32_t incl = s8;
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += t;
        }
        const uint32_t excl = incl - s8;
        if (rank >= excl && rank < incl) {
          uint32_t cum = excl;
          for (int k = 0; k < 8; k++) {
            const uint32_t c = hist[lane * 8 + k];
            if (rank < cum + c) {
              sDigit = uint32_t(lane * 8 + k);
              sCount = c;
              sRank = rank - cum;
              break;
            }
            cum += c;
          }
        }
      }
      __syncthreads();
      rank = sRank;
      cp |= sDigit << shift;
      cm |= 0xffu << shift;
      if (sCount == 1) {
        unique = true;
        break;
      }
    }
    if (!unique && tid == 0) pw[w] = cp + base;
    __syncthreads();
  }
  // the word at which the pivot became unique (w ran one past it), else
  // every word fully resolved
  const int wl = unique ? w - 1 : nwords - 1;
  if (!unique) {
    cp = pw[nwords - 1];
    cm = 0xffffffffu;
    base = 0;
  }
  if (tid == 0) {
    sPivot = 0xffffffffu;
    sNl = 0;
    sNr = 0;
  }
  __syncthreads();
  for (uint32_t i = tid; i < m; i += blockDim.x) {
    bool ok = true;
    for (int q = 0; q < wl && ok; q++) ok = word(i, q) == pw[q];
    if (ok && ((word(i, wl) - base) & cm) == cp) sPivot = i;
  }
  __syncthreads();
  // exactly one point matches; the clamp only guards memory safety
  const uint32_t piv = sPivot < m ? sPivot : 0u;
  uint32_t pk[D + 1];
#pragma unroll
  for (int x = 0; x < D + 1; x++) pk[x] = x < nwords ? word(piv, x) : 0u;
  uint32_t pkey[D];
#pragma unroll
  for (int d = 0; d < D; d++) pkey[d] = sw[d * kStageSpan + int(piv)];

  // the other points to the children, warp-contiguous runs per side
  const int64_t lchild = 2 * g + 1;
  const int lvlNext = a.level + 1;
  const int64_t lBeg = sg.base + seg_begin(lchild, lvlNext, sg.n);
  const int64_t rBeg = sg.base + seg_begin(lchild + 1, lvlNext, sg.n);
  const uint32_t lsz = r, rsz = m - 1u - r;
  const uint32_t ltMask = (1u << lane) - 1u;
  uint32_t lo[2][D], hi[2][D];
#pragma unroll
  for (int s2 = 0; s2 < 2; s2++)
#pragma unroll
    for (int d = 0; d < D; d++) {
      lo[s2][d] = 0xffffffffu;
      hi[s2][d] = 0u;
    }
  for (uint32_t i0 = 0; i0 < m; i0 += blockDim.x) {
    const uint32_t i = i0 + tid;
    const bool valid = i < m && i != piv;
    int side = 0;
    if (valid) {
      bool decided = false;
#pragma unroll
      for (int x = 0; x < D + 1; x++) {
        if (x < nwords && !decided) {
          const uint32_t v = word(i, x);
          if (v != pk[x]) {
            side = v > pk[x];
            decided = true;
          }
        }
      }
    }
    const uint32_t ml = __ballot_sync(0xffffffffu, valid && side == 0);
    const uint32_t mr = __ballot_sync(0xffffffffu, valid && side == 1);
    uint32_t bl = 0, br = 0;
    if (lane == 0) {
      if (ml) bl = atomicAdd(&sNl, uint32_t(__popc(ml)));
      if (mr) br = atomicAdd(&sNr, uint32_t(__popc(mr)));
    }
    bl = __shfl_sync(0xffffffffu, bl, 0);
    br = __shfl_sync(0xffffffffu, br, 0);
    if (valid) {
      const uint32_t pos = side ? br + __popc(mr & ltMask) : bl + __popc(ml & ltMask);
      if (pos < (side ? rsz : lsz)) {
        const int64_t dst = (side ? rBeg : lBeg) + pos;
#pragma unroll
        for (int d = 0; d < D; d++) {
          const uint32_t k = sw[d * kStageSpan + int(i)];
          b.key[nbuf][d][dst] = k;
          if (side) {
            lo[1][d] = min(lo[1][d], k);
            hi[1][d] = max(hi[1][d], k);
          } else {
            lo[0][d] = min(lo[0][d], k);
            hi[0][d] = max(hi[0][d], k);
          }
        }
        b.idx[nbuf][dst] = sw[D * kStageSpan + int(i)];
      }
    }
  }
  merge_child_bounds<D>(lo, hi, b.sbmin[1], b.sbmax[1], sg.child);
  if (tid == 0) {
    b.perm[sg.base + g] = sw[D * kStageSpan + int(piv)];
    b.ndim[sg.base + g] = uint8_t(dim);
  }
  if (tid == 0 && sg.child >= 0) {
    uint32_t bl3[D], bh3[D];
    for (int d = 0; d < D; d++) {
      bl3[d] = b.sbox[0][int64_t(seg) * 2 * D + d];
      bh3[d] = b.sbox[0][int64_t(seg) * 2 * D + D + d];
    }
    for (int s2 = 0; s2 < 2; s2++) {
      uint32_t cl[D], ch[D];
      for (int d = 0; d < D; d++) {
        cl[d] = bl3[d];
        ch[d] = bh3[d];
      }
      if (s2 == 0)
        ch[dim] = pkey[dim];
      else
        cl[dim] = pkey[dim];
      const int64_t ci = sg.child + s2;
      for (int d = 0; d < D; d++) {
        b.sbox[1][ci * 2 * D + d] = cl[d];
        b.sbox[1][ci * 2 * D + D + d] = ch[d];
      }
      b.sdim[1][ci] = explicitDims ? uint8_t(Scalar<SC>::widest(cl, ch, D))
                                   : uint8_t((a.level + 1) % D);
    }
  }
}

// the staging area exceeds the default 48 KB of dynamic shared memory for
// D >= 2: opt in (once per build, or at forest plan creation, outside any
// graph capture)
template <int SC, int D>
int partition_opt_in()
{
  CKB_CUDA(cudaFuncSetAttribute(partition_kernel<SC, D>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(partition_smem<D>())));
  CKB_CUDA(cudaFuncSetAttribute(level_fused_kernel<SC, D>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(partition_smem<D>())));
  return CUKD_OK;
}

// subtree_body's source over the working arrays: the subtree's points are
// the contiguous segment of key buffer cb at `base` + seg_begin; the result
// goes to perm / ndim; boxIndex selects the domain box in b.sbox[0]
// (explicit dims only, -1: none).
template <int D> struct WorkSrc {
  const Bufs &b;
  int64_t n, s, base, boxIndex;
  int L0, cb;
  template <class SM> __device__ void load(SM &S, int m) const
  {
    const int64_t sb = base + seg_begin(s, L0, n);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
#pragma unroll
      for (int d = 0; d < D; d++) S.key[d][i] = b.key[cb][d][sb + i];
      S.idx[i] = b.idx[cb][sb + i];
    }
    if (int(threadIdx.x) < D && boxIndex >= 0) {
      S.rootLo[threadIdx.x] = b.sbox[0][boxIndex * 2 * D + threadIdx.x];
      S.rootHi[threadIdx.x] = b.sbox[0][boxIndex * 2 * D + D + threadIdx.x];
    }
  }
  __device__ int anc_dim(int64_t a) const { return int(b.ndim[base + a]); }
  template <class SM> __device__ void settle(int64_t g, int, int piv, int dim, SM &S) const
  {
    b.perm[base + g] = S.idx[piv];
    b.ndim[base + g] = uint8_t(dim);
  }
};

template <int SC, int D>
__global__ void __launch_bounds__(kSubThreads, 4) subtree_kernel(Bufs b, int64_t n, int L0, int cb,
                                                              bool explicitDims)
{
  if (build_failed(b)) return;
  extern __shared__ __align__(16) uint8_t smem_raw[];
  SubSmem<D, kTile, kSubThreads> &S =
      *reinterpret_cast<SubSmem<D, kTile, kSubThreads> *>(smem_raw);
  const int seg = blockIdx.x;
  const int64_t s = ((int64_t(1) << L0) - 1) + seg;
  WorkSrc<D> src{b, n, s, 0, seg, L0, cb};
  subtree_body<SC, D, kTile, kSubThreads>(src, n, L0, s, explicitDims, S);
}

// Forest subtree phase, persistent: each CTA takes the next (tree, subtree)
// work item from a global counter until the list (sorted by size, largest
// first) is exhausted.  A tree whose top-down phase ran L0 levels left its
// records in key buffer L0 & 1.  Round-robin split dims.
// threads per CTA of a tile class (256 for all) and resident CTAs the
// register budget targets: 4 per SM (64 registers; measured faster than the
// 72-96 the compiler picks unbounded) for 512- and 1024-point tiles, 2 for
// 2048-point tiles, whose 108 KB of shared memory allow no more
template <int TILE> struct ForestNT {
  static constexpr int value = kSubThreads;
  static constexpr int minBlocks = TILE == 2048 ? 2 : 4;
};

template <int D, int TILE>
__global__ void __launch_bounds__(ForestNT<TILE>::value, ForestNT<TILE>::minBlocks)
    subtree_forest_kernel(Bufs b, ForestSubtrees f)
{
  if (build_failed(b)) return;
  constexpr int NT = ForestNT<TILE>::value;
  extern __shared__ __align__(16) uint8_t smem_raw[];
  SubSmem<D, TILE, NT> &S = *reinterpret_cast<SubSmem<D, TILE, NT> *>(smem_raw);
  __shared__ int next;
  for (;;) {
    if (threadIdx.x == 0) next = atomicAdd(f.counter, 1);
    __syncthreads();
    const int w = next;
    __syncthreads();
    if (w >= f.items) break;
    const int c = f.cloud[w];
    const int L0 = f.level[w];
    const int64_t s = ((int64_t(1) << L0) - 1) + f.local[w];
    WorkSrc<D> src{b, f.cloudN[c], s, f.cloudBase[c], -1, L0, L0 & 1};
    subtree_body<0, D, TILE, NT>(src, f.cloudN[c], L0, s, false, S);
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// finalize: records in node order (+ explicit dims)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) finalize_kernel(uint8_t *__restrict__ pts,
                                                       const uint8_t *__restrict__ orig,
                                                       const uint32_t *__restrict__ perm,
                                                       const uint8_t *__restrict__ ndim,
                                                       int64_t n, int stride, int doff,
                                                       int dshift, uint32_t dmask,
                                                       const uint32_t *status)
{
  if (*status) return;  // a wait gave up: leave the caller's records as they were
  const int words = stride >> 2;
  for (int64_t g = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; g < n;
       g += int64_t(gridDim.x) * blockDim.x) {
    uint32_t pi = perm[g];
    if (pi >= uint64_t(n)) pi = uint32_t(g);  // guards memory safety only
    const uint32_t *src = (const uint32_t *)(orig + int64_t(pi) * stride);
    uint32_t *dst = (uint32_t *)(pts + g * stride);
    for (int w = 0; w < words; w++) dst[w] = src[w];
    if (doff >= 0) {
      uint32_t *dw = (uint32_t *)(pts + g * stride + doff);
      *dw = (*dw & ~(dmask << dshift)) | ((uint32_t(ndim[g]) & dmask) << dshift);
    }
  }
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
static int pow2ceil(int64_t v)
{
  int p = 1;
  while (p < v && p < (1 << 30)) p <<= 1;
  return p;
}

// The builder's launch sequence; Arena provides alloc(T **, count) -- the
// caller's memory resource (TempArena) or the allocation-free builder's fixed
// device scratch (StaticCarver) -- so both entry points run the same code.
template <int SC, int D, class Arena>
int build_run(void *pts, int64_t n, const Layout &L, void *worldBounds, cudaStream_t st,
              Arena &arena)
{
  const bool explicitDims = L.doff >= 0;
  Bufs b = {};
  int G = 0;
  while (subtree_size((int64_t(1) << G) - 1, n) > kTile) G++;
  const int64_t capSeg = int64_t(1) << G;
  for (int x = 0; x < 2; x++) {
    for (int d = 0; d < D; d++) CKB_TRY(arena.alloc(&b.key[x][d], n));
    CKB_TRY(arena.alloc(&b.idx[x], n));
  }
  if (G > 0) {
    for (int d = 0; d < D; d++) CKB_TRY(arena.alloc(&b.ckey[d], n));
    CKB_TRY(arena.alloc(&b.cidx, n));
  }
  CKB_TRY(arena.alloc(&b.perm, n));
  CKB_TRY(arena.alloc(&b.ndim, n));
  uint8_t *orig = nullptr;
  CKB_TRY(arena.alloc(&orig, size_t(n) * L.stride));
  for (int x = 0; x < 2; x++) {
    CKB_TRY(arena.alloc(&b.sdim[x], capSeg));
    CKB_TRY(arena.alloc(&b.sbmin[x], capSeg * D));
    CKB_TRY(arena.alloc(&b.sbmax[x], capSeg * D));
    CKB_TRY(arena.alloc(&b.sbox[x], capSeg * 2 * D));
  }
  int64_t histCap = 64;
  for (int lvl = 0; lvl < G; lvl++) {
    const int64_t maxSeg = subtree_size((int64_t(1) << lvl) - 1, n);
    const int nb = level_bins(maxSeg);
    histCap = std::max(histCap, (int64_t(1) << lvl) * nb);
  }
  CKB_TRY(arena.alloc(&b.hist, histCap));
  CKB_TRY(arena.alloc(&b.sel, capSeg * 3));
  CKB_TRY(arena.alloc(&b.cur, capSeg * 3));
  CKB_TRY(arena.alloc(&b.wbmin, D));
  CKB_TRY(arena.alloc(&b.wbmax, D));
  CKB_TRY(arena.alloc(&b.status, 1));

  // what must start filled / zeroed is reset here, on the caller's stream
  CKB_CUDA(cudaMemsetAsync(b.status, 0, sizeof(uint32_t), st));
  CKB_CUDA(cudaMemsetAsync(b.perm, 0xff, sizeof(uint32_t) * n, st));
  CKB_CUDA(cudaMemsetAsync(b.wbmin, 0xff, sizeof(uint32_t) * D, st));
  CKB_CUDA(cudaMemsetAsync(b.wbmax, 0, sizeof(uint32_t) * D, st));
  {
    const int blocks = int(std::min<int64_t>(div_up(n, 256), kNumSMs * 8));
    extract_kernel<SC, D><<<blocks, 256, 0, st>>>((const uint8_t *)pts, n, L.stride, L.poff,
                                                  orig, b);
    CKB_CHECK_LAUNCH();
  }
  root_kernel<SC, D><<<1, 32, 0, st>>>(b, worldBounds, explicitDims);
  CKB_CHECK_LAUNCH();

  if (G > 0) CKB_TRY((partition_opt_in<SC, D>()));
  int cb = 0;
  for (int lvl = 0; lvl < G; lvl++) {
    const int nseg = 1 << lvl;
    const int64_t maxSeg = subtree_size((int64_t(1) << lvl) - 1, n);
    LevelArgs a{};
    a.n = n;
    a.level = lvl;
    a.nb = level_bins(maxSeg);
    a.chunksPerSeg = int(div_up(maxSeg, kChunk));
    a.nseg = nseg;
    a.cb = cb;
    CKB_CUDA(cudaMemsetAsync(b.sbmin[1], 0xff, sizeof(uint32_t) * 2 * nseg * D, st));
    CKB_CUDA(cudaMemsetAsync(b.sbmax[1], 0, sizeof(uint32_t) * 2 * nseg * D, st));
    if (maxSeg <= kFusedMax) {
      level_fused_kernel<SC, D><<<nseg, kGThreads, partition_smem<D>(), st>>>(b, a, explicitDims);
      CKB_CHECK_LAUNCH();
    } else {
      CKB_CUDA(cudaMemsetAsync(b.hist, 0, sizeof(uint32_t) * size_t(nseg) * a.nb, st));
      const int64_t grid = int64_t(nseg) * a.chunksPerSeg;
      hist_kernel<SC, D><<<unsigned(int64_t(nseg) * div_up(a.chunksPerSeg, kHistGroup)), kGThreads, 0,
                           st>>>(b, a);
      CKB_CHECK_LAUNCH();
      if (a.nb >= 512)
        select_block_kernel<<<unsigned(nseg), 256, 0, st>>>(b, a);
      else
        select_kernel<<<unsigned(div_up(int64_t(nseg) * 32, 256)), 256, 0, st>>>(b, a);
      CKB_CHECK_LAUNCH();
      partition_kernel<SC, D><<<unsigned(grid), kGThreads, partition_smem<D>(), st>>>(b, a);
      CKB_CHECK_LAUNCH();
      if (nseg <= kWideResolveSegs)
        resolve_kernel<SC, D, 1024><<<nseg, 1024, 0, st>>>(b, a, explicitDims);
      else
        resolve_kernel<SC, D, kGThreads><<<nseg, kGThreads, 0, st>>>(b, a, explicitDims);
      CKB_CHECK_LAUNCH();
    }
    cb ^= 1;
    std::swap(b.sdim[0], b.sdim[1]);
    std::swap(b.sbmin[0], b.sbmin[1]);
    std::swap(b.sbmax[0], b.sbmax[1]);
    std::swap(b.sbox[0], b.sbox[1]);
  }
  {
    const size_t smem = sizeof(SubSmem<D, kTile, kSubThreads>);
    CKB_CUDA(cudaFuncSetAttribute(subtree_kernel<SC, D>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    subtree_kernel<SC, D><<<unsigned(capSeg), kSubThreads, smem, st>>>(b, n, G, cb,
                                                                       explicitDims);
    CKB_CHECK_LAUNCH();
  }
  {
    const int blocks = int(std::min<int64_t>(div_up(n, 256), kNumSMs * 16));
    finalize_kernel<<<blocks, 256, 0, st>>>((uint8_t *)pts, orig, b.perm, b.ndim, n, L.stride,
                                            explicitDims ? L.doff : -1, L.dshift, L.dmask,
                                            b.status);
    CKB_CHECK_LAUNCH();
  }
  return CUKD_OK;
}

template <int SC, int D>
int build_impl(void *pts, int64_t n, const Layout &L, void *worldBounds, cudaStream_t st,
               const cukd_mem_resource *mem)
{
  TempArena arena(st, mem);
  return build_run<SC, D>(pts, n, L, worldBounds, st, arena);
}

template <int SC, int D>
__global__ void bounds_only_kernel(const uint8_t *__restrict__ pts, int64_t n, int stride,
                                   int poff, uint32_t *kmin, uint32_t *kmax)
{
  uint32_t lo[D], hi[D];
#pragma unroll
  for (int d = 0; d < D; d++) {
    lo[d] = 0xffffffffu;
    hi[d] = 0u;
  }
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const uint32_t *c = (const uint32_t *)(pts + i * stride + poff);
#pragma unroll
    for (int d = 0; d < D; d++) {
      const uint32_t k = Scalar<SC>::key(c[d]);
      lo[d] = min(lo[d], k);
      hi[d] = max(hi[d], k);
    }
  }
#pragma unroll
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

template <int SC, int D>
__global__ void bounds_write_kernel(const uint32_t *kmin, const uint32_t *kmax, uint32_t *out)
{
  if (threadIdx.x < D) {
    out[threadIdx.x] = Scalar<SC>::bits(kmin[threadIdx.x]);
    out[D + threadIdx.x] = Scalar<SC>::bits(kmax[threadIdx.x]);
  }
}

template <int SC, int D>
int bounds_impl(const void *pts, int64_t n, const Layout &L, void *out, cudaStream_t st)
{
  TempArena arena(st, nullptr);
  uint32_t *k = nullptr;
  CKB_TRY(arena.alloc(&k, 2 * D));
  CKB_CUDA(cudaMemsetAsync(k, 0xff, sizeof(uint32_t) * D, st));
  CKB_CUDA(cudaMemsetAsync(k + D, 0, sizeof(uint32_t) * D, st));
  const int blocks = int(std::max<int64_t>(1, std::min<int64_t>(div_up(n, 256), kNumSMs * 8)));
  bounds_only_kernel<SC, D><<<blocks, 256, 0, st>>>((const uint8_t *)pts, n, L.stride, L.poff,
                                                    k, k + D);
  CKB_CHECK_LAUNCH();
  bounds_write_kernel<SC, D><<<1, 32, 0, st>>>(k, k + D, (uint32_t *)out);
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

// ---------------------------------------------------------------------------
// allocation-free variant of the builder
// ---------------------------------------------------------------------------
// Some callers cannot allocate device memory at the point where they need a
// tree: code running under another framework that owns the whole device
// through its own pool and forbids allocations it does not track, real-time
// loops that cannot afford cudaMalloc's latency or its failure at run time,
// and deployments that must have a fixed device-memory footprint decided at
// load time.  For them the builder below takes all of its scratch from one
// file-scope device array of fixed size instead of a memory resource.  The
// array exists on every GPU that loads this library, until the process
// exits.  Every call shares it: calls that can overlap on the GPU (different
// streams, no ordering between them) race on it and must be serialised by
// the caller.  Everything the build needs zeroed or filled is reset by the
// call itself, so a call never sees the previous call's contents.
constexpr int64_t kNoAllocMaxPoints = 262144;  // records per call
constexpr int kNoAllocMaxStride = 64;          // bytes per record
constexpr size_t kNoAllocScratchBytes = size_t(40) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// bump allocator over the static scratch (same interface as TempArena)
struct StaticCarver {
  uint8_t *base;
  size_t cap, used;
  template <typename T>
  int alloc(T **out, size_t count)
  {
    size_t bytes = count * sizeof(T);
    if (bytes == 0) bytes = 16;
    bytes = (bytes + 255) & ~size_t(255);
    if (used + bytes > cap) return CUKD_ERR_TOO_LARGE;
    *out = (T *)(base + used);
    used += bytes;
    return CUKD_OK;
  }
};

// The driver's handle of the current context (cuCtxGetCurrent, reached
// through the runtime so the library links no driver library).
static void *current_context()
{
  using Fn = int (*)(void **);
  static Fn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return (Fn)p;
  }();
  void *ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// Device address of the scratch in the current context, looked up once per
// (device, context): host code may not use the symbol's name as a device
// address, and an address belongs to the context it was looked up in (a
// device reset or another context on the device needs a new lookup).
static int noalloc_scratch_ptr(uint8_t **out)
{
  static std::mutex mu;
  static void *ptrs[64] = {};
  static void *ctxs[64] = {};
  int dev = 0;
  CKB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return CUKD_ERR_UNSUPPORTED;
  void *ctx = current_context();
  std::lock_guard<std::mutex> lock(mu);
  if (!ptrs[dev] || !ctx || ctx != ctxs[dev]) {
    void *p = nullptr;
    // (makes the device's primary context current when none is)
    CKB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    if (!p) return CUKD_ERR_CUDA;
    ptrs[dev] = p;
    ctxs[dev] = current_context();
  }
  *out = (uint8_t *)ptrs[dev];
  return CUKD_OK;
}

// The builder's launch sequence with every buffer carved from the static
// scratch (and no memory-pool calls).
template <int SC, int D>
int build_impl_static(void *pts, int64_t n, const Layout &L, void *worldBounds, cudaStream_t st)
{
  StaticCarver arena;
  CKB_TRY(noalloc_scratch_ptr(&arena.base));
  arena.cap = kNoAllocScratchBytes;
  arena.used = 0;
  return build_run<SC, D>(pts, n, L, worldBounds, st, arena);
}

// ---------------------------------------------------------------------------
// forest builds (many clouds in one record array)
// ---------------------------------------------------------------------------
// Per cloud: its data bounds (one CTA per cloud over the extracted keys),
// the root state of clouds that start with top-down levels, and the float
// box output (lower[D] then upper[D]; an empty cloud gets +inf / -inf).
template <int D>
__global__ void __launch_bounds__(256) cloud_bounds_kernel(Bufs b, const int64_t *cBase,
                                                           const int64_t *cN,
                                                           const int32_t *rootItem,
                                                           float *boundsOut)
{
  __shared__ uint32_t sl[8][D], sh[8][D];
  const int c = blockIdx.x;
  const int64_t base = cBase[c], n = cN[c];
  uint32_t lo[D], hi[D];
#pragma unroll
  for (int d = 0; d < D; d++) {
    lo[d] = 0xffffffffu;
    hi[d] = 0u;
  }
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
#pragma unroll
    for (int d = 0; d < D; d++) {
      const uint32_t k = b.key[0][d][base + i];
      lo[d] = min(lo[d], k);
      hi[d] = max(hi[d], k);
    }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < D; d++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = min(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = max(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
    if (lane == 0) {
      sl[wid][d] = lo[d];
      sh[wid][d] = hi[d];
    }
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  for (int w = 1; w < int(blockDim.x >> 5); w++)
    for (int d = 0; d < D; d++) {
      lo[d] = min(lo[d], sl[w][d]);
      hi[d] = max(hi[d], sh[w][d]);
    }
  if (boundsOut) {
    float *o = boundsOut + int64_t(c) * 2 * D;
    for (int d = 0; d < D; d++) {
      o[d] = n > 0 ? key_float(lo[d]) : __int_as_float(0x7f800000);
      o[D + d] = n > 0 ? key_float(hi[d]) : __int_as_float(0xff800000);
    }
  }
  const int it = rootItem[c];
  if (it >= 0) {
    for (int d = 0; d < D; d++) {
      b.sbmin[0][int64_t(it) * D + d] = lo[d];
      b.sbmax[0][int64_t(it) * D + d] = hi[d];
      b.sbox[0][int64_t(it) * 2 * D + d] = lo[d];
      b.sbox[0][int64_t(it) * 2 * D + D + d] = hi[d];
    }
    b.sdim[0][it] = 0;
  }
}

struct ForestWs {
  Bufs b;
  uint8_t *orig;
  std::vector<void *> blocks;
};

template <int D>
int forest_build_impl(const ForestBuild &f, float *pts, float *boundsOut, cudaStream_t st,
                      cudaStream_t side[3], cudaEvent_t ev[4])
{
  ForestWs *ws = (ForestWs *)f.ws;
  if (!ws) return CUKD_ERR_INVALID_ARGUMENT;
  Bufs b = ws->b;
  const int64_t n = f.total;
  const int stride = 4 * D;
  if (n == 0) return CUKD_OK;
  CKB_CUDA(cudaMemsetAsync(b.status, 0, sizeof(uint32_t), st));
  CKB_CUDA(cudaMemsetAsync(b.wbmin, 0xff, sizeof(uint32_t) * D, st));
  CKB_CUDA(cudaMemsetAsync(b.wbmax, 0, sizeof(uint32_t) * D, st));
  {
    const int blocks = int(std::min<int64_t>(div_up(n, 256), kNumSMs * 8));
    extract_kernel<0, D><<<blocks, 256, 0, st>>>((const uint8_t *)pts, n, stride, 0, ws->orig, b);
    CKB_CHECK_LAUNCH();
  }
  cloud_bounds_kernel<D><<<unsigned(f.numClouds), 256, 0, st>>>(b, f.cloudBase, f.cloudN,
                                                                f.rootItem, boundsOut);
  CKB_CHECK_LAUNCH();
  int cb = 0;
  for (int lvl = 0; lvl < f.numLevels; lvl++) {
    const ForestLevel &L = f.level[lvl];
    const int nextItems = lvl + 1 < f.numLevels ? f.level[lvl + 1].items : 0;
    LevelArgs a{};
    a.n = 0;
    a.level = lvl;
    a.nb = L.nb;
    a.chunksPerSeg = L.chunksPerSeg;
    a.nseg = L.items;
    a.cb = cb;
    a.wCloud = L.cloud;
    a.wLocal = L.local;
    a.wChild = L.child;
    a.cBase = f.cloudBase;
    a.cN = f.cloudN;
    if (nextItems > 0) {
      CKB_CUDA(cudaMemsetAsync(b.sbmin[1], 0xff, sizeof(uint32_t) * size_t(nextItems) * D, st));
      CKB_CUDA(cudaMemsetAsync(b.sbmax[1], 0, sizeof(uint32_t) * size_t(nextItems) * D, st));
    }
    if (L.maxSeg <= kFusedMax) {
      level_fused_kernel<0, D><<<unsigned(L.items), kGThreads, partition_smem<D>(), st>>>(b, a,
                                                                                          false);
      CKB_CHECK_LAUNCH();
    } else {
      CKB_CUDA(cudaMemsetAsync(b.hist, 0, sizeof(uint32_t) * size_t(L.items) * L.nb, st));
      const int64_t grid = int64_t(L.items) * L.chunksPerSeg;
      hist_kernel<0, D><<<unsigned(int64_t(L.items) * div_up(L.chunksPerSeg, kHistGroup)),
                          kGThreads, 0, st>>>(b, a);
      CKB_CHECK_LAUNCH();
      if (a.nb >= 512)
        select_block_kernel<<<unsigned(L.items), 256, 0, st>>>(b, a);
      else
        select_kernel<<<unsigned(div_up(int64_t(L.items) * 32, 256)), 256, 0, st>>>(b, a);
      CKB_CHECK_LAUNCH();
      partition_kernel<0, D><<<unsigned(grid), kGThreads, partition_smem<D>(), st>>>(b, a);
      CKB_CHECK_LAUNCH();
      if (L.items <= kWideResolveSegs)
        resolve_kernel<0, D, 1024><<<unsigned(L.items), 1024, 0, st>>>(b, a, false);
      else
        resolve_kernel<0, D, kGThreads><<<unsigned(L.items), kGThreads, 0, st>>>(b, a, false);
      CKB_CHECK_LAUNCH();
    }
    cb ^= 1;
    std::swap(b.sdim[0], b.sdim[1]);
    std::swap(b.sbmin[0], b.sbmin[1]);
    std::swap(b.sbmax[0], b.sbmax[1]);
    std::swap(b.sbox[0], b.sbox[1]);
  }
  // subtree phase: one persistent launch per tile class; with side streams
  // the classes are concurrent branches (fork / join through events)
  const bool fork = side && ev;
  if (fork) CKB_CUDA(cudaEventRecord(ev[3], st));
  for (int c = 0; c < 3; c++) {
    const ForestSubtrees &S = f.sub[c];
    if (S.items == 0) continue;
    cudaStream_t s = st;
    if (fork) {
      s = side[c];
      CKB_CUDA(cudaStreamWaitEvent(s, ev[3], 0));
    }
    CKB_CUDA(cudaMemsetAsync(S.counter, 0, sizeof(int), s));
    const int grid = std::max(1, std::min(S.items, f.subGrid[c]));
    // (the shared-memory opt-in was made by forest_subtree_occupancy)
#define CKB_SUB(T_)                                                                 \
  if (kForestTiles[c] == T_) {                                                      \
    subtree_forest_kernel<D, T_><<<grid, ForestNT<T_>::value,                       \
                                   sizeof(SubSmem<D, T_, ForestNT<T_>::value>), s>>>(b, S); \
    CKB_CHECK_LAUNCH();                                                             \
  }
    CKB_SUB(512) CKB_SUB(1024) CKB_SUB(2048)
#undef CKB_SUB
    if (fork) {
      CKB_CUDA(cudaEventRecord(ev[c], s));
      CKB_CUDA(cudaStreamWaitEvent(st, ev[c], 0));
    }
  }
  {
    const int blocks = int(std::min<int64_t>(div_up(n, 256), kNumSMs * 16));
    finalize_kernel<<<blocks, 256, 0, st>>>((uint8_t *)pts, ws->orig, b.perm, b.ndim, n, stride,
                                            -1, 0, 0u, b.status);
    CKB_CHECK_LAUNCH();
  }
  return CUKD_OK;
}

template <int D, int T>
int subtree_occupancy()
{
  int blocks = 0;
  const size_t smem = sizeof(SubSmem<D, T, ForestNT<T>::value>);
  if (cudaFuncSetAttribute(subtree_forest_kernel<D, T>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, subtree_forest_kernel<D, T>,
                                                    ForestNT<T>::value, smem) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  return std::max(1, blocks);
}

}  // namespace build

// histogram bins of a global level: about kBinPoints points per bin of the
// largest subtree, 64..kMaxBins.  Fewer points per bin leave fewer pivot-bin
// candidates for resolve_kernel's radix select (one CTA per subtree); 512
// per bin measured 6.38 ms for the 10M-point build, 128 6.13 ms, 32 6.12 ms.
int level_bins(int64_t maxSeg)
{
  using namespace build;
  return std::min(kMaxBins, std::max(64, pow2ceil(maxSeg / kBinPoints)));
}

int forest_workspace_create(ForestBuild *f, int64_t maxItems, int64_t histCap)
{
  using namespace build;
  if (!f || f->D < 2 || f->D > 4) return CUKD_ERR_INVALID_ARGUMENT;
  forest_workspace_destroy(f);
  ForestWs *ws = new ForestWs();
  ws->b = Bufs{};
  const int D = f->D;
  const int64_t n = std::max<int64_t>(f->total, 1);
  const int64_t items = std::max<int64_t>(maxItems, 1);
  auto get = [&](auto **out, size_t count) -> int {
    void *p = nullptr;
    // rounded up to 256 bytes: bulk copies read whole 16-byte units
    const size_t bytes = (std::max<size_t>(16, count * sizeof(**out)) + 255) & ~size_t(255);
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      cudaGetLastError();
      return CUKD_ERR_OUT_OF_MEMORY;
    }
    ws->blocks.push_back(p);
    *out = (std::remove_reference_t<decltype(**out)> *)p;
    return CUKD_OK;
  };
  int rc = CUKD_OK;
  auto T = [&](int r) {
    if (rc == CUKD_OK) rc = r;
  };
  Bufs &b = ws->b;
  T(D == 2 ? partition_opt_in<0, 2>() : (D == 3 ? partition_opt_in<0, 3>() : partition_opt_in<0, 4>()));
  for (int x = 0; x < 2; x++) {
    for (int d = 0; d < D; d++) T(get(&b.key[x][d], n));
    T(get(&b.idx[x], n));
  }
  if (maxItems > 0) {
    for (int d = 0; d < D; d++) T(get(&b.ckey[d], n));
    T(get(&b.cidx, n));
  }
  T(get(&b.perm, n));
  T(get(&b.ndim, n));
  T(get(&ws->orig, size_t(n) * 4 * D));
  for (int x = 0; x < 2; x++) {
    T(get(&b.sdim[x], items));
    T(get(&b.sbmin[x], items * D));
    T(get(&b.sbmax[x], items * D));
    T(get(&b.sbox[x], items * 2 * D));
  }
  T(get(&b.hist, std::max<int64_t>(histCap, 64)));
  T(get(&b.sel, items * 3));
  T(get(&b.cur, items * 3));
  T(get(&b.wbmin, D));
  T(get(&b.wbmax, D));
  T(get(&b.status, 1));
  f->ws = ws;
  if (rc != CUKD_OK) forest_workspace_destroy(f);
  return rc;
}

void forest_workspace_destroy(ForestBuild *f)
{
  if (!f || !f->ws) return;
  build::ForestWs *ws = (build::ForestWs *)f->ws;
  for (void *p : ws->blocks) cudaFree(p);
  delete ws;
  f->ws = nullptr;
}

int forest_subtree_occupancy(int D, int c)
{
  using namespace build;
#define CKB_OCC(D_)                                          \
  if (D == D_) {                                             \
    if (c == 0) return subtree_occupancy<D_, 512>();         \
    if (c == 1) return subtree_occupancy<D_, 1024>();        \
    return subtree_occupancy<D_, 2048>();                    \
  }
  CKB_OCC(2) CKB_OCC(3) CKB_OCC(4)
#undef CKB_OCC
  return 1;
}

int forest_build(const ForestBuild &f, float *pts, float *boundsOut, cudaStream_t st,
                 cudaStream_t side[3], cudaEvent_t ev[4])
{
  using namespace build;
  if (f.D == 2) return forest_build_impl<2>(f, pts, boundsOut, st, side, ev);
  if (f.D == 3) return forest_build_impl<3>(f, pts, boundsOut, st, side, ev);
  if (f.D == 4) return forest_build_impl<4>(f, pts, boundsOut, st, side, ev);
  return CUKD_ERR_UNSUPPORTED;
}

int inplace_dispatch(void *pts, int64_t n, const Layout &L, void *wb, cudaStream_t st,
                     const cukd_mem_resource *mem, bool bitonic);

int build_dispatch(void *pts, int64_t n, const Layout &L, void *wb, cudaStream_t st,
                   const cukd_mem_resource *mem)
{
  using namespace build;
#define CKB_CASE(SC_, D_) \
  if (L.scalar == SC_ && L.D == D_) return build_impl<SC_, D_>(pts, n, L, wb, st, mem);
  CKB_CASE(0, 2) CKB_CASE(0, 3) CKB_CASE(0, 4) CKB_CASE(0, 5) CKB_CASE(0, 6) CKB_CASE(0, 7)
  CKB_CASE(0, 8) CKB_CASE(1, 2) CKB_CASE(1, 3) CKB_CASE(1, 4) CKB_CASE(1, 5) CKB_CASE(1, 6)
  CKB_CASE(1, 7) CKB_CASE(1, 8)
#undef CKB_CASE
  return CUKD_ERR_UNSUPPORTED;
}

int bounds_dispatch(const void *pts, int64_t n, const Layout &L, void *out, cudaStream_t st)
{
  using namespace build;
#define CKB_CASE(SC_, D_) \
  if (L.scalar == SC_ && L.D == D_) return bounds_impl<SC_, D_>(pts, n, L, out, st);
  CKB_CASE(0, 2) CKB_CASE(0, 3) CKB_CASE(0, 4) CKB_CASE(0, 5) CKB_CASE(0, 6) CKB_CASE(0, 7)
  CKB_CASE(0, 8) CKB_CASE(1, 2) CKB_CASE(1, 3) CKB_CASE(1, 4) CKB_CASE(1, 5) CKB_CASE(1, 6)
  CKB_CASE(1, 7) CKB_CASE(1, 8)
#undef CKB_CASE
  return CUKD_ERR_UNSUPPORTED;
}

int build_dispatch_static(void *pts, int64_t n, const Layout &L, void *wb, cudaStream_t st)
{
  using namespace build;
#define CKB_CASE(SC_, D_) \
  if (L.scalar == SC_ && L.D == D_) return build_impl_static<SC_, D_>(pts, n, L, wb, st);
  CKB_CASE(0, 2) CKB_CASE(0, 3) CKB_CASE(0, 4)
  CKB_CASE(1, 2) CKB_CASE(1, 3) CKB_CASE(1, 4)
#undef CKB_CASE
  return CUKD_ERR_UNSUPPORTED;
}

}  // namespace ckb

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int cukd_build_tree(void *d_points, int64_t n, const cukd_layout *layout, void *d_world_bounds,
                    int builder, cudaStream_t stream, const cukd_mem_resource *mem)
{
  ckb::Layout L;
  if (!ckb::make_layout(layout, &L)) return CUKD_ERR_INVALID_ARGUMENT;
  if (builder < CUKD_BUILDER_DEFAULT || builder > CUKD_BUILDER_INPLACE)
    return CUKD_ERR_INVALID_ARGUMENT;
  if (n < 1) return CUKD_OK;
  if (L.doff >= 0 && !d_world_bounds) return CUKD_ERR_MISSING_WORLD_BOUNDS;
  if (!d_points) return CUKD_ERR_INVALID_ARGUMENT;
  if (n > (int64_t(1) << 31) - 1) return CUKD_ERR_UNSUPPORTED;
  if (builder == CUKD_BUILDER_BITONIC || builder == CUKD_BUILDER_INPLACE)
    return ckb::inplace_dispatch(d_points, n, L, d_world_bounds, stream, mem,
                                 builder == CUKD_BUILDER_BITONIC);
  return ckb::build_dispatch(d_points, n, L, d_world_bounds, stream, mem);
}

int cukd_compute_bounds(const void *d_points, int64_t n, const cukd_layout *layout,
                        void *d_world_bounds, cudaStream_t stream)
{
  ckb::Layout L;
  if (!ckb::make_layout(layout, &L) || !d_world_bounds) return CUKD_ERR_INVALID_ARGUMENT;
  if (n < 1) return CUKD_OK;
  return ckb::bounds_dispatch(d_points, n, L, d_world_bounds, stream);
}

int cukd_build_tree_noalloc(void *d_points, int64_t n, const cukd_layout *layout,
                            void *d_world_bounds, cudaStream_t stream)
{
  ckb::Layout L;
  if (!ckb::make_layout(layout, &L)) return CUKD_ERR_INVALID_ARGUMENT;
  if (n < 1) return CUKD_OK;
  if (L.doff >= 0 && !d_world_bounds) return CUKD_ERR_MISSING_WORLD_BOUNDS;
  if (!d_points) return CUKD_ERR_INVALID_ARGUMENT;
  if (n > ckb::build::kNoAllocMaxPoints || L.stride > ckb::build::kNoAllocMaxStride)
    return CUKD_ERR_TOO_LARGE;
  return ckb::build_dispatch_static(d_points, n, L, d_world_bounds, stream);
}

#define CKB_TYPED(name, SC, D)                                                            \
  int name(void *d_points, int64_t n, void *d_world_bounds, cudaStream_t stream,          \
           const cukd_mem_resource *mem)                                                  \
  {                                                                                       \
    cukd_layout l = {SC, D, 4 * D, 0, -1, 0, 0};                                          \
    return cukd_build_tree(d_points, n, &l, d_world_bounds, CUKD_BUILDER_DEFAULT, stream, \
                           mem);                                                          \
  }
CKB_TYPED(cukd_build_float2, CUKD_FLOAT32, 2)
CKB_TYPED(cukd_build_float3, CUKD_FLOAT32, 3)
CKB_TYPED(cukd_build_float4, CUKD_FLOAT32, 4)
CKB_TYPED(cukd_build_int2, CUKD_INT32, 2)
CKB_TYPED(cukd_build_int3, CUKD_INT32, 3)
CKB_TYPED(cukd_build_int4, CUKD_INT32, 4)
#undef CKB_TYPED

const char *cukd_status_string(int status)
{
  switch (status) {
    case CUKD_OK: return "success";
    case CUKD_ERR_INVALID_ARGUMENT: return "invalid argument";
    case CUKD_ERR_MISSING_WORLD_BOUNDS:
      return "asked to build k-d tree over nodes with explicit dims, but no memory for world "
             "bounds provided";
    case CUKD_ERR_OUT_OF_MEMORY: return "out of device memory";
    case CUKD_ERR_CUDA: return "CUDA error";
    case CUKD_ERR_UNSUPPORTED: return "unsupported data layout or size";
    case CUKD_ERR_TIMEOUT: return "device-side wait timed out";
    case CUKD_ERR_STACK_OVERFLOW: return "traversal stack overflow";
    case CUKD_ERR_INTERNAL: return "a builder's internal consistency check failed";
    case CUKD_ERR_TOO_LARGE:
      return "input larger than the allocation-free builder's static scratch allows (at most "
             "262144 records of at most 64 bytes per call)";
  }
  return "unknown status";
}

const char *cukd_last_cuda_error(void) { return ckb::last_cuda_error_string(); }

unsigned long long cukd_launch_count(void) { return ckb::launch_count(); }

int cukd_async_wait_timeouts(unsigned int *count)
{
  if (!count) return CUKD_ERR_INVALID_ARGUMENT;
  CKB_CUDA(cudaMemcpyFromSymbol(count, ckb::build::g_wait_timeouts, sizeof(unsigned int)));
  return CUKD_OK;
}

int cukd_set_async_wait_polls(uint32_t polls)
{
  CKB_CUDA(cudaMemcpyToSymbol(ckb::build::g_wait_polls, &polls, sizeof(uint32_t)));
  return CUKD_OK;
}

int cukd_build_check(cudaStream_t stream)
{
  static std::mutex mu;
  static unsigned int seen[64] = {};
  int dev = 0;
  CKB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return CUKD_ERR_UNSUPPORTED;
  static unsigned int seenFaults[64] = {};
  CKB_CUDA(cudaStreamSynchronize(stream));
  unsigned int count = 0, faults = 0;
  CKB_CUDA(cudaMemcpyFromSymbol(&count, ckb::build::g_wait_timeouts, sizeof(unsigned int)));
  CKB_CUDA(cudaMemcpyFromSymbol(&faults, ckb::build::g_build_faults, sizeof(unsigned int)));
  std::lock_guard<std::mutex> lock(mu);
  const bool gaveUp = count != seen[dev];
  const bool faulted = faults != seenFaults[dev];
  seen[dev] = count;
  seenFaults[dev] = faults;
  return gaveUp ? CUKD_ERR_TIMEOUT : faulted ? CUKD_ERR_INTERNAL : CUKD_OK;
}

}  // extern "C"
