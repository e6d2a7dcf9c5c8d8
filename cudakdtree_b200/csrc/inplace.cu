// Left-balanced builders with bounded temporary memory: the reference's
// buildTree_inPlace (cukd/builder_inplace.h:82-102, 441-480: no temporary
// memory besides the world bounds) and buildTree_bitonic
// (cukd/builder_bitonic.h:263-266: one uint32 tag per point).
//
// The reference's in-place builder keeps every point at a node of its final
// subtree and, per level, swaps points between a max-heap in the left
// subtree and a min-heap in the right one (builder_inplace.h:117-320).  This
// builder keeps the same invariant -- between levels, the points of the
// subtree under node g occupy exactly that subtree's node set, so nothing
// is ever copied out of the caller's array -- and splits each subtree by
// selection instead of heaps.  The node set of subtree g is, at relative
// depth j, the run of 2^j nodes starting at (g+1)*2^j - 1: the left child's
// set is the first half of every run, the right child's the second half.
// Per level and subtree:
//   select   the point of rank leftSize(g) under the composite key: an MSD
//            radix select with 12-bit digits over the key's words, the first
//            word's digits taken over the subtree's domain span; the point is
//            swapped into node g (and, for explicit-dim layouts, given its
//            split dim);
//   split    the left set's points above the pivot are paired, k-th with
//            k-th, with the right set's points below it, and swapped.
// Levels with at most kMultiSegs subtrees spread every subtree over all
// CTAs: per-subtree digit histograms in global memory; per-chunk counts of
// misplaced points and a scan of them into ranks; for each left chunk the
// right-side position of its first rank; then each left chunk pairs its
// misplaced points with the right side's points of the same ranks.  Deeper
// levels give each subtree one CTA (histogram in shared memory, misplaced
// points of both sides streamed through two shared-memory rings).  One
// cooperative launch runs all of those levels, separated by grid barriers
// whose waits are bounded.  Subtrees of <= kTile points then finish in
// shared memory (subtree.cuh), gathered from and written back to their node
// sets.
//
// Composite key.  The word order is the one of the reference's canonical
// tree (every level a stable sort: own split coordinate, then the
// ancestors' split coordinates, nearest first, then the input position;
// builder_thrust.h:414-512): the bitonic name carries each point's input
// index in its uint32 tag array (moved with the point), so it builds the
// canonical tree, ties included.  The in-place name has no such storage:
// after the coordinates it compares the records' raw 32-bit words, so it
// builds the canonical tree whenever the coordinates decide every split
// (in particular when no two points share a coordinate value, the case the
// reference's builders agree on, testing/testBuildersSameResult.cu:96-99),
// and otherwise a valid left-balanced k-d tree that depends only on the
// input array.  Records that are byte for byte equal are interchangeable;
// the split moves as many of them as the pivot's rank requires.
//
// Every step classifies a point by comparing its own words with the pivot's
// -- a property of the record, not of its position -- so the pairing rounds
// can recount a chunk after earlier rounds swapped part of it.
//
// Temporary memory: about 5.5 MB, independent of n (in place); plus 4
// bytes per point (bitonic).
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "subtree.cuh"

namespace ckb {
namespace build {
extern __device__ unsigned int g_wait_timeouts;
extern __device__ unsigned int g_build_faults;
extern __device__ uint32_t g_wait_polls;
}  // namespace build

namespace inplace {

using build::kSubThreads;
using build::kTile;
using build::Scalar;
using build::SubSmem;

constexpr int kThreads = 256;
constexpr int kDigitBits = 12;
constexpr int kBins = 1 << kDigitBits;
constexpr int kPerThread = kBins / kThreads;
static_assert(kPerThread * kThreads == kBins, "bins per thread");
// levels with at most this many subtrees spread each subtree over all CTAs
constexpr int kMultiSegs = 128;
// record words the in-place tie-break compares after the coordinates
constexpr int kMaxRaw = 60;
constexpr int kMaxWords = kMaxDims + kMaxRaw;
constexpr int kMaxChunks = 1 << 17;  // chunks of a spread level
constexpr int kMinChunkLog = 12;     // chunks of at least 4096 points
constexpr int kQueue = 4096;         // ring of misplaced positions, per side
constexpr int kMaxLevels = 32;

// predicate on a point's comparison with the pivot
enum : int { kAbove = 0, kBelow = 1, kTwin = 2, kNone = 3 };

struct Recs {
  uint8_t *pts;
  uint32_t *idx;  // bitonic: input index of the point at each node; null: in place
  int64_t n;
  int stride, poff, doff, dshift;  // doff -1: no explicit dims
  uint32_t dmask;
};

__device__ __forceinline__ uint32_t rec_word(const Recs &R, int64_t node, int byteOff)
{
  return *(const uint32_t *)(R.pts + node * R.stride + byteOff);
}
template <int SC>
__device__ __forceinline__ uint32_t coord_key(const Recs &R, int64_t node, int d)
{
  return Scalar<SC>::key(rec_word(R, node, R.poff + 4 * d));
}
__device__ __forceinline__ int dim_at(const Recs &R, int64_t node)
{
  return int((rec_word(R, node, R.doff) >> R.dshift) & R.dmask);
}
__device__ __forceinline__ void set_dim(const Recs &R, int64_t node, int dim)
{
  uint32_t *w = (uint32_t *)(R.pts + node * R.stride + R.doff);
  *w = (*w & ~(R.dmask << R.dshift)) | ((uint32_t(dim) & R.dmask) << R.dshift);
}
// exchanges two records (and their tags); V16: records are one 16-byte
// vector each
template <bool V16>
__device__ __forceinline__ void swap_recs(const Recs &R, int64_t a, int64_t b)
{
  if (V16) {
    uint4 *pa = (uint4 *)(R.pts + a * 16);
    uint4 *pb = (uint4 *)(R.pts + b * 16);
    const uint4 x = *pa, y = *pb;
    *pa = y;
    *pb = x;
  } else {
    uint32_t *pa = (uint32_t *)(R.pts + a * R.stride);
    uint32_t *pb = (uint32_t *)(R.pts + b * R.stride);
    for (int w = 0; w < (R.stride >> 2); w++) {
      const uint32_t x = pa[w], y = pb[w];
      pa[w] = y;
      pb[w] = x;
    }
  }
  if (R.idx) {
    const uint32_t x = R.idx[a], y = R.idx[b];
    R.idx[a] = y;
    R.idx[b] = x;
  }
}

// a consistency check failed: the build stops (status) and
// cukd_build_check reports CUKD_ERR_INTERNAL; the access is skipped
__device__ __forceinline__ void build_fault(uint32_t *status)
{
  atomicOr(status, 2u);
  atomicAdd(&build::g_build_faults, 1u);
}

// word `code` of the composite key: >= 0 the key of that coordinate, -1 the
// input index, <= -2 raw record word (-code - 2)
template <int SC>
__device__ __forceinline__ uint32_t word_of(const Recs &R, int64_t node, int code)
{
  if (code >= 0) return coord_key<SC>(R, node, code);
  if (code == -1) return R.idx[node];
  // a raw word; the split-dim bits are left out (the builder writes them)
  const int off = 4 * (-code - 2);
  const uint32_t v = rec_word(R, node, off);
  return off == R.doff ? v & ~(R.dmask << R.dshift) : v;
}

// one subtree of the current level
struct Seg {
  int64_t g, m, r;  // root node, points, rank of the pivot (left subtree size)
  int dim, nwords, jmax;
  uint32_t klo, khi;  // the split dim's domain as keys
  int8_t code[kMaxWords];
};

// Subtree g (level L) from its ancestors' split dims and split coordinates
// (as keys), ancDim[k] / ancKey[k] for the ancestor on level k.
template <int SC, int D>
__device__ void seg_setup(const Recs &R, const uint32_t *wb, bool explicitDims, int L, int64_t g,
                          const int8_t *ancDim, const uint32_t *ancKey, Seg &S)
{
  uint32_t lo[D], hi[D];
  for (int d = 0; d < D; d++) {
    lo[d] = wb[d];
    hi[d] = wb[D + d];
  }
  for (int k = 0; k < L; k++) {
    const int64_t a = ((g + 1) >> (L - k)) - 1;
    const int64_t c = ((g + 1) >> (L - k - 1)) - 1;
    if (c == 2 * a + 1)
      hi[ancDim[k]] = ancKey[k];
    else
      lo[ancDim[k]] = ancKey[k];
  }
  S.g = g;
  S.m = subtree_size(g, R.n);
  S.r = left_size(g, R.n);
  S.jmax = num_levels(R.n) - 1 - L;
  S.dim = explicitDims ? Scalar<SC>::widest(lo, hi, D) : L % D;
  S.klo = lo[S.dim];
  S.khi = hi[S.dim];
  int cd[D];
  int ncd = 0;
  cd[ncd++] = S.dim;
  for (int k = L - 1; k >= 0 && ncd < D; k--) {
    const int da = ancDim[k];
    bool seen = false;
    for (int i = 0; i < ncd; i++) seen |= cd[i] == da;
    if (!seen) cd[ncd++] = da;
  }
  int nw = 0;
  for (int i = 0; i < ncd; i++) S.code[nw++] = int8_t(cd[i]);
  if (R.idx) {
    S.code[nw++] = -1;
  } else {
    for (int w = 0; w < (R.stride >> 2) && nw < kMaxWords; w++) {
      bool covered = false;
      for (int i = 0; i < ncd; i++) covered |= (w * 4 == R.poff + 4 * cd[i]);
      if (!covered) S.code[nw++] = int8_t(-2 - w);
    }
  }
  S.nwords = nw;
}

// MSD radix selection state of one subtree
struct Sel {
  uint32_t base, cp, cm, rank;
  int w, shift, width, done, twins;
  int64_t pos;
  uint32_t pw[kMaxWords];  // values of the words before w
};

// starts word s.w (skipping words that are constant over the subtree);
// past the last word the remaining candidates are byte-identical twins
__device__ void sel_begin_word(Sel &s, const Seg &S, int64_t n)
{
  while (s.w < S.nwords) {
    uint32_t span;
    if (s.w == 0) {
      s.base = S.klo <= S.khi ? S.klo : 0u;
      span = S.klo <= S.khi ? S.khi - S.klo : 0xffffffffu;
    } else {
      s.base = 0;
      span = S.code[s.w] == -1 ? uint32_t(n - 1) : 0xffffffffu;
    }
    s.cp = 0;
    s.cm = 0;
    if (span == 0) {
      s.pw[s.w] = s.base;
      s.w++;
      continue;
    }
    const int nb = 32 - __clz(span);
    s.width = nb < kDigitBits ? nb : kDigitBits;
    s.shift = nb - s.width;
    return;
  }
}

// does `node` match the resolved prefix, and its digit of the current word;
// w0 is the node's first word, already loaded
template <int SC>
__device__ __forceinline__ bool sel_digit(const Recs &R, int64_t node, const Seg &S, const Sel &s,
                                          uint32_t w0, uint32_t &dg)
{
  uint32_t v = w0;
  if (s.w > 0) {
    if (w0 != s.pw[0]) return false;
    for (int x = 1; x < s.w; x++)
      if (word_of<SC>(R, node, S.code[x]) != s.pw[x]) return false;
    v = word_of<SC>(R, node, S.code[s.w]);
  }
  v -= s.base;
  if ((v & s.cm) != s.cp) return false;
  dg = (v >> s.shift) & ((1u << s.width) - 1u);
  return true;
}

// after the digit holding the rank was found (count c, cum points below)
__device__ void sel_advance(Sel &s, const Seg &S, int64_t n, uint32_t dg, uint32_t c, uint32_t below,
                            int64_t posOfDigit)
{
  s.rank -= below;
  s.cp |= dg << s.shift;
  s.cm |= ((1u << s.width) - 1u) << s.shift;
  if (c == 1) {
    s.done = 1;
    s.pos = posOfDigit;
    return;
  }
  if (s.shift == 0) {
    s.pw[s.w] = s.cp + s.base;
    s.w++;
    sel_begin_word(s, S, n);
    if (s.w >= S.nwords) {
      s.done = 1;
      s.twins = 1;
      s.pos = posOfDigit;
    }
    return;
  }
  const int wd = s.shift < kDigitBits ? s.shift : kDigitBits;
  s.shift -= wd;
  s.width = wd;
}

// sign of (record at node) - (pivot) in the composite order; w0 is the
// node's first word, already loaded
template <int SC>
__device__ __forceinline__ int cmp_pivot(const Recs &R, int64_t node, const Seg &S,
                                         const uint32_t *pk, uint32_t w0)
{
  if (w0 != pk[0]) return w0 < pk[0] ? -1 : 1;
  for (int x = 1; x < S.nwords; x++) {
    const uint32_t v = word_of<SC>(R, node, S.code[x]);
    if (v != pk[x]) return v < pk[x] ? -1 : 1;
  }
  return 0;
}
__device__ __forceinline__ bool pred_hit(int c, int pred)
{
  return pred == kAbove ? c > 0 : pred == kBelow ? c < 0 : pred == kTwin ? c == 0 : false;
}

// half-run of side sd (0 left, 1 right) at relative depth j >= 1 of subtree
// g: first node and length (clamped to the tree)
__device__ __forceinline__ void half_run(int64_t g, int j, int sd, int64_t n, int64_t &start,
                                         int64_t &len)
{
  const int64_t half = int64_t(1) << (j - 1);
  start = ((g + 1) << j) - 1 + sd * half;
  len = n - start;
  len = len < 0 ? 0 : (len > half ? half : len);
}

// chunks of one side of one subtree on a spread level: depths 1..lc+1 give
// one chunk each, depth lc+1+i gives 2^i chunks of 2^lc points
__host__ __device__ inline int64_t chunks_per_side(int jmax, int lc)
{
  if (jmax <= lc + 1) return jmax;
  return (lc + 1) + (int64_t(1) << (jmax - lc)) - 2;
}
__device__ __forceinline__ void chunk_pos(int64_t t, int lc, int &j, int64_t &k)
{
  if (t < lc + 1) {
    j = int(t) + 1;
    k = 0;
    return;
  }
  const int64_t tp = t - (lc + 1) + 2;
  const int i = 63 - __clzll((long long)tp);
  j = lc + 1 + i;
  k = tp - (int64_t(1) << i);
}
// chunk t of side sd of subtree g: first node and length
__device__ __forceinline__ void chunk_range(int64_t g, int sd, int64_t t, int lc, int64_t n,
                                            int64_t &cs, int64_t &cl)
{
  int j;
  int64_t k;
  chunk_pos(t, lc, j, k);
  int64_t hs, hl;
  half_run(g, j, sd, n, hs, hl);
  const int64_t C = int64_t(1) << lc;
  cs = hs + (k << lc);
  cl = hl - (k << lc);
  cl = cl < 0 ? 0 : (cl > C ? C : cl);
}

// the v-th node of subtree g's node set, depth by depth
__device__ __forceinline__ int64_t set_node(int64_t g, int64_t v)
{
  const int j = 63 - __clzll((long long)(v + 1));
  return ((g + 1) << j) - 1 + (v - ((int64_t(1) << j) - 1));
}
// the v-th node of side sd (0 left, 1 right) of subtree g, depth by depth
__device__ __forceinline__ int64_t side_node(int64_t g, int sd, int64_t v)
{
  const int jj = 63 - __clzll((long long)(v + 1));  // depth - 1
  const int64_t half = int64_t(1) << jj;
  return ((g + 1) << (jj + 1)) - 1 + sd * half + (v - (half - 1));
}

// points per thread per batch in the streaming loops (independent loads in
// flight per thread)
constexpr int kU = 4;
constexpr int kBatch = kThreads * kU;
// the histogram and count passes over chunks: 16 per thread, a whole
// 4096-point chunk per batch
constexpr int kUs = 8;
constexpr int kBatchS = kThreads * kUs;

struct TopArgs {
  Recs R;
  const uint32_t *wb;  // world bounds as keys [2][D]
  int G;               // levels run by the top kernel
  bool explicitDims;
  uint32_t *status;
  unsigned int *bar;  // [0] arrivals, [1] generation
  unsigned int *active;
  Seg *seg;
  Sel *sel;
  uint32_t *hist, *hpos;  // [kMultiSegs][kBins]
  uint32_t *ccnt, *cst;   // [kMaxChunks]
  uint32_t *bnd;          // [kMaxChunks][2]: partner chunk and offset of a left chunk
  uint32_t *tot;          // [2 phases][2 * kMultiSegs]
  int8_t lc[kMaxLevels];  // log2 chunk size per spread level
};

struct TopSmem {
  union {
    struct {
      uint32_t hist[kBins];
      uint32_t hpos[kBins];
    } h;
    uint32_t q[2][kQueue];
  } u;
  Seg seg;
  Sel sel;
  uint32_t pk[kMaxWords];
  uint32_t wsum[kThreads / 32];
  uint32_t res[3];
  int cached;
  int ok;
  int pred[2];
  // rings of misplaced positions, per side: a cursor over a sequence of
  // node ranges (the side's half-runs by depth, or its chunks)
  int qHead[2], qCnt[2], qExh[2];
  int64_t qIdx[2], qEnd[2], qOff[2];
  int qChunked, qLc;
  int8_t ancDim[kMaxLevels];
  uint32_t ancKey[kMaxLevels];
};

// Grid-wide barrier of the cooperative launch.  The wait is bounded
// (build::g_wait_polls polls); one that gives up sets the build's status
// word, and every CTA returns at its next barrier.
__device__ bool grid_barrier(const TopArgs &A, TopSmem &T)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int *vgen = A.bar + 1;
    const unsigned int gen = *vgen;
    __threadfence();
    int ok = 1;
    if (atomicAdd(A.bar, 1u) == gridDim.x - 1) {
      atomicExch(A.bar, 0u);
      __threadfence();
      atomicAdd(A.bar + 1, 1u);
    } else {
      const uint32_t limit = build::g_wait_polls;
      uint32_t polls = 0;
      while (*vgen == gen) {
        if (++polls > limit) {
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    if (!ok) {
      atomicOr(A.status, 1u);
      atomicAdd(&build::g_wait_timeouts, 1u);
    }
    T.ok = ok && *(volatile uint32_t *)A.status == 0;
  }
  __syncthreads();
  return T.ok != 0;
}

// exclusive block scan of one value per thread; returns the prefix, total
// in *total (every thread)
__device__ __forceinline__ uint32_t block_scan(uint32_t v, TopSmem &T, uint32_t *total)
{
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) T.wsum[wid] = incl;
  __syncthreads();
  uint32_t before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; w++) {
    const uint32_t x = T.wsum[w];
    before += w < wid ? x : 0u;
    all += x;
  }
  __syncthreads();
  *total = all;
  return before + incl - v;
}

// the digit holding `rank` in a histogram row; T.res = {digit, count, below}
__device__ void find_digit(const uint32_t *h, uint32_t rank, TopSmem &T)
{
  uint32_t c[kPerThread];
  uint32_t s = 0;
#pragma unroll
  for (int i = 0; i < kPerThread; i++) {
    c[i] = h[threadIdx.x * kPerThread + i];
    s += c[i];
  }
  uint32_t total;
  const uint32_t before = block_scan(s, T, &total);
  if (rank >= before && rank < before + s) {
    uint32_t cum = before;
#pragma unroll
    for (int i = 0; i < kPerThread; i++) {
      if (rank >= cum && rank < cum + c[i]) {
        T.res[0] = threadIdx.x * kPerThread + i;
        T.res[1] = c[i];
        T.res[2] = cum;
      }
      cum += c[i];
    }
  }
  __syncthreads();
}

// histogram of the current digit over the nodes [cs, cs + cl) (every
// thread); true if this thread counted a point
template <int SC>
__device__ bool hist_range(const Recs &R, const Seg &S, const Sel &s, int64_t cs, int64_t cl,
                           uint32_t *hist, uint32_t *hpos)
{
  const int code0 = S.code[0];
  bool any = false;
  for (int64_t b = 0; b < cl; b += kBatchS) {
    uint32_t w[kUs];
#pragma unroll
    for (int u = 0; u < kUs; u++) {
      const int64_t e = b + u * kThreads + threadIdx.x;
      w[u] = e < cl ? word_of<SC>(R, cs + e, code0) : 0u;
    }
#pragma unroll
    for (int u = 0; u < kUs; u++) {
      const int64_t e = b + u * kThreads + threadIdx.x;
      uint32_t dg;
      if (e < cl && sel_digit<SC>(R, cs + e, S, s, w[u], dg)) {
        atomicAdd(&hist[dg], 1u);
        hpos[dg] = uint32_t(cs + e);
        any = true;
      }
    }
  }
  return any;
}

// the same over subtree S.g's whole node set, as one flat sequence
template <int SC>
__device__ void hist_set(const Recs &R, const Seg &S, const Sel &s, uint32_t *hist, uint32_t *hpos)
{
  const int64_t vEnd = (int64_t(2) << S.jmax) - 1;
  const int code0 = S.code[0];
  for (int64_t b = 0; b < vEnd; b += kBatch) {
    int64_t node[kU];
    uint32_t w[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) {
      const int64_t v = b + u * kThreads + threadIdx.x;
      node[u] = v < vEnd ? set_node(S.g, v) : R.n;
      w[u] = node[u] < R.n ? word_of<SC>(R, node[u], code0) : 0u;
    }
#pragma unroll
    for (int u = 0; u < kU; u++) {
      uint32_t dg;
      if (node[u] < R.n && sel_digit<SC>(R, node[u], S, s, w[u], dg)) {
        atomicAdd(&hist[dg], 1u);
        hpos[dg] = uint32_t(node[u]);
      }
    }
  }
}

// points of [cs, cs + cl) that satisfy pred (this thread's share)
template <int SC>
__device__ uint32_t count_range(const Recs &R, const Seg &S, const uint32_t *pk, int pred,
                                int64_t cs, int64_t cl)
{
  const int code0 = S.code[0];
  uint32_t cnt = 0;
  for (int64_t b = 0; b < cl; b += kBatchS) {
    uint32_t w[kUs];
#pragma unroll
    for (int u = 0; u < kUs; u++) {
      const int64_t e = b + u * kThreads + threadIdx.x;
      w[u] = e < cl ? word_of<SC>(R, cs + e, code0) : 0u;
    }
#pragma unroll
    for (int u = 0; u < kUs; u++) {
      const int64_t e = b + u * kThreads + threadIdx.x;
      cnt += (e < cl && pred_hit(cmp_pivot<SC>(R, cs + e, S, pk, w[u]), pred)) ? 1u : 0u;
    }
  }
  return cnt;
}

// which of this thread's kU consecutive points of the batch at offset b of
// [cs, cs + cl) satisfy pred (bit u: point b + threadIdx.x * kU + u)
template <int SC>
__device__ __forceinline__ uint32_t hit_mask(const Recs &R, const Seg &S, const uint32_t *pk,
                                             int pred, int64_t cs, int64_t cl, int64_t b)
{
  const int64_t e0 = b + int64_t(threadIdx.x) * kU;
  const int code0 = S.code[0];
  uint32_t w[kU];
#pragma unroll
  for (int u = 0; u < kU; u++) w[u] = e0 + u < cl ? word_of<SC>(R, cs + e0 + u, code0) : 0u;
  uint32_t m = 0;
#pragma unroll
  for (int u = 0; u < kU; u++)
    if (e0 + u < cl && pred_hit(cmp_pivot<SC>(R, cs + e0 + u, S, pk, w[u]), pred)) m |= 1u << u;
  return m;
}

// split dim and split coordinate (key) of every ancestor of g (level L),
// one thread per ancestor (every thread calls it)
template <int SC, int D>
__device__ void load_ancestors(const Recs &R, bool explicitDims, int L, int64_t g, int8_t *ancDim,
                               uint32_t *ancKey)
{
  __syncthreads();
  for (int k = threadIdx.x; k < L; k += blockDim.x) {
    const int64_t a = ((g + 1) >> (L - k)) - 1;
    const int da = explicitDims ? dim_at(R, a) : k % D;
    ancDim[k] = int8_t(da);
    ancKey[k] = coord_key<SC>(R, a, da);
  }
  __syncthreads();
}

template <int SC>
__device__ void place_pivot(const TopArgs &A, const Seg &S, const Sel &s)
{
  if (s.pos < 0 || s.pos >= A.R.n) {
    build_fault(A.status);
    return;
  }
  if (s.pos != S.g) swap_recs<false>(A.R, s.pos, S.g);
  if (A.explicitDims) set_dim(A.R, S.g, S.dim);
}

template <int SC>
__device__ void load_pivot_words(const TopArgs &A, TopSmem &T)
{
  for (int x = threadIdx.x; x < T.seg.nwords; x += kThreads)
    T.pk[x] = word_of<SC>(A.R, T.seg.g, T.seg.code[x]);
}

// copies subtree s's Seg (and, with withSel, its Sel) into shared memory
__device__ void load_seg(const TopArgs &A, int s, bool withSel, TopSmem &T)
{
  const uint32_t *src = (const uint32_t *)(A.seg + s);
  uint32_t *dst = (uint32_t *)&T.seg;
  for (int i = threadIdx.x; i < int(sizeof(Seg) / 4); i += kThreads) dst[i] = src[i];
  if (withSel) {
    const uint32_t *ss = (const uint32_t *)(A.sel + s);
    uint32_t *ds = (uint32_t *)&T.sel;
    for (int i = threadIdx.x; i < int(sizeof(Sel) / 4); i += kThreads) ds[i] = ss[i];
  }
}

// ---------------------------------------------------------------------------
// rings of misplaced positions
// ---------------------------------------------------------------------------
// node range idx of side sd's cursor: a half-run by depth (one CTA per
// subtree) or a chunk (spread levels)
__device__ __forceinline__ void cursor_range(const TopSmem &T, int sd, int64_t idx, int64_t n,
                                             int64_t &cs, int64_t &cl)
{
  if (T.qChunked)
    chunk_range(T.seg.g, sd, idx, T.qLc, n, cs, cl);
  else
    half_run(T.seg.g, int(idx), sd, n, cs, cl);
}

__device__ void ring_start(int sd, int pred, int64_t idx, int64_t end, int64_t off, TopSmem &T)
{
  __syncthreads();
  if (threadIdx.x == 0) {
    T.qHead[sd] = 0;
    T.qCnt[sd] = 0;
    T.qExh[sd] = 0;
    T.qIdx[sd] = idx;
    T.qEnd[sd] = end;
    T.qOff[sd] = off;
    T.pred[sd] = pred;
  }
  __syncthreads();
}

// appends the side's next misplaced positions, in node order, until the
// ring holds `want`, is nearly full, or the side is exhausted (all
// threads; uniform).  Chunked cursors walk chunk ids (qIdx) and an offset
// in the chunk; flat cursors walk the side's node set by index (qOff, up to
// qEnd).
template <int SC>
__device__ void ring_fill(const Recs &R, int sd, int64_t want, TopSmem &T)
{
  const int tid = threadIdx.x;
  for (;;) {
    __syncthreads();
    if (T.qExh[sd] || T.qCnt[sd] >= want || T.qCnt[sd] > kQueue - kBatch) break;
    const int64_t idx = T.qIdx[sd], off = T.qOff[sd];
    int64_t cs = 0, cl = T.qEnd[sd];
    bool next = false, exhausted = false;
    if (T.qChunked) {
      if (idx >= T.qEnd[sd])
        exhausted = true;
      else {
        chunk_range(T.seg.g, sd, idx, T.qLc, R.n, cs, cl);
        next = off >= cl;
      }
    } else {
      exhausted = off >= cl;
    }
    if (exhausted || next) {
      __syncthreads();
      if (tid == 0) {
        if (exhausted)
          T.qExh[sd] = 1;
        else {
          T.qIdx[sd] = idx + 1;
          T.qOff[sd] = 0;
        }
      }
      continue;
    }
    const int64_t e0 = off + int64_t(tid) * kU;
    const int code0 = T.seg.code[0];
    int64_t node[kU];
    uint32_t w[kU];
#pragma unroll
    for (int u = 0; u < kU; u++) {
      const int64_t e = e0 + u;
      node[u] = e < cl ? (T.qChunked ? cs + e : side_node(T.seg.g, sd, e)) : R.n;
      w[u] = node[u] < R.n ? word_of<SC>(R, node[u], code0) : 0u;
    }
    uint32_t m = 0;
#pragma unroll
    for (int u = 0; u < kU; u++)
      if (node[u] < R.n && pred_hit(cmp_pivot<SC>(R, node[u], T.seg, T.pk, w[u]), T.pred[sd]))
        m |= 1u << u;
    uint32_t total;
    uint32_t r = block_scan(__popc(m), T, &total);
    const int tail = T.qHead[sd] + T.qCnt[sd];
#pragma unroll
    for (int u = 0; u < kU; u++)
      if ((m >> u) & 1u) T.u.q[sd][(tail + int(r++)) % kQueue] = uint32_t(node[u]);
    __syncthreads();
    if (tid == 0) {
      T.qCnt[sd] += int(total);
      T.qOff[sd] = off + (cl - off < kBatch ? cl - off : kBatch);
    }
  }
}

// swaps the rings' first min(count0, count1, limit) pairs; returns it
template <bool V16>
__device__ int ring_pair(const Recs &R, int64_t limit, TopSmem &T)
{
  __syncthreads();
  int k = min(T.qCnt[0], T.qCnt[1]);
  if (int64_t(k) > limit) k = int(limit);
  for (int i = threadIdx.x; i < k; i += kThreads)
    swap_recs<V16>(R, T.u.q[0][(T.qHead[0] + i) % kQueue], T.u.q[1][(T.qHead[1] + i) % kQueue]);
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int sd = 0; sd < 2; sd++) {
      T.qHead[sd] = (T.qHead[sd] + k) % kQueue;
      T.qCnt[sd] -= k;
    }
  }
  __syncthreads();
  return k;
}

// ---------------------------------------------------------------------------
// spread level: every subtree over all CTAs
// ---------------------------------------------------------------------------
template <int SC, int D, bool V16>
__device__ bool spread_level(const TopArgs &A, int L, TopSmem &T)
{
  const Recs &R = A.R;
  const int nseg = 1 << L;
  const int64_t g0 = (int64_t(1) << L) - 1;
  const int lc = A.lc[L];
  const int jmax = num_levels(R.n) - 1 - L;
  const int64_t cps = chunks_per_side(jmax, lc);
  const int64_t nch = int64_t(2) * nseg * cps;
  const int tid = threadIdx.x;

  for (int s = blockIdx.x; s < nseg; s += gridDim.x) {
    load_ancestors<SC, D>(R, A.explicitDims, L, g0 + s, T.ancDim, T.ancKey);
    if (tid == 0) {
      Seg S;
      seg_setup<SC, D>(R, A.wb, A.explicitDims, L, g0 + s, T.ancDim, T.ancKey, S);
      A.seg[s] = S;
      Sel sl;
      sl.w = 0;
      sl.done = 0;
      sl.twins = 0;
      sl.pos = S.g;
      sl.rank = uint32_t(S.r);
      sel_begin_word(sl, S, R.n);
      if (sl.w >= S.nwords) {  // every point equal: any is the pivot
        sl.done = 1;
        sl.twins = 1;
      }
      A.sel[s] = sl;
      if (sl.done) place_pivot<SC>(A, S, sl);
    }
  }
  if (!grid_barrier(A, T)) return false;

  // ---- select
  for (int p = 0;; p++) {
    // pass p counts its unfinished subtrees in active[p & 1]; every CTA read
    // that counter's previous value (pass p - 2) before the barrier that
    // ended pass p - 1's histograms
    if (blockIdx.x == 0 && tid == 0) A.active[p & 1] = 0;
    if (tid == 0) T.cached = -1;
    for (int i = tid; i < kBins; i += kThreads) T.u.h.hist[i] = 0;
    __syncthreads();
    for (int64_t id = blockIdx.x; id < nch; id += gridDim.x) {
      const int s = int(id / (2 * cps));
      const int sd = int((id / cps) & 1);
      const int64_t t = id % cps;
      if (T.cached != s) {
        __syncthreads();
        load_seg(A, s, true, T);
        if (tid == 0) T.cached = s;
        __syncthreads();
      }
      if (T.sel.done) continue;
      int64_t cs, cl;
      chunk_range(T.seg.g, sd, t, lc, R.n, cs, cl);
      bool any = hist_range<SC>(R, T.seg, T.sel, cs, cl, T.u.h.hist, T.u.h.hpos);
      uint32_t dg;
      if (sd == 0 && t == 0 && tid == 0 &&
          sel_digit<SC>(R, T.seg.g, T.seg, T.sel, word_of<SC>(R, T.seg.g, T.seg.code[0]), dg)) {
        atomicAdd(&T.u.h.hist[dg], 1u);
        T.u.h.hpos[dg] = uint32_t(T.seg.g);
        any = true;
      }
      // merge into the subtree's row only if the chunk counted anything
      // (the bins are zeroed again as they are merged)
      if (__syncthreads_or(any)) {
        for (int i = tid; i < kBins; i += kThreads) {
          const uint32_t c = T.u.h.hist[i];
          if (c) {
            atomicAdd(&A.hist[int64_t(s) * kBins + i], c);
            A.hpos[int64_t(s) * kBins + i] = T.u.h.hpos[i];
            T.u.h.hist[i] = 0;
          }
        }
      }
      __syncthreads();
    }
    if (!grid_barrier(A, T)) return false;
    for (int s = blockIdx.x; s < nseg; s += gridDim.x) {
      load_seg(A, s, true, T);
      __syncthreads();
      if (!T.sel.done) {
        uint32_t *row = A.hist + int64_t(s) * kBins;
        find_digit(row, T.sel.rank, T);
        for (int i = tid; i < kBins; i += kThreads) row[i] = 0;
        if (tid == 0) {
          const uint32_t dg = T.res[0];
          sel_advance(T.sel, T.seg, R.n, dg, T.res[1], T.res[2],
                      int64_t(A.hpos[int64_t(s) * kBins + dg]));
          if (T.sel.done)
            place_pivot<SC>(A, T.seg, T.sel);
          else
            atomicAdd(A.active + (p & 1), 1u);
        }
        __syncthreads();
        uint32_t *ds = (uint32_t *)(A.sel + s);
        const uint32_t *ss = (const uint32_t *)&T.sel;
        for (int i = tid; i < int(sizeof(Sel) / 4); i += kThreads) ds[i] = ss[i];
      }
      __syncthreads();
    }
    if (!grid_barrier(A, T)) return false;
    if (*(volatile unsigned int *)(A.active + (p & 1)) == 0) break;
  }

  // ---- split: phase 0 pairs points above the pivot in the left set with
  // points below it in the right set; phase 1 (only where the pivot has
  // byte-identical twins) pairs what is left over with twins.  Per phase:
  // count each chunk's misplaced points, scan the counts per (subtree,
  // side) into ranks, find for every left chunk the right-side position of
  // its first rank, then let each left chunk swap its misplaced points with
  // the right side's points of the same ranks (disjoint positions per left
  // chunk, so no further barrier).
  bool anyUneven = false;
  for (int phase = 0; phase < 2; phase++) {
    if (phase == 1 && !anyUneven) break;
    uint32_t *tot = A.tot + phase * 2 * kMultiSegs;
    const uint32_t *tot0 = A.tot;
    if (tid == 0) T.cached = -1;
    __syncthreads();
    auto cache_seg = [&](int s) {
      if (T.cached == s) return;
      __syncthreads();
      load_seg(A, s, false, T);
      __syncthreads();
      load_pivot_words<SC>(A, T);
      if (tid == 0) {
        T.cached = s;
        if (phase == 0) {
          T.pred[0] = kAbove;
          T.pred[1] = kBelow;
        } else {
          const uint32_t a = tot0[2 * s], b = tot0[2 * s + 1];
          T.pred[0] = a > b ? kAbove : a < b ? kTwin : kNone;
          T.pred[1] = a > b ? kTwin : a < b ? kBelow : kNone;
        }
      }
      __syncthreads();
    };
    // count
    for (int64_t id = blockIdx.x; id < nch; id += gridDim.x) {
      const int s = int(id / (2 * cps));
      const int sd = int((id / cps) & 1);
      const int64_t t = id % cps;
      cache_seg(s);
      const int pred = T.pred[sd];
      uint32_t cnt = 0;
      if (pred != kNone) {
        int64_t cs, cl;
        chunk_range(T.seg.g, sd, t, lc, R.n, cs, cl);
        cnt = count_range<SC>(R, T.seg, T.pk, pred, cs, cl);
      }
      uint32_t total;
      block_scan(cnt, T, &total);
      if (tid == 0) A.ccnt[id] = total;
    }
    if (!grid_barrier(A, T)) return false;
    // scan the counts of each (subtree, side)
    for (int q = blockIdx.x; q < 2 * nseg; q += gridDim.x) {
      uint32_t carry = 0;
      for (int64_t b0 = 0; b0 < cps; b0 += kThreads) {
        const int64_t i = int64_t(q) * cps + b0 + tid;
        const uint32_t v = b0 + tid < cps ? A.ccnt[i] : 0u;
        uint32_t total;
        const uint32_t ex = block_scan(v, T, &total);
        if (b0 + tid < cps) A.cst[i] = carry + ex;
        carry += total;
      }
      if (tid == 0) tot[q] = carry;
    }
    if (!grid_barrier(A, T)) return false;
    for (int s = 0; s < nseg; s++)
      if (phase == 0 && tot[2 * s] != tot[2 * s + 1]) anyUneven = true;
    // partner position of each left chunk's first rank
    for (int64_t t = blockIdx.x; t < int64_t(nseg) * cps; t += gridDim.x) {
      const int s = int(t / cps);
      const int64_t id = int64_t(2 * s) * cps + t % cps;  // the left chunk
      const uint32_t K = min(tot[2 * s], tot[2 * s + 1]);
      const uint32_t st = A.cst[id], c = A.ccnt[id];
      if (c == 0 || st >= K) {
        if (tid == 0) A.bnd[2 * id] = 0xffffffffu;
        continue;
      }
      cache_seg(s);
      // the right chunk holding rank st: the last whose first rank is <= st
      const int64_t rb = int64_t(2 * s + 1) * cps;
      const int64_t stride = (cps + kThreads - 1) / kThreads;
      const int64_t probe = int64_t(tid) * stride;
      const int n1 = __syncthreads_count(probe < cps && A.cst[rb + probe] <= st);
      const int64_t lo = int64_t(n1 - 1) * stride;
      const int64_t p2 = lo + tid;
      const int n2 = __syncthreads_count(tid < stride && p2 < cps && A.cst[rb + p2] <= st);
      const int64_t jr = lo + n2 - 1;
      // offset of that rank's point inside the right chunk
      int64_t cs, cl;
      chunk_range(T.seg.g, 1, jr % cps, lc, R.n, cs, cl);
      uint32_t want = st - A.cst[rb + jr];
      if (tid == 0) T.res[0] = 0xffffffffu;
      __syncthreads();
      for (int64_t b = 0; b < cl; b += kBatch) {
        const uint32_t m = hit_mask<SC>(R, T.seg, T.pk, T.pred[1], cs, cl, b);
        uint32_t total;
        const uint32_t ex = block_scan(__popc(m), T, &total);
        if (want >= ex && want < ex + __popc(m)) {
          uint32_t r = ex;
#pragma unroll
          for (int u = 0; u < kU; u++)
            if ((m >> u) & 1u) {
              if (r == want) T.res[0] = uint32_t(b + int64_t(tid) * kU + u);
              r++;
            }
        }
        __syncthreads();
        if (T.res[0] != 0xffffffffu) break;
        want -= total;
      }
      if (tid == 0) {
        A.bnd[2 * id] = uint32_t(jr);
        A.bnd[2 * id + 1] = T.res[0];
        if (T.res[0] == 0xffffffffu) A.bnd[2 * id] = 0xfffffffeu;
      }
      __syncthreads();
    }
    if (!grid_barrier(A, T)) return false;
    // pair and swap, one left chunk at a time
    for (int64_t t = blockIdx.x; t < int64_t(nseg) * cps; t += gridDim.x) {
      const int s = int(t / cps);
      const int64_t id = int64_t(2 * s) * cps + t % cps;
      const uint32_t jr = A.bnd[2 * id];
      if (jr == 0xffffffffu) continue;
      cache_seg(s);
      if (jr == 0xfffffffeu) {  // the counts disagreed
        if (tid == 0) build_fault(A.status);
        continue;
      }
      const uint32_t K = min(tot[2 * s], tot[2 * s + 1]);
      const int64_t need = min(int64_t(A.ccnt[id]), int64_t(K) - A.cst[id]);
      __syncthreads();
      if (tid == 0) {
        T.qChunked = 1;
        T.qLc = lc;
      }
      ring_start(0, T.pred[0], t % cps, t % cps + 1, 0, T);
      ring_start(1, T.pred[1], jr, cps, A.bnd[2 * id + 1], T);
      int64_t done = 0;
      while (done < need) {
        ring_fill<SC>(R, 0, need - done, T);
        ring_fill<SC>(R, 1, need - done, T);
        const int k = ring_pair<V16>(R, need - done, T);
        if (k == 0) {
          if (tid == 0) build_fault(A.status);
          break;
        }
        done += k;
      }
    }
    if (!grid_barrier(A, T)) return false;
  }
  return true;
}

// ---------------------------------------------------------------------------
// CTA-per-subtree level
// ---------------------------------------------------------------------------
template <int SC, bool V16>
__device__ void cta_split(const TopArgs &A, TopSmem &T)
{
  const Recs &R = A.R;
  const int64_t unlimited = int64_t(1) << 62;
  __syncthreads();
  if (threadIdx.x == 0) T.qChunked = 0;
  const int64_t sideEnd = (int64_t(1) << T.seg.jmax) - 1;  // node slots of one side
  ring_start(0, kAbove, 0, sideEnd, 0, T);
  ring_start(1, kBelow, 0, sideEnd, 0, T);
  int twinSide = -1;  // side re-scanned for twins of the pivot, once the other is left over
  for (;;) {
    ring_fill<SC>(R, 0, unlimited, T);
    ring_fill<SC>(R, 1, unlimited, T);
    if (ring_pair<V16>(R, unlimited, T) > 0) continue;
    const bool done0 = T.qExh[0] && T.qCnt[0] == 0;
    const bool done1 = T.qExh[1] && T.qCnt[1] == 0;
    if (twinSide < 0) {
      if (done0 && done1) break;
      // one side has run out: the other's remaining points pair with twins
      // of the pivot from the side that ran out
      twinSide = done1 ? 1 : 0;
      ring_start(twinSide, kTwin, 0, sideEnd, 0, T);
      continue;
    }
    // the side paired with twins is finished (twins may be left over)
    if (twinSide == 1 ? done0 : done1) break;
    // the twins ran out first: cannot happen for a consistent pivot
    __syncthreads();
    if (threadIdx.x == 0) build_fault(A.status);
    break;
  }
  __syncthreads();
}

template <int SC, int D, bool V16>
__device__ bool cta_level(const TopArgs &A, int L, TopSmem &T)
{
  const Recs &R = A.R;
  const int nseg = 1 << L;
  const int64_t g0 = (int64_t(1) << L) - 1;
  const int tid = threadIdx.x;
  for (int s = blockIdx.x; s < nseg; s += gridDim.x) {
    load_ancestors<SC, D>(R, A.explicitDims, L, g0 + s, T.ancDim, T.ancKey);
    if (tid == 0) {
      seg_setup<SC, D>(R, A.wb, A.explicitDims, L, g0 + s, T.ancDim, T.ancKey, T.seg);
      Sel &sl = T.sel;
      sl.w = 0;
      sl.done = 0;
      sl.twins = 0;
      sl.pos = T.seg.g;
      sl.rank = uint32_t(T.seg.r);
      sel_begin_word(sl, T.seg, R.n);
      if (sl.w >= T.seg.nwords) {
        sl.done = 1;
        sl.twins = 1;
      }
    }
    __syncthreads();
    while (!T.sel.done) {
      for (int i = tid; i < kBins; i += kThreads) T.u.h.hist[i] = 0;
      __syncthreads();
      hist_set<SC>(R, T.seg, T.sel, T.u.h.hist, T.u.h.hpos);
      __syncthreads();
      find_digit(T.u.h.hist, T.sel.rank, T);
      if (tid == 0) {
        const uint32_t d = T.res[0];
        sel_advance(T.sel, T.seg, R.n, d, T.res[1], T.res[2], int64_t(T.u.h.hpos[d]));
      }
      __syncthreads();
    }
    if (tid == 0) place_pivot<SC>(A, T.seg, T.sel);
    __syncthreads();
    load_pivot_words<SC>(A, T);
    cta_split<SC, V16>(A, T);
  }
  return grid_barrier(A, T);
}

// V16: 16-byte records at a 16-byte aligned base (swapped as one vector)
template <int SC, int D, bool V16>
__global__ void __launch_bounds__(kThreads, 4) top_kernel(TopArgs A)
{
  __shared__ TopSmem T;
  for (int L = 0; L < A.G; L++) {
    const bool ok = (1 << L) <= kMultiSegs ? spread_level<SC, D, V16>(A, L, T)
                                           : cta_level<SC, D, V16>(A, L, T);
    if (!ok) return;
  }
}

// ---------------------------------------------------------------------------
// subtree phase over node sets
// ---------------------------------------------------------------------------
// subtree_body's source: the subtree's points are read from its node set
// (slot i = local level-order index i); the result is a slot per node
template <int SC, int D> struct NodeSetSrc {
  Recs R;
  const uint32_t *wb;
  int64_t s;
  int L0;
  bool explicitDims;
  uint16_t *slotOf;
  __device__ int64_t node_of(int i) const
  {
    const int j = level_of(i);
    return ((s + 1) << j) - 1 + (i - ((1 << j) - 1));
  }
  int8_t *ancDim;
  uint32_t *ancKey;
  template <class SM> __device__ void load(SM &S, int m) const
  {
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      const int64_t node = node_of(i);
#pragma unroll
      for (int d = 0; d < D; d++) S.key[d][i] = coord_key<SC>(R, node, d);
      S.idx[i] = R.idx ? R.idx[node] : uint32_t(node);
    }
    if (explicitDims) {
      load_ancestors<SC, D>(R, true, L0, s, ancDim, ancKey);
      if (threadIdx.x == 0) {
        for (int d = 0; d < D; d++) {
          S.rootLo[d] = wb[d];
          S.rootHi[d] = wb[D + d];
        }
        for (int k = 0; k < L0; k++) {
          const int64_t a = ((s + 1) >> (L0 - k)) - 1;
          const int64_t c = ((s + 1) >> (L0 - k - 1)) - 1;
          if (c == 2 * a + 1)
            S.rootHi[ancDim[k]] = ancKey[k];
          else
            S.rootLo[ancDim[k]] = ancKey[k];
        }
      }
    }
  }
  __device__ int anc_dim(int64_t a) const { return dim_at(R, a); }
  template <class SM> __device__ void settle(int64_t, int u, int piv, int, SM &) const
  {
    slotOf[u] = uint16_t(piv);
  }
};

template <int D> struct NodeSetSmem {
  SubSmem<D, kTile, kSubThreads> sub;
  uint16_t slotOf[kTile];
  uint32_t col[4][kTile];
  int8_t ancDim[kMaxLevels];
  uint32_t ancKey[kMaxLevels];
};

template <int SC, int D>
__global__ void __launch_bounds__(kSubThreads, 3) subtree_kernel(Recs R, const uint32_t *wb, int L0,
                                                                 bool explicitDims,
                                                                 const uint32_t *status)
{
  __shared__ uint32_t failed;
  if (threadIdx.x == 0) failed = *(volatile const uint32_t *)status;
  __syncthreads();
  if (failed) return;
  extern __shared__ __align__(16) uint8_t smem_raw[];
  NodeSetSmem<D> &S = *reinterpret_cast<NodeSetSmem<D> *>(smem_raw);
  const int64_t s = ((int64_t(1) << L0) - 1) + blockIdx.x;
  const int m = int(subtree_size(s, R.n));
  if (m == 0) return;
  for (int u = threadIdx.x; u < m; u += kSubThreads) S.slotOf[u] = uint16_t(u);
  NodeSetSrc<SC, D> src{R, wb, s, L0, explicitDims, S.slotOf, S.ancDim, S.ancKey};
  build::subtree_body<SC, D, kTile, kSubThreads>(src, R.n, L0, s, explicitDims, S.sub);
  __syncthreads();
  // every node takes the record of its slot, four words at a time
  const int words = R.stride >> 2;
  const int dw = explicitDims ? (R.doff >> 2) : -1;
  for (int w0 = 0; w0 < words; w0 += 4) {
    const int nw = words - w0 < 4 ? words - w0 : 4;
    for (int i = threadIdx.x; i < m; i += kSubThreads) {
      const uint32_t *r = (const uint32_t *)(R.pts + src.node_of(i) * R.stride) + w0;
      for (int c = 0; c < nw; c++) S.col[c][i] = r[c];
    }
    __syncthreads();
    for (int u = threadIdx.x; u < m; u += kSubThreads) {
      uint32_t *r = (uint32_t *)(R.pts + src.node_of(u) * R.stride) + w0;
      int from = S.slotOf[u];
      if (from >= m) from = u;  // guards memory safety only
      for (int c = 0; c < nw; c++) {
        uint32_t v = S.col[c][from];
        if (w0 + c == dw)
          v = (v & ~(R.dmask << R.dshift)) | ((uint32_t(S.sub.locDim[u]) & R.dmask) << R.dshift);
        r[c] = v;
      }
    }
    __syncthreads();
  }
}

// world bounds as keys (atomics into wb, pre-set to empty); the bitonic
// name's tags start as the input index
template <int SC, int D>
__global__ void __launch_bounds__(256) bounds_kernel(Recs R, uint32_t *wb)
{
  uint32_t lo[D], hi[D];
#pragma unroll
  for (int d = 0; d < D; d++) {
    lo[d] = 0xffffffffu;
    hi[d] = 0u;
  }
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < R.n;
       i += int64_t(gridDim.x) * blockDim.x) {
#pragma unroll
    for (int d = 0; d < D; d++) {
      const uint32_t k = coord_key<SC>(R, i, d);
      lo[d] = min(lo[d], k);
      hi[d] = max(hi[d], k);
    }
    if (R.idx) R.idx[i] = uint32_t(i);
  }
#pragma unroll
  for (int d = 0; d < D; d++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[d] = min(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
      hi[d] = max(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&wb[d], lo[d]);
      atomicMax(&wb[D + d], hi[d]);
    }
  }
}

template <int SC, int D>
__global__ void write_bounds_kernel(const uint32_t *wb, uint32_t *out)
{
  if (threadIdx.x < 2 * D) out[threadIdx.x] = Scalar<SC>::bits(wb[threadIdx.x]);
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
template <int SC, int D, bool V16>
int top_grid(int *grid)
{
  static std::mutex mu;
  static int cached[64] = {};
  int dev = 0;
  CKB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return CUKD_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(mu);
  if (!cached[dev]) {
    int perSM = 0, sms = 0;
    CKB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, top_kernel<SC, D, V16>, kThreads, 0));
    CKB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (perSM < 1) return CUKD_ERR_UNSUPPORTED;
    cached[dev] = perSM * sms;
  }
  *grid = cached[dev];
  return CUKD_OK;
}

template <int SC, int D>
int build_impl(void *pts, int64_t n, const Layout &L, void *worldBounds, cudaStream_t st,
               const cukd_mem_resource *mem, bool bitonic)
{
  const bool explicitDims = L.doff >= 0;
  TempArena arena(st, mem);
  Recs R;
  R.pts = (uint8_t *)pts;
  R.idx = nullptr;
  R.n = n;
  R.stride = L.stride;
  R.poff = L.poff;
  R.doff = explicitDims ? L.doff : -1;
  R.dshift = L.dshift;
  R.dmask = L.dmask;
  if (bitonic) CKB_TRY(arena.alloc(&R.idx, n));
  int G = 0;
  while (subtree_size((int64_t(1) << G) - 1, n) > kTile) G++;
  if (G >= kMaxLevels) return CUKD_ERR_UNSUPPORTED;

  uint32_t *small = nullptr;  // [0, 2D) world keys, [2D] status, [2D+1, +2) barrier, [+2, +2) active
  CKB_TRY(arena.alloc(&small, 2 * D + 8));
  uint32_t *wb = small;
  uint32_t *status = small + 2 * D;
  CKB_CUDA(cudaMemsetAsync(small, 0, sizeof(uint32_t) * (2 * D + 8), st));
  CKB_CUDA(cudaMemsetAsync(wb, 0xff, sizeof(uint32_t) * D, st));
  {
    const int blocks = int(std::min<int64_t>(div_up(n, 256), kNumSMs * 8));
    bounds_kernel<SC, D><<<blocks, 256, 0, st>>>(R, wb);
    CKB_CHECK_LAUNCH();
  }
  if (worldBounds) {
    write_bounds_kernel<SC, D><<<1, 32, 0, st>>>(wb, (uint32_t *)worldBounds);
    CKB_CHECK_LAUNCH();
  }
  if (G > 0) {
    TopArgs A{};
    A.R = R;
    A.wb = wb;
    A.G = G;
    A.explicitDims = explicitDims;
    A.status = status;
    A.bar = small + 2 * D + 1;
    A.active = small + 2 * D + 3;
    const int spreadLevels = std::min(G, build::ilog2_floor(kMultiSegs) + 1);
    const int nsegMax = 1 << (spreadLevels - 1);
    CKB_TRY(arena.alloc(&A.seg, nsegMax));
    CKB_TRY(arena.alloc(&A.sel, nsegMax));
    CKB_TRY(arena.alloc(&A.hist, size_t(nsegMax) * kBins));
    CKB_TRY(arena.alloc(&A.hpos, size_t(nsegMax) * kBins));
    CKB_TRY(arena.alloc(&A.tot, 4 * kMultiSegs));
    int64_t maxCh = 1;
    for (int lvl = 0; lvl < spreadLevels; lvl++) {
      const int jmax = num_levels(n) - 1 - lvl;
      int lc = kMinChunkLog;
      while ((int64_t(2) << lvl) * chunks_per_side(jmax, lc) > kMaxChunks) lc++;
      A.lc[lvl] = int8_t(lc);
      maxCh = std::max(maxCh, (int64_t(2) << lvl) * chunks_per_side(jmax, lc));
    }
    // once every spread level exists (n > 2^18) the scratch is the fixed
    // maximum; smaller trees take less
    const bool full = spreadLevels == build::ilog2_floor(kMultiSegs) + 1;
    if (full) maxCh = kMaxChunks;
    CKB_TRY(arena.alloc(&A.ccnt, maxCh));
    CKB_TRY(arena.alloc(&A.cst, maxCh));
    CKB_TRY(arena.alloc(&A.bnd, 2 * maxCh));
    CKB_CUDA(cudaMemsetAsync(A.hist, 0, sizeof(uint32_t) * size_t(nsegMax) * kBins, st));
    const bool v16 = L.stride == 16 && (reinterpret_cast<uintptr_t>(pts) & 15) == 0;
    int grid = 0;
    CKB_TRY(v16 ? (top_grid<SC, D, true>(&grid)) : (top_grid<SC, D, false>(&grid)));
    void *args[] = {&A};
    const void *fn = v16 ? (const void *)top_kernel<SC, D, true> : (const void *)top_kernel<SC, D, false>;
    CKB_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(kThreads), args, 0, st));
    count_launch();
  }
  {
    const size_t smem = sizeof(NodeSetSmem<D>);
    CKB_CUDA(cudaFuncSetAttribute(subtree_kernel<SC, D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(smem)));
    subtree_kernel<SC, D><<<unsigned(int64_t(1) << G), kSubThreads, smem, st>>>(R, wb, G, explicitDims,
                                                                               status);
    CKB_CHECK_LAUNCH();
  }
  return CUKD_OK;
}

}  // namespace inplace

int inplace_dispatch(void *pts, int64_t n, const Layout &L, void *wb, cudaStream_t st,
                     const cukd_mem_resource *mem, bool bitonic)
{
  using namespace inplace;
#define CKB_CASE(SC_, D_) \
  if (L.scalar == SC_ && L.D == D_) return build_impl<SC_, D_>(pts, n, L, wb, st, mem, bitonic);
  CKB_CASE(0, 2) CKB_CASE(0, 3) CKB_CASE(0, 4) CKB_CASE(0, 5) CKB_CASE(0, 6) CKB_CASE(0, 7)
  CKB_CASE(0, 8) CKB_CASE(1, 2) CKB_CASE(1, 3) CKB_CASE(1, 4) CKB_CASE(1, 5) CKB_CASE(1, 6)
  CKB_CASE(1, 7) CKB_CASE(1, 8)
#undef CKB_CASE
  return CUKD_ERR_UNSUPPORTED;
}

}  // namespace ckb
