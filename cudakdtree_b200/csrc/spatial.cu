// Spatial k-d tree (reference: cukd/spatial-kdtree.h) -- builder and
// traversals, sm_100a.
//
// Builder.  The reference grows the tree one level per pass: every open node
// either becomes a leaf (at most makeLeafThreshold prims, default 8) or is
// split at the centre of its prims' bounding box along the widest extent
// (first widest dim wins; a split whose centre rounds onto the box boundary
// is "degenerate" and alternates prims between the children), then every
// prim moves to a child (coord >= pos goes right) and the children's boxes
// grow atomically (:316-436).  Two of its choices depend on atomic order: the
// children's node ids (atomicAdd on a counter, :385) and which prims of a
// degenerate split go left (atomicAdd on an uninitialised counter, :424-427).
// This builder makes both canonical -- children are numbered in the order of
// their parents' ids, and the i-th prim (by prim id) of a degenerate node
// goes to side i&1 -- and otherwise follows the reference: same split rule,
// same leaf rule, node 1 kept as the reference's empty dummy, leaf prim lists
// in node-id order with prims in prim-id order (the reference's radix sort
// on node id is stable over the prim array, :577-585), bounds kept in the
// reference's int32 order-preserving float encoding (:177-192).
//
// Data layout.  Prims are kept in segments, one per open node, in prim-id
// order; a pass stably partitions each split node's segment into its two
// children's segments (two device-wide scans), so every node's prims stay
// contiguous and ordered.  One device->host read per pass decides whether
// another pass is needed (the reference reads the node count every pass).
#include <algorithm>
#include <cfloat>
#include <vector>

#include "common.cuh"
#include "query.cuh"
#include "scan.cuh"

namespace ckb {
namespace spatial {

using Node = cukd_spatial_node;

// AtomicBox encoding (spatial-kdtree.h:177-192)
__host__ __device__ inline int32_t enc(float f)
{
#ifdef __CUDA_ARCH__
  int32_t b = __float_as_int(f);
#else
  int32_t b;
  memcpy(&b, &f, 4);
#endif
  if (b & int32_t(0x80000000)) b ^= 0x7fffffff;
  return b;
}
__host__ __device__ inline float dec(int32_t b)
{
  if (b & int32_t(0x80000000)) b ^= 0x7fffffff;
#ifdef __CUDA_ARCH__
  return __int_as_float(b);
#else
  float f;
  memcpy(&f, &b, 4);
  return f;
#endif
}

struct BuildBufs {
  // per node (capacity 2n+2)
  uint32_t *count, *segBegin;
  int32_t *lo, *hi;  // [node][D], encoded
  int32_t *sdim;     // split dim of open nodes (-1 degenerate)
  float *spos;
  Node *out;
  // per open node of the current pass
  uint32_t *isSplit, *splitRank;
  // per prim position
  uint32_t *prim[2], *nodeOf[2];
  float *coord[2][4];  // the prim's coordinates, moved with it (SoA per dim)
  uint32_t *fl;        // goes-left flags -> exclusive scan
  uint32_t *total;    // scan totals / pass counters [4]
  const uint8_t *data;
  int stride, poff;
};

template <int D>
__device__ inline void load_point(const BuildBufs &b, uint32_t prim, float *p)
{
  const float *c = (const float *)(b.data + int64_t(prim) * b.stride + b.poff);
#pragma unroll
  for (int d = 0; d < D; d++) p[d] = __ldg(c + d);
}

template <int D>
__device__ inline void warp_grow(int32_t *lo, int32_t *hi, uint32_t node, bool valid,
                                 const float *p)
{
  // one atomic per (warp, node): lanes holding prims of the same node reduce
  // their encoded coordinates together
  const unsigned active = __ballot_sync(0xffffffffu, valid);
  if (!valid) return;
  const unsigned peers = __match_any_sync(active, node);
  const int leader = __ffs(peers) - 1;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 0; d < D; d++) {
    const int32_t e = enc(p[d]);
    const int32_t l = __reduce_min_sync(peers, e);
    const int32_t h = __reduce_max_sync(peers, e);
    if (lane == leader) {
      atomicMin(&lo[int64_t(node) * D + d], l);
      atomicMax(&hi[int64_t(node) * D + d], h);
    }
  }
}

// Grows the boxes of the nodes that this CTA's valid lanes carry prims to.
// When those nodes span fewer than kGrowSlots consecutive ids (always near
// the root, where every warp would otherwise hit the same few boxes), the
// warps' partial boxes are merged in shared memory first and the CTA issues
// one global atomic per (node, dim, bound); otherwise each warp issues its
// own (warp_grow).
constexpr int kGrowSlots = 64;
template <int D>
__device__ inline void block_grow(int32_t *lo, int32_t *hi, uint32_t node, bool valid,
                                  const float *p)
{
  __shared__ uint32_t nmin, nmax;
  __shared__ int32_t slo[kGrowSlots][D], shi[kGrowSlots][D];
  if (threadIdx.x == 0) {
    nmin = 0xffffffffu;
    nmax = 0u;
  }
  __syncthreads();
  if (valid) {
    atomicMin(&nmin, node);
    atomicMax(&nmax, node);
  }
  __syncthreads();
  const uint32_t n0 = nmin, n1 = nmax;
  if (n0 > n1) return;  // no valid lane in the CTA (uniform)
  if (n1 - n0 >= uint32_t(kGrowSlots)) {  // uniform
    warp_grow<D>(lo, hi, node, valid, p);
    return;
  }
  const int slots = int(n1 - n0) + 1;
  for (int i = threadIdx.x; i < slots * D; i += blockDim.x) {
    (&slo[0][0])[i] = enc(+FLT_MAX);
    (&shi[0][0])[i] = enc(-FLT_MAX);
  }
  __syncthreads();
  const unsigned active = __ballot_sync(0xffffffffu, valid);
  if (valid) {
    const unsigned peers = __match_any_sync(active, node);
    const int leader = __ffs(peers) - 1;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 0; d < D; d++) {
      const int32_t e = enc(p[d]);
      const int32_t l = __reduce_min_sync(peers, e);
      const int32_t h = __reduce_max_sync(peers, e);
      if (lane == leader) {
        atomicMin(&slo[node - n0][d], l);
        atomicMax(&shi[node - n0][d], h);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < slots * D; i += blockDim.x) {
    const int sl = i / D, d = i % D;
    const int32_t l = slo[sl][d], h = shi[sl][d];
    if (l <= h) {  // the slot's node received prims
      atomicMin(&lo[int64_t(n0 + sl) * D + d], l);
      atomicMax(&hi[int64_t(n0 + sl) * D + d], h);
    }
  }
}

template <int D>
__global__ void init_kernel(BuildBufs b, int64_t n)
{
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  const bool valid = i < n;
  float p[D];
  if (valid) {
    load_point<D>(b, uint32_t(i), p);
    b.prim[0][i] = uint32_t(i);
    b.nodeOf[0][i] = 0;
#pragma unroll
    for (int d = 0; d < D; d++) b.coord[0][d][i] = p[d];
  } else {
#pragma unroll
    for (int d = 0; d < D; d++) p[d] = 0.f;
  }
  block_grow<D>(b.lo, b.hi, 0, valid, p);
}

template <int D>
__global__ void root_setup_kernel(BuildBufs b, int64_t n)
{
  if (threadIdx.x != 0) return;
  b.count[0] = uint32_t(n);
  b.segBegin[0] = 0;
  // node 1: the reference's empty dummy (initState, :276-290)
  b.out[1].pos = 0.f;
  b.out[1].offset = 0;
  b.out[1].count = 0;
  b.out[1].dim = 0;
}

// selectSplits (:316-396) for the open nodes [pb, pe)
template <int D>
__global__ void decide_kernel(BuildBufs b, uint32_t pb, uint32_t pe, int threshold)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= pe - pb) return;
  const uint32_t node = pb + t;
  const uint32_t cnt = b.count[node];
  if (int64_t(cnt) <= threshold) {
    b.isSplit[t] = 0;
    b.out[node].offset = 0;  // leaves with prims get theirs at the end
    b.out[node].count = uint16_t(cnt);
    b.out[node].dim = 0;
    b.out[node].pos = 0.f;
    return;
  }
  float widestWidth = 0.f;
  int widestDim = -1;
  for (int d = 0; d < D; d++) {
    const float width = __fsub_rn(dec(b.hi[int64_t(node) * D + d]), dec(b.lo[int64_t(node) * D + d]));
    if (width <= widestWidth) continue;
    widestWidth = width;
    widestDim = d;
  }
  float pos = 0.f;
  if (widestDim >= 0) {
    const float l = dec(b.lo[int64_t(node) * D + widestDim]);
    const float h = dec(b.hi[int64_t(node) * D + widestDim]);
    pos = __fmul_rn(0.5f, __fadd_rn(l, h));
    if (pos == l || pos == h) widestDim = -1;
  }
  if (widestDim < 0) pos = dec(b.lo[int64_t(node) * D + 0]);
  b.sdim[node] = widestDim;
  b.spos[node] = pos;
  b.isSplit[t] = 1;
}

// children ids (parent order), split node records, empty child boxes
template <int D>
__global__ void children_kernel(BuildBufs b, uint32_t pb, uint32_t pe, uint32_t childBase)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= pe - pb || !b.isSplit[t]) return;
  const uint32_t node = pb + t;
  const uint32_t first = childBase + 2 * b.splitRank[t];
  const int dim = b.sdim[node];
  b.out[node].offset = first;
  b.out[node].count = 0;
  b.out[node].dim = int16_t(dim < 0 ? 0 : dim);
  b.out[node].pos = b.spos[node];
  for (int s = 0; s < 2; s++) {
    for (int d = 0; d < D; d++) {
      b.lo[int64_t(first + s) * D + d] = enc(+FLT_MAX);
      b.hi[int64_t(first + s) * D + d] = enc(-FLT_MAX);
    }
  }
}

// updatePrims (:398-436): side of every prim of a split node
template <int D>
__global__ void side_kernel(BuildBufs b, int64_t n, uint32_t pb, uint32_t pe, int cur)
{
  const int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= n) return;
  const uint32_t node = b.nodeOf[cur][p];
  uint32_t l = 0;
  if (node >= pb && node < pe && b.isSplit[node - pb]) {
    const int dim = b.sdim[node];
    int side;
    if (dim < 0)
      side = int((uint32_t(p) - b.segBegin[node]) & 1u);
    else
      side = b.coord[cur][dim][p] >= b.spos[node];
    l = side == 0;
  }
  b.fl[p] = l;
}

template <int D>
__global__ void move_kernel(BuildBufs b, int64_t n, uint32_t pb, uint32_t pe, int cur)
{
  const int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  const bool valid = p < n;
  bool moving = false;
  uint32_t child = 0;
  float pt[D];
#pragma unroll
  for (int d = 0; d < D; d++) pt[d] = 0.f;
  if (valid) {
    const uint32_t node = b.nodeOf[cur][p];
    const uint32_t prim = b.prim[cur][p];
    int64_t dst = p;
    uint32_t nodeOut = node;
    if (node >= pb && node < pe && b.isSplit[node - pb]) {
      const uint32_t sb = b.segBegin[node];
      const uint32_t cnt = b.count[node];
      const uint32_t nl = b.fl[sb + cnt] - b.fl[sb];
      const uint32_t first = b.out[node].offset;
      const bool isL = (b.fl[p + 1] - b.fl[p]) != 0;
      // every prim of a split node goes left or right: its right-side rank
      // is its rank in the segment minus its left-side rank
      const uint32_t lBefore = b.fl[p] - b.fl[sb];
      if (isL) {
        dst = sb + lBefore;
        nodeOut = first;
      } else {
        dst = sb + nl + (uint32_t(p) - sb - lBefore);
        nodeOut = first + 1;
      }
      moving = true;
      child = nodeOut;
#pragma unroll
      for (int d = 0; d < D; d++) {
        pt[d] = b.coord[cur][d][p];
        b.coord[cur ^ 1][d][dst] = pt[d];  // leaves' prims need no coordinates
      }
    }
    b.prim[cur ^ 1][dst] = prim;
    b.nodeOf[cur ^ 1][dst] = nodeOut;
  }
  block_grow<D>(b.lo, b.hi, child, moving, pt);
}

__global__ void child_counts_kernel(BuildBufs b, uint32_t pb, uint32_t pe)
{
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= pe - pb || !b.isSplit[t]) return;
  const uint32_t node = pb + t;
  const uint32_t sb = b.segBegin[node], cnt = b.count[node];
  const uint32_t nl = b.fl[sb + cnt] - b.fl[sb];
  const uint32_t first = b.out[node].offset;
  b.count[first] = nl;
  b.count[first + 1] = cnt - nl;
  b.segBegin[first] = sb;
  b.segBegin[first + 1] = sb + nl;
}

// leaf offsets in node-id order, then the prim list
__global__ void leaf_counts_kernel(BuildBufs b, uint32_t numNodes, uint32_t *lc)
{
  const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= numNodes) return;
  lc[node] = (node != 1 && b.out[node].count > 0) ? b.out[node].count : 0u;
}

__global__ void leaf_offsets_kernel(BuildBufs b, uint32_t numNodes, const uint32_t *off)
{
  const uint32_t node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= numNodes || node == 1) return;
  if (b.out[node].count > 0) b.out[node].offset = off[node];
}

__global__ void write_prims_kernel(BuildBufs b, int64_t n, int cur, const uint32_t *off,
                                   uint32_t *primIDs)
{
  const int64_t p = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (p >= n) return;
  const uint32_t node = b.nodeOf[cur][p];
  primIDs[off[node] + (uint32_t(p) - b.segBegin[node])] = b.prim[cur][p];
}

template <int D>
__global__ void bounds_out_kernel(BuildBufs b, float *bounds)
{
  if (threadIdx.x < D) {
    bounds[threadIdx.x] = dec(b.lo[threadIdx.x]);
    bounds[D + threadIdx.x] = dec(b.hi[threadIdx.x]);
  }
}

static int alloc_out(const cukd_mem_resource *mem, cudaStream_t st, void **p, size_t bytes)
{
  bytes = std::max<size_t>(bytes, 16);
  if (mem && mem->alloc) {
    if (mem->alloc(mem->ctx, p, bytes, st) != 0 || !*p) return CUKD_ERR_OUT_OF_MEMORY;
    return CUKD_OK;
  }
  cudaError_t e = cudaMallocAsync(p, bytes, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorMemoryAllocation ? CUKD_ERR_OUT_OF_MEMORY : CUKD_ERR_CUDA;
  }
  return CUKD_OK;
}

template <int D>
int build_impl(const void *pts, int64_t n, const Layout &L, int threshold,
               cukd_spatial_tree *tree, cudaStream_t st, const cukd_mem_resource *mem)
{
  if (threshold == 0) threshold = 8;  // spatial-kdtree.h:505-506
  if (threshold < 1 || threshold > 65535) return CUKD_ERR_INVALID_ARGUMENT;
  TempArena arena(st, mem);
  const int64_t cap = 2 * n + 2;
  BuildBufs b = {};
  b.data = (const uint8_t *)pts;
  b.stride = L.stride;
  b.poff = L.poff;
  CKB_TRY(arena.alloc(&b.count, cap));
  CKB_TRY(arena.alloc(&b.segBegin, cap));
  CKB_TRY(arena.alloc(&b.lo, cap * D));
  CKB_TRY(arena.alloc(&b.hi, cap * D));
  CKB_TRY(arena.alloc(&b.sdim, cap));
  CKB_TRY(arena.alloc(&b.spos, cap));
  CKB_TRY(arena.alloc(&b.isSplit, cap));
  CKB_TRY(arena.alloc(&b.splitRank, cap));
  for (int x = 0; x < 2; x++) {
    CKB_TRY(arena.alloc(&b.prim[x], n));
    CKB_TRY(arena.alloc(&b.nodeOf[x], n));
    for (int d = 0; d < D; d++) CKB_TRY(arena.alloc(&b.coord[x][d], n));
  }
  CKB_TRY(arena.alloc(&b.fl, n + 1));
  CKB_TRY(arena.alloc(&b.total, 4));
  Node *nodesFull = nullptr;
  CKB_TRY(arena.alloc(&nodesFull, cap));
  b.out = nodesFull;
  // the per-pass split count is read into pageable memory (a 4-byte copy
  // followed by a stream sync anyway; a pinned allocation per build cost more)
  uint32_t hostTotalVal = 0;
  uint32_t *hostTotal = &hostTotalVal;

  // root: empty box, then grown by every prim (initPrims, :300-314)
  {
    std::vector<int32_t> lo(D, enc(+FLT_MAX)), hi(D, enc(-FLT_MAX));
    CKB_CUDA(cudaMemcpyAsync(b.lo, lo.data(), sizeof(int32_t) * D, cudaMemcpyHostToDevice, st));
    CKB_CUDA(cudaMemcpyAsync(b.hi, hi.data(), sizeof(int32_t) * D, cudaMemcpyHostToDevice, st));
  }
  const unsigned nb = unsigned(std::max<int64_t>(1, div_up(n, 256)));
  init_kernel<D><<<nb, 256, 0, st>>>(b, n);
  CKB_CHECK_LAUNCH();
  root_setup_kernel<D><<<1, 32, 0, st>>>(b, n);
  CKB_CHECK_LAUNCH();

  uint32_t pb = 0, pe = 1, numNodes = 2;  // open nodes this pass: [pb, pe)
  int cur = 0;
  bool first = true;
  while (pe > pb) {
    const uint32_t m = pe - pb;
    const unsigned mb = unsigned(div_up(m, 256));
    decide_kernel<D><<<mb, 256, 0, st>>>(b, pb, pe, threshold);
    CKB_CHECK_LAUNCH();
    CKB_TRY(exclusive_scan_u32(b.isSplit, b.splitRank, m, b.total, st, &arena));
    CKB_CUDA(cudaMemcpyAsync(hostTotal, b.total, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    CKB_CUDA(cudaStreamSynchronize(st));
    const uint32_t numSplit = *hostTotal;
    if (numSplit == 0) break;
    // node 1 is the reference's dummy, so the root's children start at 2
    const uint32_t childBase = first ? 2u : pe;
    children_kernel<D><<<mb, 256, 0, st>>>(b, pb, pe, childBase);
    CKB_CHECK_LAUNCH();
    side_kernel<D><<<nb, 256, 0, st>>>(b, n, pb, pe, cur);
    CKB_CHECK_LAUNCH();
    CKB_TRY(exclusive_scan_u32(b.fl, b.fl, n + 1, nullptr, st, &arena));
    child_counts_kernel<<<mb, 256, 0, st>>>(b, pb, pe);
    CKB_CHECK_LAUNCH();
    move_kernel<D><<<nb, 256, 0, st>>>(b, n, pb, pe, cur);
    CKB_CHECK_LAUNCH();
    cur ^= 1;
    numNodes = childBase + 2 * numSplit;
    pb = childBase;
    pe = numNodes;
    first = false;
  }

  // leaf prim lists in node-id order
  uint32_t *lc = nullptr;
  CKB_TRY(arena.alloc(&lc, numNodes + 1));
  const unsigned tb = unsigned(div_up(numNodes, 256));
  leaf_counts_kernel<<<tb, 256, 0, st>>>(b, numNodes, lc);
  CKB_CHECK_LAUNCH();
  CKB_TRY(exclusive_scan_u32(lc, lc, numNodes, nullptr, st, &arena));
  leaf_offsets_kernel<<<tb, 256, 0, st>>>(b, numNodes, lc);
  CKB_CHECK_LAUNCH();

  void *nodes = nullptr, *prims = nullptr;
  CKB_TRY(alloc_out(mem, st, &nodes, sizeof(Node) * numNodes));
  const int rcP = alloc_out(mem, st, &prims, sizeof(uint32_t) * std::max<int64_t>(n, 1));
  if (rcP != CUKD_OK) {
    if (mem && mem->release) mem->release(mem->ctx, nodes, st); else cudaFreeAsync(nodes, st);
    return rcP;
  }
  write_prims_kernel<<<nb, 256, 0, st>>>(b, n, cur, lc, (uint32_t *)prims);
  CKB_CHECK_LAUNCH();
  CKB_CUDA(cudaMemcpyAsync(nodes, nodesFull, sizeof(Node) * numNodes, cudaMemcpyDeviceToDevice,
                           st));
  float *bnd = nullptr;
  CKB_TRY(arena.alloc(&bnd, 2 * D));
  bounds_out_kernel<D><<<1, 32, 0, st>>>(b, bnd);
  CKB_CHECK_LAUNCH();
  float hb[8];
  CKB_CUDA(cudaMemcpyAsync(hb, bnd, sizeof(float) * 2 * D, cudaMemcpyDeviceToHost, st));
  CKB_CUDA(cudaStreamSynchronize(st));
  tree->nodes = (Node *)nodes;
  tree->prim_ids = (uint32_t *)prims;
  tree->data = pts;
  tree->num_prims = int32_t(n);
  tree->num_nodes = int32_t(numNodes);
  tree->num_dims = D;
  for (int i = 0; i < 8; i++) tree->bounds[i] = 0.f;
  for (int d = 0; d < D; d++) {
    tree->bounds[d] = hb[d];
    tree->bounds[4 + d] = hb[D + d];
  }
  return CUKD_OK;
}

// ---------------------------------------------------------------------------
// traversals (fcp.h:256-427, knn.h:566-646 cct / 680-752 stackBased), one
// thread per query, 50-entry stack like the reference
// ---------------------------------------------------------------------------
struct SArgs {
  query::QArgs q;
  const Node *nodes;
  const uint32_t *primIDs;
  const uint8_t *data;
  int stride, poff;
  int numPrims;
  float lo[4], hi[4];
};

template <int D, int METHOD, class Res>
__global__ void __launch_bounds__(128) spatial_query_kernel(SArgs s)
{
  const query::QArgs &a = s.q;
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= a.nq) return;
  const int64_t qi = a.order ? int64_t(a.order[i]) : i;
  float q[D];
#pragma unroll
  for (int d = 0; d < D; d++) q[d] = __ldg((const float *)a.queries + qi * D + d);
  Res res(a);
  auto d2of = [&](const float *c) {
    float sum = __fmul_rn(__fsub_rn(c[0], q[0]), __fsub_rn(c[0], q[0]));
#pragma unroll
    for (int d = 1; d < D; d++)
      sum = __fadd_rn(sum, __fmul_rn(__fsub_rn(c[d], q[d]), __fsub_rn(c[d], q[d])));
    return sum;
  };
  if (s.numPrims > 0) {
    constexpr int kDepth = 50;
    int nodeSt[kDepth];
    float distSt[kDepth];
    float cornerSt[METHOD == CUKD_CCT ? kDepth : 1][D];
    int sp = 0;
    float cullDist = res.init();
    float closest[D];
    bool run = true;
    if (METHOD == CUKD_CCT) {
#pragma unroll
      for (int d = 0; d < D; d++) {
        float v = q[d];
        v = v < s.lo[d] ? s.lo[d] : v;
        v = s.hi[d] < v ? s.hi[d] : v;
        closest[d] = v;
      }
      if (d2of(closest) > cullDist) run = false;
    }
    int nodeID = 0;
    bool overflow = false;
    while (run) {
      Node node;
      for (;;) {
        node = s.nodes[nodeID];
        if (node.count) break;
        float qc = q[0];
#pragma unroll
        for (int d = 1; d < D; d++)
          if (d == node.dim) qc = q[d];
        const bool leftIsClose = qc < node.pos;
        const int lChild = int(node.offset), rChild = lChild + 1;
        const int closeChild = leftIsClose ? lChild : rChild;
        const int farChild = leftIsClose ? rChild : lChild;
        bool push;
        float fc[D];
        if (METHOD == CUKD_CCT) {
#pragma unroll
          for (int d = 0; d < D; d++) fc[d] = d == node.dim ? node.pos : closest[d];
          push = d2of(fc) < cullDist;
        } else {
          const float diff = __fsub_rn(qc, node.pos);
          const float pd2 = __fmul_rn(diff, diff);
          push = pd2 < cullDist;
          fc[0] = pd2;
        }
        if (push) {
          nodeSt[sp] = farChild;
          if (METHOD == CUKD_CCT) {
#pragma unroll
            for (int d = 0; d < D; d++) cornerSt[sp][d] = fc[d];
          } else {
            distSt[sp] = fc[0];
          }
          ++sp;
          if (sp >= kDepth) {  // the reference prints STACK OVERFLOW and returns -1
            overflow = true;
            run = false;
            break;
          }
        }
        nodeID = closeChild;
      }
      if (!run) break;
      for (int j = 0; j < node.count; j++) {
        const uint32_t primID = __ldg(s.primIDs + node.offset + j);
        float p[D];
        const float *c = (const float *)(s.data + int64_t(primID) * s.stride + s.poff);
#pragma unroll
        for (int d = 0; d < D; d++) p[d] = __ldg(c + d);
        cullDist = res.process(int32_t(primID), d2of(p));
      }
      for (;;) {
        if (sp == 0) {
          run = false;
          break;
        }
        --sp;
        if (METHOD == CUKD_CCT) {
#pragma unroll
          for (int d = 0; d < D; d++) closest[d] = cornerSt[sp][d];
          if (d2of(closest) >= cullDist) continue;
        } else {
          if (distSt[sp] >= cullDist) continue;
        }
        nodeID = nodeSt[sp];
        break;
      }
    }
    if (overflow) res.overflow();
  }
  res.write(a, qi);
}

template <class Res> struct WithOverflow : Res {
  __device__ WithOverflow(const query::QArgs &a) : Res(a) {}
  __device__ void overflow() {}
};
struct FcpOverflow : query::FcpRes<0> {
  __device__ FcpOverflow(const query::QArgs &a) : query::FcpRes<0>(a) {}
  __device__ void overflow() { id = -1; }
};

template <int D, int METHOD>
int launch_method(const SArgs &s, int kind, cudaStream_t st)
{
  using namespace query;
  const unsigned grid = unsigned(div_up(s.q.nq, 128));
#define CKB_L(...) spatial_query_kernel<D, METHOD, __VA_ARGS__><<<grid, 128, 0, st>>>(s)
  switch (kind) {
    case RES_FCP: CKB_L(FcpOverflow); break;
    case RES_FIX4: CKB_L(WithOverflow<FixedRes<0, 4>>); break;
    case RES_FIX8: CKB_L(WithOverflow<FixedRes<0, 8>>); break;
    case RES_FIX16: CKB_L(WithOverflow<FixedRes<0, 16>>); break;
    case RES_FIX32: CKB_L(WithOverflow<FixedRes<0, 32>>); break;
    case RES_HEAP128: CKB_L(WithOverflow<HeapRes<0, 128>>); break;
    case RES_HEAP1024: CKB_L(WithOverflow<HeapRes<0, 1024>>); break;
    default: return CUKD_ERR_UNSUPPORTED;
  }
#undef CKB_L
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

template <int D>
int query_impl(const SArgs &s, int method, int kind, cudaStream_t st)
{
  if (method == CUKD_CCT) return launch_method<D, CUKD_CCT>(s, kind, st);
  if (method == CUKD_STACK_BASED) return launch_method<D, CUKD_STACK_BASED>(s, kind, st);
  return CUKD_ERR_UNSUPPORTED;  // the reference has no stack-free spatial traversal
}

}  // namespace spatial

int morton_order_impl(const float *pts, int64_t n, int D, const float *bounds, int32_t *perm,
                      cudaStream_t st, const cukd_mem_resource *mem);

static int spatial_query(const cukd_spatial_tree *tree, const cukd_layout *layout,
                         const void *d_queries, int64_t nq, const cukd_query_params *p,
                         bool knn, int32_t *ids, void *d2, cudaStream_t st,
                         const cukd_mem_resource *mem)
{
  using namespace query;
  Layout L;
  if (!tree || !p || !make_layout(layout, &L) || L.scalar != CUKD_FLOAT32)
    return CUKD_ERR_INVALID_ARGUMENT;
  if (L.D != tree->num_dims) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq < 0) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq == 0) return CUKD_OK;
  if (!d_queries || !ids) return CUKD_ERR_INVALID_ARGUMENT;
  int kind = RES_FCP;
  if (knn) {
    const int k = p->k;
    if (k < 1 || k > 1024) return CUKD_ERR_INVALID_ARGUMENT;
    const bool heap = (p->flags & (CUKD_QUERY_FORCE_HEAP | CUKD_QUERY_HEAP_ORDER)) || k > 32;
    kind = heap ? (k <= 128 ? RES_HEAP128 : RES_HEAP1024)
                : (k <= 4 ? RES_FIX4 : (k <= 8 ? RES_FIX8 : (k <= 16 ? RES_FIX16 : RES_FIX32)));
  }
  spatial::SArgs s = {};
  s.q.nq = nq;
  s.q.queries = d_queries;
  s.q.k = knn ? p->k : 1;
  s.q.cutoff = p->cutoff_radius;
  s.q.heap_order = (p->flags & CUKD_QUERY_HEAP_ORDER) != 0;
  s.q.out_ids = ids;
  s.q.out_d2 = d2;
  s.nodes = tree->nodes;
  s.primIDs = tree->prim_ids;
  s.data = (const uint8_t *)tree->data;
  s.stride = L.stride;
  s.poff = L.poff;
  s.numPrims = tree->num_prims;
  for (int d = 0; d < 4; d++) {
    s.lo[d] = tree->bounds[d];
    s.hi[d] = tree->bounds[4 + d];
  }
  TempArena arena(st, mem);
  if ((p->flags & CUKD_QUERY_MORTON) && nq > 1) {
    int32_t *perm = nullptr;
    CKB_TRY(arena.alloc(&perm, nq));
    CKB_TRY(morton_order_impl((const float *)d_queries, nq, L.D, nullptr, perm, st, mem));
    s.q.order = perm;
  }
  if (L.D == 2) return spatial::query_impl<2>(s, p->method, kind, st);
  if (L.D == 3) return spatial::query_impl<3>(s, p->method, kind, st);
  if (L.D == 4) return spatial::query_impl<4>(s, p->method, kind, st);
  return CUKD_ERR_UNSUPPORTED;
}

}  // namespace ckb

extern "C" {

int cukd_spatial_build(const void *d_points, int64_t n, const cukd_layout *layout,
                       int leaf_threshold, cukd_spatial_tree *out_tree, cudaStream_t stream,
                       const cukd_mem_resource *mem)
{
  ckb::Layout L;
  if (!out_tree || !ckb::make_layout(layout, &L)) return CUKD_ERR_INVALID_ARGUMENT;
  if (L.scalar != CUKD_FLOAT32) return CUKD_ERR_UNSUPPORTED;
  if (n < 0 || n > (int64_t(1) << 30)) return CUKD_ERR_INVALID_ARGUMENT;
  if (n > 0 && !d_points) return CUKD_ERR_INVALID_ARGUMENT;
  if (L.D == 2) return ckb::spatial::build_impl<2>(d_points, n, L, leaf_threshold, out_tree, stream, mem);
  if (L.D == 3) return ckb::spatial::build_impl<3>(d_points, n, L, leaf_threshold, out_tree, stream, mem);
  if (L.D == 4) return ckb::spatial::build_impl<4>(d_points, n, L, leaf_threshold, out_tree, stream, mem);
  return CUKD_ERR_UNSUPPORTED;
}

int cukd_spatial_free(cukd_spatial_tree *tree, cudaStream_t stream, const cukd_mem_resource *mem)
{
  if (!tree) return CUKD_ERR_INVALID_ARGUMENT;
  for (void *p : {(void *)tree->nodes, (void *)tree->prim_ids}) {
    if (!p) continue;
    if (mem && mem->release)
      mem->release(mem->ctx, p, stream);
    else
      cudaFreeAsync(p, stream);
  }
  tree->nodes = nullptr;
  tree->prim_ids = nullptr;
  tree->num_nodes = 0;
  tree->num_prims = 0;
  return CUKD_OK;
}

int cukd_spatial_fcp(const cukd_spatial_tree *tree, const cukd_layout *layout,
                     const void *d_queries, int64_t nq, const cukd_query_params *params,
                     int32_t *d_out_ids, void *d_out_d2, cudaStream_t stream,
                     const cukd_mem_resource *mem)
{
  return ckb::spatial_query(tree, layout, d_queries, nq, params, false, d_out_ids, d_out_d2,
                            stream, mem);
}

int cukd_spatial_knn(const cukd_spatial_tree *tree, const cukd_layout *layout,
                     const void *d_queries, int64_t nq, const cukd_query_params *params,
                     int32_t *d_out_ids, void *d_out_d2, cudaStream_t stream,
                     const cukd_mem_resource *mem)
{
  return ckb::spatial_query(tree, layout, d_queries, nq, params, true, d_out_ids, d_out_d2,
                            stream, mem);
}

}  // extern "C"
