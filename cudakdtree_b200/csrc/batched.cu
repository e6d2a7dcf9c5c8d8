// Batched clouds: thousands of independent float clouds of uneven size,
// built and queried together (no reference counterpart; the reference
// builds one tree per call, builder.h:108-122).
//
// Plan (host, once per set of sizes): for every top-down level the list of
// (cloud, subtree) work items of the clouds that still have subtrees above
// the tile size, the links from each item to its children's items, and the
// subtree-phase items split into three tile classes (512 / 1024 / 2048
// points) sorted largest first.  All device memory is allocated here.
//
// Run (device only, no host synchronisation, no allocation):
//   extract -> per-cloud bounds -> per level: hist / select / partition /
//   resolve over all clouds' items -> one persistent subtree launch per
//   tile class (concurrent graph branches) -> finalize -> per-cloud Morton
//   keys + radix sort -> fast kNN over every query, each against its own
//   cloud -> reference-order re-run of the boundary-tie queries.
// cukd_batch_run records that sequence once as a CUDA graph and replays it.
//
// Autotuner: times the build per tile class threshold, then the query per
// (block size, queries per thread, Morton on/off), on the caller's data,
// and installs the fastest.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "fast.cuh"
#include "forest.cuh"
#include "query.cuh"
#include "sort.cuh"

namespace ckb {

namespace batch {

__global__ void fill_cloud_ids_kernel(const int64_t *__restrict__ qoff, int32_t *qcloud)
{
  const int c = blockIdx.x;
  const int64_t b = qoff[c], e = qoff[c + 1];
  for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) qcloud[i] = c;
}

// key = cloud << (bits * D) | Morton code of the query inside its cloud's box
__global__ void forest_morton_kernel(const float *__restrict__ q, int64_t nq, int D,
                                     const int32_t *__restrict__ qcloud,
                                     const float *__restrict__ cbounds, int bits,
                                     uint32_t *keys, uint32_t *vals)
{
  const float cells = float(1u << bits);
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nq;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int c = qcloud[i];
    const float *bx = cbounds + int64_t(c) * 2 * D;
    uint32_t code = 0;
    for (int d = 0; d < D; d++) {
      const float lo = bx[d], hi = bx[D + d];
      const float scale = hi > lo ? cells / (hi - lo) : 0.f;
      const float x = (q[i * D + d] - lo) * scale;
      const uint32_t cell = x >= 0.f ? (x < cells ? uint32_t(x) : (1u << bits) - 1u) : 0u;
      for (int b = 0; b < bits; b++) code |= ((cell >> b) & 1u) << (b * D + (D - 1 - d));
    }
    keys[i] = (uint32_t(c) << (bits * D)) | code;
    vals[i] = uint32_t(i);
  }
}

// Per-cloud Morton order in shared memory: one CTA per cloud sorts its
// queries' (code << 32 | local index) keys with a bitonic network and writes
// the cloud's slice of the visiting order.  Needs <= kSegSortMax queries
// per cloud (larger clouds take the global radix sort).
constexpr int kSegSortMax = 8192;
constexpr int kSegSortThreads = 512;

__global__ void __launch_bounds__(kSegSortThreads) cloud_morton_sort_kernel(
    const float *__restrict__ q, int D, const int64_t *__restrict__ qoff,
    const float *__restrict__ cbounds, int32_t *order)
{
  extern __shared__ unsigned long long keys[];
  const int c = blockIdx.x;
  const int64_t b = qoff[c];
  const int m = int(qoff[c + 1] - b);
  if (m == 0) return;
  int P = 1;
  while (P < m) P <<= 1;
  const int bits = 30 / D;
  const float cells = float(1u << bits);
  float lo[4], scale[4];
  for (int d = 0; d < D; d++) {
    const float l = cbounds[int64_t(c) * 2 * D + d], h = cbounds[int64_t(c) * 2 * D + D + d];
    lo[d] = l;
    scale[d] = h > l ? cells / (h - l) : 0.f;
  }
  for (int i = threadIdx.x; i < P; i += blockDim.x) {
    unsigned long long k = ~0ull;
    if (i < m) {
      uint32_t code = 0;
      for (int d = 0; d < D; d++) {
        const float x = (q[(b + i) * D + d] - lo[d]) * scale[d];
        const uint32_t cell = x >= 0.f ? (x < cells ? uint32_t(x) : (1u << bits) - 1u) : 0u;
        for (int bb = 0; bb < bits; bb++) code |= ((cell >> bb) & 1u) << (bb * D + (D - 1 - d));
      }
      k = ((unsigned long long)code << 32) | uint32_t(i);
    }
    keys[i] = k;
  }
  __syncthreads();
  for (int k = 2; k <= P; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < (P >> 1); t += blockDim.x) {
        const int i = 2 * j * (t / j) + (t % j);
        const int l = i + j;
        const unsigned long long x = keys[i], y = keys[l];
        const bool up = (i & k) == 0;
        if ((x > y) == up) {
          keys[i] = y;
          keys[l] = x;
        }
      }
      __syncthreads();
    }
  for (int i = threadIdx.x; i < m; i += blockDim.x)
    order[b + i] = int32_t(b + int64_t(uint32_t(keys[i])));
}

struct HostLists {
  int numLevels = 0;
  std::vector<int32_t> lvCloud[kForestMaxLevels], lvLocal[kForestMaxLevels],
      lvChild[kForestMaxLevels];
  int nb[kForestMaxLevels], cps[kForestMaxLevels];
  int64_t maxSeg[kForestMaxLevels];
  std::vector<int32_t> rootItem;
  std::vector<int32_t> subCloud[3], subLocal[3];
  std::vector<int8_t> subLevel[3];
  int64_t maxItems = 0, histCap = 0;
};

// work lists of a forest whose subtree phase takes subtrees of <= tile points
static void derive_lists(const std::vector<int64_t> &off, int tile, HostLists &h)
{
  const int64_t B = int64_t(off.size()) - 1;
  std::vector<int> G(B, 0);
  int maxG = 0;
  for (int64_t c = 0; c < B; c++) {
    const int64_t n = off[c + 1] - off[c];
    int g = 0;
    while (subtree_size((int64_t(1) << g) - 1, n) > tile) g++;
    G[c] = g;
    maxG = std::max(maxG, g);
  }
  h = HostLists();
  h.numLevels = maxG;
  h.rootItem.assign(B, -1);
  std::vector<int64_t> first(B, -1), nextFirst(B, -1);
  for (int l = 0; l < maxG; l++) {
    // items of level l, cloud by cloud; and where level l+1 starts per cloud
    int64_t cnt = 0, cntNext = 0;
    int64_t maxSeg = 0;
    for (int64_t c = 0; c < B; c++) {
      if (G[c] > l) {
        first[c] = cnt;
        cnt += int64_t(1) << l;
        maxSeg = std::max(maxSeg, subtree_size((int64_t(1) << l) - 1, off[c + 1] - off[c]));
      }
      if (G[c] > l + 1) {
        nextFirst[c] = cntNext;
        cntNext += int64_t(1) << (l + 1);
      }
    }
    auto &vc = h.lvCloud[l], &vl = h.lvLocal[l], &vh = h.lvChild[l];
    vc.reserve(cnt);
    vl.reserve(cnt);
    vh.reserve(cnt);
    for (int64_t c = 0; c < B; c++) {
      if (G[c] <= l) continue;
      if (l == 0) h.rootItem[c] = int32_t(first[c]);
      for (int64_t j = 0; j < (int64_t(1) << l); j++) {
        vc.push_back(int32_t(c));
        vl.push_back(int32_t(j));
        vh.push_back(G[c] > l + 1 ? int32_t(nextFirst[c] + 2 * j) : -1);
      }
    }
    h.nb[l] = level_bins(maxSeg);
    h.cps[l] = int(div_up(std::max<int64_t>(maxSeg, 1), kLevelChunk));
    h.maxSeg[l] = maxSeg;
    h.maxItems = std::max(h.maxItems, cnt);
    h.histCap = std::max(h.histCap, cnt * h.nb[l]);
  }
  struct Item {
    int32_t c, j;
    int8_t L0;
    int32_t m;
  };
  std::vector<Item> items[3];
  for (int64_t c = 0; c < B; c++) {
    const int64_t n = off[c + 1] - off[c];
    const int L0 = G[c];
    for (int64_t j = 0; j < (int64_t(1) << L0); j++) {
      const int64_t m = subtree_size(((int64_t(1) << L0) - 1) + j, n);
      if (m <= 0) continue;
      int cls = 0;
      while (cls < 2 && m > kForestTiles[cls]) cls++;
      items[cls].push_back(Item{int32_t(c), int32_t(j), int8_t(L0), int32_t(m)});
    }
  }
  for (int k = 0; k < 3; k++) {
    std::stable_sort(items[k].begin(), items[k].end(),
                     [](const Item &a, const Item &b) { return a.m > b.m; });
    for (const Item &it : items[k]) {
      h.subCloud[k].push_back(it.c);
      h.subLocal[k].push_back(it.j);
      h.subLevel[k].push_back(it.L0);
    }
  }
}

}  // namespace batch

}  // namespace ckb

struct cukd_batch_plan_s {
  int D = 3;
  int device = 0;
  int64_t B = 0, total = 0, nq = 0;
  cukd_query_params params{};
  bool fcp = false;
  int kind = 0;
  std::vector<int64_t> poff, qoff;
  // device arrays
  std::vector<void *> blocks;
  int64_t *d_poff = nullptr, *d_cloudN = nullptr, *d_qoff = nullptr;
  int32_t *d_qcloud = nullptr;
  float *d_bounds = nullptr;
  uint32_t *mkeys = nullptr, *mvals = nullptr, *mkeys2 = nullptr, *mvals2 = nullptr;
  uint32_t *mcounts = nullptr;
  int32_t *fb_list = nullptr;
  int64_t maxCloudQueries = 0;  // <= kSegSortMax: per-cloud Morton sort in shared memory
  int *ctr = nullptr;       // [0..1] fast-path counters, [2..4] subtree work counters
  void *lists = nullptr;    // current forest work lists (one block)
  float *tune_pts = nullptr;
  ckb::ForestBuild fb;
  int tile = 2048;
  int subGridFor[3] = {0, 0, 0};
  cukd_batch_tuning tuning{};
  unsigned long long tuningVersion = 0;
  cudaStream_t cap = nullptr, side[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaGraphExec_t exec = nullptr;
  const void *graphKey[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  unsigned long long graphVersion = ~0ull;
  long long graphKernels = 0;
};

namespace ckb {
namespace batch {

template <typename T>
static int dalloc(cukd_batch_plan_s *p, T **out, size_t count)
{
  void *q = nullptr;
  if (cudaMalloc(&q, std::max<size_t>(16, count * sizeof(T))) != cudaSuccess) {
    cudaGetLastError();
    return CUKD_ERR_OUT_OF_MEMORY;
  }
  p->blocks.push_back(q);
  *out = (T *)q;
  return CUKD_OK;
}

static void drop_graph(cukd_batch_plan_s *p)
{
  if (p->exec) cudaGraphExecDestroy(p->exec);
  p->exec = nullptr;
  p->graphVersion = ~0ull;
}

// uploads the work lists of `tile` and points the ForestBuild at them
static int install_tile(cukd_batch_plan_s *p, int tile)
{
  HostLists h;
  derive_lists(p->poff, tile, h);
  if (h.maxItems > 0 && !p->fb.ws) return CUKD_ERR_INVALID_ARGUMENT;
  size_t words = size_t(p->B);
  for (int l = 0; l < h.numLevels; l++) words += 3 * h.lvCloud[l].size();
  for (int k = 0; k < 3; k++) words += 2 * h.subCloud[k].size() + (h.subLevel[k].size() + 3) / 4;
  std::vector<int32_t> blob;
  blob.reserve(words + 8);
  std::vector<size_t> at;
  auto put = [&](const void *src, size_t bytes) {
    at.push_back(blob.size());
    const size_t w = (bytes + 3) / 4;
    const size_t o = blob.size();
    blob.resize(o + w, 0);
    if (bytes) memcpy(blob.data() + o, src, bytes);
  };
  put(h.rootItem.data(), h.rootItem.size() * 4);
  for (int l = 0; l < h.numLevels; l++) {
    put(h.lvCloud[l].data(), h.lvCloud[l].size() * 4);
    put(h.lvLocal[l].data(), h.lvLocal[l].size() * 4);
    put(h.lvChild[l].data(), h.lvChild[l].size() * 4);
  }
  for (int k = 0; k < 3; k++) {
    put(h.subCloud[k].data(), h.subCloud[k].size() * 4);
    put(h.subLocal[k].data(), h.subLocal[k].size() * 4);
    put(h.subLevel[k].data(), h.subLevel[k].size());
  }
  void *d = nullptr;
  if (cudaMalloc(&d, std::max<size_t>(16, blob.size() * 4)) != cudaSuccess) {
    cudaGetLastError();
    return CUKD_ERR_OUT_OF_MEMORY;
  }
  if (cudaMemcpy(d, blob.data(), blob.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
    set_cuda_error(cudaGetLastError());
    cudaFree(d);
    return CUKD_ERR_CUDA;
  }
  if (p->lists) cudaFree(p->lists);
  p->lists = d;
  const int32_t *base = (const int32_t *)d;
  size_t x = 0;
  ForestBuild &f = p->fb;
  f.rootItem = base + at[x++];
  f.numLevels = h.numLevels;
  for (int l = 0; l < h.numLevels; l++) {
    ForestLevel &L = f.level[l];
    L.items = int(h.lvCloud[l].size());
    L.nb = h.nb[l];
    L.chunksPerSeg = h.cps[l];
    L.maxSeg = h.maxSeg[l];
    L.cloud = base + at[x++];
    L.local = base + at[x++];
    L.child = base + at[x++];
  }
  for (int k = 0; k < 3; k++) {
    ForestSubtrees &S = f.sub[k];
    S.items = int(h.subCloud[k].size());
    S.cloud = base + at[x++];
    S.local = base + at[x++];
    S.level = (const int8_t *)(base + at[x++]);
    S.cloudBase = p->d_poff;
    S.cloudN = p->d_cloudN;
    S.counter = p->ctr + 2 + k;
    f.subGrid[k] = p->subGridFor[k];
  }
  p->tile = tile;
  return CUKD_OK;
}

static int check_tuning(const cukd_batch_tuning &t)
{
  if (t.build_tile != 512 && t.build_tile != 1024 && t.build_tile != 2048)
    return CUKD_ERR_INVALID_ARGUMENT;
  if (t.block_size < 32 || t.block_size > 512 || t.block_size % 32) return CUKD_ERR_INVALID_ARGUMENT;
  if (t.queries_per_thread != 1 && t.queries_per_thread != 2 && t.queries_per_thread != 4)
    return CUKD_ERR_INVALID_ARGUMENT;
  if (t.morton != 0 && t.morton != 1) return CUKD_ERR_INVALID_ARGUMENT;
  return CUKD_OK;
}

static int build_impl(cukd_batch_plan_s *p, float *pts, float *bounds, cudaStream_t st)
{
  if (p->total > 0 && !pts) return CUKD_ERR_INVALID_ARGUMENT;
  if (p->tile != p->tuning.build_tile) CKB_TRY(install_tile(p, p->tuning.build_tile));
  return forest_build(p->fb, pts, bounds ? bounds : p->d_bounds, st, p->side, p->ev);
}

static int query_impl(cukd_batch_plan_s *p, const float *pts, const float *bounds,
                      const float *queries, int32_t *ids, float *d2, cudaStream_t st)
{
  using namespace query;
  if (p->nq == 0) return CUKD_OK;
  if (!queries || !ids || (p->total > 0 && !pts)) return CUKD_ERR_INVALID_ARGUMENT;
  if (p->params.method == CUKD_CCT && !bounds) return CUKD_ERR_INVALID_ARGUMENT;
  const int D = p->D;
  QArgs a = {};
  a.tree = (const uint8_t *)pts;
  a.n = 0;
  a.stride = 4 * D;
  a.poff = 0;
  a.doff = -1;
  a.queries = queries;
  a.nq = p->nq;
  a.k = p->fcp ? 1 : p->params.k;
  a.cutoff = p->params.cutoff_radius;
  a.cutoff_d2 = p->params.cutoff_d2;
  a.eps = p->params.eps;
  a.heap_order = (p->params.flags & CUKD_QUERY_HEAP_ORDER) != 0;
  a.out_ids = ids;
  a.out_d2 = d2;
  a.block_size = p->tuning.block_size;
  a.q_cloud = p->d_qcloud;
  a.cloud_base = p->d_poff;
  a.cloud_bounds = bounds;
  a.queries_per_thread = p->tuning.queries_per_thread;
  // per-cloud Morton order: cloud id in the high bits, the code below
  int cloudBits = 0;
  while ((int64_t(1) << cloudBits) < p->B) cloudBits++;
  const int bits = std::min(10, (32 - cloudBits) / D);
  if (p->tuning.morton && bounds && p->nq > 1 && p->maxCloudQueries <= kSegSortMax) {
    int P = 1;
    while (P < p->maxCloudQueries) P <<= 1;
    cloud_morton_sort_kernel<<<unsigned(p->B), kSegSortThreads, size_t(P) * 8, st>>>(
        queries, D, p->d_qoff, bounds, (int32_t *)p->mvals);
    CKB_CHECK_LAUNCH();
    a.order = (const int32_t *)p->mvals;
  } else if (p->tuning.morton && bounds && p->nq > 1 && bits >= 1) {
    const int blocks = int(std::max<int64_t>(1, std::min<int64_t>(div_up(p->nq, 256), kNumSMs * 8)));
    forest_morton_kernel<<<blocks, 256, 0, st>>>(queries, p->nq, D, p->d_qcloud, bounds, bits,
                                                 p->mkeys, p->mvals);
    CKB_CHECK_LAUNCH();
    CKB_TRY(radix_sort_pairs_ws(p->mkeys, p->mvals, p->mkeys2, p->mvals2, p->nq,
                                cloudBits + bits * D, p->mcounts, st));
    a.order = (const int32_t *)p->mvals;
  }
  const bool fastOk = !p->fcp && !a.heap_order && !(p->params.flags & CUKD_QUERY_REFERENCE_ORDER) &&
                      p->params.k >= 2 &&
                      p->params.k <= 128;
  if (fastOk) {
    fast::FastArgs fa = {};
    fa.q = a;
    fa.kk = p->params.k;
    fa.fcp = false;
    CKB_CUDA(cudaMemsetAsync(p->ctr, 0, 2 * sizeof(int), st));
    fa.work = p->ctr;
    fa.fb_count = p->ctr + 1;
    fa.fb_list = p->fb_list;
    CKB_TRY(run_fast(fa, D, st));
    if (p->params.d_reordered_count)
      CKB_CUDA(cudaMemcpyAsync(p->params.d_reordered_count, fa.fb_count, sizeof(int),
                               cudaMemcpyDeviceToDevice, st));
    QArgs b = a;
    b.order = p->fb_list;
    b.count_ptr = fa.fb_count;
    b.block_size = std::min(b.block_size, 256);  // reference-order kernels: <= 256 threads
    return run_query(b, CUKD_FLOAT32, D, p->params.method, p->kind, st);
  }
  a.block_size = std::min(a.block_size, 256);
  return run_query(a, CUKD_FLOAT32, D, p->params.method, p->kind, st);
}

static float median(std::vector<float> v)
{
  std::sort(v.begin(), v.end());
  return v.empty() ? 0.f : v[v.size() / 2];
}

}  // namespace batch
}  // namespace ckb

extern "C" {

int cukd_batch_plan_create(cukd_batch_plan **out, int num_dims, int64_t num_clouds,
                           const int64_t *h_point_offsets, const int64_t *h_query_offsets,
                           const cukd_query_params *params)
{
  using namespace ckb;
  using namespace ckb::batch;
  if (!out) return CUKD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (num_dims < 2 || num_dims > 4 || num_clouds < 0 || !params) return CUKD_ERR_INVALID_ARGUMENT;
  if (num_clouds > 0 && (!h_point_offsets || !h_query_offsets)) return CUKD_ERR_INVALID_ARGUMENT;
  if (params->method < CUKD_STACK_BASED || params->method > CUKD_CCT) return CUKD_ERR_INVALID_ARGUMENT;
  if (params->k < 0 || params->k > 1024) return CUKD_ERR_INVALID_ARGUMENT;
  const int64_t lim = (int64_t(1) << 31) - 1;
  if (num_clouds > lim) return CUKD_ERR_INVALID_ARGUMENT;
  if (num_clouds > 0 && (h_point_offsets[0] != 0 || h_query_offsets[0] != 0))
    return CUKD_ERR_INVALID_ARGUMENT;
  for (int64_t c = 0; c < num_clouds; c++)
    if (h_point_offsets[c + 1] < h_point_offsets[c] || h_query_offsets[c + 1] < h_query_offsets[c])
      return CUKD_ERR_INVALID_ARGUMENT;
  const int64_t total = num_clouds ? h_point_offsets[num_clouds] : 0;
  const int64_t nq = num_clouds ? h_query_offsets[num_clouds] : 0;
  if (total > lim || nq > lim) return CUKD_ERR_UNSUPPORTED;

  cukd_batch_plan_s *p = new cukd_batch_plan_s();
  auto fail = [&](int rc) {
    cukd_batch_plan_destroy(p);
    return rc;
  };
  cudaGetDevice(&p->device);
  p->D = num_dims;
  p->B = num_clouds;
  p->total = total;
  p->nq = nq;
  p->params = *params;
  p->fcp = params->k == 0;
  if (p->fcp) {
    p->kind = query::RES_FCP;
  } else {
    const int k = params->k;
    const bool heap = (params->flags & (CUKD_QUERY_FORCE_HEAP | CUKD_QUERY_HEAP_ORDER)) || k > 32;
    if (heap)
      p->kind = k <= 128 ? query::RES_HEAP128 : query::RES_HEAP1024;
    else
      p->kind = k <= 4 ? query::RES_FIX4
                       : (k <= 8 ? query::RES_FIX8 : (k <= 16 ? query::RES_FIX16 : query::RES_FIX32));
  }
  p->poff.assign(h_point_offsets, h_point_offsets + (num_clouds + 1));
  p->qoff.assign(h_query_offsets, h_query_offsets + (num_clouds + 1));
  if (num_clouds == 0) {
    p->poff.assign(1, 0);
    p->qoff.assign(1, 0);
  }
  p->tuning.build_tile = 2048;
  p->tuning.block_size = 128;
  p->tuning.queries_per_thread = 1;
  p->tuning.morton = 1;
  int rc = CUKD_OK;
  auto T = [&](int r) {
    if (rc == CUKD_OK) rc = r;
  };
  const int64_t B = num_clouds;
  std::vector<int64_t> cn(std::max<int64_t>(B, 1), 0);
  for (int64_t c = 0; c < B; c++) cn[c] = p->poff[c + 1] - p->poff[c];
  T(dalloc(p, &p->d_poff, B + 1));
  T(dalloc(p, &p->d_qoff, B + 1));
  T(dalloc(p, &p->d_cloudN, std::max<int64_t>(B, 1)));
  T(dalloc(p, &p->d_qcloud, std::max<int64_t>(nq, 1)));
  T(dalloc(p, &p->d_bounds, std::max<int64_t>(B, 1) * 2 * num_dims));
  T(dalloc(p, &p->mkeys, std::max<int64_t>(nq, 1)));
  T(dalloc(p, &p->mvals, std::max<int64_t>(nq, 1)));
  T(dalloc(p, &p->mkeys2, std::max<int64_t>(nq, 1)));
  T(dalloc(p, &p->mvals2, std::max<int64_t>(nq, 1)));
  T(dalloc(p, &p->mcounts, radix_sort_counts(std::max<int64_t>(nq, 1))));
  T(dalloc(p, &p->fb_list, std::max<int64_t>(nq, 1)));
  T(dalloc(p, &p->ctr, 8));
  if (rc != CUKD_OK) return fail(rc);
  if (cudaMemcpy(p->d_poff, p->poff.data(), 8 * (B + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(p->d_qoff, p->qoff.data(), 8 * (B + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(p->d_cloudN, cn.data(), 8 * cn.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_cuda_error(cudaGetLastError());
    return fail(CUKD_ERR_CUDA);
  }
  if (B > 0 && nq > 0) {
    fill_cloud_ids_kernel<<<unsigned(B), 256>>>(p->d_qoff, p->d_qcloud);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
      set_cuda_error(e);
      return fail(CUKD_ERR_CUDA);
    }
    count_launch();
  }
  // forest workspace sized for the largest of the tile choices
  p->fb.D = num_dims;
  p->fb.total = total;
  p->fb.numClouds = B;
  p->fb.cloudBase = p->d_poff;
  p->fb.cloudN = p->d_cloudN;
  int64_t maxItems = 0, histCap = 0;
  for (int t = 0; t < 3; t++) {
    HostLists h;
    derive_lists(p->poff, kForestTiles[t], h);
    maxItems = std::max(maxItems, h.maxItems);
    histCap = std::max(histCap, h.histCap);
  }
  for (int64_t c = 0; c < B; c++)
    p->maxCloudQueries = std::max(p->maxCloudQueries, p->qoff[c + 1] - p->qoff[c]);
  if (cudaFuncSetAttribute(cloud_morton_sort_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           kSegSortMax * 8) != cudaSuccess) {
    set_cuda_error(cudaGetLastError());
    return fail(CUKD_ERR_CUDA);
  }
  int sms = kNumSMs;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
  for (int c = 0; c < 3; c++) p->subGridFor[c] = sms * forest_subtree_occupancy(num_dims, c);
  rc = forest_workspace_create(&p->fb, maxItems, histCap);
  if (rc != CUKD_OK) return fail(rc);
  rc = install_tile(p, p->tuning.build_tile);
  if (rc != CUKD_OK) return fail(rc);
  if (cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking) != cudaSuccess) return fail(CUKD_ERR_CUDA);
  for (int i = 0; i < 3; i++)
    if (cudaStreamCreateWithFlags(&p->side[i], cudaStreamNonBlocking) != cudaSuccess)
      return fail(CUKD_ERR_CUDA);
  for (int i = 0; i < 4; i++)
    if (cudaEventCreateWithFlags(&p->ev[i], cudaEventDisableTiming) != cudaSuccess)
      return fail(CUKD_ERR_CUDA);
  *out = p;
  return CUKD_OK;
}

int cukd_batch_plan_destroy(cukd_batch_plan *p)
{
  if (!p) return CUKD_OK;
  cudaDeviceSynchronize();
  ckb::batch::drop_graph(p);
  ckb::forest_workspace_destroy(&p->fb);
  if (p->lists) cudaFree(p->lists);
  if (p->tune_pts) cudaFree(p->tune_pts);
  for (void *b : p->blocks) cudaFree(b);
  for (int i = 0; i < 4; i++)
    if (p->ev[i]) cudaEventDestroy(p->ev[i]);
  for (int i = 0; i < 3; i++)
    if (p->side[i]) cudaStreamDestroy(p->side[i]);
  if (p->cap) cudaStreamDestroy(p->cap);
  cudaGetLastError();
  delete p;
  return CUKD_OK;
}

int cukd_batch_get_tuning(const cukd_batch_plan *p, cukd_batch_tuning *out)
{
  if (!p || !out) return CUKD_ERR_INVALID_ARGUMENT;
  *out = p->tuning;
  return CUKD_OK;
}

int cukd_batch_set_tuning(cukd_batch_plan *p, const cukd_batch_tuning *t)
{
  using namespace ckb::batch;
  if (!p || !t) return CUKD_ERR_INVALID_ARGUMENT;
  CKB_TRY(check_tuning(*t));
  const float bm = p->tuning.build_ms, qm = p->tuning.query_ms;
  p->tuning = *t;
  p->tuning.build_ms = bm;
  p->tuning.query_ms = qm;
  p->tuningVersion++;
  drop_graph(p);
  return CUKD_OK;
}

int cukd_batch_build(cukd_batch_plan *p, float *d_points, float *d_cloud_bounds,
                     cudaStream_t stream)
{
  if (!p) return CUKD_ERR_INVALID_ARGUMENT;
  return ckb::batch::build_impl(p, d_points, d_cloud_bounds, stream);
}

int cukd_batch_query(cukd_batch_plan *p, const float *d_points, const float *d_cloud_bounds,
                     const float *d_queries, int32_t *d_out_ids, float *d_out_d2,
                     cudaStream_t stream)
{
  if (!p) return CUKD_ERR_INVALID_ARGUMENT;
  return ckb::batch::query_impl(p, d_points, d_cloud_bounds, d_queries, d_out_ids, d_out_d2,
                                stream);
}

int cukd_batch_run(cukd_batch_plan *p, float *d_points, float *d_cloud_bounds,
                   const float *d_queries, int32_t *d_out_ids, float *d_out_d2,
                   cudaStream_t stream)
{
  using namespace ckb;
  using namespace ckb::batch;
  if (!p) return CUKD_ERR_INVALID_ARGUMENT;
  if ((p->total > 0 && !d_points) || (p->nq > 0 && (!d_queries || !d_out_ids)))
    return CUKD_ERR_INVALID_ARGUMENT;
  float *bounds = d_cloud_bounds ? d_cloud_bounds : p->d_bounds;
  const void *key[6] = {d_points, bounds, d_queries, d_out_ids, d_out_d2,
                        p->params.d_reordered_count};
  bool same = p->exec && p->graphVersion == p->tuningVersion;
  for (int i = 0; i < 6 && same; i++) same = key[i] == p->graphKey[i];
  if (!same) {
    drop_graph(p);
    if (p->tile != p->tuning.build_tile) CKB_TRY(install_tile(p, p->tuning.build_tile));
    const unsigned long long before = launch_count();
    CKB_CUDA(cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal));
    int rc = build_impl(p, d_points, bounds, p->cap);
    if (rc == CUKD_OK) rc = query_impl(p, d_points, bounds, d_queries, d_out_ids, d_out_d2, p->cap);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(p->cap, &g);
    add_launches(-(long long)(launch_count() - before));
    if (rc != CUKD_OK || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      if (rc == CUKD_OK) {
        set_cuda_error(e);
        rc = CUKD_ERR_CUDA;
      }
      cudaGetLastError();
      return rc;
    }
    size_t nn = 0;
    cudaGraphGetNodes(g, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if (nn) cudaGraphGetNodes(g, nodes.data(), &nn);
    long long kernels = 0;
    for (cudaGraphNode_t nd : nodes) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) kernels++;
    }
    const cudaError_t ie = cudaGraphInstantiate(&p->exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      p->exec = nullptr;
      set_cuda_error(ie);
      return CUKD_ERR_CUDA;
    }
    p->graphKernels = kernels;
    p->graphVersion = p->tuningVersion;
    for (int i = 0; i < 6; i++) p->graphKey[i] = key[i];
  }
  CKB_CUDA(cudaGraphLaunch(p->exec, stream));
  add_launches(p->graphKernels);
  return CUKD_OK;
}

int cukd_batch_autotune(cukd_batch_plan *p, const float *d_points, const float *d_queries,
                        int reps, cukd_batch_tuning *out, cudaStream_t st)
{
  using namespace ckb;
  using namespace ckb::batch;
  if (!p) return CUKD_ERR_INVALID_ARGUMENT;
  if ((p->total > 0 && !d_points) || (p->nq > 0 && !d_queries)) return CUKD_ERR_INVALID_ARGUMENT;
  reps = std::max(3, reps);
  const size_t ptsBytes = size_t(p->total) * p->D * sizeof(float);
  if (!p->tune_pts && cudaMalloc(&p->tune_pts, std::max<size_t>(16, ptsBytes)) != cudaSuccess) {
    cudaGetLastError();
    p->tune_pts = nullptr;
    return CUKD_ERR_OUT_OF_MEMORY;
  }
  const int kk = p->fcp ? 1 : p->params.k;
  int32_t *ids = nullptr;
  float *d2 = nullptr;
  if (cudaMalloc(&ids, std::max<size_t>(16, size_t(p->nq) * kk * 4)) != cudaSuccess ||
      cudaMalloc(&d2, std::max<size_t>(16, size_t(p->nq) * kk * 4)) != cudaSuccess) {
    cudaGetLastError();
    if (ids) cudaFree(ids);
    return CUKD_ERR_OUT_OF_MEMORY;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cukd_batch_tuning saved = p->tuning;
  cukd_batch_tuning best = p->tuning;
  int rc = CUKD_OK;
  auto timed = [&](auto &&fn, float *ms) -> int {
    CKB_CUDA(cudaEventRecord(e0, st));
    CKB_TRY(fn());
    CKB_CUDA(cudaEventRecord(e1, st));
    CKB_CUDA(cudaEventSynchronize(e1));
    CKB_CUDA(cudaEventElapsedTime(ms, e0, e1));
    return CUKD_OK;
  };
  auto restore = [&]() -> int {
    if (ptsBytes)
      CKB_CUDA(cudaMemcpyAsync(p->tune_pts, d_points, ptsBytes, cudaMemcpyDeviceToDevice, st));
    return CUKD_OK;
  };
  // 1. build: the subtree tile
  float bestBuild = 3.4e38f;
  for (int t = 0; t < 3 && rc == CUKD_OK; t++) {
    p->tuning.build_tile = kForestTiles[t];
    rc = install_tile(p, kForestTiles[t]);  // host work, outside the timed region
    std::vector<float> ms;
    for (int r = 0; r < reps && rc == CUKD_OK; r++) {
      rc = restore();
      float m = 0.f;
      if (rc == CUKD_OK)
        rc = timed([&]() { return build_impl(p, p->tune_pts, p->d_bounds, st); }, &m);
      ms.push_back(m);
    }
    const float med = median(ms);
    if (rc == CUKD_OK && med < bestBuild) {
      bestBuild = med;
      best.build_tile = kForestTiles[t];
    }
  }
  // clouds built with the chosen tile for the query trials
  p->tuning.build_tile = best.build_tile;
  if (rc == CUKD_OK) rc = restore();
  if (rc == CUKD_OK) rc = build_impl(p, p->tune_pts, p->d_bounds, st);
  // 2. query: Morton x block size x queries per thread
  float bestQuery = 3.4e38f;
  // 512-thread blocks only where the register-list kernel answers (k <= 32;
  // the heap and reference-order kernels take at most 256)
  const int sizes[4] = {64, 128, 256, 512};
  const bool regList = !p->fcp && !(p->params.flags & (CUKD_QUERY_HEAP_ORDER | CUKD_QUERY_REFERENCE_ORDER)) &&
                       p->params.k >= 2 && p->params.k <= 32;
  const int nSizes = regList ? 4 : 3;
  const int qpts[3] = {1, 2, 4};
  for (int mo = 1; mo >= 0 && rc == CUKD_OK; mo--)
    for (int bi = 0; bi < nSizes && rc == CUKD_OK; bi++)
      for (int qi = 0; qi < 3 && rc == CUKD_OK; qi++) {
        p->tuning.morton = mo;
        p->tuning.block_size = sizes[bi];
        p->tuning.queries_per_thread = qpts[qi];
        std::vector<float> ms;
        for (int r = 0; r < reps && rc == CUKD_OK; r++) {
          float m = 0.f;
          rc = timed([&]() { return query_impl(p, p->tune_pts, p->d_bounds, d_queries, ids, d2, st); },
                     &m);
          ms.push_back(m);
        }
        const float med = median(ms);
        if (rc == CUKD_OK && med < bestQuery) {
          bestQuery = med;
          best.morton = mo;
          best.block_size = sizes[bi];
          best.queries_per_thread = qpts[qi];
        }
      }
  cudaStreamSynchronize(st);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(ids);
  cudaFree(d2);
  if (rc != CUKD_OK) {
    p->tuning = saved;
    return rc;
  }
  best.build_ms = bestBuild;
  best.query_ms = bestQuery;
  p->tuning = best;
  p->tuningVersion++;
  drop_graph(p);
  if (out) *out = best;
  return CUKD_OK;
}

}  // extern "C"
