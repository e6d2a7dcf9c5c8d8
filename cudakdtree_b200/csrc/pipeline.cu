// kNN whose answers go to host memory, in chunks that overlap the search of
// one chunk with the device->host copy of the previous ones:
//   cukd_knn_host     host-resident queries, uploaded chunk by chunk on a
//                     side stream (three streams: up, search on the caller's
//                     stream, down);
//   cukd_knn_to_host  device-resident queries (the caller uploads them, e.g.
//                     while the tree builds), two streams.
// Three device buffer sets: a query buffer is reused once its search has
// run, a result buffer once its answers are copied down, so the uploads stay
// off the path of the result copies (the slowest stage when k is large: 128
// bytes per query at k = 16 against 12 up).  Measured on the 10M-query,
// k = 16 workload: 2^21-query chunks 27.8 ms, against 29.3 ms with two
// buffer sets; chunk sizes ramping up from chunk/16 or /4, and a second
// search stream taking every other chunk, measured 28-32 ms.  For callers
// whose queries and answers live in host memory (the reference's samples
// copy whole arrays with cudaMemcpy around one query launch,
// sample.cu:121-160); results are those of cukd_knn.
//   cukd_knn_host_async / cukd_knn_to_host_async
//                     cukd_knn_host / cukd_knn_to_host that leave the caller's stream free
//                     once the searches are queued: the answers land behind
//                     the caller's event `done` (the result buffers, up to
//                     eight sets, are released on the copy stream), so a
//                     caller can queue the next tree's build and search on
//                     the same stream while these answers are still being
//                     copied -- the compute and the device->host copies of
//                     consecutive batches then overlap, and by default a
//                     batch of up to 2^24 queries is searched in one slice.
#include <algorithm>
#include <mutex>

#include "common.cuh"

extern "C" int cukd_knn(const void *d_tree, int64_t n, const cukd_layout *layout,
                        const void *d_world_bounds, const void *d_queries, int64_t nq,
                        const cukd_query_params *params, int32_t *d_out_ids, void *d_out_d2,
                        void *d_out_max_d2, cudaStream_t stream, const cukd_mem_resource *mem);

namespace ckb {
namespace {

constexpr int kSets = 3;     // device buffer sets (queries, ids, d2)
constexpr int kMaxSets = 8;  // ... when the copies do not hold the caller's stream

struct PipeRes {
  cudaStream_t up = nullptr, down = nullptr;
  cudaEvent_t upDone[kMaxSets] = {}, searchDone[kMaxSets] = {}, downDone[kMaxSets] = {};
  cudaEvent_t start = nullptr, join[2] = {}, allocDone = nullptr;
  ~PipeRes()
  {
    for (int i = 0; i < kMaxSets; i++) {
      if (upDone[i]) cudaEventDestroy(upDone[i]);
      if (searchDone[i]) cudaEventDestroy(searchDone[i]);
      if (downDone[i]) cudaEventDestroy(downDone[i]);
    }
    if (start) cudaEventDestroy(start);
    if (allocDone) cudaEventDestroy(allocDone);
    for (cudaEvent_t e : join)
      if (e) cudaEventDestroy(e);
    if (up) cudaStreamDestroy(up);
    if (down) cudaStreamDestroy(down);
  }
};

// The result buffers of the asynchronous calls (no caller's resource) come
// from a pool of their own that never makes an allocation wait for a
// release queued on another stream: the device's default pool may hand a
// call the buffers that the previous call releases behind its device->host
// copies, and the call's searches would then wait for those copies.  This
// pool reuses memory whose release has run, or whose release the copy
// stream already follows (a caller that waited for an earlier call's `done`
// before this call), else it grows; it keeps what it holds for the next
// call, like the default pool does for this library's other temporaries.
cudaMemPool_t result_pool()
{
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;  // the default pool then
    }
    uint64_t keep = UINT64_MAX;
    int no = 0;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no);
    cudaGetLastError();
    pools[dev] = pool;
  }
  return pools[dev];
}

// On every exit, success or error: the caller's stream waits for all work
// queued on the side streams (only the upload stream when the answers land
// behind the caller's event instead), so that the buffers released on it
// afterwards (stream-ordered) are no longer in use.
struct JoinSideStreams {
  PipeRes &r;
  cudaStream_t stream;
  bool down = true;
  ~JoinSideStreams()
  {
    cudaStream_t side[2] = {r.up, down ? r.down : nullptr};
    for (int i = 0; i < 2; i++) {
      if (!side[i] || !r.join[i]) continue;
      if (cudaEventRecord(r.join[i], side[i]) == cudaSuccess)
        cudaStreamWaitEvent(stream, r.join[i], 0);
    }
    // the other way round when the result buffers are released on the copy
    // stream: after every search queued on the caller's stream (also on an
    // error midway, when some search has no copy behind it)
    if (!down && r.down && r.join[1] && cudaEventRecord(r.join[1], stream) == cudaSuccess)
      cudaStreamWaitEvent(r.down, r.join[1], 0);
  }
};

}  // namespace
}  // namespace ckb

namespace ckb {
namespace {

// The chunked pipeline behind cukd_knn_host (h_queries set: chunks are
// uploaded on a side stream) and cukd_knn_to_host (d_queries set: the
// chunks are read in place).
int knn_pipeline(const void *d_tree, int64_t n, const cukd_layout *layout,
                 const void *d_world_bounds, const void *h_queries, const void *d_queries,
                 int64_t nq, const cukd_query_params *params, int32_t *h_out_ids, void *h_out_d2,
                 int64_t chunk, cudaStream_t stream, const cukd_mem_resource *mem,
                 cudaEvent_t done = nullptr)
{
  Layout L;
  if (!make_layout(layout, &L) || !params) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq < 0 || params->k < 1 || params->k > 1024) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq == 0) return CUKD_OK;
  if ((!h_queries && !d_queries) || !h_out_ids) return CUKD_ERR_INVALID_ARGUMENT;
  const bool upload = d_queries == nullptr;
  const int k = params->k;
  const int64_t qBytes = int64_t(L.D) * 4;
  const int64_t d2Bytes = L.scalar == CUKD_FLOAT32 ? 4 : 8;
  // the asynchronous calls overlap one call's copies with the next call's
  // build and search, so slicing a batch only adds per-search cost (10M
  // queries, k = 16, back to back: 23.8 ms a batch in one slice, 24.6 in
  // 5M-query slices, 26.8 in 2^21): one slice up to 2^24 queries
  if (chunk <= 0) chunk = done ? int64_t(1) << 24 : int64_t(1) << 20;
  chunk = std::min(chunk, nq);

  PipeRes r;
  if ((upload && cudaStreamCreateWithFlags(&r.up, cudaStreamNonBlocking) != cudaSuccess) ||
      cudaStreamCreateWithFlags(&r.down, cudaStreamNonBlocking) != cudaSuccess) {
    set_cuda_error(cudaGetLastError());
    return CUKD_ERR_CUDA;
  }
  const int64_t chunks = div_up(nq, chunk);
  const int sets = done ? int(std::min<int64_t>(kMaxSets, chunks)) : kSets;
  for (int i = 0; i < sets; i++) {
    CKB_CUDA(cudaEventCreateWithFlags(&r.upDone[i], cudaEventDisableTiming));
    CKB_CUDA(cudaEventCreateWithFlags(&r.searchDone[i], cudaEventDisableTiming));
    CKB_CUDA(cudaEventCreateWithFlags(&r.downDone[i], cudaEventDisableTiming));
  }
  CKB_CUDA(cudaEventCreateWithFlags(&r.start, cudaEventDisableTiming));
  CKB_CUDA(cudaEventCreateWithFlags(&r.allocDone, cudaEventDisableTiming));
  for (cudaEvent_t &e : r.join) CKB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));

  // the side streams start after the work already queued on `stream` --
  // also the result buffers' allocations on the copy stream: memory that an
  // earlier call released before its `done`, which the caller's stream has
  // waited for, is then reused without waiting for anything else
  CKB_CUDA(cudaEventRecord(r.start, stream));
  if (upload) CKB_CUDA(cudaStreamWaitEvent(r.up, r.start, 0));
  CKB_CUDA(cudaStreamWaitEvent(r.down, r.start, 0));
  TempArena arena(stream, mem);
  // the result buffers: released on the copy stream when the answers land
  // behind `done` (after the copies), else on the caller's stream
  TempArena downArena(done ? r.down : stream, mem,
                      done && !(mem && mem->alloc) ? result_pool() : nullptr);
  uint8_t *dq[kMaxSets] = {};
  int32_t *di[kMaxSets];
  uint8_t *dd[kMaxSets] = {};
  for (int b = 0; b < sets; b++) {
    if (upload) CKB_TRY(arena.alloc(&dq[b], size_t(chunk * qBytes)));
    CKB_TRY(downArena.alloc(&di[b], size_t(chunk * k)));
    if (h_out_d2) CKB_TRY(downArena.alloc(&dd[b], size_t(chunk * k * d2Bytes)));
  }
  // declared after the arenas: joins the side streams before they release
  JoinSideStreams joiner{r, stream, done == nullptr};
  // result buffers taken on the copy stream are written first by the
  // searches on the caller's stream: that stream waits for the allocations
  if (done) {
    CKB_CUDA(cudaEventRecord(r.allocDone, r.down));
    CKB_CUDA(cudaStreamWaitEvent(stream, r.allocDone, 0));
  }
  for (int64_t c = 0; c < chunks; c++) {
    const int b = int(c % sets);
    const int64_t q0 = c * chunk, m = std::min(chunk, nq - q0);
    const void *qs = (const uint8_t *)d_queries + q0 * qBytes;
    if (upload) {
      // query buffer b: free once the search of chunk c - sets has run
      if (c >= sets) CKB_CUDA(cudaStreamWaitEvent(r.up, r.searchDone[b], 0));
      CKB_CUDA(cudaMemcpyAsync(dq[b], (const uint8_t *)h_queries + q0 * qBytes,
                               size_t(m * qBytes), cudaMemcpyHostToDevice, r.up));
      CKB_CUDA(cudaEventRecord(r.upDone[b], r.up));
      CKB_CUDA(cudaStreamWaitEvent(stream, r.upDone[b], 0));
      qs = dq[b];
    }
    // result buffers b: free once chunk c - sets' answers are copied down
    if (c >= sets) CKB_CUDA(cudaStreamWaitEvent(stream, r.downDone[b], 0));
    CKB_TRY(cukd_knn(d_tree, n, layout, d_world_bounds, qs, m, params, di[b], dd[b], nullptr,
                     stream, mem));
    CKB_CUDA(cudaEventRecord(r.searchDone[b], stream));
    CKB_CUDA(cudaStreamWaitEvent(r.down, r.searchDone[b], 0));
    CKB_CUDA(cudaMemcpyAsync(h_out_ids + q0 * k, di[b], size_t(m * k * 4), cudaMemcpyDeviceToHost,
                             r.down));
    if (h_out_d2)
      CKB_CUDA(cudaMemcpyAsync((uint8_t *)h_out_d2 + q0 * k * d2Bytes, dd[b],
                               size_t(m * k * d2Bytes), cudaMemcpyDeviceToHost, r.down));
    CKB_CUDA(cudaEventRecord(r.downDone[b], r.down));
  }
  // the caller's stream completes after the last copy (the joiner), and the
  // buffers are released behind it -- or the answers land behind `done`
  // (every search has its copies queued behind it on the copy stream, so
  // the result buffers are released there before `done`)
  if (done) {
    downArena.release_all();
    CKB_CUDA(cudaEventRecord(done, r.down));
  }
  return CUKD_OK;
}

}  // namespace
}  // namespace ckb

extern "C" int cukd_knn_host(const void *d_tree, int64_t n, const cukd_layout *layout,
                             const void *d_world_bounds, const void *h_queries, int64_t nq,
                             const cukd_query_params *params, int32_t *h_out_ids,
                             void *h_out_d2, int64_t chunk, cudaStream_t stream,
                             const cukd_mem_resource *mem)
{
  if (nq > 0 && !h_queries) return CUKD_ERR_INVALID_ARGUMENT;
  return ckb::knn_pipeline(d_tree, n, layout, d_world_bounds, h_queries, nullptr, nq, params,
                           h_out_ids, h_out_d2, chunk, stream, mem);
}

extern "C" int cukd_knn_host_async(const void *d_tree, int64_t n, const cukd_layout *layout,
                                   const void *d_world_bounds, const void *h_queries, int64_t nq,
                                   const cukd_query_params *params, int32_t *h_out_ids,
                                   void *h_out_d2, int64_t chunk, cudaEvent_t done,
                                   cudaStream_t stream, const cukd_mem_resource *mem)
{
  if ((nq > 0 && !h_queries) || !done) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq == 0) {
    CKB_CUDA(cudaEventRecord(done, stream));
    return CUKD_OK;
  }
  return ckb::knn_pipeline(d_tree, n, layout, d_world_bounds, h_queries, nullptr, nq, params,
                           h_out_ids, h_out_d2, chunk, stream, mem, done);
}

extern "C" int cukd_knn_to_host(const void *d_tree, int64_t n, const cukd_layout *layout,
                                const void *d_world_bounds, const void *d_queries, int64_t nq,
                                const cukd_query_params *params, int32_t *h_out_ids,
                                void *h_out_d2, int64_t chunk, cudaStream_t stream,
                                const cukd_mem_resource *mem)
{
  if (nq > 0 && !d_queries) return CUKD_ERR_INVALID_ARGUMENT;
  return ckb::knn_pipeline(d_tree, n, layout, d_world_bounds, nullptr, d_queries, nq, params,
                           h_out_ids, h_out_d2, chunk, stream, mem);
}

extern "C" int cukd_knn_to_host_async(const void *d_tree, int64_t n, const cukd_layout *layout,
                                      const void *d_world_bounds, const void *d_queries,
                                      int64_t nq, const cukd_query_params *params,
                                      int32_t *h_out_ids, void *h_out_d2, int64_t chunk,
                                      cudaEvent_t done, cudaStream_t stream,
                                      const cukd_mem_resource *mem)
{
  if ((nq > 0 && !d_queries) || !done) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq == 0) {
    CKB_CUDA(cudaEventRecord(done, stream));
    return CUKD_OK;
  }
  return ckb::knn_pipeline(d_tree, n, layout, d_world_bounds, nullptr, d_queries, nq, params,
                           h_out_ids, h_out_d2, chunk, stream, mem, done);
}
