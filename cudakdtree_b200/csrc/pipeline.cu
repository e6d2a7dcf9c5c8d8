// kNN with host-resident queries and results: the queries are cut into
// chunks that flow through three streams -- host->device copy, search
// (cukd_knn on the caller's stream), device->host copy -- with two device
// buffers per kind, so that copies of one chunk overlap the search of the
// next.  For callers whose queries and answers live in host memory (the
// reference's samples copy whole arrays with cudaMemcpy around one query
// launch, sample.cu:121-160); results are those of cukd_knn.
#include <algorithm>

#include "common.cuh"

extern "C" int cukd_knn(const void *d_tree, int64_t n, const cukd_layout *layout,
                        const void *d_world_bounds, const void *d_queries, int64_t nq,
                        const cukd_query_params *params, int32_t *d_out_ids, void *d_out_d2,
                        void *d_out_max_d2, cudaStream_t stream, const cukd_mem_resource *mem);

namespace ckb {
namespace {

struct PipeRes {
  cudaStream_t up = nullptr, down = nullptr;
  cudaEvent_t ev[8] = {};
  ~PipeRes()
  {
    for (cudaEvent_t &e : ev)
      if (e) cudaEventDestroy(e);
    if (up) cudaStreamDestroy(up);
    if (down) cudaStreamDestroy(down);
  }
};

}  // namespace
}  // namespace ckb

extern "C" int cukd_knn_host(const void *d_tree, int64_t n, const cukd_layout *layout,
                             const void *d_world_bounds, const void *h_queries, int64_t nq,
                             const cukd_query_params *params, int32_t *h_out_ids,
                             void *h_out_d2, int64_t chunk, cudaStream_t stream,
                             const cukd_mem_resource *mem)
{
  using namespace ckb;
  Layout L;
  if (!make_layout(layout, &L) || !params) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq < 0 || params->k < 1 || params->k > 1024) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq == 0) return CUKD_OK;
  if (!h_queries || !h_out_ids) return CUKD_ERR_INVALID_ARGUMENT;
  const int k = params->k;
  const int64_t qBytes = int64_t(L.D) * 4;
  const int64_t d2Bytes = L.scalar == CUKD_FLOAT32 ? 4 : 8;
  if (chunk <= 0) chunk = int64_t(1) << 20;
  chunk = std::min(chunk, nq);

  PipeRes r;
  if (cudaStreamCreateWithFlags(&r.up, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&r.down, cudaStreamNonBlocking) != cudaSuccess) {
    set_cuda_error(cudaGetLastError());
    return CUKD_ERR_CUDA;
  }
  for (cudaEvent_t &e : r.ev)
    CKB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  cudaEvent_t *upDone = r.ev, *searchDone = r.ev + 2, *downDone = r.ev + 4, *start = r.ev + 6;
  // buffers: [2] queries, ids, d2
  TempArena arena(stream, mem);
  uint8_t *dq[2];
  int32_t *di[2];
  uint8_t *dd[2] = {nullptr, nullptr};
  for (int b = 0; b < 2; b++) {
    CKB_TRY(arena.alloc(&dq[b], size_t(chunk * qBytes)));
    CKB_TRY(arena.alloc(&di[b], size_t(chunk * k)));
    if (h_out_d2) CKB_TRY(arena.alloc(&dd[b], size_t(chunk * k * d2Bytes)));
  }
  // the side streams start after the work already queued on `stream`
  CKB_CUDA(cudaEventRecord(start[0], stream));
  CKB_CUDA(cudaStreamWaitEvent(r.up, start[0], 0));
  CKB_CUDA(cudaStreamWaitEvent(r.down, start[0], 0));
  const int64_t chunks = div_up(nq, chunk);
  for (int64_t c = 0; c < chunks; c++) {
    const int b = int(c & 1);
    const int64_t q0 = c * chunk, m = std::min(chunk, nq - q0);
    if (c >= 2) CKB_CUDA(cudaStreamWaitEvent(r.up, downDone[b], 0));  // buffer b drained
    CKB_CUDA(cudaMemcpyAsync(dq[b], (const uint8_t *)h_queries + q0 * qBytes, size_t(m * qBytes),
                             cudaMemcpyHostToDevice, r.up));
    CKB_CUDA(cudaEventRecord(upDone[b], r.up));
    CKB_CUDA(cudaStreamWaitEvent(stream, upDone[b], 0));
    CKB_TRY(cukd_knn(d_tree, n, layout, d_world_bounds, dq[b], m, params, di[b], dd[b], nullptr,
                     stream, mem));
    CKB_CUDA(cudaEventRecord(searchDone[b], stream));
    CKB_CUDA(cudaStreamWaitEvent(r.down, searchDone[b], 0));
    CKB_CUDA(cudaMemcpyAsync(h_out_ids + q0 * k, di[b], size_t(m * k * 4), cudaMemcpyDeviceToHost,
                             r.down));
    if (h_out_d2)
      CKB_CUDA(cudaMemcpyAsync((uint8_t *)h_out_d2 + q0 * k * d2Bytes, dd[b],
                               size_t(m * k * d2Bytes), cudaMemcpyDeviceToHost, r.down));
    CKB_CUDA(cudaEventRecord(downDone[b], r.down));
  }
  // the caller's stream completes after the last copy (and the buffers are
  // released behind it)
  CKB_CUDA(cudaEventRecord(start[1], r.down));
  CKB_CUDA(cudaStreamWaitEvent(stream, start[1], 0));
  return CUKD_OK;
}
