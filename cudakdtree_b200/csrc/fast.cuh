// Fast exact kNN / FCP path (fast.cu): arguments and launcher.
#pragma once

#include "query.cuh"

namespace ckb {
namespace fast {

struct FastArgs {
  query::QArgs q;       // tree / queries / outputs (ids, d2 [nq][k], max [nq])
  int kk;               // k (1 for FCP)
  bool fcp;             // FCP semantics (strict minimum, -1 beyond the cut-off)
  int *work;            // global chunk counter (zeroed before the launch)
  int *fb_count;        // fallback queue length (zeroed before the launch)
  int32_t *fb_list;     // fallback queue (query indices), capacity nq
  const float *radius;  // optional per-query initial cull radius (before scaling)
  int32_t *status;      // optional per-query outcome: 0 answered, 1 queued
  float radius_scale;   // multiplies `radius`
};

}  // namespace fast

// Launches the fast kernel for float trees with D = 2..4 and k <= 128
// (register list up to k = 32, local-memory heap above).
int run_fast(const fast::FastArgs &fa, int D, cudaStream_t st);

// The warp-cooperative traversal (packet.cu): float kNN, k = 2..32, no
// forest, no device-side query count.
int run_packet(const fast::FastArgs &fa, int D, cudaStream_t st);

// The same for int32 trees (exact int64 distances), kNN with k = 2..128
// (fast_int.cu).
int run_fast_int(const fast::FastArgs &fa, int D, cudaStream_t st);

}  // namespace ckb
