// Learned kNN-radius proposal (no reference counterpart; the reference's
// queries start from the caller's cut-off radius, cukd/knn.h:503-511).
//
// A small MLP predicts each query's k-th-neighbour distance from its
// normalised coordinates and a coarse density feature, log(1 + points in a
// cell of a res^3 occupancy grid of the tree's points), interpolated
// trilinearly between the 8 cell centres around the query:
//     f (4) -> 64 ReLU -> 64 ReLU -> 1   (the log of the distance,
//                                         standardised over the training set)
// Weights are kept in BF16 for every forward/backward pass (FP32 master
// copy for the optimiser); the inputs and the first hidden layer enter the
// products as bf16, and every sum accumulates in FP32.  Training uses
// exact k-th distances the plain traversal computes, Adam, minibatches.
//
// The learned kNN predicts each query's radius inside its search kernel
// (knn_learned_kernel: the network on the tensor cores, then the fast exact
// traversal of fast_one.cuh from an initial cull radius r_hat * scale).
// A query that finds at least k points strictly
// inside that radius has its exact answer (every point nearer than its k-th
// neighbour was examined); any other query -- fewer than k inside, or a
// distance tie at the k-th boundary -- is re-run by the plain unbounded
// traversal, and a boundary tie there by the reference's own visiting
// order.  So the learned path returns the same bits as the plain one.
//
// Kernels (all hand-written, FP32 accumulate over BF16 weights):
//   grid_count_kernel   occupancy grid of the tree's points
//   features_kernel     4 features per query
//   train_kernel        fused forward + backward of a minibatch slice per
//                       CTA; per-CTA gradient sums merged with atomics
//   adam_kernel         Adam update of the FP32 master weights, refresh of
//                       the BF16 copy, gradient reset
//   infer_kernel        forward pass of 32 queries per warp on the tensor
//                       cores (mma.sync bf16, FP32 accumulate) -> radius
//   knn_learned_kernel  the same forward pass fused with the seeded kNN
//                       traversal (pass 1 of cukd_knn_learned)
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "fast.cuh"
#include "fast_one.cuh"
#include "learned.cuh"
#include "query.cuh"

struct cukd_radius_model_s;

namespace ckb {
namespace learned {

constexpr int S = 32;             // samples per CTA in training
constexpr int kTrainThreads = 256;

struct ModelDev {
  float *params;          // FP32 master
  __nv_bfloat16 *wbf;     // BF16 copy used by every pass
  float *m, *v, *grad;    // Adam state, gradient accumulator
  uint32_t *grid;         // res^D counts
  float *dens;            // res^D log1pf(count): the density feature's cells
  float *loss;            // per-step loss sums
};

// a coordinate word of scalar type SC (0 float, 1 int32) as a float
template <int SC> __device__ __forceinline__ float coord_f(uint32_t bits)
{
  return SC == 0 ? __uint_as_float(bits) : float(int32_t(bits));
}

// ---------------------------------------------------------------------------
template <int D, int SC>
__global__ void grid_count_kernel(const uint8_t *__restrict__ pts, int64_t n, int stride,
                                  int poff, Norm nm, uint32_t *grid)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const uint32_t *c = (const uint32_t *)(pts + i * stride + poff);
    int cell = 0;
#pragma unroll
    for (int d = 0; d < D; d++) {
      const float x = coord_f<SC>(__ldg(c + d));
      const float u = __fmul_rn(__fsub_rn(x, nm.lo[d]), nm.invext[d]);
      const float cc = __fmul_rn(u, float(nm.res));
      const int ci = cc >= 0.f ? (cc < float(nm.res) ? int(cc) : nm.res - 1) : 0;
      cell = cell * nm.res + ci;
    }
    atomicAdd(&grid[cell], 1u);
  }
}

// query i's coordinates (scalar type SC, D per query) as floats
template <int D, int SC>
__device__ __forceinline__ void query_f(const void *q, int64_t i, float *out)
{
  const uint32_t *w = (const uint32_t *)q + i * D;
#pragma unroll
  for (int d = 0; d < D; d++) out[d] = coord_f<SC>(__ldg(w + d));
}

__global__ void density_kernel(const uint32_t *grid, int64_t cells, float *dens)
{
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < cells;
       i += int64_t(gridDim.x) * blockDim.x)
    dens[i] = log1pf(float(grid[i]));
}

__global__ void grid_max_kernel(const uint32_t *grid, int64_t cells, uint32_t *out)
{
  uint32_t m = 0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < cells;
       i += int64_t(gridDim.x) * blockDim.x)
    m = max(m, grid[i]);
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

template <int D, int SC>
__global__ void features_kernel(const void *__restrict__ q, int64_t nq, Norm nm,
                                const float *dens, float *feat)
{
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nq) return;
  float qq[D];
  query_f<D, SC>(q, i, qq);
  float f[kIn];
  features<D>(nm, dens, qq, f);
#pragma unroll
  for (int d = 0; d < kIn; d++) feat[i * kIn + d] = f[d];
}

// targets: standardised log of the k-th distance (from squared distances:
// float for float trees, int64 for int trees)
template <int SC>
__global__ void targets_kernel(const void *kth_d2, int64_t nq, float *t)
{
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nq) return;
  const float d2 = SC == 0 ? ((const float *)kth_d2)[i] : float(((const long long *)kth_d2)[i]);
  t[i] = __fmul_rn(0.5f, logf(fmaxf(d2, 1e-30f)));
}

__global__ void normalize_targets_kernel(float *t, int64_t nq, float mean, float invstd)
{
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i >= nq) return;
  t[i] = __fmul_rn(__fsub_rn(t[i], mean), invstd);
}

// ---------------------------------------------------------------------------
// fused forward + backward over one slice of S samples per CTA
// ---------------------------------------------------------------------------
struct TrainSmem {
  float w1[H][kIn], b1[H], w2[H][H], b2[H], w3[H], b3;
  float f[S][kIn], h1[S][H], h2[S][H], dh2[S][H], dh1[S][H];
  float y[S], dy[S];
};

// quantile == 0: mean squared error; 0 < quantile < 1: pinball loss, whose
// minimiser is that quantile of the target given the features
__global__ void __launch_bounds__(kTrainThreads) train_kernel(
    const __nv_bfloat16 *__restrict__ wbf, const float *__restrict__ feat,
    const float *__restrict__ tgt, int64_t begin, int64_t count, float gradScale, float *grad,
    float *lossOut, float quantile)
{
  extern __shared__ __align__(16) uint8_t smem_raw[];
  TrainSmem &M = *reinterpret_cast<TrainSmem *>(smem_raw);
  const int tid = threadIdx.x;
  for (int i = tid; i < NP; i += kTrainThreads) {
    const float w = __bfloat162float(wbf[i]);
    if (i < OB1) M.w1[(i - OW1) / kIn][(i - OW1) % kIn] = w;
    else if (i < OW2) M.b1[i - OB1] = w;
    else if (i < OB2) M.w2[(i - OW2) / H][(i - OW2) % H] = w;
    else if (i < OW3) M.b2[i - OB2] = w;
    else if (i < OB3) M.w3[i - OW3] = w;
    else M.b3 = w;
  }
  const int64_t s0 = begin + int64_t(blockIdx.x) * S;
  const int64_t left = begin + count - s0;
  const int ns = left <= 0 ? 0 : (left < S ? int(left) : S);
  for (int i = tid; i < S * kIn; i += kTrainThreads) {
    const int s = i / kIn;
    M.f[s][i % kIn] = s < ns ? bf16_round(feat[(s0 + s) * kIn + i % kIn]) : 0.f;
  }
  __syncthreads();
  if (ns == 0) return;
  // layer 1
  for (int i = tid; i < S * H; i += kTrainThreads) {
    const int s = i / H, j = i % H;
    float z = M.b1[j];
#pragma unroll
    for (int c = 0; c < kIn; c++) z = __fmaf_rn(M.w1[j][c], M.f[s][c], z);
    M.h1[s][j] = bf16_round(fmaxf(z, 0.f));  // as the tensor cores see it
  }
  __syncthreads();
  // layer 2
  for (int i = tid; i < S * H; i += kTrainThreads) {
    const int s = i / H, j = i % H;
    float z = M.b2[j];
#pragma unroll 16
    for (int c = 0; c < H; c++) z = __fmaf_rn(M.w2[j][c], M.h1[s][c], z);
    M.h2[s][j] = fmaxf(z, 0.f);
  }
  __syncthreads();
  // output, loss, dL/dy  (one warp per sample group)
  {
    const int lane = tid & 31, wid = tid >> 5;
    for (int s = wid; s < S; s += kTrainThreads / 32) {
      float p = __fmul_rn(M.w3[lane], M.h2[s][lane]);
      p = __fmaf_rn(M.w3[lane + 32], M.h2[s][lane + 32], p);
      for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
      if (lane == 0) {
        const float y = p + M.b3;
        const float e = s < ns ? y - tgt[s0 + s] : 0.f;
        M.y[s] = y;
        float dl, l;
        if (quantile > 0.f) {  // pinball: slope 1 - q above the target, -q below
          dl = e > 0.f ? 1.f - quantile : (e < 0.f ? -quantile : 0.f);
          l = e > 0.f ? (1.f - quantile) * e : -quantile * e;
        } else {
          dl = 2.f * e;
          l = e * e;
        }
        M.dy[s] = dl * gradScale;
        if (s < ns && lossOut) atomicAdd(lossOut, l);
      }
    }
  }
  __syncthreads();
  for (int i = tid; i < S * H; i += kTrainThreads) {
    const int s = i / H, j = i % H;
    M.dh2[s][j] = M.h2[s][j] > 0.f ? M.dy[s] * M.w3[j] : 0.f;
  }
  __syncthreads();
  for (int i = tid; i < S * H; i += kTrainThreads) {
    const int s = i / H, k = i % H;
    float g = 0.f;
#pragma unroll 16
    for (int j = 0; j < H; j++) g = __fmaf_rn(M.w2[j][k], M.dh2[s][j], g);
    M.dh1[s][k] = M.h1[s][k] > 0.f ? g : 0.f;
  }
  __syncthreads();
  // gradient sums over the slice, merged into the global accumulator
  for (int i = tid; i < NP; i += kTrainThreads) {
    float g = 0.f;
    if (i < OB1) {
      const int j = (i - OW1) / kIn, c = (i - OW1) % kIn;
      for (int s = 0; s < S; s++) g = __fmaf_rn(M.dh1[s][j], M.f[s][c], g);
    } else if (i < OW2) {
      const int j = i - OB1;
      for (int s = 0; s < S; s++) g += M.dh1[s][j];
    } else if (i < OB2) {
      const int j = (i - OW2) / H, k = (i - OW2) % H;
      for (int s = 0; s < S; s++) g = __fmaf_rn(M.dh2[s][j], M.h1[s][k], g);
    } else if (i < OW3) {
      const int j = i - OB2;
      for (int s = 0; s < S; s++) g += M.dh2[s][j];
    } else if (i < OB3) {
      const int j = i - OW3;
      for (int s = 0; s < S; s++) g = __fmaf_rn(M.dy[s], M.h2[s][j], g);
    } else {
      for (int s = 0; s < S; s++) g += M.dy[s];
    }
    if (g != 0.f) atomicAdd(&grad[i], g);
  }
}

__global__ void adam_kernel(float *params, __nv_bfloat16 *wbf, float *m, float *v, float *grad,
                            float lr, float b1, float b2, float eps, float c1, float c2)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NP) return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float p = params[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  params[i] = p;
  wbf[i] = __float2bfloat16_rn(p);
  grad[i] = 0.f;
}

// ---------------------------------------------------------------------------
// inference: 32 queries per warp through mlp_forward_warp (tensor cores)
// ---------------------------------------------------------------------------
template <int D, int SC>
__global__ void __launch_bounds__(128, 4) infer_kernel(const __nv_bfloat16 *__restrict__ wbf,
                                                    const void *__restrict__ q, int64_t nq,
                                                    Norm nm, const float *dens, float *radius)
{
  const int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  if (i - (threadIdx.x & 31) >= nq) return;  // whole warps only: they run the mma together
  const bool live = i < nq;
  const int64_t qi = live ? i : 0;
  float qq[D];
  query_f<D, SC>(q, qi, qq);
  float f[kIn];
  features<D>(nm, dens, qq, f);
  const float y = mlp_forward_warp(wbf, f);
  if (live) radius[i] = expf(__fmaf_rn(y, nm.tstd, nm.tmean));
}

// ---------------------------------------------------------------------------
// Pass 1 of the learned kNN, fused: each warp predicts the radii of 32
// consecutive queries of the visiting order on the tensor cores, then every
// lane runs the fast traversal (fast_one.cuh) of its query from its radius.
// The prediction never leaves registers; the traversal is latency-bound, so
// the network's instructions mostly fill issue slots the traversal leaves
// idle.
// ---------------------------------------------------------------------------
template <int D, bool EXPL, bool VEC16, int KC>
__global__ void __launch_bounds__(256, KC <= 17 ? 4 : 2)
    knn_learned_kernel(fast::FastArgs fa, const __nv_bfloat16 *__restrict__ wbf,
                       const float *__restrict__ dens, Norm nm)
{
  const int lane = threadIdx.x & 31;
  const int64_t nq = fa.q.nq;
  const int64_t warps = int64_t(gridDim.x) * (blockDim.x >> 5);
  for (int64_t w = int64_t(blockIdx.x) * (blockDim.x >> 5) + (threadIdx.x >> 5); w * 32 < nq;
       w += warps) {
    const int64_t i = w * 32 + lane;
    const bool live = i < nq;
    // lanes past the end (last warp) predict query 0's radius and stop
    const int64_t myq = live ? (fa.q.order ? int64_t(__ldg(fa.q.order + i)) : i) : 0;
    float qq[D];
    query_f<D, 0>(fa.q.queries, myq, qq);
    float f[kIn];
    features<D>(nm, dens, qq, f);
    __syncwarp();
    const float y = mlp_forward_warp(wbf, f);
    const float r = expf(__fmaf_rn(y, nm.tstd, nm.tmean));
    if (live) fast::knn_fast_one<D, EXPL, VEC16, KC>(fa, i, myq, true, r);
  }
}

template <int D, bool EXPL, bool VEC16>
int launch_learned(const fast::FastArgs &fa, const __nv_bfloat16 *wbf, const float *dens,
                   const Norm &nm, cudaStream_t st)
{
  const int bs = 256;
  const unsigned grid = unsigned(std::max<int64_t>(1, div_up(fa.q.nq, bs)));
  const int slots = fa.kk + 1;
  if (slots <= 5)
    knn_learned_kernel<D, EXPL, VEC16, 5><<<grid, bs, 0, st>>>(fa, wbf, dens, nm);
  else if (slots <= 9)
    knn_learned_kernel<D, EXPL, VEC16, 9><<<grid, bs, 0, st>>>(fa, wbf, dens, nm);
  else if (slots <= 17)
    knn_learned_kernel<D, EXPL, VEC16, 17><<<grid, bs, 0, st>>>(fa, wbf, dens, nm);
  else if (slots <= 33)
    knn_learned_kernel<D, EXPL, VEC16, 33><<<grid, bs, 0, st>>>(fa, wbf, dens, nm);
  else
    return CUKD_ERR_UNSUPPORTED;
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

template <int D>
int launch_learned_layout(const fast::FastArgs &fa, const Layout &L, const __nv_bfloat16 *wbf,
                          const float *dens, const Norm &nm, cudaStream_t st)
{
  const bool expl = L.doff >= 0;
  const bool vec16 = L.stride == 16 && L.poff == 0 && (!expl || L.doff == 12) && D <= 3;
  if (expl)
    return vec16 ? launch_learned<D, true, true>(fa, wbf, dens, nm, st)
                 : launch_learned<D, true, false>(fa, wbf, dens, nm, st);
  return vec16 ? launch_learned<D, false, true>(fa, wbf, dens, nm, st)
               : launch_learned<D, false, false>(fa, wbf, dens, nm, st);
}

// (D, scalar) dispatch of the per-query model kernels
#define CKB_MODEL_DISPATCH(D_, SC_, CALL)                          \
  do {                                                            \
    if ((D_) == 2 && (SC_) == 0) { constexpr int D = 2, SC = 0; CALL; } \
    else if ((D_) == 3 && (SC_) == 0) { constexpr int D = 3, SC = 0; CALL; } \
    else if ((D_) == 4 && (SC_) == 0) { constexpr int D = 4, SC = 0; CALL; } \
    else if ((D_) == 2 && (SC_) == 1) { constexpr int D = 2, SC = 1; CALL; } \
    else if ((D_) == 3 && (SC_) == 1) { constexpr int D = 3, SC = 1; CALL; } \
    else if ((D_) == 4 && (SC_) == 1) { constexpr int D = 4, SC = 1; CALL; } \
    else return CUKD_ERR_UNSUPPORTED;                             \
  } while (0)

// deterministic initialisation (He-uniform over the D + 1 real inputs), a
// 64-bit LCG seeded by the caller
static void init_params(std::vector<float> &p, uint64_t seed, int D)
{
  uint64_t x = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    x = x * 6364136223846793005ull + 1442695040888963407ull;
    return float((x >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
  };
  p.assign(NP, 0.f);
  for (int i = 0; i < kIn * H; i++) p[OW1 + i] = uni() * std::sqrt(6.f / float(D + 1));
  for (int i = 0; i < H * H; i++) p[OW2 + i] = uni() * std::sqrt(6.f / float(H));
  for (int i = 0; i < H; i++) p[OW3 + i] = uni() * std::sqrt(3.f / float(H));
}

}  // namespace learned

int run_fast(const fast::FastArgs &fa, int D, cudaStream_t st);

}  // namespace ckb

// opaque model handle
struct cukd_radius_model_s {
  int device;
  int scalar;  // coordinate type of the tree the grid was built from
  ckb::learned::Norm norm;
  ckb::learned::ModelDev d;
  int trained;
  float last_loss;
  float quantile;  // training loss: 0 = mean squared error, else pinball at this quantile
};

using namespace ckb;
using namespace ckb::learned;

static int64_t grid_cells(int res, int D)
{
  int64_t c = 1;
  for (int d = 0; d < D; d++) c *= res;
  return c;
}

static int model_alloc(cukd_radius_model_s *m, int64_t cells)
{
  CKB_CUDA(cudaMalloc(&m->d.params, sizeof(float) * NP));
  CKB_CUDA(cudaMalloc(&m->d.wbf, sizeof(__nv_bfloat16) * NP));
  CKB_CUDA(cudaMalloc(&m->d.m, sizeof(float) * NP));
  CKB_CUDA(cudaMalloc(&m->d.v, sizeof(float) * NP));
  CKB_CUDA(cudaMalloc(&m->d.grad, sizeof(float) * NP));
  CKB_CUDA(cudaMalloc(&m->d.grid, sizeof(uint32_t) * size_t(cells)));
  CKB_CUDA(cudaMalloc(&m->d.dens, sizeof(float) * size_t(cells)));
  CKB_CUDA(cudaMalloc(&m->d.loss, sizeof(float) * 2));
  return CUKD_OK;
}

extern "C" {

int cukd_radius_model_create_nd(cukd_radius_model **out, int grid_res, int num_dims,
                                uint64_t seed)
{
  if (!out || num_dims < 2 || num_dims > 4 || grid_res < 1 ||
      grid_cells(grid_res, num_dims) > (int64_t(1) << 24))
    return CUKD_ERR_INVALID_ARGUMENT;
  auto *m = new cukd_radius_model_s();
  CKB_CUDA(cudaGetDevice(&m->device));
  m->norm.res = grid_res;
  m->norm.D = num_dims;
  m->trained = 0;
  const int rc = model_alloc(m, grid_cells(grid_res, num_dims));
  if (rc != CUKD_OK) {
    cukd_radius_model_destroy((cukd_radius_model *)m);
    return rc;
  }
  std::vector<float> p;
  init_params(p, seed, num_dims);
  std::vector<__nv_bfloat16> pb(NP);
  for (int i = 0; i < NP; i++) pb[i] = __float2bfloat16_rn(p[i]);
  CKB_CUDA(cudaMemcpy(m->d.params, p.data(), sizeof(float) * NP, cudaMemcpyHostToDevice));
  CKB_CUDA(cudaMemcpy(m->d.wbf, pb.data(), sizeof(__nv_bfloat16) * NP, cudaMemcpyHostToDevice));
  CKB_CUDA(cudaMemset(m->d.m, 0, sizeof(float) * NP));
  CKB_CUDA(cudaMemset(m->d.v, 0, sizeof(float) * NP));
  CKB_CUDA(cudaMemset(m->d.grad, 0, sizeof(float) * NP));
  *out = (cukd_radius_model *)m;
  return CUKD_OK;
}

int cukd_radius_model_create(cukd_radius_model **out, int grid_res, uint64_t seed)
{
  return cukd_radius_model_create_nd(out, grid_res, 3, seed);
}

int cukd_radius_model_set_loss(cukd_radius_model *model, float quantile)
{
  auto *m = (cukd_radius_model_s *)model;
  if (!m || !(quantile == 0.f || (quantile > 0.f && quantile < 1.f)))
    return CUKD_ERR_INVALID_ARGUMENT;
  m->quantile = quantile;
  return CUKD_OK;
}

int cukd_radius_model_destroy(cukd_radius_model *model)
{
  auto *m = (cukd_radius_model_s *)model;
  if (!m) return CUKD_OK;
  for (void *p : {(void *)m->d.params, (void *)m->d.wbf, (void *)m->d.m, (void *)m->d.v,
                  (void *)m->d.grad, (void *)m->d.grid, (void *)m->d.dens,
                  (void *)m->d.loss})
    if (p) cudaFree(p);
  delete m;
  return CUKD_OK;
}

// Occupancy grid of the tree's points inside the world bounds.
int cukd_radius_model_set_grid(cukd_radius_model *model, const void *d_points, int64_t n,
                               const cukd_layout *layout, const float *h_world_bounds,
                               cudaStream_t st)
{
  auto *m = (cukd_radius_model_s *)model;
  ckb::Layout L;
  if (!m || !make_layout(layout, &L) || L.D != m->norm.D || !h_world_bounds)
    return CUKD_ERR_INVALID_ARGUMENT;
  Norm &nm = m->norm;
  const int D = L.D;
  m->scalar = L.scalar;
  for (int d = 0; d < D; d++) {
    const float lo = h_world_bounds[d], hi = h_world_bounds[D + d];
    nm.lo[d] = lo;
    nm.invext[d] = hi > lo ? 1.f / (hi - lo) : 0.f;
  }
  const int64_t cells = grid_cells(nm.res, D);
  CKB_CUDA(cudaMemsetAsync(m->d.grid, 0, sizeof(uint32_t) * cells, st));
  const int blocks = int(std::max<int64_t>(1, std::min<int64_t>(div_up(n, 256), kNumSMs * 8)));
  CKB_MODEL_DISPATCH(D, L.scalar, (grid_count_kernel<D, SC><<<blocks, 256, 0, st>>>(
                                      (const uint8_t *)d_points, n, L.stride, L.poff, nm,
                                      m->d.grid)));
  CKB_CHECK_LAUNCH();
  uint32_t *mx = nullptr;
  CKB_CUDA(cudaMallocAsync(&mx, sizeof(uint32_t), st));
  CKB_CUDA(cudaMemsetAsync(mx, 0, sizeof(uint32_t), st));
  density_kernel<<<std::max<int64_t>(1, std::min<int64_t>(div_up(cells, 256), 1024)), 256, 0,
                   st>>>(m->d.grid, cells, m->d.dens);
  CKB_CHECK_LAUNCH();
  grid_max_kernel<<<std::max<int64_t>(1, std::min<int64_t>(div_up(cells, 256), 1024)), 256, 0,
                    st>>>(m->d.grid, cells, mx);
  CKB_CHECK_LAUNCH();
  uint32_t hm = 0;
  CKB_CUDA(cudaMemcpyAsync(&hm, mx, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  CKB_CUDA(cudaFreeAsync(mx, st));
  CKB_CUDA(cudaStreamSynchronize(st));
  nm.invLogMax = 1.f / std::log1p(float(std::max<uint32_t>(hm, 1)));
  return CUKD_OK;
}

static int features_launch(const cukd_radius_model_s *m, const void *q, int64_t nq, float *feat,
                           cudaStream_t st)
{
  const unsigned nb = unsigned(div_up(nq, 256));
  CKB_MODEL_DISPATCH(m->norm.D, m->scalar, (features_kernel<D, SC><<<nb, 256, 0, st>>>(
                                               q, nq, m->norm, m->d.dens, feat)));
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

static int infer_launch(const cukd_radius_model_s *m, const void *q, int64_t nq, float *radius,
                        cudaStream_t st)
{
  const unsigned nb = unsigned(div_up(nq, 128));
  CKB_MODEL_DISPATCH(m->norm.D, m->scalar, (infer_kernel<D, SC><<<nb, 128, 0, st>>>(
                                               m->d.wbf, q, nq, m->norm, m->d.dens, radius)));
  CKB_CHECK_LAUNCH();
  return CUKD_OK;
}

// Trains on (queries, exact k-th squared distances): standardises the log
// distances, then `epochs` passes of Adam over minibatches of `batch`.
int cukd_radius_model_train(cukd_radius_model *model, const void *d_queries,
                            const void *d_kth_d2, int64_t nq, int epochs, int batch, float lr,
                            float *h_final_loss, cudaStream_t st)
{
  auto *m = (cukd_radius_model_s *)model;
  if (!m || !d_queries || !d_kth_d2 || nq < 2 || epochs < 1 || batch < S || lr <= 0.f)
    return CUKD_ERR_INVALID_ARGUMENT;
  TempArena arena(st, nullptr);
  float *feat = nullptr, *tgt = nullptr;
  CKB_TRY(arena.alloc(&feat, nq * kIn));
  CKB_TRY(arena.alloc(&tgt, nq));
  const unsigned nb = unsigned(div_up(nq, 256));
  CKB_TRY(features_launch(m, d_queries, nq, feat, st));
  if (m->scalar == CUKD_FLOAT32)
    targets_kernel<0><<<nb, 256, 0, st>>>(d_kth_d2, nq, tgt);
  else
    targets_kernel<1><<<nb, 256, 0, st>>>(d_kth_d2, nq, tgt);
  CKB_CHECK_LAUNCH();
  // standardise targets (host statistics; one read of nq floats)
  std::vector<float> ht(nq);
  CKB_CUDA(cudaMemcpyAsync(ht.data(), tgt, sizeof(float) * nq, cudaMemcpyDeviceToHost, st));
  CKB_CUDA(cudaStreamSynchronize(st));
  double s1 = 0, s2 = 0;
  for (float v : ht) {
    s1 += v;
    s2 += double(v) * v;
  }
  const double mean = s1 / nq, var = std::max(1e-12, s2 / nq - mean * mean);
  m->norm.tmean = float(mean);
  m->norm.tstd = float(std::sqrt(var));
  normalize_targets_kernel<<<nb, 256, 0, st>>>(tgt, nq, m->norm.tmean, 1.f / m->norm.tstd);
  CKB_CHECK_LAUNCH();
  const size_t smem = sizeof(TrainSmem);
  CKB_CUDA(cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(smem)));
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  int step = 0;
  CKB_CUDA(cudaMemsetAsync(m->d.loss, 0, sizeof(float) * 2, st));
  for (int e = 0; e < epochs; e++) {
    const bool last = e == epochs - 1;
    for (int64_t b0 = 0; b0 < nq; b0 += batch) {
      const int64_t cnt = std::min<int64_t>(batch, nq - b0);
      train_kernel<<<unsigned(div_up(cnt, S)), kTrainThreads, smem, st>>>(
          m->d.wbf, feat, tgt, b0, cnt, 1.f / float(cnt), m->d.grad, last ? m->d.loss : nullptr,
          m->quantile);
      CKB_CHECK_LAUNCH();
      step++;
      const float c1 = 1.f - std::pow(b1, float(step)), c2 = 1.f - std::pow(b2, float(step));
      adam_kernel<<<div_up(NP, 256), 256, 0, st>>>(m->d.params, m->d.wbf, m->d.m, m->d.v,
                                                   m->d.grad, lr, b1, b2, eps, c1, c2);
      CKB_CHECK_LAUNCH();
    }
  }
  float hl = 0.f;
  CKB_CUDA(cudaMemcpyAsync(&hl, m->d.loss, sizeof(float), cudaMemcpyDeviceToHost, st));
  CKB_CUDA(cudaStreamSynchronize(st));
  m->last_loss = hl / float(nq);
  if (h_final_loss) *h_final_loss = m->last_loss;
  m->trained = 1;
  return CUKD_OK;
}

// Per-query predicted k-th-neighbour distance (before the safety scale).
int cukd_radius_model_predict(const cukd_radius_model *model, const void *d_queries, int64_t nq,
                              float *d_out_radius, cudaStream_t st)
{
  auto *m = (const cukd_radius_model_s *)model;
  if (!m || (nq > 0 && (!d_queries || !d_out_radius))) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq == 0) return CUKD_OK;
  return infer_launch(m, d_queries, nq, d_out_radius, st);
}

// Gradient of the mean squared error over one batch of (features, standardised
// targets) at the current BF16 weights -- for checking against a CPU oracle.
int cukd_radius_model_gradients(cukd_radius_model *model, const float *d_features,
                                const float *d_targets, int64_t n, float *h_grad,
                                float *h_params_bf16, float *h_loss, cudaStream_t st)
{
  auto *m = (cukd_radius_model_s *)model;
  if (!m || !d_features || !d_targets || n < 1) return CUKD_ERR_INVALID_ARGUMENT;
  const size_t smem = sizeof(TrainSmem);
  CKB_CUDA(cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(smem)));
  CKB_CUDA(cudaMemsetAsync(m->d.grad, 0, sizeof(float) * NP, st));
  CKB_CUDA(cudaMemsetAsync(m->d.loss, 0, sizeof(float) * 2, st));
  train_kernel<<<unsigned(div_up(n, S)), kTrainThreads, smem, st>>>(
      m->d.wbf, d_features, d_targets, 0, n, 1.f / float(n), m->d.grad, m->d.loss, m->quantile);
  CKB_CHECK_LAUNCH();
  if (h_grad)
    CKB_CUDA(cudaMemcpyAsync(h_grad, m->d.grad, sizeof(float) * NP, cudaMemcpyDeviceToHost, st));
  if (h_params_bf16) {
    std::vector<__nv_bfloat16> pb(NP);
    CKB_CUDA(cudaMemcpyAsync(pb.data(), m->d.wbf, sizeof(__nv_bfloat16) * NP,
                             cudaMemcpyDeviceToHost, st));
    CKB_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < NP; i++) h_params_bf16[i] = __bfloat162float(pb[i]);
  }
  float hl = 0.f;
  CKB_CUDA(cudaMemcpyAsync(&hl, m->d.loss, sizeof(float), cudaMemcpyDeviceToHost, st));
  CKB_CUDA(cudaStreamSynchronize(st));
  if (h_loss) *h_loss = hl / float(n);
  CKB_CUDA(cudaMemsetAsync(m->d.grad, 0, sizeof(float) * NP, st));
  return CUKD_OK;
}

// Features of a batch of queries (the model's input), for inspection/tests.
int cukd_radius_model_features(const cukd_radius_model *model, const void *d_queries,
                               int64_t nq, float *d_out_features, cudaStream_t st)
{
  auto *m = (const cukd_radius_model_s *)model;
  if (!m || nq < 0) return CUKD_ERR_INVALID_ARGUMENT;
  if (nq == 0) return CUKD_OK;
  return features_launch(m, d_queries, nq, d_out_features, st);
}

// kNN with the learned radius: same results as cukd_knn (plain), see the
// file header.  d_out_fallback (optional, device int[2]): queries re-run by
// the plain traversal, and by the reference's visiting order.  d_visits
// (optional, device int64[nq], zeroed by the caller): nodes visited per
// query over all passes.
int cukd_knn_learned(const void *d_tree, int64_t n, const cukd_layout *layout,
                     const void *d_world_bounds, const void *d_queries, int64_t nq,
                     const cukd_query_params *p, const cukd_radius_model *model,
                     float radius_scale, int32_t *d_out_ids, void *d_out_d2,
                     int32_t *d_out_fallback, int32_t *d_status, int64_t *d_visits,
                     cudaStream_t st, const cukd_mem_resource *mem)
{
  auto *m = (const cukd_radius_model_s *)model;
  ckb::Layout L;
  if (!m || !p || !make_layout(layout, &L) || L.D != m->norm.D || L.scalar != m->scalar)
    return CUKD_ERR_INVALID_ARGUMENT;
  if (p->k < 2 || p->k > 128 || (p->flags & CUKD_QUERY_HEAP_ORDER) || radius_scale <= 0.f ||
      n > kMaxQueryTree)
    return CUKD_ERR_UNSUPPORTED;
  if (nq == 0) return CUKD_OK;
  if (!d_queries || !d_out_ids || (n > 0 && !d_tree)) return CUKD_ERR_INVALID_ARGUMENT;
  TempArena arena(st, mem);
  query::QArgs a = {};
  a.tree = (const uint8_t *)d_tree;
  a.n = n;
  a.stride = L.stride;
  a.poff = L.poff;
  a.doff = L.doff;
  a.dshift = L.dshift;
  a.dmask = L.dmask;
  a.bounds = d_world_bounds;
  a.queries = d_queries;
  a.nq = nq;
  a.k = p->k;
  a.cutoff = p->cutoff_radius;
  a.cutoff_d2 = p->cutoff_d2;
  a.eps = 0.f;
  a.out_ids = d_out_ids;
  a.out_d2 = d_out_d2;
  a.visits = d_visits;
  a.block_size = p->block_size;
  if ((p->flags & CUKD_QUERY_MORTON) && nq > 1 && L.scalar == CUKD_FLOAT32) {
    int32_t *perm = nullptr;
    CKB_TRY(arena.alloc(&perm, nq));
    CKB_TRY(cukd_morton_order((const float *)d_queries, nq, L.D, (const float *)d_world_bounds,
                              perm, st, mem));
    a.order = perm;
  }
  int *ctr = nullptr;
  CKB_TRY(arena.alloc(&ctr, 4));
  CKB_CUDA(cudaMemsetAsync(ctr, 0, 4 * sizeof(int), st));
  int32_t *fb1 = nullptr, *fb2 = nullptr;
  CKB_TRY(arena.alloc(&fb1, nq));
  CKB_TRY(arena.alloc(&fb2, nq));
  fast::FastArgs fa = {};
  fa.q = a;
  fa.kk = p->k;
  fa.work = ctr;
  fa.fb_count = ctr + 1;
  fa.fb_list = fb1;
  fa.radius_scale = radius_scale;
  fa.status = d_status;
  const bool isFloat = L.scalar == CUKD_FLOAT32;
  const bool packet = (p->flags & CUKD_QUERY_WARP_PACKET) && isFloat && p->k <= 32;
  if (isFloat && p->k <= 32 && !packet) {
    // pass 1: radii predicted and searched in one kernel
    const int D = L.D;
    const int rc = D == 2 ? launch_learned_layout<2>(fa, L, m->d.wbf, m->d.dens, m->norm, st)
                 : D == 3 ? launch_learned_layout<3>(fa, L, m->d.wbf, m->d.dens, m->norm, st)
                          : launch_learned_layout<4>(fa, L, m->d.wbf, m->d.dens, m->norm, st);
    CKB_TRY(rc);
  } else {
    // pass 1: the radii predicted for every query, then the seeded traversal
    // (the local-memory heap for k > 32, or the integer kernel)
    float *radius = nullptr;
    CKB_TRY(arena.alloc(&radius, nq));
    CKB_TRY(infer_launch(m, d_queries, nq, radius, st));
    fa.radius = radius;
    CKB_TRY(packet ? run_packet(fa, L.D, st)
                   : (isFloat ? run_fast(fa, L.D, st) : run_fast_int(fa, L.D, st)));
  }
  // pass 2: plain unbounded traversal of the queries pass 1 could not answer
  fast::FastArgs fb = fa;
  fb.radius = nullptr;
  fb.status = nullptr;
  fb.q.order = fb1;
  fb.q.count_ptr = ctr + 1;
  fb.fb_count = ctr + 2;
  fb.fb_list = fb2;
  CKB_TRY(isFloat ? run_fast(fb, L.D, st) : run_fast_int(fb, L.D, st));
  // pass 3: boundary ties in the reference's visiting order
  query::QArgs c = a;
  c.order = fb2;
  c.count_ptr = ctr + 2;
  c.visits = nullptr;
  const int kind = p->k > 32 ? query::RES_HEAP128
                 : p->k <= 4 ? query::RES_FIX4
                             : (p->k <= 8 ? query::RES_FIX8
                                          : (p->k <= 16 ? query::RES_FIX16 : query::RES_FIX32));
  CKB_TRY(query::run_query(c, L.scalar, L.D, p->method, kind, st));
  if (d_out_fallback)
    CKB_CUDA(cudaMemcpyAsync(d_out_fallback, ctr + 1, 2 * sizeof(int), cudaMemcpyDeviceToDevice,
                             st));
  return CUKD_OK;
}

}  // extern "C"
