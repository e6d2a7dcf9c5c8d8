// Learned kNN-radius model: parameter layout, input features and the
// warp-level tensor-core forward pass of the inference kernel (learned.cu).
// No reference counterpart: the
// reference's queries start from the caller's cut-off radius
// (cukd/knn.h:503-511).
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"

namespace ckb {
namespace learned {

constexpr int H = 64;
// network input: the query's D normalised coordinates (D = 2..4), its
// density feature, zeros up to kIn (the first layer's input is padded to 8,
// one k-pair per lane group of the tensor-core fragment)
constexpr int kIn = 8;
constexpr int OW1 = 0;              // [H][kIn]  W1[j][i]
constexpr int OB1 = OW1 + kIn * H;  // [H]
constexpr int OW2 = OB1 + H;        // [H][H]  W2[j][k]: output j, input k
constexpr int OB2 = OW2 + H * H;    // [H]
constexpr int OW3 = OB2 + H;        // [H]
constexpr int OB3 = OW3 + H;        // [1]
constexpr int NP = OB3 + 1;         // 4801 parameters
// every block the forward pass reads as bf16 pairs starts on an even index
static_assert(OB1 % 2 == 0 && OW2 % 2 == 0 && OB2 % 2 == 0 && OW3 % 2 == 0, "pair alignment");

struct Norm {
  float lo[4], invext[4];  // world box: coordinates -> [0, 1]
  int D;                   // dimensions of the tree's points
  int res;                 // grid cells per dimension (res^D cells)
  float invLogMax;         // 1 / log(1 + max cell count)
  float tmean, tstd;       // standardisation of the log k-th distance
};

// Features of one query (coordinates already as floats): f[0..D) the
// coordinates mapped to [-1, 1] over the world box, f[D] log(1 + cell count)
// interpolated multilinearly between the centres of the 2^D cells around the
// query (a smooth density estimate at grid scale), the rest 0.  `dens` holds
// log1pf(count) per cell, computed once per grid; cells are row-major with
// dimension 0 the slowest.
template <int D>
__device__ inline void features(const Norm &nm, const float *dens, const float *q, float *f)
{
  int c0[D];
  float w[D];
#pragma unroll
  for (int d = 0; d < D; d++) {
    const float u = __fmul_rn(__fsub_rn(q[d], nm.lo[d]), nm.invext[d]);
    f[d] = __fsub_rn(__fmul_rn(u, 2.f), 1.f);
    // position in cell-centre coordinates
    float c = __fsub_rn(__fmul_rn(u, float(nm.res)), 0.5f);
    c = fminf(fmaxf(c, 0.f), float(nm.res - 1));
    int ci = int(c);
    ci = ci < nm.res - 1 ? ci : nm.res - 1;
    c0[d] = ci;
    w[d] = __fsub_rn(c, float(ci));
  }
  float acc = 0.f;
#pragma unroll
  for (int corner = 0; corner < (1 << D); corner++) {
    int cell = 0;
    float wt = 1.f;
#pragma unroll
    for (int d = 0; d < D; d++) {
      const int bit = (corner >> d) & 1;
      const int ci = min(c0[d] + bit, nm.res - 1);
      cell = cell * nm.res + ci;
      wt = __fmul_rn(wt, bit ? w[d] : __fsub_rn(1.f, w[d]));
    }
    acc = __fmaf_rn(wt, __ldg(dens + cell), acc);
  }
  f[D] = __fmul_rn(acc, nm.invLogMax);
#pragma unroll
  for (int d = D + 1; d < kIn; d++) f[d] = 0.f;
}

// bf16 rounding of an activation as the tensor-core operands see it
__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi)
{
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // lo in the low half
  return *reinterpret_cast<const uint32_t *>(&v);
}
__device__ __forceinline__ float2 ld_bf16x2(const __nv_bfloat16 *w, int idx)
{
  const uint32_t u = __ldg(reinterpret_cast<const unsigned int *>(w + idx));
  return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u));
}
__device__ __forceinline__ uint32_t ld_u32(const __nv_bfloat16 *w, int idx)
{
  return __ldg(reinterpret_cast<const unsigned int *>(w + idx));
}

// D += A * B for one 16x8x16 tile: A 16x16 bf16 (row), B 16x8 bf16 (col),
// FP32 accumulators (PTX ISA, mma.sync.aligned.m16n8k16 fragment layouts)
__device__ __forceinline__ void mma_16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                          uint32_t b1)
{
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Forward pass of 32 queries on the tensor cores, one query per lane (all
// 32 lanes must take part).  `f` holds this lane's kIn features; returns the
// standardised network output of this lane's query.
//
// Rows of the 32x64 activation tile are the lanes: m-tile 0 = lanes 0..15,
// m-tile 1 = lanes 16..31.  Fragment ownership (groupID g = lane/4,
// t = lane%4): an A fragment holds rows g and g+8 at columns 2t,2t+1 (and
// +8); B holds k = 2t,2t+1 (and +8) of column g; C holds rows g and g+8 at
// columns 2t,2t+1.  So the C fragments of n-tiles 2j and 2j+1 of one layer,
// after bias + ReLU, are exactly the A fragment of k-tile j of the next
// layer: activations never leave registers.  Inputs and hidden activations
// enter the tensor cores as bf16 (the training forward pass rounds them
// the same way); every product is accumulated in FP32.
//   layer 1: [32 x 16 (8 inputs, zero padded)] x W1^T:  2 x 8 mma
//   layer 2: [32 x 64] x W2^T:                           2 x 8 x 4 mma
//   layer 3: 64-wide dot per row on the FP32 cores, reduced over the 4
//            lanes that share a row
__device__ __forceinline__ float mlp_forward_warp(const __nv_bfloat16 *__restrict__ w,
                                                  const float f[kIn])
{
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  // this lane's input pair for column pair t of the A fragment
  const uint32_t pair[4] = {pack_bf16x2(f[0], f[1]), pack_bf16x2(f[2], f[3]),
                            pack_bf16x2(f[4], f[5]), pack_bf16x2(f[6], f[7])};
  const float b3 = __bfloat162float(w[OB3]);
  float y00 = 0.f, y01 = 0.f, y10 = 0.f, y11 = 0.f;  // [m-tile][row g / g+8]
  // rolled loops over m-tiles and layer-2 n-tiles keep one accumulator tile
  // and the 16-register hidden fragment live (the caller may be register-capped)
#pragma unroll 1
  for (int mt = 0; mt < 2; mt++) {
    const int r0 = 16 * mt + g;
    // A fragment: rows r0 and r0 + 8, columns 2t and 2t+1 (inputs); columns
    // 8..15 are zero padding
    uint32_t s0 = 0u, s1 = 0u;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const uint32_t v0 = __shfl_sync(full, pair[j], r0), v1 = __shfl_sync(full, pair[j], r0 + 8);
      s0 = t == j ? v0 : s0;
      s1 = t == j ? v1 : s1;
    }
    const uint32_t a1[4] = {s0, s1, 0u, 0u};
    uint32_t h1[4][4];  // A fragments of layer 2, one per k-tile
#pragma unroll
    for (int nt = 0; nt < 8; nt++) {
      const int col = 8 * nt + 2 * t;
      const float2 bb = ld_bf16x2(w, OB1 + col);
      float c[4] = {bb.x, bb.y, bb.x, bb.y};
      const uint32_t b0 = ld_u32(w, OW1 + kIn * (8 * nt + g) + 2 * t);
      mma_16816(c, a1, b0, 0u);
      const uint32_t lo = pack_bf16x2(fmaxf(c[0], 0.f), fmaxf(c[1], 0.f));
      const uint32_t hi = pack_bf16x2(fmaxf(c[2], 0.f), fmaxf(c[3], 0.f));
      h1[nt >> 1][(nt & 1) * 2 + 0] = lo;
      h1[nt >> 1][(nt & 1) * 2 + 1] = hi;
    }
    float y0 = 0.f, y1 = 0.f;
#pragma unroll 1
    for (int nt = 0; nt < 8; nt++) {
      const int col = 8 * nt + 2 * t;
      const float2 bb = ld_bf16x2(w, OB2 + col);
      float c[4] = {bb.x, bb.y, bb.x, bb.y};
      const int row = OW2 + H * (8 * nt + g);
#pragma unroll
      for (int kt = 0; kt < 4; kt++)
        mma_16816(c, h1[kt], ld_u32(w, row + 16 * kt + 2 * t), ld_u32(w, row + 16 * kt + 8 + 2 * t));
      const float2 w3 = ld_bf16x2(w, OW3 + col);
      y0 = __fmaf_rn(w3.x, fmaxf(c[0], 0.f), y0);
      y0 = __fmaf_rn(w3.y, fmaxf(c[1], 0.f), y0);
      y1 = __fmaf_rn(w3.x, fmaxf(c[2], 0.f), y1);
      y1 = __fmaf_rn(w3.y, fmaxf(c[3], 0.f), y1);
    }
    y0 += __shfl_xor_sync(full, y0, 1);
    y0 += __shfl_xor_sync(full, y0, 2);
    y1 += __shfl_xor_sync(full, y1, 1);
    y1 += __shfl_xor_sync(full, y1, 2);
    if (mt == 0) {
      y00 = y0 + b3;
      y01 = y1 + b3;
    } else {
      y10 = y0 + b3;
      y11 = y1 + b3;
    }
  }
  // lane l's row: m-tile l/16, row (l%16) -> held by lanes 4*(l%8) (+0..3)
  const int src = 4 * (lane & 7);
  const float v0 = __shfl_sync(full, y00, src), v1 = __shfl_sync(full, y01, src);
  const float v2 = __shfl_sync(full, y10, src), v3 = __shfl_sync(full, y11, src);
  const int sel = lane >> 3;
  return sel == 0 ? v0 : (sel == 1 ? v1 : (sel == 2 ? v2 : v3));
}

}  // namespace learned
}  // namespace ckb
