// mlp_mma.cuh -- warp-level tensor-core inference of the 10-64-64-64-5 SiLU
// surrogate for the 32 droplets of a warp.
//
// BF16 weights, FP32 accumulation: mma.sync.m16n8k16 (bf16 x bf16 -> f32).
// The warp's 32 droplets form two 16-row M tiles.  The input row of each
// droplet is staged once through shared memory as a hi/lo pair of bf16
// values (x = hi + lo to ~16 bits); every later activation stays in
// registers: the FP32 accumulator fragment of an m16n8 tile is exactly the
// register layout of the bf16 A fragment of the next layer, so bias, SiLU and
// the bf16 repacking happen in place.  Only the 5 outputs go back through
// shared memory to the lane that owns the droplet.
//
// Shared-memory weight layout (bf16, row = output unit, padded rows so the
// B-fragment loads of the 8 row groups fall in distinct banks):
//   W1: 64 rows x 40 (cols 0-9 = W1[:,0:10], cols 16-25 = the same again for
//       the lo half of the input, other columns 0)
//   W2, W3: 64 x 72 (cols 0-63)      W4: 8 x 72 (rows 0-4 used)
// Biases FP32: b1[64] b2[64] b3[64] b4[8].
#pragma once

#include <cuda_bf16.h>

namespace pmp {

constexpr int kW1Stride = 40;
constexpr int kWStride = 72;
constexpr int kXStride = 40;  // per-warp input staging row (bf16)
constexpr int kYStride = 9;   // per-warp output staging row (fp32)

struct MlpSmem {
  __nv_bfloat16 w1[64 * kW1Stride];
  __nv_bfloat16 w2[64 * kWStride];
  __nv_bfloat16 w3[64 * kWStride];
  __nv_bfloat16 w4[8 * kWStride];
  float b1[64];
  float b2[64];
  float b3[64];
  float b4[8];
};

struct MlpWarpScratch {
  __nv_bfloat16 x[32 * kXStride];
  float y[32 * kYStride];
};

__device__ __forceinline__ void mma_bf16(float* c, const unsigned* a, unsigned b0, unsigned b1)
{
  asm volatile(
    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
    "{%0,%1,%2,%3};\n"
    : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
    : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi)
{
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&v);
}

// SiLU with the SFU tanh: x * (1 + tanh(x/2)) / 2
__device__ __forceinline__ float silu_fast(float x)
{
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * x));
  return 0.5f * x * (1.f + t);
}

__device__ __forceinline__ unsigned lds32(const __nv_bfloat16* p)
{
  return *reinterpret_cast<const unsigned*>(p);
}

// One hidden layer for one M tile: acc[nt][4] = bias + A(16x64) * W^T, then
// SiLU and repack into the A fragments of the next layer.
__device__ __forceinline__ void hidden_layer(
  const __nv_bfloat16* w, const float* bias, const unsigned (&a)[4][4], unsigned (&out)[4][4], int g, int t)
{
#pragma unroll
  for (int kb2 = 0; kb2 < 4; ++kb2) {
    float acc[2][4];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int nt = 2 * kb2 + h;
      const float bl = bias[8 * nt + 2 * t];
      const float bh = bias[8 * nt + 2 * t + 1];
      acc[h][0] = bl;
      acc[h][1] = bh;
      acc[h][2] = bl;
      acc[h][3] = bh;
      const __nv_bfloat16* row = w + (8 * nt + g) * kWStride + 2 * t;
#pragma unroll
      for (int kb = 0; kb < 4; ++kb) {
        mma_bf16(acc[h], a[kb], lds32(row + 16 * kb), lds32(row + 16 * kb + 8));
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        acc[h][i] = silu_fast(acc[h][i]);
      }
    }
    out[kb2][0] = pack_bf16(acc[0][0], acc[0][1]);
    out[kb2][1] = pack_bf16(acc[0][2], acc[0][3]);
    out[kb2][2] = pack_bf16(acc[1][0], acc[1][1]);
    out[kb2][3] = pack_bf16(acc[1][2], acc[1][3]);
  }
}

// Evaluate the network for the warp.  xin: this lane's 10 normalised inputs;
// yout: this lane's 5 normalised outputs.  All 32 lanes must call it.
__device__ __forceinline__ void mlp_warp(
  const MlpSmem& S, MlpWarpScratch& W, const float* xin, float* yout)
{
  const int lane = threadIdx.x & 31;
  const int g = lane >> 2;
  const int t = lane & 3;
  // stage the input row: hi in cols 0-9, lo in cols 16-25
  __nv_bfloat16* xr = W.x + lane * kXStride;
#pragma unroll
  for (int k = 0; k < 10; ++k) {
    const __nv_bfloat16 hi = __float2bfloat16_rn(xin[k]);
    xr[k] = hi;
    xr[16 + k] = __float2bfloat16_rn(xin[k] - __bfloat162float(hi));
  }
#pragma unroll
  for (int k = 10; k < 16; ++k) {
    xr[k] = __float2bfloat16_rn(0.f);
    xr[16 + k] = __float2bfloat16_rn(0.f);
  }
  __syncwarp();
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    const int r0 = 16 * mt + g;
    unsigned a1[2][4];
#pragma unroll
    for (int kb = 0; kb < 2; ++kb) {
      a1[kb][0] = lds32(W.x + r0 * kXStride + 16 * kb + 2 * t);
      a1[kb][1] = lds32(W.x + (r0 + 8) * kXStride + 16 * kb + 2 * t);
      a1[kb][2] = lds32(W.x + r0 * kXStride + 16 * kb + 2 * t + 8);
      a1[kb][3] = lds32(W.x + (r0 + 8) * kXStride + 16 * kb + 2 * t + 8);
    }
    // layer 1: K = 32 (hi + lo halves)
    unsigned h1[4][4];
#pragma unroll
    for (int kb2 = 0; kb2 < 4; ++kb2) {
      float acc[2][4];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int nt = 2 * kb2 + h;
        const float bl = S.b1[8 * nt + 2 * t];
        const float bh = S.b1[8 * nt + 2 * t + 1];
        acc[h][0] = bl;
        acc[h][1] = bh;
        acc[h][2] = bl;
        acc[h][3] = bh;
        const __nv_bfloat16* row = S.w1 + (8 * nt + g) * kW1Stride + 2 * t;
#pragma unroll
        for (int kb = 0; kb < 2; ++kb) {
          mma_bf16(acc[h], a1[kb], lds32(row + 16 * kb), lds32(row + 16 * kb + 8));
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          acc[h][i] = silu_fast(acc[h][i]);
        }
      }
      h1[kb2][0] = pack_bf16(acc[0][0], acc[0][1]);
      h1[kb2][1] = pack_bf16(acc[0][2], acc[0][3]);
      h1[kb2][2] = pack_bf16(acc[1][0], acc[1][1]);
      h1[kb2][3] = pack_bf16(acc[1][2], acc[1][3]);
    }
    unsigned h2[4][4];
    hidden_layer(S.w2, S.b2, h1, h2, g, t);
    hidden_layer(S.w3, S.b3, h2, h1, g, t);
    // output layer: one n tile of 8 (5 used)
    float acc[4];
    acc[0] = S.b4[2 * t];
    acc[1] = S.b4[2 * t + 1];
    acc[2] = acc[0];
    acc[3] = acc[1];
    const __nv_bfloat16* row = S.w4 + g * kWStride + 2 * t;
#pragma unroll
    for (int kb = 0; kb < 4; ++kb) {
      mma_bf16(acc, h1[kb], lds32(row + 16 * kb), lds32(row + 16 * kb + 8));
    }
    W.y[r0 * kYStride + 2 * t] = acc[0];
    W.y[r0 * kYStride + 2 * t + 1] = acc[1];
    W.y[(r0 + 8) * kYStride + 2 * t] = acc[2];
    W.y[(r0 + 8) * kYStride + 2 * t + 1] = acc[3];
  }
  __syncwarp();
#pragma unroll
  for (int o = 0; o < 5; ++o) {
    yout[o] = W.y[lane * kYStride + o];
  }
  __syncwarp();
}

}  // namespace pmp
