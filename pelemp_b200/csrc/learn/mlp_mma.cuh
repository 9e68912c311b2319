// mlp_mma.cuh -- warp-level tensor-core inference of the 10-64-64-64-5 SiLU
// surrogate for the 32 droplets of a warp.
//
// BF16 weights and activations, FP32 accumulation: mma.sync.m16n8k16
// (bf16 x bf16 -> f32).  The warp's 32 droplets form two 16-row M tiles.  The
// input row of each droplet is staged once through shared memory as a hi/lo
// pair of bf16 values (x = hi + lo to ~16 bits); every later activation stays
// in registers: the FP32 accumulator fragment of an m16n8 tile is the register
// layout of the bf16 A fragment of the next layer, so bias, SiLU and the
// repacking happen in place.  Weight (B) and input (A) fragments are read with
// ldmatrix.x4.  Only the 5 outputs go back through shared memory to the lane
// that owns the droplet.
//
// SiLU in packed bf16x2: the hidden layers' weights and biases are stored
// pre-multiplied by 1/2 (exact in bf16), so a layer produces h = x/2 and
//   silu(x) = x sigmoid(x) = h (1 + tanh h) = fma(h, tanh h, h),
// three bf16x2 instructions per pair: cvt (round h to bf16), tanh.approx,
// fma.rn.  The training forward pass rounds the same way
// (pmp_learn.cu, k_bias_act) so the trained network is the one evaluated here.
//
// Shared-memory weight layout (bf16, row = output unit, rows padded so the
// eight row addresses of an ldmatrix phase fall in distinct banks):
//   W1: 64 rows x 40 (cols 0-9 = W1[:,0:10]/2, cols 16-25 = the same again
//       for the lo half of the input, other columns 0)
//   W2, W3: 64 x 72 (cols 0-63, halved)      W4: 8 x 72 (rows 0-4 used)
// Biases FP32: b1[64]/2 b2[64]/2 b3[64]/2 b4[8].
#pragma once

#include <cuda_bf16.h>

namespace pmp {

constexpr int kW1Stride = 40;
constexpr int kWStride = 72;
constexpr int kXStride = 40;  // per-warp input staging row (bf16)
constexpr int kYStride = 9;   // per-warp output staging row (fp32)

struct __align__(16) MlpSmem {
  __nv_bfloat16 w1[64 * kW1Stride];
  __nv_bfloat16 w2[64 * kWStride];
  __nv_bfloat16 w3[64 * kWStride];
  __nv_bfloat16 w4[8 * kWStride];
  float b1[64];
  float b2[64];
  float b3[64];
  float b4[8];
};

struct __align__(16) MlpWarpScratch {
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

// Four 8x8 b16 matrices; lane l supplies the address of row (l & 7) of matrix
// (l >> 3) and receives, in r[m], row l/4, elements 2(l%4) and 2(l%4)+1 of
// matrix m.
__device__ __forceinline__ void ldsm_x4(unsigned (&r)[4], const void* p)
{
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a)
               : "memory");
}

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi)
{
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<unsigned*>(&v);
}

// silu of the pair (2 h0, 2 h1) as packed bf16x2: fma(h, tanh h, h)
__device__ __forceinline__ unsigned silu_pair(float h0, float h1)
{
  const unsigned p = pack_bf16(h0, h1);
  unsigned t, r;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(p));
  asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(r) : "r"(p), "r"(t));
  return r;
}

// One hidden layer (K = 64) for one M tile: h = bias/2 + A(16x64) (W/2)^T, then
// SiLU, repacked as the A fragments of the next layer.
__device__ __forceinline__ void hidden_layer(
  const __nv_bfloat16* w, const float* bias, const unsigned (&a)[4][4], unsigned (&out)[4][4], int lane)
{
  const int t = lane & 3;
  const __nv_bfloat16* wrow = w + (lane & 7) * kWStride + 8 * (lane >> 3);
#pragma unroll
  for (int kb2 = 0; kb2 < 4; ++kb2) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int nt = 2 * kb2 + h;
      const float2 bb = *reinterpret_cast<const float2*>(bias + 8 * nt + 2 * t);
      float acc[4] = {bb.x, bb.y, bb.x, bb.y};
      unsigned b0[4], b1[4];
      ldsm_x4(b0, wrow + 8 * nt * kWStride);       // k 0..31
      ldsm_x4(b1, wrow + 8 * nt * kWStride + 32);  // k 32..63
      mma_bf16(acc, a[0], b0[0], b0[1]);
      mma_bf16(acc, a[1], b0[2], b0[3]);
      mma_bf16(acc, a[2], b1[0], b1[1]);
      mma_bf16(acc, a[3], b1[2], b1[3]);
      out[kb2][2 * h] = silu_pair(acc[0], acc[1]);      // row g
      out[kb2][2 * h + 1] = silu_pair(acc[2], acc[3]);  // row g + 8
    }
  }
}

// Evaluate the network for the warp.  xin: this lane's 10 normalised inputs;
// yout: this lane's 5 normalised outputs.  All 32 lanes must call it.
__device__ __forceinline__ void mlp_warp(
  const MlpSmem& S, MlpWarpScratch& W, const float* xin, float* yout)
{
  const int lane = threadIdx.x & 31;
  const int t = lane & 3;
  // stage the input row: hi in cols 0-9, lo in cols 16-25, zeros elsewhere
  {
    unsigned hi[8], lo[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float x0 = 2 * j < 10 ? xin[2 * j] : 0.f;
      const float x1 = 2 * j + 1 < 10 ? xin[2 * j + 1] : 0.f;
      const __nv_bfloat162 h = __floats2bfloat162_rn(x0, x1);
      const float2 hf = __bfloat1622float2(h);
      hi[j] = *reinterpret_cast<const unsigned*>(&h);
      lo[j] = pack_bf16(x0 - hf.x, x1 - hf.y);
    }
    uint4* xr = reinterpret_cast<uint4*>(W.x + lane * kXStride);
    xr[0] = make_uint4(hi[0], hi[1], hi[2], hi[3]);
    xr[1] = make_uint4(hi[4], hi[5], hi[6], hi[7]);
    xr[2] = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    xr[3] = make_uint4(lo[4], lo[5], lo[6], lo[7]);
  }
  __syncwarp();
  const int r = lane & 7, mi = lane >> 3;
  const __nv_bfloat16* w1row = S.w1 + r * kW1Stride + 8 * mi;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt) {
    unsigned a1[2][4];
    {
      const __nv_bfloat16* xrow = W.x + (16 * mt + (mi & 1) * 8 + r) * kXStride + (mi >> 1) * 8;
      ldsm_x4(a1[0], xrow);       // hi, k 0..15
      ldsm_x4(a1[1], xrow + 16);  // lo, k 16..31
    }
    // layer 1: K = 32 (hi + lo halves)
    unsigned h1[4][4];
#pragma unroll
    for (int kb2 = 0; kb2 < 4; ++kb2) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int nt = 2 * kb2 + h;
        const float2 bb = *reinterpret_cast<const float2*>(S.b1 + 8 * nt + 2 * t);
        float acc[4] = {bb.x, bb.y, bb.x, bb.y};
        unsigned b[4];
        ldsm_x4(b, w1row + 8 * nt * kW1Stride);
        mma_bf16(acc, a1[0], b[0], b[1]);
        mma_bf16(acc, a1[1], b[2], b[3]);
        h1[kb2][2 * h] = silu_pair(acc[0], acc[1]);
        h1[kb2][2 * h + 1] = silu_pair(acc[2], acc[3]);
      }
    }
    unsigned h2[4][4];
    hidden_layer(S.w2, S.b2, h1, h2, lane);
    hidden_layer(S.w3, S.b3, h2, h1, lane);
    // output layer: one n tile of 8 (5 used), weights not halved
    float acc[4];
    {
      const float2 bb = *reinterpret_cast<const float2*>(S.b4 + 2 * t);
      acc[0] = bb.x;
      acc[1] = bb.y;
      acc[2] = bb.x;
      acc[3] = bb.y;
      const __nv_bfloat16* w4row = S.w4 + r * kWStride + 8 * mi;
      unsigned b0[4], b1[4];
      ldsm_x4(b0, w4row);
      ldsm_x4(b1, w4row + 32);
      mma_bf16(acc, h1[0], b0[0], b0[1]);
      mma_bf16(acc, h1[1], b0[2], b0[3]);
      mma_bf16(acc, h1[2], b1[0], b1[1]);
      mma_bf16(acc, h1[3], b1[2], b1[3]);
    }
    const int r0 = 16 * mt + (lane >> 2);
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
