// pmp_learn.cu -- the learned form (PMP_MODE_LEARNED): tuple generation by the
// FP64 teacher, GPU training with the project's own kernels, tensor-core
// inference inside the spray update, the input-range / output gate with the
// FP64 fallback, and the audit that measures the surrogate's error online.
//
// Network: 10 -> 64 -> 64 -> 64 -> 5, SiLU, FP32 master weights trained with
// Adam; the forward pass of training rounds weights and hidden activations to
// bf16 (straight-through gradients) so the trained net is the one the bf16
// tensor-core inference evaluates.  See learn/learn_common.cuh for the
// inputs and targets and learn/mlp_mma.cuh for the inference.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "learn/learn_common.cuh"
#include "learn/mlp_mma.cuh"
#include "learn/mlp_tc.cuh"
#include "pmp_handle.h"
#include "spray_kernels.cuh"

namespace pmp {

// flat parameter layout
constexpr int kP_W1 = 0;               // 64 x 16 (inputs padded to 16)
constexpr int kP_B1 = kP_W1 + 64 * 16;
constexpr int kP_W2 = kP_B1 + 64;      // 64 x 64
constexpr int kP_B2 = kP_W2 + 64 * 64;
constexpr int kP_W3 = kP_B2 + 64;      // 64 x 64
constexpr int kP_B3 = kP_W3 + 64 * 64;
constexpr int kP_W4 = kP_B3 + 64;      // 8 x 64 (outputs padded to 8)
constexpr int kP_B4 = kP_W4 + 8 * 64;
constexpr int kP_N = kP_B4 + 8;
constexpr int kTupleW = 16;            // x[10], y[5], pad

struct LearnParams {
  LearnNorm norm;
  const MlpSmem* mlp;        // warp-level layout (audit)
  const tc::TcMlp* mlp_tc;   // tcgen05 operand layout (the update kernel)
  long long audit_stride;
  long long audit_offset;
  double* audit;  // [0] count, [1..5] sum of squared errors, [6..10] sum of squared targets
  int ncta;       // items of the CTA map
};

struct LearnState {
  // tuples
  float* tuples = nullptr;
  long long cap = 0;
  unsigned long long* d_count = nullptr;
  // parameters and optimiser
  float* params = nullptr;
  float* wq = nullptr;
  float* grads = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  // training work buffers
  int bcap = 0;
  float *X = nullptr, *Yt = nullptr, *H1 = nullptr, *A1 = nullptr, *H2 = nullptr, *A2 = nullptr;
  float *H3 = nullptr, *A3 = nullptr, *Yp = nullptr, *dY = nullptr, *dA = nullptr, *dH = nullptr;
  double* d_stats = nullptr;
  double* d_loss = nullptr;
  // inference
  MlpSmem* d_mlp = nullptr;
  tc::TcMlp* d_mlp_tc = nullptr;
  LearnNorm norm;
  bool trained = false;
  double gate_margin = 0.05;
  double audit_fraction = 0.0;
  double* d_audit = nullptr;
  unsigned long long seed = 1;
  double target_std[kLearnOut] = {1., 1., 1., 1., 1.};  // of the raw targets (report)
};

// ---------------------------------------------------------------------------
// helpers

__host__ __device__ inline unsigned long long mix64(unsigned long long z)
{
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

__host__ __device__ inline double u01(unsigned long long a, unsigned long long b, unsigned long long c)
{
  return (double)(mix64(a ^ mix64(b ^ mix64(c))) >> 11) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

static float host_bf16r(float x)
{
  unsigned u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) {
    return x;
  }
  const unsigned lsb = (u >> 16) & 1u;
  u += 0x7fffu + lsb;
  u &= 0xffff0000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

static __nv_bfloat16 host_bf16(float x)
{
  const float r = host_bf16r(x);
  unsigned u;
  memcpy(&u, &r, 4);
  const unsigned short s = (unsigned short)(u >> 16);
  __nv_bfloat16 b;
  memcpy(&b, &s, 2);
  return b;
}

// ---------------------------------------------------------------------------
// tuple generation

template <int NS, int NF>
__global__ void k_learn_tuples(
  const __grid_constant__ KParams P, long long total, long long stride, long long offset, int augment,
  unsigned long long seed, float* out, unsigned long long* count, long long cap)
{
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= total || (s % stride) != offset) {
    return;
  }
  if (!(P.parts.id[s] > 0)) {
    return;
  }
  const int b = box_of_slot(P, s);
  const BoxEntry& B = P.boxes[b];
  double pos[3], vel[3], Y[NF];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    pos[d] = P.parts.pos[d][s];
    vel[d] = P.parts.rd[PMP_PSTATE_VEL + d][s];
  }
  double T = P.parts.rd[PMP_PSTATE_T][s];
  double dia = P.parts.rd[PMP_PSTATE_DIA][s];
  if (dia < kMixedMinDia) {
    return;
  }
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    Y[f] = P.parts.rd[PMP_PSTATE_Y + f][s];
  }
  GasVals<NS, NF> gpv;
  double cBoilT[NF];
  if (!learn_gas_fp64<NS, NF>(P, B, pos, gpv, cBoilT)) {
    return;
  }
  double Tmax = cBoilT[0];
#pragma unroll
  for (int f = 1; f < NF; ++f) {
    Tmax = dmin(Tmax, cBoilT[f]);
  }
  for (int k = 0; k <= augment; ++k) {
    double Tk = T, dk = dia, vk[3] = {vel[0], vel[1], vel[2]}, Yk[NF];
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      Yk[f] = Y[f];
    }
    if (k > 0) {
      // perturbed state around the droplet: temperature up to near boiling,
      // diameter x e^[-0.6,0.6], slip x e^[-1.5,1.5], composition resampled
      Tk = T + u01(seed, s, 4 * k) * dmax(0.97 * Tmax - T, 0.);
      dk = dmin(80e-6, dmax(2e-6, dia * exp(0.6 * (2. * u01(seed, s, 4 * k + 1) - 1.))));
      const double sc = exp(1.5 * (2. * u01(seed, s, 4 * k + 2) - 1.));
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        vk[d] = gpv.vel[d] + (vel[d] - gpv.vel[d]) * sc;
      }
      if (NF > 1) {
        const double u = u01(seed, s, 4 * k + 3);
        Yk[0] = u;
        Yk[NF > 1 ? 1 : 0] = 1. - u;
      }
    }
    double slip = 0.;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      slip += (gpv.vel[d] - vk[d]) * (gpv.vel[d] - vk[d]);
    }
    slip = sqrt(slip);
    float x[kLearnIn];
    float y[kLearnOut];
    double Yfv[NF];
    if (!learn_teacher<NS, NF>(P, gpv, cBoilT, Tk, dk, Yk, vk, y, Yfv)) {
      continue;
    }
    learn_inputs<NF>(x, dk, Tk, gpv.T, gpv.p, sel(gpv.Y, P.f.dep[0]),
                     NF > 1 ? sel(gpv.Y, P.f.dep[NF > 1 ? 1 : 0]) : 0., gpv.rho, slip, Yk, Yfv);
    const unsigned long long i = atomicAdd(count, 1ULL);
    if ((long long)i < cap) {
      float* o = out + i * kTupleW;
#pragma unroll
      for (int j = 0; j < kLearnIn; ++j) {
        o[j] = x[j];
      }
#pragma unroll
      for (int j = 0; j < kLearnOut; ++j) {
        o[kLearnIn + j] = y[j];
      }
      o[15] = 0.f;
    }
  }
}

// ---------------------------------------------------------------------------
// training kernels

// column statistics: sum, sum of squares, min, max of the 15 tuple columns
__global__ void k_tuple_stats(const float* t, long long n, double* st)
{
  __shared__ double ssum[15], ssq[15];
  __shared__ float smin[15], smax[15];
  if (threadIdx.x < 15) {
    ssum[threadIdx.x] = 0.;
    ssq[threadIdx.x] = 0.;
    smin[threadIdx.x] = 3.4e38f;
    smax[threadIdx.x] = -3.4e38f;
  }
  __syncthreads();
  double ls[15], lq[15];
  float lmin[15], lmax[15];
  for (int c = 0; c < 15; ++c) {
    ls[c] = 0.;
    lq[c] = 0.;
    lmin[c] = 3.4e38f;
    lmax[c] = -3.4e38f;
  }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    for (int c = 0; c < 15; ++c) {
      const float v = t[i * kTupleW + c];
      ls[c] += v;
      lq[c] += (double)v * v;
      lmin[c] = fminf(lmin[c], v);
      lmax[c] = fmaxf(lmax[c], v);
    }
  }
  for (int c = 0; c < 15; ++c) {
    atomicAdd(&ssum[c], ls[c]);
    atomicAdd(&ssq[c], lq[c]);
    // float min/max through the ordered integer view
    const float mn = lmin[c], mx = lmax[c];
    if (mn >= 0.f) {
      atomicMin(reinterpret_cast<int*>(&smin[c]), __float_as_int(mn));
    } else {
      atomicMax(reinterpret_cast<unsigned*>(&smin[c]), __float_as_uint(mn));
    }
    if (mx >= 0.f) {
      atomicMax(reinterpret_cast<int*>(&smax[c]), __float_as_int(mx));
    } else {
      atomicMin(reinterpret_cast<unsigned*>(&smax[c]), __float_as_uint(mx));
    }
  }
  __syncthreads();
  if (threadIdx.x < 15) {
    const int c = threadIdx.x;
    atomicAdd(&st[c], ssum[c]);
    atomicAdd(&st[15 + c], ssq[c]);
    // global min/max kept as doubles through a CAS loop
    unsigned long long* pmn = reinterpret_cast<unsigned long long*>(&st[30 + c]);
    unsigned long long* pmx = reinterpret_cast<unsigned long long*>(&st[45 + c]);
    unsigned long long old = *pmn, assumed;
    do {
      assumed = old;
      if (__longlong_as_double(assumed) <= (double)smin[c]) {
        break;
      }
      old = atomicCAS(pmn, assumed, __double_as_longlong((double)smin[c]));
    } while (old != assumed);
    old = *pmx;
    do {
      assumed = old;
      if (__longlong_as_double(assumed) >= (double)smax[c]) {
        break;
      }
      old = atomicCAS(pmx, assumed, __double_as_longlong((double)smax[c]));
    } while (old != assumed);
  }
}

// Normal equations of the baseline fit in FP64: the upper triangle of F^T F
// (kBaseTerms x kBaseTerms) and F^T Y (kBaseTerms x kLearnOut) over every
// stride-th tuple, F the baseline features of the normalised inputs and Y the
// raw targets.  A block of 256 threads stages 128 tuples' features and
// targets in shared memory; each thread sums fixed entries over them.
constexpr int kBaseCols = kBaseTerms + kLearnOut;
constexpr int kBaseTri = kBaseTerms * (kBaseTerms + 1) / 2;
constexpr int kBaseEntries = kBaseTri + kBaseTerms * kLearnOut;
__global__ void __launch_bounds__(256) k_base_normal(const float* t, long long n, long long stride,
                                                     LearnNorm nrm, double* out)
{
  constexpr int kChunk = 128;  // tuples staged per pass (shared memory)
  __shared__ float F[kChunk][kBaseCols + 1];
  constexpr int kPer = (kBaseEntries + 255) / 256;
  int ea[kPer], eb[kPer];
  double acc[kPer];
#pragma unroll
  for (int q = 0; q < kPer; ++q) {
    const int e = threadIdx.x + 256 * q;
    int a = -1, b = -1;
    if (e < kBaseTri) {
      int r = e;
      a = 0;
      while (r >= kBaseTerms - a) {
        r -= kBaseTerms - a;
        ++a;
      }
      b = a + r;
    } else if (e < kBaseEntries) {
      const int r = e - kBaseTri;
      a = r / kLearnOut;
      b = kBaseTerms + r % kLearnOut;
    }
    ea[q] = a;
    eb[q] = b;
    acc[q] = 0.;
  }
  const long long m = (n + stride - 1) / stride;
  for (long long c0 = (long long)blockIdx.x * kChunk; c0 < m; c0 += (long long)gridDim.x * kChunk) {
    const long long i = c0 + threadIdx.x;
    float* row = F[threadIdx.x % kChunk];
    if (threadIdx.x >= kChunk) {
      // the second half of the block only sums
    } else if (i < m) {
      const float* o = t + (i * stride) * kTupleW;
      float xn[kLearnIn];
      for (int k = 0; k < kLearnIn; ++k) {
        xn[k] = (o[k] - nrm.x_mean[k]) * nrm.x_inv_std[k];
      }
      base_features(xn, base_vars(o, nrm), row);
      for (int k = 0; k < kLearnOut; ++k) {
        row[kBaseTerms + k] = o[kLearnIn + k];
      }
    } else {
      for (int k = 0; k < kBaseCols; ++k) {
        row[k] = 0.f;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      if (ea[q] >= 0) {
        double s = 0.;
        for (int r = 0; r < kChunk; ++r) {
          s = fma((double)F[r][ea[q]], (double)F[r][eb[q]], s);
        }
        acc[q] += s;
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < kPer; ++q) {
    if (ea[q] >= 0) {
      atomicAdd(&out[threadIdx.x + 256 * q], acc[q]);
    }
  }
}

// Sum and sum of squares of each target's residual about the baseline
// (st[0..4], st[5..9]).
__global__ void k_resid_stats(const float* t, long long n, LearnNorm nrm, double* st)
{
  __shared__ double ss[2 * kLearnOut];
  if (threadIdx.x < 2 * kLearnOut) {
    ss[threadIdx.x] = 0.;
  }
  __syncthreads();
  double ls[kLearnOut], lq[kLearnOut];
  for (int k = 0; k < kLearnOut; ++k) {
    ls[k] = 0.;
    lq[k] = 0.;
  }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float* o = t + i * kTupleW;
    float xn[kLearnIn];
    for (int k = 0; k < kLearnIn; ++k) {
      xn[k] = (o[k] - nrm.x_mean[k]) * nrm.x_inv_std[k];
    }
    const BaseVars bv = base_vars(o, nrm);
    for (int k = 0; k < kLearnOut; ++k) {
      const double r = (double)o[kLearnIn + k] - (double)learn_base(nrm, k, xn, bv);
      ls[k] += r;
      lq[k] += r * r;
    }
  }
  for (int k = 0; k < kLearnOut; ++k) {
    atomicAdd(&ss[k], ls[k]);
    atomicAdd(&ss[kLearnOut + k], lq[k]);
  }
  __syncthreads();
  if (threadIdx.x < 2 * kLearnOut) {
    atomicAdd(&st[threadIdx.x], ss[threadIdx.x]);
  }
}

// float min / max through the ordered integer view (mn, mx start at +/-3.4e38)
__device__ __forceinline__ void atomic_min_max_f(float* mn, float* mx, float lo, float hi)
{
  if (lo >= 0.f) {
    atomicMin(reinterpret_cast<int*>(mn), __float_as_int(lo));
  } else {
    atomicMax(reinterpret_cast<unsigned*>(mn), __float_as_uint(lo));
  }
  if (hi >= 0.f) {
    atomicMax(reinterpret_cast<int*>(mx), __float_as_int(hi));
  } else {
    atomicMin(reinterpret_cast<unsigned*>(mx), __float_as_uint(hi));
  }
}

// Range of each target's normalised residual about the baseline over the
// tuples (mm[0..4] min, mm[5..9] max): the residual gate's bounds.
__global__ void k_resid_range(const float* t, long long n, LearnNorm nrm, float* mm)
{
  float lo[kLearnOut], hi[kLearnOut];
  for (int k = 0; k < kLearnOut; ++k) {
    lo[k] = 3.4e38f;
    hi[k] = -3.4e38f;
  }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float* o = t + i * kTupleW;
    float xn[kLearnIn];
    for (int k = 0; k < kLearnIn; ++k) {
      xn[k] = (o[k] - nrm.x_mean[k]) * nrm.x_inv_std[k];
    }
    const BaseVars bv = base_vars(o, nrm);
    for (int k = 0; k < kLearnOut; ++k) {
      const float r = (o[kLearnIn + k] - learn_base(nrm, k, xn, bv) - nrm.y_mean[k]) / nrm.y_std[k];
      lo[k] = fminf(lo[k], r);
      hi[k] = fmaxf(hi[k], r);
    }
  }
  for (int k = 0; k < kLearnOut; ++k) {
    for (int off = 16; off > 0; off >>= 1) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], off));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], off));
    }
    if ((threadIdx.x & 31) == 0) {
      atomic_min_max_f(&mm[k], &mm[kLearnOut + k], lo[k], hi[k]);
    }
  }
}

// batch rows: normalised inputs (16 columns, 10 used) and normalised
// residual targets about the baseline (8, 5 used)
__global__ void k_gather_batch(
  const float* t, long long ntrain, long long base, int B, unsigned long long seed, long long step, int random,
  LearnNorm nrm, float* X, float* Y)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B) {
    return;
  }
  long long i;
  if (random) {
    i = (long long)(mix64(seed ^ mix64((unsigned long long)step * 1315423911ULL + r)) % (unsigned long long)ntrain);
  } else {
    i = base + r;
  }
  const float* o = t + i * kTupleW;
  float xn[kLearnIn];
  for (int k = 0; k < kLearnIn; ++k) {
    xn[k] = (o[k] - nrm.x_mean[k]) * nrm.x_inv_std[k];
  }
  for (int k = 0; k < 16; ++k) {
    X[r * 16 + k] = k < kLearnIn ? xn[k] : 0.f;
  }
  const BaseVars bv = base_vars(o, nrm);
  for (int k = 0; k < 8; ++k) {
    Y[r * 8 + k] = k < kLearnOut ? (o[kLearnIn + k] - learn_base(nrm, k, xn, bv) - nrm.y_mean[k]) / nrm.y_std[k] : 0.f;
  }
}

// C[MxN] (+)= op(A) op(B); A is MxK (TA: stored KxM), B is KxN (TB: stored NxK).
// blockIdx.z splits K; with more than one split the partial sums are atomically added.
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_gemm(
  int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc, int kchunk)
{
  __shared__ float As[16][68];
  __shared__ float Bs[16][68];
  const int tx = threadIdx.x & 15;
  const int ty = threadIdx.x >> 4;
  const int row0 = blockIdx.y * 64;
  const int col0 = blockIdx.x * 64;
  const int kbeg = blockIdx.z * kchunk;
  const int kend = min(K, kbeg + kchunk);
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      acc[i][j] = 0.f;
    }
  }
  for (int k0 = kbeg; k0 < kend; k0 += 16) {
    for (int i = threadIdx.x; i < 1024; i += 256) {
      int r, kk;
      if (TA) {
        r = i & 63;
        kk = i >> 6;
      } else {
        r = i >> 4;
        kk = i & 15;
      }
      const int gr = row0 + r;
      const int gk = k0 + kk;
      float v = 0.f;
      if (gr < M && gk < kend) {
        v = TA ? A[(size_t)gk * lda + gr] : A[(size_t)gr * lda + gk];
      }
      As[kk][r] = v;
    }
    for (int i = threadIdx.x; i < 1024; i += 256) {
      int c, kk;
      if (TB) {
        c = i >> 4;
        kk = i & 15;
      } else {
        c = i & 63;
        kk = i >> 6;
      }
      const int gc = col0 + c;
      const int gk = k0 + kk;
      float v = 0.f;
      if (gc < N && gk < kend) {
        v = TB ? B[(size_t)gc * ldb + gk] : B[(size_t)gk * ldb + gc];
      }
      Bs[kk][c] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        a[i] = As[kk][ty * 4 + i];
        b[i] = Bs[kk][tx * 4 + i];
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = row0 + ty * 4 + i;
    if (r >= M) {
      continue;
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int cc = col0 + tx * 4 + j;
      if (cc < N) {
        if (gridDim.z > 1) {
          atomicAdd(&C[(size_t)r * ldc + cc], acc[i][j]);
        } else {
          C[(size_t)r * ldc + cc] = acc[i][j];
        }
      }
    }
  }
}

__device__ __forceinline__ float silu_exact(float x) { return x / (1.f + expf(-x)); }

// silu(x) as the inference kernel rounds it (mlp_mma.cuh): h = bf16(x/2),
// bf16(fma(h, bf16(tanh h), h))
__device__ __forceinline__ float silu_bf16(float x)
{
  const float h = bf16r(0.5f * x);
  return bf16r(fmaf(h, bf16r(tanhf(h)), h));
}

// H += bias; A = silu(H), with the inference's bf16 roundings when quant
__global__ void k_bias_act(float* H, float* A, const float* bias, int B, int N, int act, int quant)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= (long long)B * N) {
    return;
  }
  const int n = (int)(i % N);
  const float h = H[i] + bias[n];
  H[i] = h;
  if (act) {
    A[i] = quant ? silu_bf16(h) : silu_exact(h);
  }
}

// dY = 2 (Yp - Y) / (B * 5) on the 5 used outputs; loss partial sums
__global__ void k_mse(const float* Yp, const float* Y, float* dY, int B, double* loss)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (i < B * 8) {
    const int k = i & 7;
    if (k < kLearnOut) {
      const float d = Yp[i] - Y[i];
      dY[i] = 2.f * d / (float)(B * kLearnOut);
      l = d * d;
    } else {
      dY[i] = 0.f;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    l += __shfl_down_sync(0xffffffffu, l, o);
  }
  if ((threadIdx.x & 31) == 0 && loss) {
    atomicAdd(loss, (double)l);
  }
}

// dH = dA * silu'(H)
__global__ void k_act_bwd(const float* dA, const float* H, float* dH, long long n)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) {
    return;
  }
  const float h = H[i];
  const float s = 1.f / (1.f + expf(-h));
  dH[i] = dA[i] * s * (1.f + h * (1.f - s));
}

// db[n] += sum over rows of dH[:, n]
__global__ void k_colsum(const float* dH, float* db, int B, int N)
{
  const int n = blockIdx.x;
  float s = 0.f;
  for (int r = threadIdx.x; r < B; r += blockDim.x) {
    s += dH[(size_t)r * N + n];
  }
  __shared__ float red[256];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) {
      red[threadIdx.x] += red[threadIdx.x + o];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    db[n] += red[0];
  }
}

// Adam; wq = the bf16-rounded weights used by the forward pass (biases exact)
__global__ void k_adam(
  float* p, float* wq, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
  float bc1, float bc2, int quant)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) {
    return;
  }
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  p[i] = pi;
  const bool is_bias = (i >= kP_B1 && i < kP_W2) || (i >= kP_B2 && i < kP_W3) || (i >= kP_B3 && i < kP_W4) ||
                       (i >= kP_B4);
  wq[i] = (quant && !is_bias) ? bf16r(pi) : pi;
}

__global__ void k_quantize(const float* p, float* wq, int n, int quant)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) {
    return;
  }
  const bool is_bias = (i >= kP_B1 && i < kP_W2) || (i >= kP_B2 && i < kP_W3) || (i >= kP_B3 && i < kP_W4) ||
                       (i >= kP_B4);
  wq[i] = (quant && !is_bias) ? bf16r(p[i]) : p[i];
}

// ---------------------------------------------------------------------------
// host-side training driver

template <bool TA, bool TB>
static void gemm(int M, int N, int K, const float* A, int lda, const float* Bm, int ldb, float* C, int ldc,
                 cudaStream_t st, bool accumulate_split)
{
  const int kchunk = accumulate_split ? 256 : ((K + 15) / 16) * 16;
  dim3 grid((N + 63) / 64, (M + 63) / 64, accumulate_split ? (K + kchunk - 1) / kchunk : 1);
  k_gemm<TA, TB><<<grid, 256, 0, st>>>(M, N, K, A, lda, Bm, ldb, C, ldc, kchunk);
}

static unsigned nb(long long n, int b = 256) { return (unsigned)((n + b - 1) / b); }

// forward of a batch in the training buffers (X -> Yp); quant rounds activations
static void forward(LearnState* L, const float* w, int B, int quant, cudaStream_t st)
{
  gemm<false, true>(B, 64, 16, L->X, 16, w + kP_W1, 16, L->H1, 64, st, false);
  k_bias_act<<<nb((long long)B * 64), 256, 0, st>>>(L->H1, L->A1, w + kP_B1, B, 64, 1, quant);
  gemm<false, true>(B, 64, 64, L->A1, 64, w + kP_W2, 64, L->H2, 64, st, false);
  k_bias_act<<<nb((long long)B * 64), 256, 0, st>>>(L->H2, L->A2, w + kP_B2, B, 64, 1, quant);
  gemm<false, true>(B, 64, 64, L->A2, 64, w + kP_W3, 64, L->H3, 64, st, false);
  k_bias_act<<<nb((long long)B * 64), 256, 0, st>>>(L->H3, L->A3, w + kP_B3, B, 64, 1, quant);
  gemm<false, true>(B, 8, 64, L->A3, 64, w + kP_W4, 64, L->Yp, 8, st, false);
  k_bias_act<<<nb((long long)B * 8), 256, 0, st>>>(L->Yp, nullptr, w + kP_B4, B, 8, 0, 0);
}

// backward of the MSE loss into L->grads (zeroed here)
static void backward(LearnState* L, const float* w, int B, cudaStream_t st)
{
  cudaMemsetAsync(L->grads, 0, sizeof(float) * kP_N, st);
  // output layer
  gemm<true, false>(8, 64, B, L->dY, 8, L->A3, 64, L->grads + kP_W4, 64, st, true);
  k_colsum<<<8, 256, 0, st>>>(L->dY, L->grads + kP_B4, B, 8);
  gemm<false, false>(B, 64, 8, L->dY, 8, w + kP_W4, 64, L->dA, 64, st, false);
  k_act_bwd<<<nb((long long)B * 64), 256, 0, st>>>(L->dA, L->H3, L->dH, (long long)B * 64);
  // layer 3
  gemm<true, false>(64, 64, B, L->dH, 64, L->A2, 64, L->grads + kP_W3, 64, st, true);
  k_colsum<<<64, 256, 0, st>>>(L->dH, L->grads + kP_B3, B, 64);
  gemm<false, false>(B, 64, 64, L->dH, 64, w + kP_W3, 64, L->dA, 64, st, false);
  k_act_bwd<<<nb((long long)B * 64), 256, 0, st>>>(L->dA, L->H2, L->dH, (long long)B * 64);
  // layer 2
  gemm<true, false>(64, 64, B, L->dH, 64, L->A1, 64, L->grads + kP_W2, 64, st, true);
  k_colsum<<<64, 256, 0, st>>>(L->dH, L->grads + kP_B2, B, 64);
  gemm<false, false>(B, 64, 64, L->dH, 64, w + kP_W2, 64, L->dA, 64, st, false);
  k_act_bwd<<<nb((long long)B * 64), 256, 0, st>>>(L->dA, L->H1, L->dH, (long long)B * 64);
  // layer 1
  gemm<true, false>(64, 16, B, L->dH, 64, L->X, 16, L->grads + kP_W1, 16, st, true);
  k_colsum<<<64, 256, 0, st>>>(L->dH, L->grads + kP_B1, B, 64);
}

static int ensure_batch(LearnState* L, int B)
{
  if (L->bcap >= B) {
    return 0;
  }
  float** bufs[] = {&L->X, &L->Yt, &L->H1, &L->A1, &L->H2, &L->A2, &L->H3, &L->A3, &L->Yp, &L->dY, &L->dA, &L->dH};
  const int widths[] = {16, 8, 64, 64, 64, 64, 64, 64, 8, 8, 64, 64};
  for (int i = 0; i < 12; ++i) {
    cudaFree(*bufs[i]);
    *bufs[i] = nullptr;
    if (cudaMalloc(bufs[i], sizeof(float) * (size_t)B * widths[i]) != cudaSuccess) {
      return -1;
    }
  }
  L->bcap = B;
  return 0;
}

static int ensure_params(LearnState* L)
{
  if (L->params) {
    return 0;
  }
  float** bufs[] = {&L->params, &L->wq, &L->grads, &L->adam_m, &L->adam_v};
  for (auto b : bufs) {
    if (cudaMalloc(b, sizeof(float) * kP_N) != cudaSuccess) {
      return -1;
    }
  }
  if (cudaMalloc(&L->d_stats, sizeof(double) * 64) != cudaSuccess ||
      cudaMalloc(&L->d_loss, sizeof(double)) != cudaSuccess ||
      cudaMalloc(&L->d_mlp, sizeof(MlpSmem)) != cudaSuccess ||
      cudaMalloc(&L->d_mlp_tc, sizeof(tc::TcMlp)) != cudaSuccess ||
      cudaMalloc(&L->d_audit, sizeof(double) * 16) != cudaSuccess) {
    return -1;
  }
  return 0;
}

static void init_params(std::vector<float>& p, unsigned long long seed)
{
  p.assign(kP_N, 0.f);
  auto fill = [&](int off, int rows, int cols, int used_cols, int used_rows) {
    const double bound = sqrt(6.0 / (double)used_cols);  // He-uniform for SiLU
    for (int r = 0; r < rows; ++r) {
      for (int c = 0; c < cols; ++c) {
        if (r < used_rows && c < used_cols) {
          p[off + r * cols + c] = (float)((2.0 * u01(seed, off, r * cols + c) - 1.0) * bound);
        }
      }
    }
  };
  fill(kP_W1, 64, 16, kLearnIn, 64);
  fill(kP_W2, 64, 64, 64, 64);
  fill(kP_W3, 64, 64, 64, 64);
  fill(kP_W4, 8, 64, 64, kLearnOut);
  for (int i = 0; i < 8 * 64; ++i) {
    p[kP_W4 + i] *= 0.1f;
  }
}

// inference weights in the shared-memory layout of mlp_mma.cuh
static void build_mlp(const std::vector<float>& p, MlpSmem& S)
{
  memset(&S, 0, sizeof(S));
  const __nv_bfloat16 z = host_bf16(0.f);
  for (int i = 0; i < 64 * kW1Stride; ++i) {
    S.w1[i] = z;
  }
  for (int i = 0; i < 64 * kWStride; ++i) {
    S.w2[i] = z;
    S.w3[i] = z;
  }
  for (int i = 0; i < 8 * kWStride; ++i) {
    S.w4[i] = z;
  }
  // hidden layers halved (exact): the kernel's SiLU takes h = x/2
  for (int o = 0; o < 64; ++o) {
    for (int k = 0; k < kLearnIn; ++k) {
      S.w1[o * kW1Stride + k] = host_bf16(0.5f * p[kP_W1 + o * 16 + k]);
      S.w1[o * kW1Stride + 16 + k] = host_bf16(0.5f * p[kP_W1 + o * 16 + k]);
    }
    for (int k = 0; k < 64; ++k) {
      S.w2[o * kWStride + k] = host_bf16(0.5f * p[kP_W2 + o * 64 + k]);
      S.w3[o * kWStride + k] = host_bf16(0.5f * p[kP_W3 + o * 64 + k]);
    }
    S.b1[o] = 0.5f * p[kP_B1 + o];
    S.b2[o] = 0.5f * p[kP_B2 + o];
    S.b3[o] = 0.5f * p[kP_B3 + o];
  }
  for (int o = 0; o < 8; ++o) {
    for (int k = 0; k < 64; ++k) {
      S.w4[o * kWStride + k] = host_bf16(o < kLearnOut ? p[kP_W4 + o * 64 + k] : 0.f);
    }
    S.b4[o] = o < kLearnOut ? p[kP_B4 + o] : 0.f;
  }
}

// inference weights in the canonical tcgen05 operand layout of mlp_tc.cuh
static void build_mlp_tc(const std::vector<float>& p, tc::TcMlp& S)
{
  memset(&S, 0, sizeof(S));  // bf16 zero is all-zero bits
  for (int o = 0; o < 64; ++o) {
    for (int k = 0; k < kLearnIn; ++k) {
      S.w1[tc::tc_off(o, k, tc::kK1)] = host_bf16(0.5f * p[kP_W1 + o * 16 + k]);
      S.w1[tc::tc_off(o, 16 + k, tc::kK1)] = host_bf16(0.5f * p[kP_W1 + o * 16 + k]);
    }
    for (int k = 0; k < 64; ++k) {
      S.w2[tc::tc_off(o, k, tc::kHid)] = host_bf16(0.5f * p[kP_W2 + o * 64 + k]);
      S.w3[tc::tc_off(o, k, tc::kHid)] = host_bf16(0.5f * p[kP_W3 + o * 64 + k]);
    }
    S.b1[o] = 0.5f * p[kP_B1 + o];
    S.b2[o] = 0.5f * p[kP_B2 + o];
    S.b3[o] = 0.5f * p[kP_B3 + o];
  }
  for (int o = 0; o < kLearnOut; ++o) {
    for (int k = 0; k < 64; ++k) {
      S.w4[tc::tc_off(o, k, tc::kHid)] = host_bf16(p[kP_W4 + o * 64 + k]);
    }
    S.b4[o] = p[kP_B4 + o];
  }
}

static void upload_mlp_tc(LearnState* L, const std::vector<float>& p)
{
  tc::TcMlp* S = new tc::TcMlp;
  build_mlp_tc(p, *S);
  cudaMemcpy(L->d_mlp_tc, S, sizeof(tc::TcMlp), cudaMemcpyHostToDevice);
  delete S;
}

// ---------------------------------------------------------------------------
// the learned update kernel

// 256 threads, 2 CTAs per SM (128 registers): one copy of the weights in
// shared memory serves 8 warps (measured against 128 threads x 4 CTAs and
// 256 x 3 or 4 CTAs, whose register caps spill more than they gain)
#ifndef PMP_LEARNED_THREADS
#define PMP_LEARNED_THREADS 128  /* one M tile per CTA: 4 warps per barrier (measured against 256) */
#endif
#ifndef PMP_LEARNED_GRID_CAP
/* > 0: at most this many CTAs per SM (the resident ones), each looping over
   map items, so that a CTA allocates tensor memory and loads the weights
   once; 0: one CTA per item.  4 measured against 0: config 5 (calls of one
   sub-cycle) 4.88e9 vs 4.31e9 droplet-substeps/s, config 2 equal */
#define PMP_LEARNED_GRID_CAP 4
#endif
#ifndef PMP_LEARNED_MIN_BLOCKS
#define PMP_LEARNED_MIN_BLOCKS 4  /* 128 registers; 4 CTAs of 47 KB shared memory per SM */
#endif
constexpr int kLearnThreads = PMP_LEARNED_THREADS;  // threads per CTA, a multiple of kBlock
// shared-memory doubles per thread (position, parcel count, start mass, composition)
__host__ __device__ constexpr int learn_stash(int nf) { return 5 + nf; }

// The CTA's droplets step together (a CTA-wide loop over the inner sub-steps)
// so that every sub-step evaluates the network for all of them at once:
// kBlock = 128 droplets per tcgen05 M tile, BLOCK / kBlock tiles per CTA.
template <int NS, int NF, int BLOCK, bool FF>
__global__ void __launch_bounds__(BLOCK, PMP_LEARNED_MIN_BLOCKS)
  spray_update_learned(const __grid_constant__ KParams P, const __grid_constant__ LearnParams L)
{
  constexpr int TILES = BLOCK / tc::kTile;
  static_assert(BLOCK % tc::kTile == 0 && tc::kTile == kBlock, "one M tile per CTA-map item");
  static_assert(TILES == 1 || TILES == 2 || TILES == 4, "TMEM is allocated in powers of 2 columns");
  // dynamic shared memory: the network's weights (tcgen05 operand layout),
  // one A operand per tile, then per thread the values the droplet physics
  // does not read (learn_stash(NF) doubles, stride BLOCK)
  extern __shared__ __align__(128) unsigned char learn_smem[];
  tc::TcMlp& S = *reinterpret_cast<tc::TcMlp*>(learn_smem);
  tc::TcTileA* A = reinterpret_cast<tc::TcTileA*>(learn_smem + sizeof(tc::TcMlp));
  double* sx = reinterpret_cast<double*>(learn_smem + sizeof(tc::TcMlp) + sizeof(tc::TcTileA) * TILES) +
               threadIdx.x;
  __shared__ uint32_t tmem_slot;
  __shared__ unsigned long long mbar_slot;
  __shared__ unsigned long long wbar_slot;
  // the weights arrive by one bulk copy while the droplets are read and the
  // first gather runs; the first network evaluation waits for them
  static_assert(sizeof(tc::TcMlp) % 16 == 0, "bulk copies move multiples of 16 bytes");
  // a failed call since the last status read: leave the droplets (before any
  // copy is issued or tensor memory allocated)
  if (cta_call_failed(P)) {
    return;
  }
  const uint32_t wbar = tc::smem_u32(&wbar_slot);
  if (threadIdx.x == 0) {
    tc::mbar_init(wbar);
    tc::bulk_load(&S, L.mlp_tc, (uint32_t)sizeof(tc::TcMlp), wbar);
  }
  tc::TcCta tcs = tc::tc_setup(&tmem_slot, &mbar_slot, TILES * tc::kCols);
  bool weights_in = false;  // uniform over the CTA
  const DevMechF& m = P.mf;
  const DevFuelF& ff = P.ff;
  const DevFuel& fdat = P.f;
  // each group of kBlock threads takes one kBlock-slot item of the CTA map;
  // a CTA takes TILES items, and loops to the next TILES items gridDim.x
  // apart when the grid is smaller than the map
  __shared__ BoxEntry sB[TILES];
  Counters c;
  bool tc_dead = false;  // a timed-out MMA wait stops the CTA (uniform)
  for (int it = blockIdx.x; it * TILES < L.ncta && !tc_dead; it += gridDim.x) {
    const int item = it * TILES + threadIdx.x / kBlock;
    const bool item_ok = item < L.ncta;
    const int b = item_ok ? P.cta_box[item] : 0;
    // this item's box entry, staged in shared memory (after the previous
    // item's readers are done)
    __syncthreads();
    {
      const int h = threadIdx.x / kBlock;
      const int* src = reinterpret_cast<const int*>(P.boxes + b);
      int* dst = reinterpret_cast<int*>(&sB[h]);
      for (int i = threadIdx.x % kBlock; i < (int)(sizeof(BoxEntry) / 4); i += kBlock) {
        dst[i] = src[i];
      }
    }
    __syncthreads();
    const BoxEntry& B = sB[threadIdx.x / kBlock];
    const long long s = item_ok ? P.cta_start[item] + threadIdx.x % kBlock : 0;
    bool valid = item_ok && s < B.p_end;
    int id = valid ? P.parts.id[s] : 0;
    valid = valid && id > 0;
    double dia = valid ? P.parts.rd[PMP_PSTATE_DIA][s] : 1e-5;
    if (valid && dia < P.mixed_min_dia) {
      if (!P.fb_pre) {
        push_fallback(P, s);
      }
      valid = false;
    }
    double pos[3] = {0., 0., 0.}, vel[3] = {0., 0., 0.}, Y[NF];
    double T = 300.;
#pragma unroll
    for (int f = 0; f < NF; ++f) {
      Y[f] = 0.;
    }
    double num_ppp = 0., film = 0.;
    if (valid) {
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        pos[d] = P.parts.pos[d][s];
        vel[d] = P.parts.rd[PMP_PSTATE_VEL + d][s];
      }
      T = P.parts.rd[PMP_PSTATE_T][s];
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        Y[f] = P.parts.rd[PMP_PSTATE_Y + f][s];
      }
      num_ppp = P.parts.rd[PMP_PSTATE_NUMDENS(NF)][s];
      film = P.parts.rd[PMP_PSTATE_FILMHGHT(NF)][s];
    }
    int bflags[3] = {0, 0, 0};
    bool ok = true;
    if (valid && B.at_bounds) {
      if (check_bounds(P, pos, bflags)) {
        set_error(P, PMP_ERR_LEFT_DOMAIN, b, s);
        ok = false;
      }
    }
    // a wall-film droplet stops the first sub-cycle (the film height never
    // changes here, so the check is made once)
    if (valid && ok && P.num_iter > 0 && id > 0 && film > 0.) {
      set_error(P, PMP_ERR_UNSUPPORTED, b, s);
      ok = false;
    }
    sx[3 * BLOCK] = num_ppp;
    for (int cur_iter = 0; cur_iter < P.num_iter; ++cur_iter) {
      // cell of the droplet (recomputed from the position each sub-cycle, so
      // the stencil indices are not live across the network evaluation)
      double lx[3];
      int ijk[3], ijkc[3];
      cell_of(P, pos, lx, ijk, ijkc);
      bool active = valid && ok && id > 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        sx[d * BLOCK] = pos[d];
      }
      GasF<NS> g;
      float cBoilT[NF];
      g.T = 0.f;
      g.rho = 1.f;
      g.p = 1.f;
      g.mw_mix = 1.f;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        g.vel[d] = 0.f;
      }
#pragma unroll
      for (int n = 0; n < NS; ++n) {
        g.Y[n] = 0.f;
      }
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        cBoilT[f] = 400.f;
      }
      if (active) {
        double ssv[2][3];
#pragma unroll
        for (int dir = 0; dir < 3; ++dir) {
          const double sx_hi = __dsub_rn(lx[dir], static_cast<double>(ijk[dir]));
          const double sx_lo = __dsub_rn(1., sx_hi);
          ssv[0][dir] = bflags[dir] > 1 ? 1. : (bflags[dir] < -1 ? 0. : sx_lo);
          ssv[1][dir] = bflags[dir] > 1 ? 0. : (bflags[dir] < -1 ? 1. : sx_hi);
        }
        constexpr int R4 = gas_rec4(NS);
        float rho = 0.f, Tg = 0.f, vg[3] = {0.f, 0.f, 0.f}, Yg[NS];
#pragma unroll
        for (int n = 0; n < NS; ++n) {
          Yg[n] = 0.f;
        }
        bool state_ok = true;
        // FP32 weights, corners chosen by the FP64 factors' signs, one bounds
        // check for the whole stencil (as the mixed form's gather)
        float wf[2][3];
#pragma unroll
        for (int dir = 0; dir < 3; ++dir) {
          wf[0][dir] = (float)ssv[0][dir];
          wf[1][dir] = (float)ssv[1][dir];
        }
        const bool stencil_in = in_box(B.state_lo, B.state_hi, ijk[0] - 1, ijk[1] - 1, ijk[2] - 1) &&
                                in_box(B.state_lo, B.state_hi, ijk[0], ijk[1], ijk[2]);
#pragma unroll
        for (int kk = -1; kk < 1; ++kk) {
#pragma unroll
          for (int jj = -1; jj < 1; ++jj) {
#pragma unroll
            for (int ii = -1; ii < 1; ++ii) {
              if (ssv[ii + 1][0] > 0. && ssv[jj + 1][1] > 0. && ssv[kk + 1][2] > 0.) {
                const int ci = ijk[0] + ii, cj = ijk[1] + jj, ck = ijk[2] + kk;
                if (!stencil_in && !in_box(B.state_lo, B.state_hi, ci, cj, ck)) {
                  state_ok = false;
                } else {
                  float rec[4 * R4];
                  load_gas_rec<R4>(B, ci, cj, ck, rec);
                  const float w = wf[ii + 1][0] * wf[jj + 1][1] * wf[kk + 1][2];
                  rho = fmaf(w, rec[0], rho);
                  Tg = fmaf(w, rec[1], Tg);
#pragma unroll
                  for (int dir = 0; dir < 3; ++dir) {
                    vg[dir] = fmaf(w, rec[2 + dir], vg[dir]);
                  }
#pragma unroll
                  for (int n = 0; n < NS; ++n) {
                    Yg[n] = fmaf(w, rec[5 + n], Yg[n]);
                  }
                }
              }
            }
          }
        }
        if (!state_ok) {
          set_error(P, PMP_ERR_STATE_BOX, b, s);
          ok = false;
          active = false;
        } else {
          g.rho = rho;
          g.T = Tg;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            g.vel[d] = vg[d];
          }
          float mwinv = 0.f;
#pragma unroll
          for (int n = 0; n < NS; ++n) {
            g.Y[n] = Yg[n];
            mwinv = fmaf(g.Y[n], m.inv_mw_kg[n], mwinv);
          }
          g.p = g.rho * (float)(kRuCgs * kRuConv) * mwinv * g.T;
          g.mw_mix = fdiv(1.f, mwinv);
          const float lp = flog(fdiv((float)(kPatmCgs * kPresConv), g.p));
#pragma unroll
          for (int spf = 0; spf < NF; ++spf) {
            cBoilT[spf] = fminf(ff.critT[spf], fdiv(1.f, fmaf(lp, ff.hb[spf], ff.inv_boilT[spf])));
          }
        }
      }
      // calculateSpraySource with the surrogate for the evaporation sub-step
      SrcD<NF> src;
      double Y_part[NF];
      double vel_part[3] = {vel[0], vel[1], vel[2]};
      if (fdat.fixed_parts) {
        vel_part[0] = vel_part[1] = vel_part[2] = 0.;
      }
      double T_part = T, dia_part = dia;
#pragma unroll
      for (int spf = 0; spf < NF; ++spf) {
        Y_part[spf] = Y[spf];
      }
      double rho_part = mixed_rho_liquid<NF>(fdat, Y_part, T_part, cBoilT);
      double dt = P.sub_dt;
      const double flow_dt = P.sub_dt;
      int isub = 1, nsub = 1;
      double pmass = PMP_PI / 6. * rho_part * (dia_part * dia_part * dia_part);
      sx[4 * BLOCK] = pmass;
#pragma unroll
      for (int spf = 0; spf < NF; ++spf) {
        sx[(5 + spf) * BLOCK] = Y[spf];
      }
      // sums over the inner sub-steps in FP32; times the parcel count in FP64 at the end
      float eng_acc = 0.f, mom_acc[3] = {0.f, 0.f, 0.f};
      float T_h = (float)T_part;
      bool pending = active;
      bool fell_back = false;
      while (__syncthreads_or(pending)) {
        // closed-form vapor state, then the surrogate inputs
        float xin[kLearnIn];
        float xn[kLearnIn];
        float L_fuel[NF], X_vapor[NF], Yfv[NF];
        float sumXVap, B_M;
        bool in_range = true;
        vapor_state_f<NS, NF, FF>(m, ff, fdat, g, cBoilT, (float)T_part, Y_part, L_fuel, X_vapor, Yfv, sumXVap, B_M);
        {
          double slip = 0.;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const double dv = (double)g.vel[d] - vel_part[d];
            slip += dv * dv;
          }
          slip = sqrt(slip);
          xin[0] = flog((float)dia_part);
          xin[1] = (float)T_part;
          xin[2] = g.T;
          xin[3] = flog(g.p * (float)(1. / (kPatmCgs * kPresConv)));
          xin[4] = fsel(g.Y, dep_sp<FF>(fdat, 0));
          xin[5] = NF > 1 ? fsel(g.Y, dep_sp<FF>(fdat, NF > 1 ? 1 : 0)) : 0.f;
          xin[6] = flog((float)(g.rho * slip * dia_part) + 1e-12f);
          xin[7] = (float)Y_part[0];
          xin[8] = Yfv[0];
          xin[9] = NF > 1 ? Yfv[NF > 1 ? 1 : 0] : 0.f;
#pragma unroll
          for (int k = 0; k < kLearnIn; ++k) {
            xn[k] = pending ? (xin[k] - L.norm.x_mean[k]) * L.norm.x_inv_std[k] : 0.f;
            in_range = in_range && xin[k] >= L.norm.x_lo[k] && xin[k] <= L.norm.x_hi[k];
          }
        }
        // the targets' baseline plus the residual mean; the network adds the
        // residual (outputs 1 unused with one fuel)
        float yb[kLearnOut];
        {
          const BaseVars bv = base_vars(xin, L.norm);
#pragma unroll
          for (int k = 0; k < kLearnOut; ++k) {
            yb[k] = (NF > 1 || k != 1) && pending ? learn_base(L.norm, k, xn, bv) + L.norm.y_mean[k] : 0.f;
          }
        }
        float yo[kLearnOut];
        if (!weights_in) {
          weights_in = true;
          if (__syncthreads_and(tc::mbar_wait(wbar, 0)) == 0) {
            // the weights never landed: stop the CTA (the copy is waited for
            // once more before the exit)
            tc_dead = true;
            pending = false;
            active = false;
            valid = false;
            weights_in = false;
            if (threadIdx.x == 0) {
              set_error(P, PMP_ERR_TIMEOUT, b, s);
            }
            continue;
          }
        }
        if (!tc::mlp_cta_tc<TILES>(S, A, tcs, xn, yo)) {
          // an MMA completion wait timed out (uniformly over the CTA): stop, no
          // further droplet of the CTA is written
          tc_dead = true;
          pending = false;
          active = false;
          valid = false;
          if (threadIdx.x == 0) {
            set_error(P, PMP_ERR_TIMEOUT, b, s);
          }
          tc::mbar_wait(tcs.mbar, tcs.phase ^ 1u);  // the MMAs the timed-out wait was for
          continue;
        }
        if (pending) {
          float yv[kLearnOut];
#pragma unroll
          for (int k = 0; k < kLearnOut; ++k) {
            yv[k] = fmaf(yo[k], L.norm.y_std[k], yb[k]);
          }
          if (cur_iter == 0 && isub == 1) {
            // gate: some fuel evaporates, inputs inside the (widened)
            // training range, outputs finite, and the predicted residuals
            // about the baseline inside the (widened) training range
            bool in = sumXVap > 0.f && in_range;
#pragma unroll
            for (int k = 0; k < kLearnOut; ++k) {
              in = in && isfinite(yv[k]) &&
                   ((k == 1 && NF == 1) || (yo[k] >= L.norm.r_lo[k] && yo[k] <= L.norm.r_hi[k]));
            }
            if (!in) {
              push_fallback_back(P, s);
              fell_back = true;
              valid = false;
              active = false;
              pending = false;
            }
          }
        }
        if (pending) {
          float yv[kLearnOut];
#pragma unroll
          for (int k = 0; k < kLearnOut; ++k) {
            yv[k] = fmaf(yo[k], L.norm.y_std[k], yb[k]);
          }
          const float Tp_f = (float)T_part;
          T_h = Tp_f;
          const float dia_f = (float)dia_part;
          float cp_part = 0.f;
          double Tboil = 0.;
#pragma unroll
          for (int spf = 0; spf < NF; ++spf) {
            Tboil += Y_part[spf] * (double)cBoilT[spf];
            cp_part += (float)Y_part[spf] * ff.cp[spf];
          }
          const float delT = fmaxf(g.T - Tp_f, 0.f);
          float mi_dot[NF];
          float m_dot = 0.f, sumL = 0.f;
          if (sumXVap > 0.f) {
            // mdot_f = -pi d (rhoD_f Sh*) (X_v,f / sum X_v) ln(1 + B_M), clipped at 0
            const float coef = (float)PMP_PI * dia_f * flog1p(B_M) * fdiv(1.f, sumXVap);
#pragma unroll
            for (int spf = 0; spf < NF; ++spf) {
              mi_dot[spf] = -fmaxf(fexp(yv[spf < 2 ? spf : 0]) * X_vapor[spf] * coef, 0.f);
              m_dot += mi_dot[spf];
              sumL += mi_dot[spf] * L_fuel[spf];
            }
          } else {
#pragma unroll
            for (int spf = 0; spf < NF; ++spf) {
              mi_dot[spf] = 0.f;
            }
          }
          const float conv_src = (float)PMP_PI * dia_f * delT * fexp(yv[2]);
          const float mu_skin = fexp(yv[3]);
          const float rho_skin = fexp(yv[4]);
          float diff_vel[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            diff_vel[d] = g.vel[d] - (float)vel_part[d];
          }
          const float diff_vel_mag =
            sqrtf(diff_vel[0] * diff_vel[0] + diff_vel[1] * diff_vel[1] + diff_vel[2] * diff_vel[2]);
          const float Reyn = fdiv(rho_skin * diff_vel_mag * dia_f, mu_skin);
          const float inv_pmass = __frcp_rn((float)pmass);  // consumed in FP32
          float drag_coef = 0.f;
          if (Reyn > 1000.f) {
            drag_coef = 0.424f;
          } else if (Reyn > 1.f) {
            drag_coef = fdiv(24.f, Reyn) * (1.f + fcbrt(Reyn * Reyn) * (1.f / 6.f));
          } else if (Reyn > 0.f) {
            drag_coef = fdiv(24.f, Reyn);
          }
          const float drag_force = 0.125f * rho_skin * drag_coef * (float)PMP_PI * dia_f * dia_f * diff_vel_mag;
          const float drag_force_p = fdiv(0.75f * rho_skin * drag_coef * diff_vel_mag, dia_f * (float)rho_part);
          float part_vel_src[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            part_vel_src[d] = drag_force_p * diff_vel[d] + ff.body_force[d];
          }
          if (fdat.mom_trans) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              mom_acc[d] = fmaf(drag_force, diff_vel[d], mom_acc[d]);
            }
            if (isub == 1) {
              nsub = min(max(nsub, static_cast<int>((float)flow_dt * drag_force_p) + 1), 100);
            }
          }
          eng_acc += conv_src;
          const float part_temp_src = fdiv((sumL + conv_src) * inv_pmass, cp_part);
          if (isub == 1 && delT > 1e-15f) {
            const float inv_tau_d = fdiv(-m_dot, 0.2f * (float)pmass);
            const float inv_tau_T = fdiv(conv_src * inv_pmass, cp_part * delT);
            nsub = min(max(nsub, max(static_cast<int>((float)flow_dt * inv_tau_d),
                                     static_cast<int>((float)flow_dt * inv_tau_T)) + 1),
                       100);
          }
          if (isub == 1) {
            dt = nsub == 1 ? flow_dt : flow_dt / static_cast<double>(nsub);
          }
          const double part_dt = fdat.dtmod * dt;
          if (!fdat.fixed_parts) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
              vel_part[d] += part_dt * (double)part_vel_src[d];
            }
          }
          const double newT = T_part + part_dt * (double)part_temp_src;
          const double new_mass = pmass + (double)m_dot * part_dt;
          if (new_mass > 1.E-13 * kMassConv && newT < Tboil) {
            T_part = newT;
            if (NF > 1) {
              mixed_new_composition<NF>(Y_part, pmass, mi_dot, part_dt, new_mass);
            }
            pmass = new_mass;
            mixed_rho_dia<NF>(fdat, Y_part, T_part, cBoilT, pmass, rho_part, dia_part);
          } else {
            pmass = 0.;
            id = -1;
            nsub = isub;
            isub = nsub + 1;
          }
          ++isub;
          pending = isub <= nsub;
        }
      }
      // back from shared memory (volatile: read there, not kept in registers
      // across the sub-steps), and the cell the position gives
      const volatile double* vx = sx;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        pos[d] = vx[d * BLOCK];
      }
      num_ppp = vx[3 * BLOCK];
      const double startmass = vx[4 * BLOCK];
#pragma unroll
      for (int spf = 0; spf < NF; ++spf) {
        Y[spf] = vx[(5 + spf) * BLOCK];
      }
      cell_of(P, pos, lx, ijk, ijkc);
      if (fell_back) {
        continue;
      }
      if (active) {
        src.eng = num_ppp * (double)eng_acc;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          src.mom[d] = num_ppp * (double)mom_acc[d];
        }
        if (nsub > 1) {
          src.eng /= static_cast<double>(nsub);
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            src.mom[d] /= static_cast<double>(nsub);
          }
        }
        const double inv_dtf = P.inv_dtf;  // 1 / (dtmod sub_dt), computed on the host
        const double mdot_total = (pmass - startmass) * inv_dtf;
        src.mass = num_ppp * mdot_total;
        if (fdat.mom_trans) {
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            src.mom[d] += num_ppp * vel_part[d] * mdot_total;
          }
        }
#pragma unroll
        for (int spf = 0; spf < NF; ++spf) {
          const double midot = (Y_part[spf] * pmass - Y[spf] * startmass) * inv_dtf;
          src.Ydot[spf] = num_ppp * midot;
          src.eng += num_ppp * midot * (double)hf(m, dep_sp<FF>(fdat, spf), T_h);
          Y[spf] = Y_part[spf];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          vel[d] = vel_part[d];
        }
        T = T_part;
        dia = dia_part;
        c.sub += 1;
        c.inner += static_cast<unsigned>(nsub);
        // deposit into the cell holding the droplet (SprayParticles.cpp:419-441)
        const double cur_coef = P.cur_coef;  // -(1/V) sub_dt / flow_dt, computed on the host
        bool src_ok = in_box(B.src_lo, B.src_hi, ijkc[0], ijkc[1], ijkc[2]) ||
                      (P.is_ghost && in_box(B.sr_alo, B.sr_ahi, ijkc[0], ijkc[1], ijkc[2]));
        if (!src_ok) {
          set_error(P, PMP_ERR_SOURCE_BOX, b, s);
          ok = false;
        } else {
          double* q = B.sr + ((ijkc[0] - B.sr_lo[0]) + (ijkc[1] - B.sr_lo[1]) * B.sr_j32 + (ijkc[2] - B.sr_lo[2]) * B.sr_k32);
          deposit<NF>(P, q, B.sr_n32, cur_coef, src.mom, src.mass, src.Ydot, src.eng);
          if (P.do_move && !fdat.fixed_parts && id > 0) {
#pragma unroll
            for (int dir = 0; dir < 3; ++dir) {
              pos[dir] = __dadd_rn(pos[dir], __dmul_rn(P.sub_dt, vel[dir]));
            }
            if (B.at_bounds) {
              if (check_bounds(P, pos, bflags)) {
                id = -1;
              } else {
                impose_wall(P, pos, vel, bflags);
              }
            }
            cell_of(P, pos, lx, ijk, ijkc);
          }
          if (P.is_ghost && !in_box(B.src_lo, B.src_hi, ijkc[0], ijkc[1], ijkc[2])) {
            id = -1;
          }
        }
      }
    }
    if (valid && ok) {
      if (P.do_move) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          P.parts.pos[d][s] = pos[d];
        }
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        P.parts.rd[PMP_PSTATE_VEL + d][s] = vel[d];
      }
      P.parts.rd[PMP_PSTATE_T][s] = T;
      P.parts.rd[PMP_PSTATE_DIA][s] = dia;
#pragma unroll
      for (int f = 0; f < NF; ++f) {
        P.parts.rd[PMP_PSTATE_Y + f][s] = Y[f];
      }
      if (id <= 0) {
        P.parts.id[s] = id;
        c.killed += 1;
      }
    }
  }  // items
  if (!weights_in) {
    tc::mbar_wait(wbar, 0);  // no network evaluation waited for the weight copy: it must land before the exit
  }
  tc::tc_teardown(tcs, TILES * tc::kCols);
  flush_counters(P, c);
}

// silu from the halved pre-activation h2 = x/2, rounded as the kernel does
__device__ __forceinline__ float silu_half_bf16(float h2)
{
  const float h = bf16r(h2);
  return bf16r(fmaf(h, bf16r(tanhf(h)), h));
}

// SIMT FP32 forward with the inference weights (audit)
__device__ void mlp_simt(const MlpSmem& S, const float* xn, float* y)
{
  float h[64], h2[64];
  for (int o = 0; o < 64; ++o) {
    float a = S.b1[o];
    for (int k = 0; k < kLearnIn; ++k) {
      const float hi = bf16r(xn[k]);
      const float lo = bf16r(xn[k] - hi);
      a = fmaf(__bfloat162float(S.w1[o * kW1Stride + k]), hi + lo, a);
    }
    h[o] = silu_half_bf16(a);
  }
  for (int o = 0; o < 64; ++o) {
    float a = S.b2[o];
    for (int k = 0; k < 64; ++k) {
      a = fmaf(__bfloat162float(S.w2[o * kWStride + k]), h[k], a);
    }
    h2[o] = silu_half_bf16(a);
  }
  for (int o = 0; o < 64; ++o) {
    float a = S.b3[o];
    for (int k = 0; k < 64; ++k) {
      a = fmaf(__bfloat162float(S.w3[o * kWStride + k]), h2[k], a);
    }
    h[o] = silu_half_bf16(a);
  }
  for (int o = 0; o < kLearnOut; ++o) {
    float a = S.b4[o];
    for (int k = 0; k < 64; ++k) {
      a = fmaf(__bfloat162float(S.w4[o * kWStride + k]), h[k], a);
    }
    y[o] = a;
  }
}

// The audit: on every audit_stride-th droplet, compare the surrogate with the
// FP64 teacher at the droplet's state at call entry.
template <int NS, int NF>
__global__ void k_learn_audit(const __grid_constant__ KParams P, const __grid_constant__ LearnParams L, long long total)
{
  const long long s = (blockIdx.x * (long long)blockDim.x + threadIdx.x) * L.audit_stride + L.audit_offset;
  if (s >= total || !(P.parts.id[s] > 0)) {
    return;
  }
  const double dia = P.parts.rd[PMP_PSTATE_DIA][s];
  if (dia < P.mixed_min_dia) {  // the droplets the FP64 kernel updates
    return;
  }
  const BoxEntry& B = P.boxes[box_of_slot(P, s)];
  double pos[3], vel[3], Y[NF];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    pos[d] = P.parts.pos[d][s];
    vel[d] = P.parts.rd[PMP_PSTATE_VEL + d][s];
  }
  const double T = P.parts.rd[PMP_PSTATE_T][s];
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    Y[f] = P.parts.rd[PMP_PSTATE_Y + f][s];
  }
  GasVals<NS, NF> gpv;
  double cBoilT[NF];
  if (!learn_gas_fp64<NS, NF>(P, B, pos, gpv, cBoilT)) {
    return;
  }
  double slip = 0.;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    slip += (gpv.vel[d] - vel[d]) * (gpv.vel[d] - vel[d]);
  }
  slip = sqrt(slip);
  float x[kLearnIn], xn[kLearnIn], yt[kLearnOut], yp[kLearnOut];
  double Yfv[NF];
  if (!learn_teacher<NS, NF>(P, gpv, cBoilT, T, dia, Y, vel, yt, Yfv)) {
    return;  // no fuel evaporates: the gate sends it to the FP64 kernel
  }
  learn_inputs<NF>(x, dia, T, gpv.T, gpv.p, sel(gpv.Y, P.f.dep[0]),
                   NF > 1 ? sel(gpv.Y, P.f.dep[NF > 1 ? 1 : 0]) : 0., gpv.rho, slip, Y, Yfv);
  for (int k = 0; k < kLearnIn; ++k) {
    if (!(x[k] >= L.norm.x_lo[k] && x[k] <= L.norm.x_hi[k])) {
      return;  // the gate sends it to the FP64 kernel
    }
    xn[k] = (x[k] - L.norm.x_mean[k]) * L.norm.x_inv_std[k];
  }
  mlp_simt(*L.mlp, xn, yp);
  atomicAdd(&L.audit[0], 1.);
  for (int k = 0; k < kLearnOut; ++k) {
    const double yk = (double)fmaf(yp[k], L.norm.y_std[k], L.norm.y_mean[k] + learn_base(L.norm, k, xn, base_vars(x, L.norm)));
    const double e = yk - (double)yt[k];
    atomicAdd(&L.audit[1 + k], e * e);
    atomicAdd(&L.audit[6 + k], (double)yt[k] * (double)yt[k]);
  }
}

template <int NS, int NF>
static int launch_learned_t(pmp_spray* h, const KParams& P, const LearnParams& LP, cudaStream_t st)
{
  if (LP.audit_stride > 0 && LP.ncta == h->ncta) {
    const long long n = (h->total + LP.audit_stride - 1) / LP.audit_stride;
    if (n > 0) {
      k_learn_audit<NS, NF><<<nb(n, 128), 128, 0, st>>>(P, LP, h->total);
    }
  }
  constexpr int per = kLearnThreads / kBlock;
  int grid = (LP.ncta + per - 1) / per;
#if PMP_LEARNED_GRID_CAP > 0
  {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    grid = std::min(grid, sms * PMP_LEARNED_GRID_CAP);
  }
#endif
  constexpr size_t smem = sizeof(tc::TcMlp) + sizeof(tc::TcTileA) * (kLearnThreads / tc::kTile) +
                          sizeof(double) * learn_stash(NF) * kLearnThreads;
  auto kern = P.fuel_first ? spray_update_learned<NS, NF, kLearnThreads, true>
                           : spray_update_learned<NS, NF, kLearnThreads, false>;
  if (smem > 48 * 1024) {
    const cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
      return PMP_ERR_CUDA;
    }
  }
  // the resident CTAs loop over the items (PMP_LEARNED_GRID_CAP); a
  // shared-memory carveout preference measured no help
  kern<<<grid, kLearnThreads, smem, st>>>(P, LP);
  return PMP_OK;
}

int launch_learned(pmp_spray* h, const KParams& P, cudaStream_t st, int first, int count)
{
  if (count < 0) {
    first = 0;
    count = h->ncta;
  }
  if (count == 0) {
    return PMP_OK;
  }
  KParams Q = P;
  Q.cta_box = P.cta_box + first;
  Q.cta_start = P.cta_start + first;
  LearnState* L = h->learn;
  if (!L || !L->trained) {
    return PMP_ERR_INVALID;
  }
  if (!h->data.mass_trans) {
    return PMP_ERR_UNSUPPORTED;
  }
  LearnParams LP;
  memset(&LP, 0, sizeof(LP));
  LP.norm = L->norm;
  LP.mlp = L->d_mlp;
  LP.mlp_tc = L->d_mlp_tc;
  LP.audit = L->d_audit;
  LP.ncta = count;
  LP.audit_stride = 0;
  if (L->audit_fraction > 0. && count == h->ncta) {
    LP.audit_stride = std::max(1LL, (long long)llround(1.0 / L->audit_fraction));
    LP.audit_offset = (long long)(mix64(L->seed++) % (unsigned long long)LP.audit_stride);
    cudaMemsetAsync(L->d_audit, 0, sizeof(double) * 16, st);
  }
  const int ns = h->nspec, nf = h->nfuel;
#define PMP_LCASE(S, F)                              \
  if (ns == S && nf == F) {                          \
    return launch_learned_t<S, F>(h, Q, LP, st);     \
  }
  PMP_LCASE(3, 1)
  PMP_LCASE(5, 1)
  PMP_LCASE(5, 2)
  PMP_LCASE(4, 1)
  PMP_LCASE(4, 2)
#undef PMP_LCASE
  return PMP_ERR_UNSUPPORTED;
}

bool learn_ready(const pmp_spray* h) { return h->learn && h->learn->trained; }

bool learn_audit_on(const pmp_spray* h) { return h->learn && h->learn->audit_fraction > 0.; }

static void free_state(LearnState* L)
{
  void* bufs[] = {L->tuples, L->d_count, L->params, L->wq, L->grads, L->adam_m, L->adam_v, L->X, L->Yt,
                  L->H1, L->A1, L->H2, L->A2, L->H3, L->A3, L->Yp, L->dY, L->dA, L->dH, L->d_stats,
                  L->d_loss, L->d_mlp, L->d_mlp_tc, L->d_audit};
  for (void* p : bufs) {
    cudaFree(p);
  }
  delete L;
}

void learn_free(pmp_spray* h)
{
  if (h->learn) {
    free_state(h->learn);
    h->learn = nullptr;
  }
}

static LearnState* learn_state(pmp_spray* h)
{
  if (!h->learn) {
    h->learn = new LearnState();
  }
  return h->learn;
}

}  // namespace pmp

using namespace pmp;

extern "C" int pmp_spray_learn_audit(const pmp_spray* h, long long* audited, double rel_rms[5])
{
  if (!h || !audited || !rel_rms) {
    return PMP_ERR_INVALID;
  }
  *audited = 0;
  for (int k = 0; k < kLearnOut; ++k) {
    rel_rms[k] = 0.;
  }
  const LearnState* L = h->learn;
  if (!L || !L->d_audit || L->audit_fraction <= 0.) {
    return PMP_OK;
  }
  cudaSetDevice(h->device);
  double a[16];
  if (cudaMemcpy(a, L->d_audit, sizeof(a), cudaMemcpyDeviceToHost) != cudaSuccess) {
    return PMP_ERR_CUDA;
  }
  *audited = (long long)a[0];
  for (int k = 0; k < kLearnOut; ++k) {
    // the outputs are logarithms: their absolute error is the relative error
    rel_rms[k] = a[0] > 0. ? sqrt(a[1 + k] / a[0]) : 0.;
  }
  return PMP_OK;
}

// ===========================================================================
// C ABI of the learned form

extern "C" int pmp_spray_learn_generate(
  pmp_spray* h, const pmp_box_view* state, int nboxes, double flow_dt, int state_ghosts, int do_move,
  double spray_cfl_lev, long long sample_stride, int augment, unsigned long long seed, void* stream)
{
  if (!h || !state || sample_stride < 1 || augment < 0) {
    return PMP_ERR_INVALID;
  }
  cudaSetDevice(h->device);
  pmp::quiesce(h);
  cudaStream_t st = (cudaStream_t)stream;
  // prepare_update validates source views too: pass the state views, which
  // cover the boxes and are never written here.  The teacher needs no trained
  // network, so the mode check of the learned form is bypassed.
  KParams P;
  const int saved_mode = h->mode;
  h->mode = PMP_MODE_FP64;
  const int rc = prepare_update(h, state, state, nboxes, flow_dt, state_ghosts, 0, 0, do_move, spray_cfl_lev, st, P);
  h->mode = saved_mode;
  if (rc != PMP_OK) {
    return rc;
  }
  LearnState* L = learn_state(h);
  const long long per_call = (h->total / sample_stride + 1) * (augment + 1);
  long long have = 0;
  if (L->d_count) {
    unsigned long long c = 0;
    cudaMemcpy(&c, L->d_count, sizeof(c), cudaMemcpyDeviceToHost);
    have = std::min((long long)c, L->cap);
  } else if (cudaMalloc(&L->d_count, sizeof(unsigned long long)) != cudaSuccess) {
    return set_err(h, PMP_ERR_CUDA, "allocation failed");
  } else {
    cudaMemset(L->d_count, 0, sizeof(unsigned long long));
  }
  if (have + per_call > L->cap) {
    const long long ncap = std::max(have + per_call, L->cap * 2);
    float* nt = nullptr;
    if (cudaMalloc(&nt, sizeof(float) * kTupleW * (size_t)ncap) != cudaSuccess) {
      return set_err(h, PMP_ERR_CUDA, "tuple buffer allocation failed");
    }
    if (have > 0) {
      cudaMemcpy(nt, L->tuples, sizeof(float) * kTupleW * (size_t)have, cudaMemcpyDeviceToDevice);
    }
    cudaFree(L->tuples);
    L->tuples = nt;
    L->cap = ncap;
    const unsigned long long c = (unsigned long long)have;
    cudaMemcpy(L->d_count, &c, sizeof(c), cudaMemcpyHostToDevice);
  }
  const long long offset = (long long)(seed % (unsigned long long)sample_stride);
  const int ns = h->nspec, nf = h->nfuel;
  const unsigned grid = nb(h->total, 128);
  if (h->total > 0) {
#define PMP_GCASE(S, F)                                                                                  \
  if (ns == S && nf == F) {                                                                              \
    k_learn_tuples<S, F><<<grid, 128, 0, st>>>(P, h->total, sample_stride, offset, augment, seed, L->tuples, \
                                              L->d_count, L->cap);                                       \
  }
    PMP_GCASE(3, 1)
    PMP_GCASE(5, 1)
    PMP_GCASE(5, 2)
    PMP_GCASE(4, 1)
    PMP_GCASE(4, 2)
#undef PMP_GCASE
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    return set_err(h, PMP_ERR_CUDA, "tuple generation failed");
  }
  return PMP_OK;
}

extern "C" int pmp_spray_learn_count(const pmp_spray* h, long long* n)
{
  if (!h || !n) {
    return PMP_ERR_INVALID;
  }
  *n = 0;
  if (h->learn && h->learn->d_count) {
    unsigned long long c = 0;
    cudaMemcpy(&c, h->learn->d_count, sizeof(c), cudaMemcpyDeviceToHost);
    *n = std::min((long long)c, h->learn->cap);
  }
  return PMP_OK;
}

extern "C" int pmp_spray_learn_tuples(const pmp_spray* h, float* buf, long long* n)
{
  if (!h || !n) {
    return PMP_ERR_INVALID;
  }
  long long have = 0;
  pmp_spray_learn_count(h, &have);
  if (!buf) {
    *n = have;
    return PMP_OK;
  }
  const long long m = std::min(*n, have);
  if (m > 0) {
    cudaSetDevice(h->device);
    if (cudaMemcpy(buf, h->learn->tuples, sizeof(float) * kTupleW * (size_t)m, cudaMemcpyDeviceToHost) !=
        cudaSuccess) {
      return PMP_ERR_CUDA;
    }
  }
  *n = m;
  return PMP_OK;
}

static bool solve_baseline(const double* acc, LearnNorm& nrm);

// Least-squares fit of the targets' polynomial baseline (LearnNorm::base) on
// the tuples, with the input normalisation already in nrm: FP64 normal
// equations over at most 8M tuples (k_base_normal), a ridge of 1e-10 of each
// feature's diagonal (features that never vary get no weight), Cholesky on
// the host.
static bool fit_baseline(LearnState* L, long long n, LearnNorm& nrm)
{
  const long long stride = std::max(1LL, (n + 8000000LL - 1) / 8000000LL);
  double* d_acc = nullptr;
  if (cudaMalloc(&d_acc, sizeof(double) * kBaseEntries) != cudaSuccess) {
    return false;
  }
  cudaMemset(d_acc, 0, sizeof(double) * kBaseEntries);
  k_base_normal<<<592, 256>>>(L->tuples, n, stride, nrm, d_acc);
  std::vector<double> acc(kBaseEntries);
  const bool ok = cudaMemcpy(acc.data(), d_acc, sizeof(double) * kBaseEntries, cudaMemcpyDeviceToHost) == cudaSuccess;
  cudaFree(d_acc);
  return ok && solve_baseline(acc.data(), nrm);
}

// The baseline's coefficients from the accumulated normal equations acc
// (k_base_normal's layout: the upper triangle of F^T F row by row, then
// F^T Y row by row): ridge and Cholesky in FP64 on the host.
static bool solve_baseline(const double* acc, LearnNorm& nrm)
{
  constexpr int T = kBaseTerms;
  std::vector<double> G(T * T), R(T * kLearnOut);
  int e = 0;
  for (int a = 0; a < T; ++a) {
    for (int b = a; b < T; ++b, ++e) {
      G[a * T + b] = G[b * T + a] = acc[e];
    }
  }
  for (int a = 0; a < T; ++a) {
    for (int k = 0; k < kLearnOut; ++k) {
      R[a * kLearnOut + k] = acc[kBaseTri + a * kLearnOut + k];
    }
  }
  double dmax = 0.;
  for (int a = 0; a < T; ++a) {
    dmax = std::max(dmax, G[a * T + a]);
  }
  if (!(dmax > 0.)) {
    return false;
  }
  // ridge relative to each feature's own scale (a ridge scaled by the
  // largest diagonal over-damped the small features: the viscosity
  // residual doubled), plus a floor for features that never vary
  for (int a = 0; a < T; ++a) {
    G[a * T + a] += 1e-10 * G[a * T + a] + 1e-14 * dmax;
  }
  // G = C C^T (lower C in place)
  for (int j = 0; j < T; ++j) {
    double d = G[j * T + j];
    for (int k = 0; k < j; ++k) {
      d -= G[j * T + k] * G[j * T + k];
    }
    if (!(d > 0.)) {
      return false;
    }
    d = sqrt(d);
    G[j * T + j] = d;
    for (int i = j + 1; i < T; ++i) {
      double v = G[i * T + j];
      for (int k = 0; k < j; ++k) {
        v -= G[i * T + k] * G[j * T + k];
      }
      G[i * T + j] = v / d;
    }
  }
  for (int o = 0; o < kLearnOut; ++o) {
    std::vector<double> y(T);
    for (int i = 0; i < T; ++i) {  // C y = r
      double v = R[i * kLearnOut + o];
      for (int k = 0; k < i; ++k) {
        v -= G[i * T + k] * y[k];
      }
      y[i] = v / G[i * T + i];
    }
    for (int i = T - 1; i >= 0; --i) {  // C^T c = y
      double v = y[i];
      for (int k = i + 1; k < T; ++k) {
        v -= G[k * T + i] * y[k];
      }
      y[i] = v / G[i * T + i];
    }
    for (int i = 0; i < T; ++i) {
      nrm.base[o][i] = (float)y[i];
    }
  }
  return true;
}

extern "C" int pmp_spray_learn_train(pmp_spray* h, const pmp_learn_config* cfg, pmp_learn_report* rep)
{
  if (!h || !cfg) {
    return PMP_ERR_INVALID;
  }
  cudaSetDevice(h->device);
  pmp::quiesce(h);
  LearnState* L = learn_state(h);
  long long n = 0;
  pmp_spray_learn_count(h, &n);
  if (n < 1000) {
    return set_err(h, PMP_ERR_INVALID, "too few tuples: call pmp_spray_learn_generate first");
  }
  if (ensure_params(L) != 0) {
    return set_err(h, PMP_ERR_CUDA, "allocation failed");
  }
  const int B = cfg->batch > 0 ? cfg->batch : 8192;
  if (ensure_batch(L, B) != 0) {
    return set_err(h, PMP_ERR_CUDA, "allocation failed");
  }
  cudaStream_t st = nullptr;
  const auto t0 = std::chrono::steady_clock::now();
  // normalisation from all tuples
  std::vector<double> init(64, 0.);
  for (int c = 0; c < 15; ++c) {
    init[30 + c] = 1e300;
    init[45 + c] = -1e300;
  }
  cudaMemcpy(L->d_stats, init.data(), sizeof(double) * 64, cudaMemcpyHostToDevice);
  k_tuple_stats<<<592, 256>>>(L->tuples, n, L->d_stats);
  double stt[64];
  if (cudaMemcpy(stt, L->d_stats, sizeof(stt), cudaMemcpyDeviceToHost) != cudaSuccess) {
    return set_err(h, PMP_ERR_CUDA, "statistics failed");
  }
  const double margin = cfg->gate_margin > 0. ? cfg->gate_margin : 0.05;
  LearnNorm& nrm = L->norm;
  for (int k = 0; k < kLearnIn; ++k) {
    const double mean = stt[k] / n;
    const double var = std::max(0., stt[15 + k] / n - mean * mean);
    const double sd = sqrt(var);
    const double lo = stt[30 + k], hi = stt[45 + k];
    const double span = hi - lo;
    nrm.x_mean[k] = (float)mean;
    nrm.x_inv_std[k] = (float)(sd > 1e-12 * (fabs(mean) + 1e-30) && sd > 0. ? 1. / sd : 1.);
    const double w = span > 0. ? margin * span : 1e-6 * (fabs(lo) + 1e-12);
    nrm.x_lo[k] = (float)(lo - w);
    nrm.x_hi[k] = (float)(hi + w);
  }
  // the baseline of the targets, then the statistics of the residuals
  if (!fit_baseline(L, n, nrm)) {
    return set_err(h, PMP_ERR_CUDA, "baseline fit failed");
  }
  for (int k = 0; k < kLearnOut; ++k) {
    const double mean = stt[kLearnIn + k] / n;
    const double var = std::max(0., stt[15 + kLearnIn + k] / n - mean * mean);
    L->target_std[k] = var > 0. ? sqrt(var) : 1.;
  }
  cudaMemset(L->d_stats, 0, sizeof(double) * 64);
  k_resid_stats<<<592, 256>>>(L->tuples, n, nrm, L->d_stats);
  if (cudaMemcpy(stt, L->d_stats, sizeof(double) * 2 * kLearnOut, cudaMemcpyDeviceToHost) != cudaSuccess) {
    return set_err(h, PMP_ERR_CUDA, "statistics failed");
  }
  for (int k = 0; k < kLearnOut; ++k) {
    const double mean = stt[k] / n;
    const double var = std::max(0., stt[kLearnOut + k] / n - mean * mean);
    nrm.y_mean[k] = (float)mean;
    nrm.y_std[k] = (float)(var > 0. ? sqrt(var) : 1.);
  }
  // the residual gate's range: the training residuals', widened by the margin
  {
    float mm[2 * kLearnOut];
    for (int k = 0; k < kLearnOut; ++k) {
      mm[k] = 3.4e38f;
      mm[kLearnOut + k] = -3.4e38f;
    }
    float* d_mm = reinterpret_cast<float*>(L->d_stats);
    cudaMemcpy(d_mm, mm, sizeof(mm), cudaMemcpyHostToDevice);
    k_resid_range<<<592, 256>>>(L->tuples, n, nrm, d_mm);
    if (cudaMemcpy(mm, d_mm, sizeof(mm), cudaMemcpyDeviceToHost) != cudaSuccess) {
      return set_err(h, PMP_ERR_CUDA, "statistics failed");
    }
    for (int k = 0; k < kLearnOut; ++k) {
      const double span = std::max(0., (double)mm[kLearnOut + k] - (double)mm[k]);
      nrm.r_lo[k] = (float)(mm[k] - margin * span);
      nrm.r_hi[k] = (float)(mm[kLearnOut + k] + margin * span);
    }
  }
  L->gate_margin = margin;
  L->audit_fraction = cfg->audit_fraction;
  L->seed = cfg->seed ? cfg->seed : 1;
  // parameters
  std::vector<float> p;
  init_params(p, L->seed);
  cudaMemcpy(L->params, p.data(), sizeof(float) * kP_N, cudaMemcpyHostToDevice);
  cudaMemset(L->adam_m, 0, sizeof(float) * kP_N);
  cudaMemset(L->adam_v, 0, sizeof(float) * kP_N);
  const int quant = cfg->no_quant ? 0 : 1;
  k_quantize<<<nb(kP_N), 256>>>(L->params, L->wq, kP_N, quant);
  const long long nval = std::max(1000LL, n / 100);
  const long long ntrain = n - nval;
  const int epochs = cfg->epochs > 0 ? cfg->epochs : 20;
  const long long steps = std::max(1LL, (ntrain / B) * epochs);
  const double lr0 = cfg->lr > 0. ? cfg->lr : 2e-3;
  const double lr_end = lr0 * 0.01;
  double loss_first = -1., loss_last = -1.;
  for (long long it = 0; it < steps; ++it) {
    k_gather_batch<<<nb(B), 256>>>(L->tuples, ntrain, 0, B, L->seed, it, 1, nrm, L->X, L->Yt);
    forward(L, L->wq, B, quant, st);
    const bool track = (it == 0 || it == steps - 1 || (it % 200) == 0);
    if (track) {
      cudaMemsetAsync(L->d_loss, 0, sizeof(double), st);
    }
    k_mse<<<nb((long long)B * 8), 256>>>(L->Yp, L->Yt, L->dY, B, track ? L->d_loss : nullptr);
    backward(L, L->wq, B, st);
    const double lr = lr0 * pow(lr_end / lr0, (double)it / (double)steps);
    const double b1 = 0.9, b2 = 0.999;
    const double bc1 = 1. - pow(b1, (double)(it + 1));
    const double bc2 = 1. - pow(b2, (double)(it + 1));
    k_adam<<<nb(kP_N), 256>>>(L->params, L->wq, L->grads, L->adam_m, L->adam_v, kP_N, (float)lr, (float)b1,
                              (float)b2, 1e-8f, (float)bc1, (float)bc2, quant);
    if (track) {
      double l = 0.;
      cudaMemcpy(&l, L->d_loss, sizeof(double), cudaMemcpyDeviceToHost);
      l /= (double)B * kLearnOut;
      if (loss_first < 0.) {
        loss_first = l;
      }
      loss_last = l;
    }
  }
  if (cudaDeviceSynchronize() != cudaSuccess) {
    return set_err(h, PMP_ERR_CUDA, "training failed");
  }
  // validation: normalised RMSE per output on the held-out tuples
  double se[kLearnOut] = {0}, sy[kLearnOut] = {0};
  std::vector<float> yp((size_t)B * 8), yt((size_t)B * 8);
  long long done = 0;
  while (done < nval) {
    const int bb = (int)std::min((long long)B, nval - done);
    k_gather_batch<<<nb(bb), 256>>>(L->tuples, n, ntrain + done, bb, 0, 0, 0, nrm, L->X, L->Yt);
    forward(L, L->wq, bb, quant, st);
    cudaMemcpy(yp.data(), L->Yp, sizeof(float) * bb * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(yt.data(), L->Yt, sizeof(float) * bb * 8, cudaMemcpyDeviceToHost);
    for (int r = 0; r < bb; ++r) {
      for (int k = 0; k < kLearnOut; ++k) {
        const double a = yp[r * 8 + k] * nrm.y_std[k] + nrm.y_mean[k];
        const double t = yt[r * 8 + k] * nrm.y_std[k] + nrm.y_mean[k];
        se[k] += (a - t) * (a - t);
        sy[k] += t * t;
      }
    }
    done += bb;
  }
  // inference weights
  std::vector<float> pw(kP_N);
  cudaMemcpy(pw.data(), L->params, sizeof(float) * kP_N, cudaMemcpyDeviceToHost);
  MlpSmem S;
  build_mlp(pw, S);
  cudaMemcpy(L->d_mlp, &S, sizeof(S), cudaMemcpyHostToDevice);
  upload_mlp_tc(L, pw);
  L->trained = true;
  const auto t1 = std::chrono::steady_clock::now();
  if (rep) {
    memset(rep, 0, sizeof(*rep));
    rep->tuples = n;
    rep->steps = steps;
    rep->loss_first = loss_first;
    rep->loss_last = loss_last;
    for (int k = 0; k < kLearnOut; ++k) {
      rep->val_rel_rms[k] = sqrt(se[k] / (double)nval);
    }
    rep->train_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    for (int k = 0; k < kLearnOut; ++k) {
      rep->base_resid_frac[k] = (double)nrm.y_std[k] / L->target_std[k];
    }
  }
  return PMP_OK;
}

extern "C" int pmp_spray_learn_weights(pmp_spray* h, int get, float* buf, long long* count)
{
  // layout: kP_N parameters, then x_mean[10] x_inv_std[10] x_lo[10] x_hi[10] y_mean[5] y_std[5]
  // base[5][kBaseTerms] r_lo[5] r_hi[5]
  const long long total = kP_N + 4 * kLearnIn + 4 * kLearnOut + kLearnOut * kBaseTerms;
  if (!h || !count) {
    return PMP_ERR_INVALID;
  }
  if (!buf) {
    *count = total;
    return PMP_OK;
  }
  if (*count < total) {
    return PMP_ERR_INVALID;
  }
  cudaSetDevice(h->device);
  pmp::quiesce(h);
  LearnState* L = learn_state(h);
  if (ensure_params(L) != 0) {
    return PMP_ERR_CUDA;
  }
  LearnNorm& nrm = L->norm;
  float* tail = buf + kP_N;
  if (get) {
    if (!L->trained) {
      return PMP_ERR_INVALID;
    }
    cudaMemcpy(buf, L->params, sizeof(float) * kP_N, cudaMemcpyDeviceToHost);
    memcpy(tail, nrm.x_mean, sizeof(float) * kLearnIn);
    memcpy(tail + 10, nrm.x_inv_std, sizeof(float) * kLearnIn);
    memcpy(tail + 20, nrm.x_lo, sizeof(float) * kLearnIn);
    memcpy(tail + 30, nrm.x_hi, sizeof(float) * kLearnIn);
    memcpy(tail + 40, nrm.y_mean, sizeof(float) * kLearnOut);
    memcpy(tail + 45, nrm.y_std, sizeof(float) * kLearnOut);
    memcpy(tail + 50, nrm.base, sizeof(float) * kLearnOut * kBaseTerms);
    memcpy(tail + 50 + kLearnOut * kBaseTerms, nrm.r_lo, sizeof(float) * kLearnOut);
    memcpy(tail + 55 + kLearnOut * kBaseTerms, nrm.r_hi, sizeof(float) * kLearnOut);
  } else {
    cudaMemcpy(L->params, buf, sizeof(float) * kP_N, cudaMemcpyHostToDevice);
    memcpy(nrm.x_mean, tail, sizeof(float) * kLearnIn);
    memcpy(nrm.x_inv_std, tail + 10, sizeof(float) * kLearnIn);
    memcpy(nrm.x_lo, tail + 20, sizeof(float) * kLearnIn);
    memcpy(nrm.x_hi, tail + 30, sizeof(float) * kLearnIn);
    memcpy(nrm.y_mean, tail + 40, sizeof(float) * kLearnOut);
    memcpy(nrm.y_std, tail + 45, sizeof(float) * kLearnOut);
    memcpy(nrm.base, tail + 50, sizeof(float) * kLearnOut * kBaseTerms);
    memcpy(nrm.r_lo, tail + 50 + kLearnOut * kBaseTerms, sizeof(float) * kLearnOut);
    memcpy(nrm.r_hi, tail + 55 + kLearnOut * kBaseTerms, sizeof(float) * kLearnOut);
    std::vector<float> pw(buf, buf + kP_N);
    MlpSmem S;
    build_mlp(pw, S);
    cudaMemcpy(L->d_mlp, &S, sizeof(S), cudaMemcpyHostToDevice);
    upload_mlp_tc(L, pw);
    L->trained = true;
  }
  *count = total;
  return PMP_OK;
}

extern "C" int pmp_spray_learn_set_audit(pmp_spray* h, double audit_fraction)
{
  if (!h || audit_fraction < 0. || audit_fraction > 1.) {
    return PMP_ERR_INVALID;
  }
  learn_state(h)->audit_fraction = audit_fraction;
  return PMP_OK;
}

// Training-kernel check: loss and gradients of the MSE on n given rows
// (normalised inputs x[n][10], targets y[n][5]) with the given parameters;
// quant = 0 runs the plain FP32 network.  Allocates its own buffers.
extern "C" int pmp_learn_debug_grad(
  const float* params, const float* x, const float* y, int n, int quant, float* grads, double* loss)
{
  if (!params || !x || !y || n < 1 || !grads) {
    return PMP_ERR_INVALID;
  }
  LearnState* L = new LearnState();
  if (ensure_params(L) != 0 || ensure_batch(L, n) != 0) {
    free_state(L);
    return PMP_ERR_CUDA;
  }
  std::vector<float> X((size_t)n * 16, 0.f), Y((size_t)n * 8, 0.f);
  for (int r = 0; r < n; ++r) {
    for (int k = 0; k < kLearnIn; ++k) {
      X[r * 16 + k] = x[r * kLearnIn + k];
    }
    for (int k = 0; k < kLearnOut; ++k) {
      Y[r * 8 + k] = y[r * kLearnOut + k];
    }
  }
  cudaMemcpy(L->X, X.data(), sizeof(float) * X.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(L->Yt, Y.data(), sizeof(float) * Y.size(), cudaMemcpyHostToDevice);
  cudaMemcpy(L->params, params, sizeof(float) * kP_N, cudaMemcpyHostToDevice);
  k_quantize<<<nb(kP_N), 256>>>(L->params, L->wq, kP_N, quant);
  cudaMemset(L->d_loss, 0, sizeof(double));
  forward(L, L->wq, n, quant, nullptr);
  k_mse<<<nb((long long)n * 8), 256>>>(L->Yp, L->Yt, L->dY, n, L->d_loss);
  backward(L, L->wq, n, nullptr);
  int rc = PMP_OK;
  if (cudaDeviceSynchronize() != cudaSuccess) {
    rc = PMP_ERR_CUDA;
  } else {
    cudaMemcpy(grads, L->grads, sizeof(float) * kP_N, cudaMemcpyDeviceToHost);
    double l = 0.;
    cudaMemcpy(&l, L->d_loss, sizeof(double), cudaMemcpyDeviceToHost);
    if (loss) {
      *loss = l / ((double)n * kLearnOut);
    }
  }
  free_state(L);
  return rc;
}

extern "C" int pmp_learn_param_count(void) { return kP_N; }

extern "C" int pmp_learn_base_terms(void) { return kBaseTerms; }

// Host instantiation of the baseline's term layout and its FP32 nested
// evaluation (the code the kernels run): feats[kBaseTerms] for normalised
// inputs xn[10] and the derived variables (ell, g); value = the polynomial
// with coefficients coef[kBaseTerms].  No GPU needed.
extern "C" int pmp_learn_debug_base(const float* xn, float ell, float g, const float* coef, double* feats,
                                    float* value)
{
  if (!xn || !coef || !feats || !value) {
    return PMP_ERR_INVALID;
  }
  BaseVars v;
  v.ell = ell;
  v.g = g;
  base_features(xn, v, feats);
  LearnNorm nrm;
  memset(&nrm, 0, sizeof(nrm));
  memcpy(nrm.base[0], coef, sizeof(float) * kBaseTerms);
  *value = learn_base(nrm, 0, xn, v);
  return PMP_OK;
}

// The host solve of the baseline fit: acc[kBaseTerms (kBaseTerms + 1) / 2 +
// 5 kBaseTerms] in k_base_normal's layout (upper triangle of F^T F row by
// row, then F^T Y row by row) -> coef[5][kBaseTerms].  No GPU needed.
extern "C" int pmp_learn_debug_solve_baseline(const double* acc, float* coef)
{
  if (!acc || !coef) {
    return PMP_ERR_INVALID;
  }
  LearnNorm nrm;
  memset(&nrm, 0, sizeof(nrm));
  if (!solve_baseline(acc, nrm)) {
    return PMP_ERR_INVALID;
  }
  memcpy(coef, nrm.base, sizeof(float) * kLearnOut * kBaseTerms);
  return PMP_OK;
}

namespace {

// mlp_warp over n rows of normalised inputs (rows padded to whole warps)
__global__ void k_debug_infer(const MlpSmem* mlp, const float* xn, int n, float* y)
{
  __shared__ MlpSmem S;
  __shared__ MlpWarpScratch WS[4];
  {
    const int4* src = reinterpret_cast<const int4*>(mlp);
    int4* dst = reinterpret_cast<int4*>(&S);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpSmem) / 16); i += blockDim.x) {
      dst[i] = src[i];
    }
  }
  __syncthreads();
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  float x[kLearnIn], o[kLearnOut];
  for (int k = 0; k < kLearnIn; ++k) {
    x[k] = r < n ? xn[(size_t)r * kLearnIn + k] : 0.f;
  }
  mlp_warp(S, WS[threadIdx.x >> 5], x, o);
  if (r < n) {
    for (int k = 0; k < kLearnOut; ++k) {
      y[(size_t)r * kLearnOut + k] = o[k];
    }
  }
}

// mlp_cta_tc over n rows of normalised inputs, TILES x 128 rows per CTA
template <int TILES>
__global__ void __launch_bounds__(TILES * tc::kTile) k_debug_infer_tc(const tc::TcMlp* mlp, const float* xn, int n,
                                                                      float* y, int* status)
{
  extern __shared__ __align__(128) unsigned char tc_smem[];
  tc::TcMlp& S = *reinterpret_cast<tc::TcMlp*>(tc_smem);
  tc::TcTileA* A = reinterpret_cast<tc::TcTileA*>(tc_smem + sizeof(tc::TcMlp));
  __shared__ uint32_t tmem_slot;
  __shared__ unsigned long long mbar_slot;
  {
    const int4* src = reinterpret_cast<const int4*>(mlp);
    int4* dst = reinterpret_cast<int4*>(&S);
    for (int i = threadIdx.x; i < (int)(sizeof(tc::TcMlp) / 16); i += blockDim.x) {
      dst[i] = src[i];
    }
  }
  tc::TcCta c = tc::tc_setup(&tmem_slot, &mbar_slot, TILES * tc::kCols);
  const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float x[kLearnIn], o[kLearnOut];
  for (int k = 0; k < kLearnIn; ++k) {
    x[k] = r < n ? xn[r * kLearnIn + k] : 0.f;
  }
  const bool ok = tc::mlp_cta_tc<TILES>(S, A, c, x, o);
  if (!ok) {
    if (threadIdx.x == 0) {
      atomicExch(status, 1);
    }
    tc::mbar_wait(c.mbar, c.phase ^ 1u);  // the MMAs the timed-out wait was for
  } else if (r < n) {
    for (int k = 0; k < kLearnOut; ++k) {
      y[r * kLearnOut + k] = o[k];
    }
  }
  tc::tc_teardown(c, TILES * tc::kCols);
}

}  // namespace

namespace {

// The timeout path of the tcgen05 waits: one CTA allocates its tensor memory
// and waits on an mbarrier that nothing arrives on; the bounded wait must give
// up, the CTA agree on it and free the tensor memory.
__global__ void __launch_bounds__(tc::kTile) k_debug_wait_timeout(int* status, long long* cycles)
{
  __shared__ uint32_t tmem_slot;
  __shared__ unsigned long long mbar_slot;
  tc::TcCta c = tc::tc_setup(&tmem_slot, &mbar_slot, tc::kCols);
  const long long t0 = clock64();
  const bool ok = __syncthreads_and(tc::mbar_wait(c.mbar, c.phase)) != 0;
  if (threadIdx.x == 0) {
    *status = ok ? 0 : 1;
    *cycles = clock64() - t0;
  }
  tc::tc_teardown(c, tc::kCols);
}

}  // namespace

extern "C" int pmp_learn_debug_wait_timeout(long long* cycles)
{
  if (!cycles) {
    return PMP_ERR_INVALID;
  }
  int* d_status = nullptr;
  long long* d_cycles = nullptr;
  int rc = PMP_OK;
  if (cudaMalloc(&d_status, sizeof(int)) != cudaSuccess || cudaMalloc(&d_cycles, sizeof(long long)) != cudaSuccess) {
    rc = PMP_ERR_CUDA;
  } else {
    k_debug_wait_timeout<<<1, tc::kTile>>>(d_status, d_cycles);
    int status = 0;
    if (cudaDeviceSynchronize() != cudaSuccess) {
      rc = PMP_ERR_CUDA;
    } else {
      cudaMemcpy(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost);
      cudaMemcpy(cycles, d_cycles, sizeof(long long), cudaMemcpyDeviceToHost);
      rc = status ? PMP_ERR_TIMEOUT : PMP_OK;
    }
  }
  cudaFree(d_status);
  cudaFree(d_cycles);
  return rc;
}

extern "C" int pmp_learn_debug_infer_tc(const float* params, const float* xn, int n, float* y)
{
  if (!params || !xn || !y || n < 1) {
    return PMP_ERR_INVALID;
  }
  std::vector<float> pw(params, params + kP_N);
  tc::TcMlp S;
  build_mlp_tc(pw, S);
  tc::TcMlp* d_mlp = nullptr;
  float *d_x = nullptr, *d_y = nullptr;
  int* d_status = nullptr;
  int rc = PMP_OK;
  constexpr int kTiles = 2;
  const size_t smem = sizeof(tc::TcMlp) + kTiles * sizeof(tc::TcTileA);
  if (cudaMalloc(&d_mlp, sizeof(S)) != cudaSuccess ||
      cudaMalloc(&d_x, sizeof(float) * (size_t)n * kLearnIn) != cudaSuccess ||
      cudaMalloc(&d_y, sizeof(float) * (size_t)n * kLearnOut) != cudaSuccess ||
      cudaMalloc(&d_status, sizeof(int)) != cudaSuccess ||
      cudaFuncSetAttribute(k_debug_infer_tc<kTiles>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess) {
    rc = PMP_ERR_CUDA;
  } else {
    cudaMemcpy(d_mlp, &S, sizeof(S), cudaMemcpyHostToDevice);
    cudaMemcpy(d_x, xn, sizeof(float) * (size_t)n * kLearnIn, cudaMemcpyHostToDevice);
    cudaMemset(d_status, 0, sizeof(int));
    const int rows = kTiles * tc::kTile;
    k_debug_infer_tc<kTiles><<<(n + rows - 1) / rows, rows, smem>>>(d_mlp, d_x, n, d_y, d_status);
    int status = 0;
    if (cudaDeviceSynchronize() != cudaSuccess) {
      rc = PMP_ERR_CUDA;
    } else {
      cudaMemcpy(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost);
      cudaMemcpy(y, d_y, sizeof(float) * (size_t)n * kLearnOut, cudaMemcpyDeviceToHost);
      rc = status ? PMP_ERR_TIMEOUT : PMP_OK;
    }
  }
  cudaFree(d_mlp);
  cudaFree(d_x);
  cudaFree(d_y);
  cudaFree(d_status);
  return rc;
}

// Inference check: the tensor-core network of the learned kernel on n rows of
// normalised inputs xn[n][10] with the flat parameters params; y[n][5].
extern "C" int pmp_learn_debug_infer(const float* params, const float* xn, int n, float* y)
{
  if (!params || !xn || !y || n < 1) {
    return PMP_ERR_INVALID;
  }
  std::vector<float> pw(params, params + kP_N);
  MlpSmem S;
  build_mlp(pw, S);
  MlpSmem* d_mlp = nullptr;
  float *d_x = nullptr, *d_y = nullptr;
  int rc = PMP_OK;
  if (cudaMalloc(&d_mlp, sizeof(S)) != cudaSuccess ||
      cudaMalloc(&d_x, sizeof(float) * (size_t)n * kLearnIn) != cudaSuccess ||
      cudaMalloc(&d_y, sizeof(float) * (size_t)n * kLearnOut) != cudaSuccess) {
    rc = PMP_ERR_CUDA;
  } else {
    cudaMemcpy(d_mlp, &S, sizeof(S), cudaMemcpyHostToDevice);
    cudaMemcpy(d_x, xn, sizeof(float) * (size_t)n * kLearnIn, cudaMemcpyHostToDevice);
    k_debug_infer<<<(n + 127) / 128, 128>>>(d_mlp, d_x, n, d_y);
    if (cudaDeviceSynchronize() != cudaSuccess) {
      rc = PMP_ERR_CUDA;
    } else {
      cudaMemcpy(y, d_y, sizeof(float) * (size_t)n * kLearnOut, cudaMemcpyDeviceToHost);
    }
  }
  cudaFree(d_mlp);
  cudaFree(d_x);
  cudaFree(d_y);
  return rc;
}
