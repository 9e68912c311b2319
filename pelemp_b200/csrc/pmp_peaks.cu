// pmp_peaks.cu -- measured compute peaks of the device, for the compute
// roofline of the update kernels (no counterpart in the reference).
//
// Three loop kernels, each thread running 8 independent dependency chains in
// registers (enough instruction-level parallelism to keep the pipe busy at
// full occupancy), over a grid of 8 CTAs of 256 threads per SM:
//  - FP64 fused multiply-adds (DFMA), 2 FLOP each;
//  - FP32 fused multiply-adds (FFMA), 2 FLOP each;
//  - SFU base-2 exponentials (ex2.approx.ftz.f32), the transcendental unit
//    the mixed and learned forms use for exp, log and pow.
// Each is timed with CUDA events after a warm-up launch; the result is the
// best of a few launches.  Nothing is changed on the device (no clock or
// power setting): the figures are those of the clocks the GPU runs at.
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/pmp_spray.h"

namespace {

constexpr int kThreads = 256;
constexpr int kChains = 8;

__global__ void __launch_bounds__(kThreads) k_peak_dfma(int iters, double a, double* sink)
{
  double x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    x[c] = threadIdx.x * 1e-3 + c;
  }
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
      x[c] = fma(x[c], a, 0.25);
    }
  }
  double s = 0.;
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    s += x[c];
  }
  if (s == -1.2345) {  // never true: keeps the loop
    *sink = s;
  }
}

__global__ void __launch_bounds__(kThreads) k_peak_ffma(int iters, float a, float* sink)
{
  float x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    x[c] = threadIdx.x * 1e-3f + c;
  }
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
      x[c] = fmaf(x[c], a, 0.25f);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    s += x[c];
  }
  if (s == -1.2345f) {
    *sink = s;
  }
}

__global__ void __launch_bounds__(kThreads) k_peak_ex2(int iters, float* sink)
{
  float x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    x[c] = -1e-3f * (threadIdx.x + c);
  }
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) {
      float r;
      asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x[c]));
      x[c] = r - 1.0f;  // stays in (-1, 0]
    }
  }
  float s = 0.f;
#pragma unroll
  for (int c = 0; c < kChains; ++c) {
    s += x[c];
  }
  if (s == -1.2345f) {
    *sink = s;
  }
}

}  // namespace

extern "C" int pmp_measure_peaks(int device, double* fp64_tflops, double* fp32_tflops, double* sfu_gops)
{
  if (!fp64_tflops || !fp32_tflops || !sfu_gops) {
    return PMP_ERR_INVALID;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev || cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return PMP_ERR_NO_DEVICE;
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    return PMP_ERR_CUDA;
  }
  const int grid = 8 * sms;
  double* sink = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaMalloc(&sink, 16) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess) {
    cudaFree(sink);
    return PMP_ERR_CUDA;
  }
  const double lanes = (double)grid * kThreads * kChains;
  double best[3] = {0., 0., 0.};
  const int iters[3] = {4096, 16384, 4096};
  for (int kind = 0; kind < 3; ++kind) {
    for (int rep = 0; rep < 4; ++rep) {  // the first launch warms up
      cudaEventRecord(e0);
      if (kind == 0) {
        k_peak_dfma<<<grid, kThreads>>>(iters[0], 0.9999, sink);
      } else if (kind == 1) {
        k_peak_ffma<<<grid, kThreads>>>(iters[1], 0.9999f, reinterpret_cast<float*>(sink));
      } else {
        k_peak_ex2<<<grid, kThreads>>>(iters[2], reinterpret_cast<float*>(sink));
      }
      cudaEventRecord(e1);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        cudaFree(sink);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return PMP_ERR_CUDA;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      const double ops = lanes * iters[kind] / (ms * 1e-3);  // operations per second
      if (rep > 0 && ops > best[kind]) {
        best[kind] = ops;
      }
    }
  }
  cudaFree(sink);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *fp64_tflops = 2. * best[0] * 1e-12;
  *fp32_tflops = 2. * best[1] * 1e-12;
  *sfu_gops = best[2] * 1e-9;
  return PMP_OK;
}
