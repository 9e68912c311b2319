// batch_kernels.cuh -- launch-shape variants of the FP64 update for many boxes
// with uneven droplet counts (the batched form).
//
// The per-droplet work is update_one<..., Form::FP64>, the same function the
// default launch runs, so every variant gives bit-identical droplet states;
// only the order of the atomic deposits differs.  What varies:
//  * grid: one CTA per work item of BLOCK slots, the hardware block
//    scheduler balancing the boxes;
//  * persistent: a grid of (resident CTAs per SM) x (SMs) CTAs; each CTA takes
//    work items of `chunk` slots from a device counter (atomicAdd, no waiting
//    on other CTAs) until none are left;
//  * the thread count per CTA and the register cap (launch bounds).
// The work items are the (box, first slot) chunks of the packed, cell-sorted
// droplet arrays, so a chunk never spans two boxes.
#pragma once

#include "../spray_kernels.cuh"

namespace pmp {

struct WorkArgs {
  const int* box;         // work item -> box
  const long long* start; // work item -> first slot
  int nitems;
  int chunk;              // slots per work item
  int* counter;           // persistent: next work item (zeroed before the launch)
};

template <int NS, int NF, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
  spray_update_fp64_grid(const __grid_constant__ KParams P, const WorkArgs W)
{
  __shared__ BoxEntry sB;
  const int item = blockIdx.x;
  const int b = W.box[item];
  if (stage_box(P, b, sB)) {
    return;
  }
  const long long s = W.start[item] + threadIdx.x;
  Counters c;
  if (s < sB.p_end) {
    update_one<NS, NF, Form::FP64>(P, sB, b, s, c);
  }
  flush_counters(P, c);
}

template <int NS, int NF, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB)
  spray_update_fp64_persistent(const __grid_constant__ KParams P, const WorkArgs W)
{
  __shared__ int s_item;
  Counters c;
  if (cta_call_failed(P)) {
    return;
  }
  for (;;) {
    if (threadIdx.x == 0) {
      s_item = atomicAdd(W.counter, 1);
    }
    __syncthreads();
    const int item = s_item;
    __syncthreads();
    if (item >= W.nitems) {
      break;
    }
    const int b = W.box[item];
    const long long end = min(W.start[item] + W.chunk, P.boxes[b].p_end);
    for (long long s = W.start[item] + threadIdx.x; s < end; s += BLOCK) {
      update_one<NS, NF, Form::FP64>(P, P.boxes[b], b, s, c);
    }
  }
  flush_counters(P, c);
}

// Launch one variant; returns false when (ns, nf) has no instantiation.
// grid = number of CTAs (grid kind: W.nitems; persistent: resident CTAs).
template <int BLOCK, int MINB, bool PERSISTENT>
bool launch_fp64_variant(int ns, int nf, const KParams& P, const WorkArgs& W, int grid, cudaStream_t st)
{
#define PMP_BCASE(S, F)                                                                   \
  if (ns == S && nf == F) {                                                               \
    if (PERSISTENT) {                                                                     \
      spray_update_fp64_persistent<S, F, BLOCK, MINB><<<grid, BLOCK, 0, st>>>(P, W);      \
    } else {                                                                              \
      spray_update_fp64_grid<S, F, BLOCK, MINB><<<grid, BLOCK, 0, st>>>(P, W);            \
    }                                                                                     \
    return true;                                                                          \
  }
  PMP_BCASE(3, 1)
  PMP_BCASE(5, 1)
  PMP_BCASE(5, 2)
  PMP_BCASE(4, 1)
  PMP_BCASE(4, 2)
#undef PMP_BCASE
  return false;
}

// Resident CTAs per SM of a variant (occupancy calculator)
template <int BLOCK, int MINB, bool PERSISTENT>
int occupancy_fp64_variant(int ns, int nf)
{
  int n = 0;
#define PMP_OCASE(S, F)                                                                          \
  if (ns == S && nf == F) {                                                                      \
    if (PERSISTENT) {                                                                            \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, spray_update_fp64_persistent<S, F, BLOCK, MINB>, \
                                                    BLOCK, 0);                                   \
    } else {                                                                                     \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, spray_update_fp64_grid<S, F, BLOCK, MINB>, BLOCK, 0); \
    }                                                                                            \
  }
  PMP_OCASE(3, 1)
  PMP_OCASE(5, 1)
  PMP_OCASE(5, 2)
  PMP_OCASE(4, 1)
  PMP_OCASE(4, 2)
#undef PMP_OCASE
  return n;
}

// Per block size translation unit: launch / occupancy of its variants.
// regs is the register cap (96 or 128); returns false if the variant is not built.
bool batch_launch_b64(int ns, int nf, int regs, bool persistent, const KParams& P, const WorkArgs& W, int grid,
                      cudaStream_t st);
bool batch_launch_b128(int ns, int nf, int regs, bool persistent, const KParams& P, const WorkArgs& W, int grid,
                       cudaStream_t st);
bool batch_launch_b256(int ns, int nf, int regs, bool persistent, const KParams& P, const WorkArgs& W, int grid,
                       cudaStream_t st);
int batch_occupancy_b64(int ns, int nf, int regs, bool persistent);
int batch_occupancy_b128(int ns, int nf, int regs, bool persistent);
int batch_occupancy_b256(int ns, int nf, int regs, bool persistent);

}  // namespace pmp
