// pmp_mixed.cu -- launches of the mixed-precision update kernel.
//
// Its own translation unit so that it is compiled with multiply-add
// contraction enabled (the FP32 physics benefits; the FP64 kernels in
// pmp_spray.cu are compiled without it to stay bit-identical to the oracle).
#include <cuda_runtime.h>

#include <algorithm>

#include "spray_kernels.cuh"

namespace pmp {

int launch_mixed(int ns, int nf, const KParams& P, int ncta, int block, cudaStream_t st)
{
  if (block != 128) {
    return PMP_ERR_INVALID;
  }
#define PMP_MIXED_CASE(S, F)                                                  \
  if (ns == S && nf == F) {                                                   \
    if (P.pelec) {                                                            \
      if (P.fuel_first) {                                                     \
        spray_update_mixed<S, F, 128, true, true><<<ncta, 128, 0, st>>>(P);   \
      } else {                                                                \
        spray_update_mixed<S, F, 128, false, true><<<ncta, 128, 0, st>>>(P);  \
      }                                                                       \
    } else if (P.fuel_first) {                                                \
      spray_update_mixed<S, F, 128, true><<<ncta, 128, 0, st>>>(P);           \
    } else {                                                                  \
      spray_update_mixed<S, F, 128, false><<<ncta, 128, 0, st>>>(P);          \
    }                                                                         \
    return PMP_OK;                                                            \
  }
  PMP_MIXED_CASE(3, 1)
  PMP_MIXED_CASE(5, 1)
  PMP_MIXED_CASE(5, 2)
  PMP_MIXED_CASE(4, 1)
  PMP_MIXED_CASE(4, 2)
#undef PMP_MIXED_CASE
  return PMP_ERR_UNSUPPORTED;
}

int launch_select_small(const KParams& P, long long s0, long long s1, cudaStream_t st)
{
  const long long n = s1 - s0;
  if (n <= 0) {
    return PMP_OK;
  }
  const int grid = (int)std::min<long long>((n + 255) / 256, 148LL * 8);
  k_select_small<<<grid, 256, 0, st>>>(P, s0, s1);
  return PMP_OK;
}

int launch_gas_records(int ns, const KParams& P, int b0, int nb, int max_cells, cudaStream_t st)
{
  if (nb <= 0 || max_cells <= 0) {
    return PMP_OK;
  }
  const dim3 grid((unsigned)std::min((max_cells + 255) / 256, 128), (unsigned)nb);
#define PMP_REC_CASE(S)                                     \
  if (ns == S) {                                            \
    if (P.pelec) {                                          \
      k_gas_records<S, true><<<grid, 256, 0, st>>>(P, b0);  \
    } else {                                                \
      k_gas_records<S><<<grid, 256, 0, st>>>(P, b0);        \
    }                                                       \
    return PMP_OK;                                          \
  }
  PMP_REC_CASE(3)
  PMP_REC_CASE(4)
  PMP_REC_CASE(5)
#undef PMP_REC_CASE
  return PMP_ERR_UNSUPPORTED;
}

}  // namespace pmp
