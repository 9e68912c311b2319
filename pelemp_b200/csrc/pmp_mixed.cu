// pmp_mixed.cu -- launches of the mixed-precision update kernel.
//
// Its own translation unit so that it is compiled with multiply-add
// contraction enabled (the FP32 physics benefits; the FP64 kernels in
// pmp_spray.cu are compiled without it to stay bit-identical to the oracle).
#include <cuda_runtime.h>

#include "spray_kernels.cuh"

namespace pmp {

int launch_mixed(int ns, int nf, const KParams& P, int ncta, int block, cudaStream_t st)
{
  if (block != 128) {
    return PMP_ERR_INVALID;
  }
#define PMP_MIXED_CASE(S, F)                                          \
  if (ns == S && nf == F) {                                           \
    if (P.fuel_first) {                                                \
      spray_update_mixed<S, F, 128, true><<<ncta, 128, 0, st>>>(P);    \
    } else {                                                           \
      spray_update_mixed<S, F, 128, false><<<ncta, 128, 0, st>>>(P);   \
    }                                                                  \
    return PMP_OK;                                                    \
  }
  PMP_MIXED_CASE(3, 1)
  PMP_MIXED_CASE(5, 1)
  PMP_MIXED_CASE(5, 2)
  PMP_MIXED_CASE(4, 1)
  PMP_MIXED_CASE(4, 2)
#undef PMP_MIXED_CASE
  return PMP_ERR_UNSUPPORTED;
}

}  // namespace pmp
