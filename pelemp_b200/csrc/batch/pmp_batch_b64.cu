// 64-thread variants of the batched FP64 update (96-register cap).
#include "batch_kernels.cuh"

namespace pmp {

bool batch_launch_b64(int ns, int nf, int regs, bool persistent, const KParams& P, const WorkArgs& W, int grid,
                      cudaStream_t st)
{
  if (regs != 96) {
    return false;
  }
  return persistent ? launch_fp64_variant<64, 10, true>(ns, nf, P, W, grid, st)
                    : launch_fp64_variant<64, 10, false>(ns, nf, P, W, grid, st);
}

int batch_occupancy_b64(int ns, int nf, int regs, bool persistent)
{
  if (regs != 96) {
    return 0;
  }
  return persistent ? occupancy_fp64_variant<64, 10, true>(ns, nf) : occupancy_fp64_variant<64, 10, false>(ns, nf);
}

}  // namespace pmp
