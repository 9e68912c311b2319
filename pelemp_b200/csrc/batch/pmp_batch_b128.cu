// 128-thread variants of the batched FP64 update (96- and 128-register caps).
#include "batch_kernels.cuh"

namespace pmp {

bool batch_launch_b128(int ns, int nf, int regs, bool persistent, const KParams& P, const WorkArgs& W, int grid,
                       cudaStream_t st)
{
  if (regs == 96) {
    return persistent ? launch_fp64_variant<128, 5, true>(ns, nf, P, W, grid, st)
                      : launch_fp64_variant<128, 5, false>(ns, nf, P, W, grid, st);
  }
  if (regs == 128) {
    return persistent ? launch_fp64_variant<128, 4, true>(ns, nf, P, W, grid, st)
                      : launch_fp64_variant<128, 4, false>(ns, nf, P, W, grid, st);
  }
  return false;
}

int batch_occupancy_b128(int ns, int nf, int regs, bool persistent)
{
  if (regs == 96) {
    return persistent ? occupancy_fp64_variant<128, 5, true>(ns, nf) : occupancy_fp64_variant<128, 5, false>(ns, nf);
  }
  if (regs == 128) {
    return persistent ? occupancy_fp64_variant<128, 4, true>(ns, nf) : occupancy_fp64_variant<128, 4, false>(ns, nf);
  }
  return 0;
}

}  // namespace pmp
