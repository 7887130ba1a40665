// stage_inst.cu — the fused stage kernels of one precision and one mode (every
// flux and tile shape). The build compiles this file six times, with
// CFD_STAGE_PREC = 0 (double) / 1 (float) and CFD_STAGE_MODE = 0 (rhs) /
// 1 (limited) / 2 (unlimited), so the kernels' template instantiations build in
// parallel objects; kernels.cu calls them through launch_stage_part.
#include "common.cuh"

#if !defined(CFD_STAGE_PREC) || !defined(CFD_STAGE_MODE)
#error "compile with -DCFD_STAGE_PREC=<0|1> -DCFD_STAGE_MODE=<0|1|2>"
#endif

namespace cfd {
#if CFD_STAGE_PREC == 0
template void launch_stage_part<double, CFD_STAGE_MODE>(const StageParams&, int, int, int, cudaStream_t);
#else
template void launch_stage_part<float, CFD_STAGE_MODE>(const StageParams&, int, int, int, cudaStream_t);
#endif
}  // namespace cfd
