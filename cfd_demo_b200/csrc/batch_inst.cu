// batch_inst.cu — the persistent batch kernel of one precision and one flux
// (every limiter). The build compiles this file six times, with
// CFD_BATCH_PREC = 0 (double) / 1 (float) and CFD_BATCH_FLUX = 0 / 1 / 2
// (rusanov / roe / hllc); kernels.cu calls them through launch_batch_part.
#include "common.cuh"

#if !defined(CFD_BATCH_PREC) || !defined(CFD_BATCH_FLUX)
#error "compile with -DCFD_BATCH_PREC=<0|1> -DCFD_BATCH_FLUX=<0|1|2>"
#endif

namespace cfd {
#if CFD_BATCH_PREC == 0
template cudaError_t launch_batch_part<double, CFD_BATCH_FLUX>(const BatchParams&, int, cudaStream_t);
#else
template cudaError_t launch_batch_part<float, CFD_BATCH_FLUX>(const BatchParams&, int, cudaStream_t);
#endif
}  // namespace cfd
