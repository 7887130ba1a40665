// batch.cuh — the persistent form of the run loop for many instances: ONE
// cooperative launch whose blocks stay resident and loop over the element
// tiles of every instance, advancing `attempts` passes of (SSP-RK3 attempt +
// run-loop control). The phases of an attempt are separated by grid-wide
// barriers (cooperative groups; the cooperative launch guarantees that every
// block is resident, and every block takes every barrier):
//   zero the reduction slots and limiter counters | stage 1 | limiter scan |
//   limiter rewrite | stage 2 | ... | stage 3 | ... | report + control
// Finished instances are skipped by the bodies; the loop ends early once no
// instance is active. The per-tile and per-element work is exactly the
// stage / limiter / control code of the separate launches, so the results are
// theirs: bit for bit in FP32-mixed, to an ulp in FP64 (the compiler may
// contract a multiply-add of the plain form differently in the two kernels).
// Included by common.cuh inside namespace cfd.
#pragma once


struct BatchParams {
  CfdSolver s;
  void* x0;
  void* x1;
  void* stage;
  int attempts;
};

// Tile shape of the persistent kernel per precision: FP32 the autotuned
// shape 9 (64 elements, staged base rows, packed contractions, out-of-line
// flux), FP64 shape 3 (64 elements).
template <typename R> struct BatchShape;
template <> struct BatchShape<float> {
  static constexpr int EPB = 64, MINB = 4;
  static constexpr bool SB = true, UF = true, PK = true, CF = true;
};
template <> struct BatchShape<double> {
  static constexpr int EPB = 64, MINB = 3;
  static constexpr bool SB = false, UF = true, PK = false, CF = false;
};

template <typename R, int FLUX, int PHI>
__global__ void __launch_bounds__(2 * BatchShape<R>::EPB, BatchShape<R>::MINB)
    batch_persistent_kernel(const BatchParams B) {
  using SH = BatchShape<R>;
  constexpr int EPB = SH::EPB, BS = 2 * EPB;
  constexpr int MODE = PHI == LIM_UNLIMITED ? MODE_UNLIMITED : MODE_LIMITED;
  namespace cgr = cooperative_groups;
  cgr::grid_group grid = cgr::this_grid();
  const CfdSolver& s = B.s;
  const int n = s.mesh.num_instances;
  const int K = s.mesh.num_elements;
  const int ntiles = (K + EPB - 1) / EPB;
  const int gtid = blockIdx.x * BS + threadIdx.x;
  const int gthreads = gridDim.x * BS;

  StageParams p;
  memset(&p, 0, sizeof(p));
  p.m = s.mesh;
  p.ctl = s.control;
  p.x0 = B.x0;
  p.x1 = B.x1;
  p.stage = B.stage;
  p.gamma = s.gamma;
  p.avg = s.averages;
  p.aux = s.element_aux;
  p.acc = s.acc;
  LimitParams lp;
  memset(&lp, 0, sizeof(lp));
  lp.m = s.mesh;
  lp.ctl = s.control;
  lp.x0 = B.x0;
  lp.x1 = B.x1;
  lp.stage = B.stage;
  lp.gamma = s.gamma;
  lp.avg = s.averages;
  lp.aux = s.element_aux;
  lp.acc = s.acc;
  lp.list = s.limit_list + LIMIT_LIST_HEADER;

  for (int it = 0; it < B.attempts; ++it) {
    for (int i = gtid; i < 3 * n; i += gthreads) reset_acc_one(s.acc, i);
    if (gtid < 4) s.limit_list[gtid] = 0;
    grid.sync();
    for (int k = 1; k <= 3; ++k) {
      p.stage_idx = k;
      for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        stage_tile_body<R, FLUX, MODE, EPB, SH::SB, SH::UF, SH::PK, SH::CF>(p, t);
        __syncthreads();  // the next tile reuses the block's shared memory
      }
      grid.sync();
      if constexpr (PHI != LIM_UNLIMITED) {
        lp.stage_idx = k;
        lp.count = s.limit_list + k;
        for (int e0 = blockIdx.x * BS; e0 < K; e0 += gridDim.x * BS) limit_scan_body<R, PHI, BS>(lp, e0);
        grid.sync();
        limit_rewrite_body<R, PHI>(lp);
        grid.sync();
      }
    }
    for (int i = gtid; i < n; i += gthreads) {
      report_one(s.acc, s.control, s.report, i, s.cfl);
      control_one(s.control, s.report, i, s.max_rejections);
    }
    grid.sync();
    // every block reads the same loop states here, so all leave together
    int active = 0;
    for (int i = threadIdx.x; i < n; i += BS)
      active |= ((const volatile CfdControl*)s.control)[i].status == CFD_RUN_ACTIVE;
    if (!__syncthreads_or(active)) break;
  }
}

// Host side: one persistent launch of a precision and flux, every limiter:
// as many blocks as are resident on the GPU, or as there are element tiles
// if that is fewer.
template <typename R, int FLUX, int PHI>
cudaError_t launch_batch_phi(const BatchParams& b, cudaStream_t st) {
  // b.attempts == 0: only the per-device lookup below, no launch
  using SH = BatchShape<R>;
  using L = TileLayout<R, SH::EPB, SH::SB>;
  auto kern = batch_persistent_kernel<R, FLUX, PHI>;
  // per device: the shared-memory opt-in and the resident grid size, looked
  // up once (before any stream capture, on the first call)
  constexpr int MAX_DEV = 64;
  static int grid_of[MAX_DEV] = {};
  int dev = 0;
  cudaError_t rc = cudaGetDevice(&dev);
  if (rc != cudaSuccess) return rc;
  if (dev < 0 || dev >= MAX_DEV) return cudaErrorInvalidDevice;
  if (!grid_of[dev]) {
    if ((rc = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES)) != cudaSuccess)
      return rc;
    int per_sm = 0, sms = 0;
    if ((rc = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 2 * SH::EPB, L::BYTES)) != cudaSuccess)
      return rc;
    if ((rc = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return rc;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    grid_of[dev] = per_sm * sms;
  }
  if (b.attempts == 0) return cudaSuccess;
  // no more blocks than element tiles: every phase strides over its work, and
  // a grid barrier over fewer blocks is cheaper for a small batch
  const int ntiles = (b.s.mesh.num_elements + SH::EPB - 1) / SH::EPB;
  const int grid = ntiles < 1 ? 1 : (ntiles < grid_of[dev] ? ntiles : grid_of[dev]);
  void* args[] = {const_cast<BatchParams*>(&b)};
  return cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3(2 * SH::EPB), args, L::BYTES, st);
}

template <typename R, int FLUX>
cudaError_t launch_batch_part(const BatchParams& b, int limiter, cudaStream_t st) {
  switch (limiter) {
    case 0: return launch_batch_phi<R, FLUX, 0>(b, st);
    case 1: return launch_batch_phi<R, FLUX, 1>(b, st);
    case 2: return launch_batch_phi<R, FLUX, 2>(b, st);
    case 3: return launch_batch_phi<R, FLUX, 3>(b, st);
    default: return launch_batch_phi<R, FLUX, 4>(b, st);
  }
}
#define CFD_DECLARE_BATCH_PART(R, FLUX) \
  extern template cudaError_t launch_batch_part<R, FLUX>(const BatchParams&, int, cudaStream_t);
CFD_DECLARE_BATCH_PART(double, 0)
CFD_DECLARE_BATCH_PART(double, 1)
CFD_DECLARE_BATCH_PART(double, 2)
CFD_DECLARE_BATCH_PART(float, 0)
CFD_DECLARE_BATCH_PART(float, 1)
CFD_DECLARE_BATCH_PART(float, 2)
