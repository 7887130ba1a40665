// kernels.cu — sm_100a kernels and C ABI of the degree-4 nodal DG Euler hot
// path (the operator of CFD-demo's src/cfd_demo/dg.py, limiting.py and
// time_integration.py, driven by the run loop of solver.py).
//
// Design: one thread per element, element-major SoA state q[(c*15+j)*ld+e], so
// every per-node load and store of a warp is one coalesced 256 B (double) or
// 128 B (float) transaction. The 15x30 [Dr|Ds] contraction and the 15x15 LIFT
// are compile-time constants (tables.cuh) applied as register-blocked FMAs:
// each thread streams over the nodes j computing the contravariant fluxes
// once and accumulating into a 15x4 register tile, then streams over its 15
// face nodes (neighbour trace gathered from the neighbour's column, or a
// boundary state), evaluates the interface flux and lifts the jump into the
// same tile. The RK stage combine, the cell averages and — when the limiter
// is `unlimited` — the positivity limiter, the stage minima and the CFL
// reduction all happen in the same kernel, so one stage reads the state once
// and writes it once. With slope limiting, a second light kernel per stage
// (limit_kernel) reads the averages of the element and its neighbours plus
// six midpoint traces and rewrites only troubled or non-positive elements.
// Global reductions go through ordered 64-bit keys and one atomic per block.
#include "common.cuh"

#include <nvtx3/nvToolsExt.h>

namespace {
// Host-side NVTX range over an entry point's launches (visible to Nsight
// tools when one is attached; a no-op check otherwise).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};
}  // namespace

namespace cfd {

// Averages + per-element minima of q_in, copied to q_out (cfd_limit prologue).
template <typename R, int BS>
__global__ void __launch_bounds__(BS) prep_kernel(CfdMesh m, const R* __restrict__ qin, R* __restrict__ qout,
                                                   double* avg, double* aux, double gamma) {
  const int e = blockIdx.x * BS + threadIdx.x;
  if (e >= m.num_elements) return;
  const int ld = m.ld;
  R s[NP][4];
#pragma unroll
  for (int i = 0; i < NP; ++i)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      s[i][c] = qin[(c * NP + i) * ld + e];
      if (qout != qin) qout[(c * NP + i) * ld + e] = s[i][c];
    }
  double a[4];
  cell_average<R>(s, a);
#pragma unroll
  for (int c = 0; c < 4; ++c) avg[c * ld + e] = a[c];
  double rmin, pmin, lam;
  bool finite;
  element_stats<R>(s, gamma - 1.0, gamma, rmin, pmin, lam, finite);
  aux[e] = rmin;
  aux[ld + e] = pmin;
  aux[2 * ld + e] = lam;
}

#include "adjoint.cuh"

// ---------------------------------------------------------- small kernels ---
template <typename R, int BS>
__global__ void __launch_bounds__(BS) dt_kernel(CfdMesh m, const R* __restrict__ q, CfdStageAcc* acc, double gamma,
                                                 double* minima) {
  const int e = blockIdx.x * BS + threadIdx.x;
  const int inst_raw = (e < m.num_elements && m.instance) ? m.instance[e] : 0;
  const bool live = e < m.num_elements && inst_raw >= 0;
  const int inst = live ? inst_raw : 0;
  Red red;
  red.init();
  if (live) {
    const int ld = m.ld;
    R s[NP][4];
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c) s[i][c] = q[(c * NP + i) * ld + e];
    double rmin, pmin, lam;
    bool finite;
    element_stats<R>(s, gamma - 1.0, gamma, rmin, pmin, lam, finite);
    // time_integration.py:41 — the min propagates NaN: a NaN element poisons dt
    const double d = m.dt_geo[e] / lam;
    red.kd = dkey(d);
    if (d != d) red.fl |= FLAG_NAN_DT;
    red.kr = dkey(rmin);
    red.kp = dkey(pmin);
    if (!finite) red.fl |= FLAG_NONFINITE;
  }
  block_commit<BS>(red, live, inst, acc, 3, 2);
}

__global__ void reset_acc_kernel(CfdStageAcc* acc, int n, int* list_counters) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < 4 && list_counters) list_counters[i] = 0;  // the two-pass limiter's per-stage counters
  if (i < n) reset_acc_one(acc, i);
}

__global__ void report_kernel(const CfdStageAcc* acc, const CfdControl* ctl, CfdStepReport* rep, int n, double cfl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) report_one(acc, ctl, rep, i, cfl);
}

__global__ void run_control_kernel(CfdControl* ctl, const CfdStepReport* rep, int n, int max_rejections) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) control_one(ctl, rep, i, max_rejections);
}

__global__ void run_init_kernel(CfdControl* ctl, const CfdStageAcc* acc, const double* final_time, int n, double cfl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  CfdControl c;
  memset(&c, 0, sizeof(c));
  c.final_time = final_time[i];
  const CfdStageAcc a = acc[3 * i + 2];
  c.min_density = key_min_value(a.min_rho_key);
  c.min_pressure = key_min_value(a.min_p_key);
  c.status = CFD_RUN_ACTIVE;
  if (!(c.time < c.final_time)) {
    c.status = CFD_RUN_DONE;
  } else {
    const double dt = (a.flags & FLAG_NAN_DT) ? (double)NAN : cfl * dkey_decode(a.dt_key);
    if (!isfinite(dt) || dt <= 0.0) {
      c.status = CFD_RUN_BAD_DT;
      c.dt = dt;
    } else {
      const double remaining = c.final_time - c.time;
      c.reaches_end = dt >= remaining;
      c.dt = c.reaches_end ? remaining : dt;
    }
  }
  ctl[i] = c;
}

// Loop state of a fixed-size step (cfd_rk3_step_fixed): every instance
// active, its state in x0, the step size given per instance.
__global__ void fixed_control_kernel(CfdControl* ctl, const double* dt, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  CfdControl c;
  memset(&c, 0, sizeof(c));
  c.final_time = INFINITY;
  c.dt = dt[i];
  c.min_density = INFINITY;
  c.min_pressure = INFINITY;
  c.status = CFD_RUN_ACTIVE;
  ctl[i] = c;
}

__global__ void dt_out_kernel(const CfdStageAcc* acc, double* dt, int n, double cfl) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dt[i] = (acc[3 * i + 2].flags & FLAG_NAN_DT) ? (double)NAN : cfl * dkey_decode(acc[3 * i + 2].dt_key);
}

__global__ void check_out_kernel(const CfdStageAcc* acc, double* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const CfdStageAcc a = acc[3 * i + 2];
  out[3 * i + 0] = key_min_value(a.min_rho_key);
  out[3 * i + 1] = key_min_value(a.min_p_key);
  out[3 * i + 2] = (a.flags & FLAG_NONFINITE) ? 0.0 : 1.0;
}

// (Np, K, 4) double  <->  [(c*15+j)*ld + e] of R
template <typename R>
__global__ void pack_kernel(const double* __restrict__ in, R* __restrict__ out, int K, int ld) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)NP * K) return;
  const int j = (int)(t / K), e = (int)(t % K);
  const double4 v = reinterpret_cast<const double4*>(in)[t];
  out[(0 * NP + j) * (long long)ld + e] = (R)v.x;
  out[(1 * NP + j) * (long long)ld + e] = (R)v.y;
  out[(2 * NP + j) * (long long)ld + e] = (R)v.z;
  out[(3 * NP + j) * (long long)ld + e] = (R)v.w;
}
template <typename R>
__global__ void unpack_kernel(const R* __restrict__ in, double* __restrict__ out, int K, int ld) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)NP * K) return;
  const int j = (int)(t / K), e = (int)(t % K);
  double4 v;
  v.x = (double)in[(0 * NP + j) * (long long)ld + e];
  v.y = (double)in[(1 * NP + j) * (long long)ld + e];
  v.z = (double)in[(2 * NP + j) * (long long)ld + e];
  v.w = (double)in[(3 * NP + j) * (long long)ld + e];
  reinterpret_cast<double4*>(out)[t] = v;
}

template <typename R>
__global__ void averages_kernel(CfdMesh m, const R* __restrict__ q, double* avg) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.num_elements) return;
  const int ld = m.ld;
  if (m.instance && m.instance[e] < 0) return;  // padding between instances
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < NP; ++i) s = fma(tab::AVG_W[i], (double)q[(c * NP + i) * ld + e], s);
    avg[c * ld + e] = s;
  }
}

// Domain integral per instance (dg.py:174-176): J_k sum_i w_i q_ik, summed
// over the warp before one atomic per warp and variable when the warp's
// elements belong to one instance (one atomic per element would serialise
// on the four addresses).
template <typename R>
__global__ void integral_kernel(CfdMesh m, const R* __restrict__ q, double* integral) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int ld = m.ld;
  int inst = (e < m.num_elements) ? (m.instance ? m.instance[e] : 0) : -1;
  double v[4] = {0.0, 0.0, 0.0, 0.0};
  if (inst >= 0) {
    const double jac = m.jacobian[e];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      double s = 0.0;
#pragma unroll
      for (int i = 0; i < NP; ++i) s = fma(tab::CELL_W[i], (double)q[(c * NP + i) * ld + e], s);
      v[c] = jac * s;
    }
  }
  const int lane = threadIdx.x & 31;
  const int first = __reduce_max_sync(0xffffffffu, (unsigned)(inst + 1)) - 1;  // an instance present in the warp
  const bool uniform = __all_sync(0xffffffffu, inst < 0 || inst == first) && first >= 0;
  if (uniform) {
#pragma unroll
    for (int c = 0; c < 4; ++c) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(0xffffffffu, v[c], o);
    }
    if (lane == 0)
      for (int c = 0; c < 4; ++c) atomicAdd(&integral[first * 4 + c], v[c]);
  } else if (inst >= 0) {
    for (int c = 0; c < 4; ++c) atomicAdd(&integral[inst * 4 + c], v[c]);
  }
}

template <int FLUX>
__global__ void flux_pointwise_kernel(int n, const double* qm, const double* qp, const double* nx, const double* ny,
                                      double gamma, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a[4], b[4], fh[4], fm[4];
  for (int c = 0; c < 4; ++c) {
    a[c] = qm[4 * i + c];
    b[c] = qp[4 * i + c];
  }
  interface_flux<double, FLUX>(a, b, nx[i], ny[i], gamma, fh, fm);
  for (int c = 0; c < 4; ++c) out[4 * i + c] = fh[c];
}

template <int PHI>
__global__ void phi_pointwise_kernel(int n, const double* r, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = phi<double, PHI>(r[i]);
}

}  // namespace cfd

// ================================================================= C ABI ===
using namespace cfd;

static thread_local char g_err[512] = "";

static int fail(int code, const char* msg) {
  snprintf(g_err, sizeof(g_err), "%s", msg);
  return code;
}
int cfd::cfd_fail(int code, const char* msg) { return fail(code, msg); }
static int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
    return CFD_E_CUDA;
  }
  return CFD_OK;
}

static int validate(const CfdSolver* s) {
  if (!s) return fail(CFD_E_ARG, "null solver");
  const CfdMesh& m = s->mesh;
  if (m.num_elements <= 0 || m.ld < m.num_elements || m.num_instances < 1) return fail(CFD_E_ARG, "bad mesh sizes");
  if (!m.metric || !m.face_geo || !m.face_hlen || !m.dt_geo || !m.jacobian || !m.cs_coef || !m.neighbor || !m.face_info)
    return fail(CFD_E_ARG, "mesh table pointer is null");
  if (m.num_instances > 1 && !m.instance) return fail(CFD_E_ARG, "instance table needed for several instances");
  if (s->flux < 0 || s->flux > 2) return fail(CFD_E_ARG, "unknown flux id");
  if (s->limiter < 0 || s->limiter > 4) return fail(CFD_E_ARG, "unknown limiter id");
  if (s->precision != CFD_FP64 && s->precision != CFD_FP32_MIXED) return fail(CFD_E_ARG, "unknown precision id");
  if (s->precision == CFD_FP32_MIXED && (!m.metric32 || !m.face_geo32 || !m.cs_coef32))
    return fail(CFD_E_ARG, "FP32 mesh tables missing for the mixed precision");
  if (!(s->gamma > 1.0)) return fail(CFD_E_ARG, "gamma must be greater than one");
  if (s->block_size != 0 && s->block_size != 64 && s->block_size != 128 && s->block_size != 256)
    return fail(CFD_E_ARG, "block_size must be 0, 64, 128 or 256");
  if (s->variant < 0 || s->variant > 14) return fail(CFD_E_ARG, "variant must be 0..14");
  if (s->variant != 2 && s->mesh.instance && s->mesh.num_instances > 1 && (s->mesh.flags & 1) == 0)
    return fail(CFD_E_ARG, "tiled stage kernels need instance ranges aligned to 64 elements (CfdMesh.flags bit 0)");
  return CFD_OK;
}

static inline int bs_of(const CfdSolver* s) { return s->block_size ? s->block_size : 128; }

static void launch_stage(const CfdSolver* s, const StageParams& p, int mode, cudaStream_t st) {
  const int bs = bs_of(s);
  const int v = s->variant;
  if (s->precision == CFD_FP64) {
    if (mode == MODE_RHS) launch_stage_part<double, MODE_RHS>(p, s->flux, v, bs, st);
    else if (mode == MODE_LIMITED) launch_stage_part<double, MODE_LIMITED>(p, s->flux, v, bs, st);
    else launch_stage_part<double, MODE_UNLIMITED>(p, s->flux, v, bs, st);
  } else {
    if (mode == MODE_RHS) launch_stage_part<float, MODE_RHS>(p, s->flux, v, bs, st);
    else if (mode == MODE_LIMITED) launch_stage_part<float, MODE_LIMITED>(p, s->flux, v, bs, st);
    else launch_stage_part<float, MODE_UNLIMITED>(p, s->flux, v, bs, st);
  }
}
template <typename R, int PHI>
static void launch_limit_bs(const LimitParams& p, int bs, cudaStream_t st) {
  const unsigned g = blocks_for(p.m.num_elements, bs);
  if (bs == 64) limit_kernel<R, PHI, 64><<<g, 64, 0, st>>>(p);
  else if (bs == 256) limit_kernel<R, PHI, 256><<<g, 256, 0, st>>>(p);
  else limit_kernel<R, PHI, 128><<<g, 128, 0, st>>>(p);
}
template <typename R>
static void launch_limit_phi(const LimitParams& p, int lim, int bs, cudaStream_t st) {
  switch (lim) {
    case 0: launch_limit_bs<R, 0>(p, bs, st); break;
    case 1: launch_limit_bs<R, 1>(p, bs, st); break;
    case 2: launch_limit_bs<R, 2>(p, bs, st); break;
    case 3: launch_limit_bs<R, 3>(p, bs, st); break;
    default: launch_limit_bs<R, 4>(p, bs, st); break;
  }
}
template <typename R, int PHI>
static void launch_limit_two_pass(const LimitParams& p, int bs, cudaStream_t st) {
  const unsigned g = blocks_for(p.m.num_elements, bs);
  if (bs == 64) limit_scan_kernel<R, PHI, 64><<<g, 64, 0, st>>>(p);
  else if (bs == 256) limit_scan_kernel<R, PHI, 256><<<g, 256, 0, st>>>(p);
  else limit_scan_kernel<R, PHI, 128><<<g, 128, 0, st>>>(p);
  // the list's length is only known on the device: four threads per listed
  // element, enough for a sixteenth of the elements in one sweep (blocks
  // beyond the list end exit at once; a longer list is swept grid-stride)
  const unsigned full = blocks_for(p.m.num_elements, 64), cap = 32 * 148;
  limit_rewrite_kernel<R, PHI><<<full < cap ? full : cap, 64, 0, st>>>(p);
}
template <typename R>
static void launch_limit_two_pass_phi(const LimitParams& p, int lim, int bs, cudaStream_t st) {
  switch (lim) {
    case 0: launch_limit_two_pass<R, 0>(p, bs, st); break;
    case 1: launch_limit_two_pass<R, 1>(p, bs, st); break;
    case 2: launch_limit_two_pass<R, 2>(p, bs, st); break;
    case 3: launch_limit_two_pass<R, 3>(p, bs, st); break;
    default: launch_limit_two_pass<R, 4>(p, bs, st); break;
  }
}
// With a limit_list scratch the limiter runs in two passes (scan + rewrite
// of the listed elements); without one, in one pass.
static void launch_limit(const CfdSolver* s, LimitParams p, cudaStream_t st) {
  if (s->limit_list) {
    p.count = s->limit_list + (p.stage_idx >= 0 && p.stage_idx <= 3 ? p.stage_idx : 0);
    p.list = s->limit_list + LIMIT_LIST_HEADER;
    if (s->precision == CFD_FP64) launch_limit_two_pass_phi<double>(p, s->limiter, bs_of(s), st);
    else launch_limit_two_pass_phi<float>(p, s->limiter, bs_of(s), st);
    return;
  }
  if (s->precision == CFD_FP64) launch_limit_phi<double>(p, s->limiter, bs_of(s), st);
  else launch_limit_phi<float>(p, s->limiter, bs_of(s), st);
}
template <typename R>
static void launch_dt(const CfdSolver* s, const void* q, cudaStream_t st) {
  const int bs = 128;
  dt_kernel<R, 128><<<blocks_for(s->mesh.num_elements, bs), bs, 0, st>>>(s->mesh, (const R*)q, s->acc, s->gamma, nullptr);
}
static void reset_acc(const CfdSolver* s, cudaStream_t st) {
  const int n = 3 * s->mesh.num_instances;
  reset_acc_kernel<<<blocks_for(n > 4 ? n : 4, 128), 128, 0, st>>>(s->acc, n, s->limit_list);
}

extern "C" {

int cfd_abi_version(void) { return CFD_ABI_VERSION; }

int cfd_struct_sizes(int32_t* out, int32_t n) {
  if (!out || n < 5) return fail(CFD_E_ARG, "cfd_struct_sizes: need room for 5 sizes");
  out[0] = (int32_t)sizeof(CfdMesh);
  out[1] = (int32_t)sizeof(CfdStageAcc);
  out[2] = (int32_t)sizeof(CfdStepReport);
  out[3] = (int32_t)sizeof(CfdControl);
  out[4] = (int32_t)sizeof(CfdSolver);
  return CFD_OK;
}
const char* cfd_last_error(void) { return g_err; }

int cfd_pack_state(const double* q_nk4, void* q_dev, int32_t K, int32_t ld, int32_t precision, void* stream) {
  if (!q_nk4 || !q_dev || K <= 0 || ld < K) return fail(CFD_E_ARG, "cfd_pack_state: bad arguments");
  if (((uintptr_t)q_nk4) % 32) return fail(CFD_E_ARG, "cfd_pack_state: input must be 32-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  const long long n = (long long)NP * K;
  if (precision == CFD_FP64) pack_kernel<double><<<blocks_for(n, 256), 256, 0, st>>>(q_nk4, (double*)q_dev, K, ld);
  else if (precision == CFD_FP32_MIXED) pack_kernel<float><<<blocks_for(n, 256), 256, 0, st>>>(q_nk4, (float*)q_dev, K, ld);
  else return fail(CFD_E_ARG, "cfd_pack_state: unknown precision");
  return check_launch("cfd_pack_state");
}

int cfd_unpack_state(const void* q_dev, double* q_nk4, int32_t K, int32_t ld, int32_t precision, void* stream) {
  if (!q_nk4 || !q_dev || K <= 0 || ld < K) return fail(CFD_E_ARG, "cfd_unpack_state: bad arguments");
  if (((uintptr_t)q_nk4) % 32) return fail(CFD_E_ARG, "cfd_unpack_state: output must be 32-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  const long long n = (long long)NP * K;
  if (precision == CFD_FP64) unpack_kernel<double><<<blocks_for(n, 256), 256, 0, st>>>((const double*)q_dev, q_nk4, K, ld);
  else if (precision == CFD_FP32_MIXED) unpack_kernel<float><<<blocks_for(n, 256), 256, 0, st>>>((const float*)q_dev, q_nk4, K, ld);
  else return fail(CFD_E_ARG, "cfd_unpack_state: unknown precision");
  return check_launch("cfd_unpack_state");
}

int cfd_rhs(const CfdSolver* s, const void* q, void* rhs, double* bflux, void* stream) {
  NvtxRange nvtx_range("cfd_rhs");
  int rc = validate(s);
  if (rc) return rc;
  if (!q || !rhs || !bflux) return fail(CFD_E_ARG, "cfd_rhs: null pointer");
  if (q == rhs) return fail(CFD_E_ARG, "cfd_rhs: rhs must not alias q");
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(bflux, 0, sizeof(double) * 4 * s->mesh.num_instances, st) != cudaSuccess)
    return check_launch("cfd_rhs: memset");
  StageParams p;
  memset(&p, 0, sizeof(p));
  p.m = s->mesh;
  p.gamma = s->gamma;
  p.q_in = q;
  p.q_out = rhs;
  p.bflux_out = bflux;
  launch_stage(s, p, MODE_RHS, st);
  return check_launch("cfd_rhs");
}

int cfd_limit(const CfdSolver* s, const void* q_in, void* q_out, int32_t* troubled, void* stream) {
  NvtxRange nvtx_range("cfd_limit");
  int rc = validate(s);
  if (rc) return rc;
  if (!q_in || !q_out || !troubled || !s->averages || !s->element_aux) return fail(CFD_E_ARG, "cfd_limit: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(troubled, 0, sizeof(int32_t) * s->mesh.num_instances, st) != cudaSuccess)
    return check_launch("cfd_limit: memset");
  if (s->limit_list && cudaMemsetAsync(s->limit_list, 0, sizeof(int32_t), st) != cudaSuccess)
    return check_launch("cfd_limit: memset");
  const int bs = 128;
  const unsigned g = blocks_for(s->mesh.num_elements, bs);
  if (s->precision == CFD_FP64)
    prep_kernel<double, 128><<<g, bs, 0, st>>>(s->mesh, (const double*)q_in, (double*)q_out, s->averages, s->element_aux, s->gamma);
  else
    prep_kernel<float, 128><<<g, bs, 0, st>>>(s->mesh, (const float*)q_in, (float*)q_out, s->averages, s->element_aux, s->gamma);
  LimitParams p;
  memset(&p, 0, sizeof(p));
  p.m = s->mesh;
  p.stage_idx = 0;
  p.q_io = q_out;
  p.gamma = s->gamma;
  p.avg = s->averages;
  p.aux = s->element_aux;
  p.troubled_out = troubled;
  p.flags = s->troubled_flags;
  launch_limit(s, p, st);
  return check_launch("cfd_limit");
}

int cfd_time_step(const CfdSolver* s, const void* q, double* dt, void* stream) {
  NvtxRange nvtx_range("cfd_time_step");
  int rc = validate(s);
  if (rc) return rc;
  if (!q || !dt || !s->acc) return fail(CFD_E_ARG, "cfd_time_step: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  reset_acc(s, st);
  if (s->precision == CFD_FP64) launch_dt<double>(s, q, st);
  else launch_dt<float>(s, q, st);
  const int n = s->mesh.num_instances;
  dt_out_kernel<<<blocks_for(n, 128), 128, 0, st>>>(s->acc, dt, n, s->cfl);
  return check_launch("cfd_time_step");
}

int cfd_check_state(const CfdSolver* s, const void* q, double* out, void* stream) {
  int rc = validate(s);
  if (rc) return rc;
  if (!q || !out || !s->acc) return fail(CFD_E_ARG, "cfd_check_state: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  reset_acc(s, st);
  if (s->precision == CFD_FP64) launch_dt<double>(s, q, st);
  else launch_dt<float>(s, q, st);
  const int n = s->mesh.num_instances;
  check_out_kernel<<<blocks_for(n, 128), 128, 0, st>>>(s->acc, out, n);
  return check_launch("cfd_check_state");
}

int cfd_cell_averages(const CfdSolver* s, const void* q, double* avg, void* stream) {
  int rc = validate(s);
  if (rc) return rc;
  if (!q || !avg) return fail(CFD_E_ARG, "cfd_cell_averages: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned g = blocks_for(s->mesh.num_elements, 128);
  if (s->precision == CFD_FP64) averages_kernel<double><<<g, 128, 0, st>>>(s->mesh, (const double*)q, avg);
  else averages_kernel<float><<<g, 128, 0, st>>>(s->mesh, (const float*)q, avg);
  return check_launch("cfd_cell_averages");
}

int cfd_integrate(const CfdSolver* s, const void* q, double* integral, void* stream) {
  int rc = validate(s);
  if (rc) return rc;
  if (!q || !integral) return fail(CFD_E_ARG, "cfd_integrate: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemsetAsync(integral, 0, sizeof(double) * 4 * s->mesh.num_instances, st) != cudaSuccess)
    return check_launch("cfd_integrate: memset");
  const unsigned g = blocks_for(s->mesh.num_elements, 128);
  if (s->precision == CFD_FP64) integral_kernel<double><<<g, 128, 0, st>>>(s->mesh, (const double*)q, integral);
  else integral_kernel<float><<<g, 128, 0, st>>>(s->mesh, (const float*)q, integral);
  return check_launch("cfd_integrate");
}

static int attempt_args(const CfdSolver* s, void* x0, void* x1, void* stage) {
  int rc = validate(s);
  if (rc) return rc;
  if (!x0 || !x1 || !stage || !s->acc || !s->control || !s->report) return fail(CFD_E_ARG, "cfd_rk3: null pointer");
  if (s->limiter != CFD_LIMITER_UNLIMITED && (!s->averages || !s->element_aux))
    return fail(CFD_E_ARG, "cfd_rk3: averages / element_aux scratch missing");
  if (x0 == x1 || x0 == stage || x1 == stage) return fail(CFD_E_ARG, "cfd_rk3: state buffers must be distinct");
  return CFD_OK;
}

int cfd_rk3_begin(const CfdSolver* s, void* stream) {
  int rc = validate(s);
  if (rc) return rc;
  if (!s->acc) return fail(CFD_E_ARG, "cfd_rk3_begin: null pointer");
  reset_acc(s, (cudaStream_t)stream);
  return check_launch("cfd_rk3_begin");
}

int cfd_rk3_stage(const CfdSolver* s, void* x0, void* x1, void* stage, int32_t k, void* stream) {
  NvtxRange nvtx_range("cfd_rk3_stage");
  int rc = attempt_args(s, x0, x1, stage);
  if (rc) return rc;
  if (k < 1 || k > 3) return fail(CFD_E_ARG, "cfd_rk3_stage: stage must be 1, 2 or 3");
  cudaStream_t st = (cudaStream_t)stream;
  const bool limited = s->limiter != CFD_LIMITER_UNLIMITED;
  StageParams p;
  memset(&p, 0, sizeof(p));
  p.m = s->mesh;
  p.ctl = s->control;
  p.x0 = x0;
  p.x1 = x1;
  p.stage = stage;
  p.stage_idx = k;
  p.gamma = s->gamma;
  p.avg = s->averages;
  p.aux = s->element_aux;
  p.acc = s->acc;
  launch_stage(s, p, limited ? MODE_LIMITED : MODE_UNLIMITED, st);
  if (limited) {
    LimitParams lp;
    memset(&lp, 0, sizeof(lp));
    lp.m = s->mesh;
    lp.ctl = s->control;
    lp.x0 = x0;
    lp.x1 = x1;
    lp.stage = stage;
    lp.stage_idx = k;
    lp.gamma = s->gamma;
    lp.avg = s->averages;
    lp.aux = s->element_aux;
    lp.acc = s->acc;
    lp.flags = s->troubled_flags ? s->troubled_flags + (size_t)(k - 1) * s->mesh.ld : nullptr;
    launch_limit(s, lp, st);
  }
  return check_launch("cfd_rk3_stage");
}

int cfd_rk3_finish(const CfdSolver* s, void* stream) {
  int rc = validate(s);
  if (rc) return rc;
  if (!s->acc || !s->control || !s->report) return fail(CFD_E_ARG, "cfd_rk3_finish: null pointer");
  const int n = s->mesh.num_instances;
  report_kernel<<<blocks_for(n, 128), 128, 0, (cudaStream_t)stream>>>(s->acc, s->control, s->report, n, s->cfl);
  return check_launch("cfd_rk3_finish");
}

int cfd_rk3_attempt(const CfdSolver* s, void* x0, void* x1, void* stage, void* stream) {
  NvtxRange nvtx_range("cfd_rk3_attempt");
  int rc = attempt_args(s, x0, x1, stage);
  if (rc) return rc;
  if ((rc = cfd_rk3_begin(s, stream))) return rc;
  for (int k = 1; k <= 3; ++k)
    if ((rc = cfd_rk3_stage(s, x0, x1, stage, k, stream))) return rc;
  return cfd_rk3_finish(s, stream);
}

int cfd_run_control(const CfdSolver* s, void* stream) {
  NvtxRange nvtx_range("cfd_run_control");
  int rc = validate(s);
  if (rc) return rc;
  if (!s->control || !s->report) return fail(CFD_E_ARG, "cfd_run_control: null pointer");
  const int n = s->mesh.num_instances;
  run_control_kernel<<<blocks_for(n, 128), 128, 0, (cudaStream_t)stream>>>(s->control, s->report, n, s->max_rejections);
  return check_launch("cfd_run_control");
}

int cfd_batch_advance(const CfdSolver* s, void* x0, void* x1, void* stage, int32_t attempts, void* stream) {
  NvtxRange nvtx_range("cfd_batch_advance");
  int rc = attempt_args(s, x0, x1, stage);
  if (rc) return rc;
  if (!s->limit_list) return fail(CFD_E_ARG, "cfd_batch_advance: limit_list scratch is required");
  if (attempts < 0) return fail(CFD_E_ARG, "cfd_batch_advance: attempts must be nonnegative");
  BatchParams b;
  memset(&b, 0, sizeof(b));
  b.s = *s;
  b.x0 = x0;
  b.x1 = x1;
  b.stage = stage;
  b.attempts = attempts;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (s->precision == CFD_FP64) {
    e = s->flux == 0 ? launch_batch_part<double, 0>(b, s->limiter, st)
        : s->flux == 1 ? launch_batch_part<double, 1>(b, s->limiter, st)
                       : launch_batch_part<double, 2>(b, s->limiter, st);
  } else {
    e = s->flux == 0 ? launch_batch_part<float, 0>(b, s->limiter, st)
        : s->flux == 1 ? launch_batch_part<float, 1>(b, s->limiter, st)
                       : launch_batch_part<float, 2>(b, s->limiter, st);
  }
  if (e != cudaSuccess) {
    snprintf(g_err, sizeof(g_err), "cfd_batch_advance: %s", cudaGetErrorString(e));
    return CFD_E_CUDA;
  }
  return check_launch("cfd_batch_advance");
}

int cfd_run_init(const CfdSolver* s, const void* x0, const double* final_time, void* stream) {
  int rc = validate(s);
  if (rc) return rc;
  if (!x0 || !final_time || !s->control || !s->acc) return fail(CFD_E_ARG, "cfd_run_init: null pointer");
  cudaStream_t st = (cudaStream_t)stream;
  reset_acc(s, st);
  if (s->precision == CFD_FP64) launch_dt<double>(s, x0, st);
  else launch_dt<float>(s, x0, st);
  const int n = s->mesh.num_instances;
  run_init_kernel<<<blocks_for(n, 128), 128, 0, st>>>(s->control, s->acc, final_time, n, s->cfl);
  return check_launch("cfd_run_init");
}

int cfd_interface_flux(int32_t flux, int32_t n, const double* q_minus, const double* q_plus, const double* nx,
                       const double* ny, double gamma, double* out, void* stream) {
  if (n < 0 || (n > 0 && (!q_minus || !q_plus || !nx || !ny || !out))) return fail(CFD_E_ARG, "cfd_interface_flux: bad arguments");
  if (n == 0) return CFD_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned g = blocks_for(n, 128);
  if (flux == 0) flux_pointwise_kernel<0><<<g, 128, 0, st>>>(n, q_minus, q_plus, nx, ny, gamma, out);
  else if (flux == 1) flux_pointwise_kernel<1><<<g, 128, 0, st>>>(n, q_minus, q_plus, nx, ny, gamma, out);
  else if (flux == 2) flux_pointwise_kernel<2><<<g, 128, 0, st>>>(n, q_minus, q_plus, nx, ny, gamma, out);
  else return fail(CFD_E_ARG, "cfd_interface_flux: unknown flux id");
  return check_launch("cfd_interface_flux");
}

int cfd_limiter_phi(int32_t limiter, int32_t n, const double* r, double* out, void* stream) {
  if (n < 0 || (n > 0 && (!r || !out))) return fail(CFD_E_ARG, "cfd_limiter_phi: bad arguments");
  if (n == 0) return CFD_OK;
  cudaStream_t st = (cudaStream_t)stream;
  const unsigned g = blocks_for(n, 128);
  switch (limiter) {
    case 0: phi_pointwise_kernel<0><<<g, 128, 0, st>>>(n, r, out); break;
    case 1: phi_pointwise_kernel<1><<<g, 128, 0, st>>>(n, r, out); break;
    case 2: phi_pointwise_kernel<2><<<g, 128, 0, st>>>(n, r, out); break;
    case 3: phi_pointwise_kernel<3><<<g, 128, 0, st>>>(n, r, out); break;
    case 4: phi_pointwise_kernel<4><<<g, 128, 0, st>>>(n, r, out); break;
    default: return fail(CFD_E_ARG, "cfd_limiter_phi: unknown limiter id");
  }
  return check_launch("cfd_limiter_phi");
}

}  // extern "C"

// ------------------------------------------------ fixed-size step + adjoint ---
// Tape of one step (sizes in elements of ld): the pre-limiting stage states
// qt1, qt2, qt3 and the limited stage states q1, q2 (60 rows each, solver
// precision) in the order qt1 q1 qt2 q2 qt3, then per stage k = 1..3 nine rows
// of double: the cell averages of qt_k (4), its nodal density / pressure
// minima and wave speed (3), and the positivity limiter's pressure-scaling
// theta and critical node (2, written for the elements it processed).
namespace {
constexpr int TAPE_ROWS_PER_STAGE = 9;
size_t state_bytes(int ld, int precision) { return (size_t)60 * ld * (precision == CFD_FP64 ? 8 : 4); }
size_t tape_bytes(int ld, int precision) {
  return 5 * state_bytes(ld, precision) + (size_t)3 * TAPE_ROWS_PER_STAGE * ld * 8;
}
char* tape_state(void* tape, int ld, int precision, int slot) { return (char*)tape + slot * state_bytes(ld, precision); }
double* tape_avg(void* tape, int ld, int precision, int k) {
  return (double*)((char*)tape + 5 * state_bytes(ld, precision)) + (size_t)(k - 1) * TAPE_ROWS_PER_STAGE * ld;
}
double* tape_aux(void* tape, int ld, int precision, int k) { return tape_avg(tape, ld, precision, k) + (size_t)4 * ld; }
double* tape_pos(void* tape, int ld, int precision, int k) { return tape_avg(tape, ld, precision, k) + (size_t)7 * ld; }
// adjoint scratch: qt_bar, face-node adjoints w, neighbour-average adjoints,
// the adjoints of q1 and q2 (60 + 60 + 12 + 60 + 60 rows of the solver
// precision), the list of elements for the full limiter replay (ld ints), its
// counter (in a 256-byte slot) and the per-element listed flags (ld bytes)
size_t adjoint_reals_bytes(int ld, int precision) { return (size_t)252 * ld * (precision == CFD_FP64 ? 8 : 4); }
size_t adjoint_work_bytes(int ld, int precision) {
  return adjoint_reals_bytes(ld, precision) + (size_t)4 * ld + 256 + (((size_t)ld + 255) & ~(size_t)255);
}

template <typename R, int PHI>
void launch_adj_limit_phi(const AdjParams& p, int n, cudaStream_t st) {
  adj_limit_scan_kernel<R, PHI><<<blocks_for(n, 128), 128, 0, st>>>(p);
  // four lanes per listed element; the list's length is only known on the
  // device, so the grid covers up to 37,888 elements per sweep (16 blocks of
  // 64 threads per SM) and strides over the rest
  const unsigned want = blocks_for(4LL * n, 64), hb = want < 16 * 148 ? want : 16 * 148;
  adj_limit_heavy_kernel<R, PHI><<<hb, 64, 0, st>>>(p);
}
template <typename R>
void launch_adj_limit(const AdjParams& p, int lim, int n, cudaStream_t st) {
  switch (lim) {
    case 0: launch_adj_limit_phi<R, 0>(p, n, st); break;
    case 1: launch_adj_limit_phi<R, 1>(p, n, st); break;
    case 2: launch_adj_limit_phi<R, 2>(p, n, st); break;
    case 3: launch_adj_limit_phi<R, 3>(p, n, st); break;
    default: launch_adj_limit_phi<R, 4>(p, n, st); break;
  }
}
template <typename R>
void launch_adj_rhs(const AdjParams& p, int flux, int n, cudaStream_t st) {
  adj_lift_kernel<R><<<dim3(blocks_for(n, 128), 4), 128, 0, st>>>(p);
  const dim3 grid(blocks_for(n, ADJ_EPB)), block(ADJ_EPB, NP);
  switch (flux) {
    case 0: adj_rhs_node_kernel<R, 0><<<grid, block, 0, st>>>(p); break;
    case 1: adj_rhs_node_kernel<R, 1><<<grid, block, 0, st>>>(p); break;
    default: adj_rhs_node_kernel<R, 2><<<grid, block, 0, st>>>(p); break;
  }
}
}  // namespace

extern "C" {

int64_t cfd_tape_bytes(int32_t ld, int32_t precision) {
  if (ld <= 0 || (precision != CFD_FP64 && precision != CFD_FP32_MIXED)) return -1;
  return (int64_t)tape_bytes(ld, precision);
}

int64_t cfd_adjoint_work_bytes(int32_t ld, int32_t precision) {
  if (ld <= 0 || (precision != CFD_FP64 && precision != CFD_FP32_MIXED)) return -1;
  return (int64_t)adjoint_work_bytes(ld, precision);
}

int cfd_rk3_step_fixed(const CfdSolver* s, const void* q_in, void* q_out, void* stage, const double* dt, void* tape,
                       void* stream) {
  NvtxRange nvtx_range("cfd_rk3_step_fixed");
  int rc = validate(s);
  if (rc) return rc;
  if (!q_in || !q_out || !stage || !dt || !s->acc || !s->control || !s->report || !s->averages || !s->element_aux)
    return fail(CFD_E_ARG, "cfd_rk3_step_fixed: null pointer");
  if (q_in == q_out || q_in == stage || q_out == stage) return fail(CFD_E_ARG, "cfd_rk3_step_fixed: state buffers must be distinct");
  cudaStream_t st = (cudaStream_t)stream;
  const int n = s->mesh.num_instances, ld = s->mesh.ld, prec = s->precision;
  fixed_control_kernel<<<blocks_for(n, 128), 128, 0, st>>>(s->control, dt, n);
  reset_acc(s, st);
  // with a tape, the tiled stage kernel writes its input tile and its result
  // into the tape as it goes (the register-only pair kernel cannot copy its
  // input), and the averages / minima / positivity theta land there directly
  CfdSolver sv = *s;
  if (tape && sv.variant == 2) sv.variant = 0;
  for (int k = 1; k <= 3; ++k) {
    StageParams p;
    memset(&p, 0, sizeof(p));
    p.m = s->mesh;
    p.ctl = s->control;
    p.x0 = q_in;
    p.x1 = q_out;
    p.stage = stage;
    p.stage_idx = k;
    p.gamma = s->gamma;
    p.avg = tape ? tape_avg(tape, ld, prec, k) : s->averages;
    p.aux = tape ? tape_aux(tape, ld, prec, k) : s->element_aux;
    p.acc = s->acc;
    if (tape) {
      p.tape_dst = tape_state(tape, ld, prec, 2 * (k - 1));
      p.tape_src = k >= 2 ? tape_state(tape, ld, prec, 2 * k - 3) : nullptr;
    }
    // the limited path for every limiter: positivity runs in limit_kernel on
    // the stored stage state, so the tape sees the state before limiting
    launch_stage(&sv, p, MODE_LIMITED, st);
    LimitParams lp;
    memset(&lp, 0, sizeof(lp));
    lp.m = s->mesh;
    lp.ctl = s->control;
    lp.x0 = q_in;
    lp.x1 = q_out;
    lp.stage = stage;
    lp.stage_idx = k;
    lp.gamma = s->gamma;
    lp.avg = p.avg;
    lp.aux = p.aux;
    lp.acc = s->acc;
    lp.pos_out = tape ? tape_pos(tape, ld, prec, k) : nullptr;
    lp.flags = s->troubled_flags ? s->troubled_flags + (size_t)(k - 1) * ld : nullptr;
    launch_limit(s, lp, st);
  }
  report_kernel<<<blocks_for(n, 128), 128, 0, st>>>(s->acc, s->control, s->report, n, s->cfl);
  return check_launch("cfd_rk3_step_fixed");
}

int cfd_rk3_step_adjoint(const CfdSolver* s, const void* q_in, const void* tape, const double* dt, const void* g_out,
                         void* g_in, double* bc_bar, int32_t flags, void* work, void* stream) {
  NvtxRange nvtx_range("cfd_rk3_step_adjoint");
  int rc = validate(s);
  if (rc) return rc;
  if (!q_in || !tape || !dt || !g_out || !g_in || !work) return fail(CFD_E_ARG, "cfd_rk3_step_adjoint: null pointer");
  if (g_out == g_in) return fail(CFD_E_ARG, "cfd_rk3_step_adjoint: g_in must not alias g_out");
  cudaStream_t st = (cudaStream_t)stream;
  const int ld = s->mesh.ld, prec = s->precision;
  const size_t sb = state_bytes(ld, prec), es = prec == CFD_FP64 ? 8 : 4;
  char* wk = (char*)work;
  void* qtb = wk;
  void* w = wk + sb;
  void* nab = wk + 2 * sb;
  void* b1 = wk + 2 * sb + (size_t)12 * ld * es;  // adjoint of q1
  void* b2 = (char*)b1 + sb;                      // adjoint of q2
  int* list = (int*)(wk + adjoint_reals_bytes(ld, prec));
  int* count = (int*)(wk + adjoint_reals_bytes(ld, prec) + (size_t)4 * ld);
  uint8_t* listed = (uint8_t*)(wk + adjoint_reals_bytes(ld, prec) + (size_t)4 * ld + 256);
  void* tp = const_cast<void*>(tape);
  if (cudaMemsetAsync(g_in, 0, sb, st) != cudaSuccess) return check_launch("cfd_rk3_step_adjoint: memset");
  const int n = s->mesh.num_elements;
  static const double A[4] = {0.0, 0.0, 0.75, 1.0 / 3.0}, B[4] = {0.0, 1.0, 0.25, 2.0 / 3.0};
  for (int k = 3; k >= 1; --k) {
    AdjParams p;
    memset(&p, 0, sizeof(p));
    p.m = s->mesh;
    p.gamma = s->gamma;
    p.dt = dt;
    p.qt = tape_state(tp, ld, prec, 2 * (k - 1));
    p.avg = tape_avg(tp, ld, prec, k);
    p.aux = tape_aux(tp, ld, prec, k);
    p.pos = tape_pos(tp, ld, prec, k);
    p.qs = k == 1 ? q_in : tape_state(tp, ld, prec, 2 * k - 3);
    p.g = k == 3 ? g_out : (k == 2 ? b2 : b1);
    p.qtb = qtb;
    p.w = w;
    p.nab = nab;
    p.src_bar = k == 3 ? b2 : (k == 2 ? b1 : g_in);
    p.base_bar = k == 1 ? nullptr : g_in;
    p.bc_bar = bc_bar;
    p.a = A[k];
    p.b = B[k];
    p.accumulate_src = k == 1;
    p.limited = s->limiter != CFD_LIMITER_UNLIMITED;
    p.hold_theta = (flags & CFD_ADJ_HOLD_THETA) != 0;
    p.list = list;
    p.count = count;
    p.listed = listed;
    if (cudaMemsetAsync(count, 0, sizeof(int), st) != cudaSuccess) return check_launch("cfd_rk3_step_adjoint: memset");
    if (prec == CFD_FP64) {
      launch_adj_limit<double>(p, s->limiter, n, st);
      launch_adj_rhs<double>(p, s->flux, n, st);
    } else {
      launch_adj_limit<float>(p, s->limiter, n, st);
      launch_adj_rhs<float>(p, s->flux, n, st);
    }
  }
  return check_launch("cfd_rk3_step_adjoint");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free RK3 step (no counterpart in the reference).
//
// For callers that cannot allocate device memory themselves: a foreign-language
// binding that holds only the pointers it was given and has no CUDA allocator,
// or an application whose memory pool must not see outside cudaMalloc calls
// once it has started. All scratch of one step lives in the file-scope array
// below, which every GPU that loads this library keeps until process exit.
// ---------------------------------------------------------------------------
constexpr size_t NOALLOC_LD_MAX = CFD_NOALLOC_MAX_ELEMENTS;  // leading-dimension bound (elements)
constexpr size_t NOALLOC_STAGE_BYTES = sizeof(double) * 60 * NOALLOC_LD_MAX;  // stage state (f64 or f32)
constexpr size_t NOALLOC_AVG_BYTES = sizeof(double) * 4 * NOALLOC_LD_MAX;     // stage cell averages
constexpr size_t NOALLOC_AUX_BYTES = sizeof(double) * 3 * NOALLOC_LD_MAX;     // per-element minima, wave speed
constexpr size_t NOALLOC_SMALL_BYTES = 1024;  // reduction slots, report, loop state (256-aligned pieces)
constexpr size_t NOALLOC_BYTES = NOALLOC_STAGE_BYTES + NOALLOC_AVG_BYTES + NOALLOC_AUX_BYTES + NOALLOC_SMALL_BYTES;
static_assert(3 * sizeof(CfdStageAcc) <= 256 && sizeof(CfdStepReport) <= 256 && sizeof(CfdControl) <= 256,
              "scratch layout of the allocation-free step");

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
// Device address of g_noalloc_scratch, per device, looked up on the first call
// on that device under a lock (host threads making their first calls at once
// would otherwise race on the cache). A cudaDeviceReset in the same process
// invalidates the address; the cache does not notice, so a process that resets
// a device must not call the allocation-free step on it again.
std::atomic<unsigned char*> g_noalloc_ptr[NOALLOC_MAX_DEVICES];
std::mutex g_noalloc_lock;
}  // namespace

__global__ void noalloc_control_kernel(CfdControl* ctl, double dt) {
  CfdControl c;
  memset(&c, 0, sizeof(c));
  c.final_time = INFINITY;
  c.dt = dt;
  c.status = CFD_RUN_ACTIVE;
  *ctl = c;
}

__global__ void noalloc_report_kernel(const CfdStepReport* src, CfdStepReport* dst) { *dst = *src; }

extern "C" int cfd_rk3_step_noalloc(const CfdMesh* mesh, int32_t flux, int32_t limiter, int32_t precision, double gamma,
                                    double cfl, const void* q_in, void* q_out, double dt, CfdStepReport* report,
                                    void* stream) {
  if (!mesh || !q_in || !q_out || !report) return fail(CFD_E_ARG, "cfd_rk3_step_noalloc: null pointer");
  if (q_in == q_out) return fail(CFD_E_ARG, "cfd_rk3_step_noalloc: q_out must not alias q_in");
  if (mesh->num_instances != 1 || mesh->instance)
    return fail(CFD_E_ARG, "cfd_rk3_step_noalloc: one mesh instance only");
  if (mesh->ld < 0 || (size_t)mesh->ld > NOALLOC_LD_MAX) {
    snprintf(g_err, sizeof(g_err),
             "cfd_rk3_step_noalloc: mesh leading dimension %d exceeds the static scratch limit of %d elements",
             (int)mesh->ld, (int)NOALLOC_LD_MAX);
    return CFD_E_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("cfd_rk3_step_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(CFD_E_ARG, "cfd_rk3_step_noalloc: device index out of range");
  // Once per device, with that device current: the device address of the
  // static array (its host-side name is only a stand-in for it).
  unsigned char* base = g_noalloc_ptr[dev].load(std::memory_order_acquire);
  if (!base) {
    std::lock_guard<std::mutex> guard(g_noalloc_lock);
    base = g_noalloc_ptr[dev].load(std::memory_order_relaxed);
    if (!base) {
      void* ptr = nullptr;
      const cudaError_t rc = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (rc != cudaSuccess || !ptr) {
        snprintf(g_err, sizeof(g_err), "cfd_rk3_step_noalloc: cudaGetSymbolAddress failed: %s",
                 cudaGetErrorString(rc));
        return CFD_E_CUDA;
      }
      base = (unsigned char*)ptr;
      g_noalloc_ptr[dev].store(base, std::memory_order_release);
    }
  }
  CfdSolver s;
  memset(&s, 0, sizeof(s));
  s.mesh = *mesh;
  s.flux = flux;
  s.limiter = limiter;
  s.precision = precision;
  s.max_rejections = 0;
  s.gamma = gamma;
  s.cfl = cfl;
  void* stage = base;
  s.averages = (double*)(base + NOALLOC_STAGE_BYTES);
  s.element_aux = (double*)(base + NOALLOC_STAGE_BYTES + NOALLOC_AVG_BYTES);
  unsigned char* small = base + NOALLOC_STAGE_BYTES + NOALLOC_AVG_BYTES + NOALLOC_AUX_BYTES;
  s.acc = (CfdStageAcc*)small;
  s.report = (CfdStepReport*)(small + 256);
  s.control = (CfdControl*)(small + 512);
  s.block_size = 0;
  int rc = validate(&s);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // The loop state is written fresh on every call; the reduction slots are
  // zeroed by the attempt itself; averages and aux are written before read.
  noalloc_control_kernel<<<1, 1, 0, st>>>(s.control, dt);
  if ((rc = check_launch("cfd_rk3_step_noalloc"))) return rc;
  if ((rc = cfd_rk3_attempt(&s, const_cast<void*>(q_in), q_out, stage, stream))) return rc;
  noalloc_report_kernel<<<1, 1, 0, st>>>(s.report, report);
  return check_launch("cfd_rk3_step_noalloc");
}
