// common.cuh — device code shared by every object of libcfd_b200.so: the
// physics, reductions, positivity scaling and the fused stage kernels, plus the
// host templates that launch a stage kernel. The stage kernels' many template
// instantiations (precision x mode x flux x shape) are compiled in six objects
// (stage_inst.cu, one per precision and mode) beside kernels.cu, which holds
// the limiter, adjoint and small kernels and the C ABI.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <mutex>

#include "cfd_b200.h"
#include "physics.cuh"
#include "tables.cuh"

namespace cfd {

constexpr int NP = 15;
constexpr int NFP = 5;
constexpr double NEIGHBOR_FACTOR = 1.5;      // limiting.py:22
constexpr double DETECTION_TOLERANCE = 1e-10; // limiting.py:24
// FP32-mixed form: the troubled-cell test compares with ~100 single-precision
// ulps of the average (1e-10 lies far below the state's own round-off there)
constexpr double DETECTION_TOLERANCE_FP32 = 1e-5;
constexpr double POSITIVITY_FLOOR = 1e-13;    // limiting.py:28
constexpr int BISECTION_STEPS = 60;           // limiting.py:29

enum { MODE_RHS = 0, MODE_LIMITED = 1, MODE_UNLIMITED = 2 };
// CfdSolver.limit_list: [LIMIT_LIST_HEADER] counters (index = RK stage, 0 for
// cfd_limit), then the element list
constexpr int LIMIT_LIST_HEADER = CFD_LIMIT_LIST_HEADER;
// bits 0-1 decide admissibility; bit 2 marks a NaN CFL step (time_step -> NaN)
enum { FLAG_NONFINITE = 1, FLAG_BAD_AVERAGE = 2, FLAG_NAN_DT = 4, FLAG_ADMISSIBILITY = 3 };

// ---------------------------------------------------------------- helpers ---
// Monotone map double -> uint64 so that unsigned integer order equals float order.
__device__ __forceinline__ unsigned long long dkey(double x) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ __forceinline__ double dkey_decode(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double d;
  memcpy(&d, &b, sizeof(d));
  return d;
}
constexpr unsigned long long KEY_EMPTY = ~0ull;

__device__ __forceinline__ bool finite_(double x) { return isfinite(x); }
__device__ __forceinline__ bool finite_(float x) { return isfinite(x); }

// Face node k of face f, packed 4 bits per entry (tab::FACE_NODES_PACKED).
constexpr unsigned long long FN_PACK = tab::FACE_NODES_PACKED;

// FP32 form: skip the [Dr|Ds] entries that are round-off zeros of the
// construction (|D| < 1e-13: 65 of 225 per matrix). The FP64 form keeps all.
template <typename R> __host__ __device__ constexpr bool keep_entry(double v) {
  return sizeof(R) == 8 ? true : (v > 1e-13 || v < -1e-13);
}
__device__ __forceinline__ int face_node_rt(int f, int k) { return (int)((FN_PACK >> (4 * (f * NFP + k))) & 15ull); }


template <typename R> struct GeoPtr;
template <> struct GeoPtr<double> {
  static __device__ __forceinline__ const double* metric(const CfdMesh& m) { return m.metric; }
  static __device__ __forceinline__ const double* face(const CfdMesh& m) { return m.face_geo; }
  static __device__ __forceinline__ const double* cs(const CfdMesh& m) { return m.cs_coef; }
};
template <> struct GeoPtr<float> {
  static __device__ __forceinline__ const float* metric(const CfdMesh& m) { return m.metric32; }
  static __device__ __forceinline__ const float* face(const CfdMesh& m) { return m.face_geo32; }
  static __device__ __forceinline__ const float* cs(const CfdMesh& m) { return m.cs_coef32; }
};

// Per-thread contribution to the per-instance stage reductions.
struct Red {
  double b[4];
  unsigned long long kr, kp, kd;
  int tr, fl;
  __device__ void init() {
    b[0] = b[1] = b[2] = b[3] = 0.0;
    kr = kp = kd = KEY_EMPTY;
    tr = 0;
    fl = 0;
  }
};

// Appends e to list[] where flag is set, with one atomic per warp on the
// shared counter (when a large share of the elements is listed, per-thread
// atomics on one address serialise). All 32 lanes of the warp must call it.
__device__ __forceinline__ void warp_list_append(int* list, int* count, bool flag, int e) {
  const unsigned mask = __ballot_sync(0xffffffffu, flag);
  if (!mask) return;
  const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(count, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (flag) list[base + __popc(mask & ((1u << lane) - 1u))] = e;
}

__device__ __forceinline__ void commit_one(const Red& r, CfdStageAcc* a) {
#pragma unroll
  for (int c = 0; c < 4; ++c)
    if (r.b[c] != 0.0) atomicAdd(&a->boundary_flux[c], r.b[c]);
  if (r.kr != KEY_EMPTY) atomicMin(&a->min_rho_key, r.kr);
  if (r.kp != KEY_EMPTY) atomicMin(&a->min_p_key, r.kp);
  if (r.kd != KEY_EMPTY) atomicMin(&a->dt_key, r.kd);
  if (r.tr) atomicAdd(&a->troubled, r.tr);
  if (r.fl) atomicOr(&a->flags, r.fl);
}

// Reduce over the block and commit with one set of atomics when every live
// thread belongs to the same instance (else each thread commits its own).
// `slot(inst)` -> CfdStageAcc*. All threads of the block must call this.
template <int BS>
__device__ __forceinline__ void block_commit(Red r, bool live, int inst, CfdStageAcc* acc, int stride, int offset) {
  __shared__ int s_inst;
  __shared__ double s_b[BS / 32][4];
  __shared__ unsigned long long s_k[BS / 32][3];
  __shared__ int s_i[BS / 32][2];
  if (threadIdx.x == 0) s_inst = live ? inst : -1;
  __syncthreads();
  const int inst0 = s_inst;
  const bool uniform = __syncthreads_and(!live || inst == inst0) && inst0 >= 0;
  if (!uniform) {
    if (live) commit_one(r, acc + inst * stride + offset);
    return;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int c = 0; c < 4; ++c) r.b[c] += __shfl_xor_sync(0xffffffffu, r.b[c], o);
    r.kr = min(r.kr, __shfl_xor_sync(0xffffffffu, r.kr, o));
    r.kp = min(r.kp, __shfl_xor_sync(0xffffffffu, r.kp, o));
    r.kd = min(r.kd, __shfl_xor_sync(0xffffffffu, r.kd, o));
    r.tr += __shfl_xor_sync(0xffffffffu, r.tr, o);
    r.fl |= __shfl_xor_sync(0xffffffffu, r.fl, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
#pragma unroll
    for (int c = 0; c < 4; ++c) s_b[w][c] = r.b[c];
    s_k[w][0] = r.kr;
    s_k[w][1] = r.kp;
    s_k[w][2] = r.kd;
    s_i[w][0] = r.tr;
    s_i[w][1] = r.fl;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    Red t;
    t.init();
    for (int i = 0; i < BS / 32; ++i) {
      for (int c = 0; c < 4; ++c) t.b[c] += s_b[i][c];
      t.kr = min(t.kr, s_k[i][0]);
      t.kp = min(t.kp, s_k[i][1]);
      t.kd = min(t.kd, s_k[i][2]);
      t.tr += s_i[i][0];
      t.fl |= s_i[i][1];
    }
    commit_one(t, acc + inst0 * stride + offset);
  }
}

// Pressure in double of a (possibly float) state: fast form (reciprocal,
// contracted) and the reference's exact operation order (euler.py:21-27).
__device__ __forceinline__ double pressure_d(double q0, double q1, double q2, double q3, double gm1) {
  const double ir = __drcp_rn(q0);
  return gm1 * (q3 - 0.5 * (q1 * (q1 * ir) + q2 * (q2 * ir)));
}
__device__ __forceinline__ double pressure_x(double q0, double q1, double q2, double q3, double gm1) {
  return xmul(gm1, xsub(q3, xmul(0.5, xadd(xmul(q1, xdiv(q1, q0)), xmul(q2, xdiv(q2, q0))))));
}
// The fast form, replaced by the exact one wherever the two could fall on
// different sides of `bound` (they differ by a few ulps of |E| + |m.u|).
__device__ __forceinline__ double pressure_near(double q0, double q1, double q2, double q3, double gm1, double bound) {
  const double ir = __drcp_rn(q0);
  const double k = 0.5 * (q1 * (q1 * ir) + q2 * (q2 * ir));
  const double p = gm1 * (q3 - k);
  const double margin = 1e-13 * (fabs(q3) + fabs(k)) + 1e-300;
  return (p - bound > margin || p != p) ? p : pressure_x(q0, q1, q2, q3, gm1);
}

// Constant-bank operator tables in the arithmetic type (warp-uniform index).
template <typename R> struct tabv;
template <> struct tabv<double> {
  static __device__ __forceinline__ double dr(int i, int j) { return ctab::DR[i][j]; }
  static __device__ __forceinline__ double ds(int i, int j) { return ctab::DS[i][j]; }
  static __device__ __forceinline__ double lift(int i, int j) { return ctab::LIFT[i][j]; }
};
template <> struct tabv<float> {
  static __device__ __forceinline__ float dr(int i, int j) { return ctab::DR32[i][j]; }
  static __device__ __forceinline__ float ds(int i, int j) { return ctab::DS32[i][j]; }
  static __device__ __forceinline__ float lift(int i, int j) { return ctab::LIFT32[i][j]; }
};

// |u| + c of a node (time_integration.py:39-40). The plain form follows the
// reference's operation order exactly (divisions, unfused), so the CFL step
// of a given state is the reference's to the last bit.
template <typename R>
__device__ __forceinline__ double wave_speed(R q0, R q1, R q2, R q3, double gamma) {
  if (sizeof(R) == 8) {
    const double u = xdiv(q1, q0), v = xdiv(q2, q0);
    const double p = xmul(gamma - 1.0, xsub(q3, xmul(0.5, xadd(xmul(q1, u), xmul(q2, v)))));
    return xadd(__dsqrt_rn(xadd(xmul(u, u), xmul(v, v))), __dsqrt_rn(xdiv(xmul(gamma, p), q0)));
  }
  // FP32 form: single precision, except that a pressure lost to cancellation
  // (near vacuum) is recovered in double before the sound speed is taken
  const float ir = rcp<float>((float)q0);
  const float u = (float)q1 * ir, v = (float)q2 * ir;
  const float kin = 0.5f * ((float)q1 * u + (float)q2 * v);
  float p = (float)(gamma - 1.0) * ((float)q3 - kin);
  if (!(p > 1e-4f * (fabsf((float)q3) + kin)))
    p = (float)pressure_x((double)q0, (double)q1, (double)q2, (double)q3, gamma - 1.0);
  return (double)(sqrt_<float>(u * u + v * v) + sqrt_<float>((float)gamma * p * ir));
}

// Exact-order pressure of a node for the positivity test and the minima:
// the fast form unless it lies within rounding of `bound`.
template <typename R>
__device__ __forceinline__ double node_pressure(R q0, R q1, R q2, R q3, double gm1, double bound) {
  if (sizeof(R) == 8) return pressure_near(q0, q1, q2, q3, gm1, bound);
  const float ir = __frcp_rn((float)q0);
  const float k = 0.5f * ((float)q1 * ((float)q1 * ir) + (float)q2 * ((float)q2 * ir));
  const float p = (float)gm1 * ((float)q3 - k);
  const float margin = 1e-5f * (fabsf((float)q3) + fabsf(k));
  return ((double)p - bound > (double)margin || p != p) ? (double)p : pressure_x(q0, q1, q2, q3, gm1);
}

// Pressure target of the positivity limiter: the reference's eps
// (limiting.py:173-176) in the plain form; in the FP32-mixed form eps plus a
// margin covering the rounding of the repaired state to single precision
// (|dp| <= ~2e-7 (gamma-1) |E|), capped at half the average pressure so that
// the average itself stays admissible.
template <typename R>
__device__ __forceinline__ double pressure_target(double eps, double pa, double e_avg, double gm1) {
  if (sizeof(R) == 8) return eps;
  return eps + jmin(2e-6 * gm1 * fabs(e_avg), 0.5 * pa);
}

// Cell average in double, sequential and unfused like NumPy's einsum
// (limiting.py:209, dg.py:168-171).
template <typename R>
__device__ __forceinline__ void cell_average(const R (&q)[NP][4], double a[4]) {
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    double s = xmul(tab::AVG_W[0], (double)q[0][c]);
#pragma unroll
    for (int i = 1; i < NP; ++i) s = xadd(s, xmul(tab::AVG_W[i], (double)q[i][c]));
    a[c] = s;
  }
}

// Zhang-Shu positivity scaling of one element toward its average, in double
// and in the reference's operation order (limiting.py:166-200). q is the
// element's nodal state in registers. Returns true if q changed.
template <typename R>
__device__ __forceinline__ bool positivity(R (&q)[NP][4], const double a[4], double gm1, double* theta_out = nullptr,
                                           int* node_out = nullptr) {
  const double pa = pressure_x(a[0], a[1], a[2], a[3], gm1);
  const double eps = jmin(POSITIVITY_FLOOR, jmin(a[0], pa));
  const double pt = pressure_target<R>(eps, pa, a[3], gm1);
  double rmin = (double)q[0][0];
#pragma unroll
  for (int i = 1; i < NP; ++i) rmin = jmin(rmin, (double)q[i][0]);
  bool changed = false;
  if (rmin < eps) {
    const double span = xsub(a[0], rmin);
    const double theta = jmin(jmax(xdiv(xsub(a[0], eps), span), 0.0), 1.0);
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c) q[i][c] = (R)xadd(a[c], xmul(theta, xsub((double)q[i][c], a[c])));
    changed = true;
  }
  unsigned need = 0;
#pragma unroll
  for (int i = 0; i < NP; ++i)
    if (pressure_near(q[i][0], q[i][1], q[i][2], q[i][3], gm1, pt) < pt) need |= 1u << i;
  if (theta_out) {
    *theta_out = 1.0;
    *node_out = -1;
  }
  if (!need) return changed;
  double theta = 1.0;
#pragma unroll 1
  for (int i = 0; i < NP; ++i) {
    if (!((need >> i) & 1u)) continue;
    double qi[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      // select node i without dynamic register indexing
      double v = 0.0;
#pragma unroll
      for (int j = 0; j < NP; ++j) v = (j == i) ? (double)q[j][c] : v;
      qi[c] = v;
    }
    const double d0 = xsub(qi[0], a[0]), d1 = xsub(qi[1], a[1]), d2 = xsub(qi[2], a[2]), d3 = xsub(qi[3], a[3]);
    double lo = 0.0, hi = 1.0;
#pragma unroll 1
    for (int it = 0; it < BISECTION_STEPS; ++it) {
      const double mid = xmul(0.5, xadd(lo, hi));
      const bool ok = pressure_x(xadd(a[0], xmul(mid, d0)), xadd(a[1], xmul(mid, d1)), xadd(a[2], xmul(mid, d2)),
                                 xadd(a[3], xmul(mid, d3)), gm1) >= pt;
      lo = ok ? mid : lo;
      hi = ok ? hi : mid;
    }
    if (theta_out && lo < theta) *node_out = i;
    theta = jmin(theta, lo);
  }
  if (theta_out) *theta_out = theta;
  if (theta < 1.0) {
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c) q[i][c] = (R)xadd(a[c], xmul(theta, xsub((double)q[i][c], a[c])));
    changed = true;
  }
  return changed;
}

// Nodal minima (density, pressure; NaN ignored), max wave speed and finiteness.
template <typename R>
__device__ __forceinline__ void element_stats(const R (&q)[NP][4], double gm1, double gamma, double& rmin, double& pmin,
                                              double& lam, bool& finite) {
  rmin = INFINITY;
  pmin = INFINITY;
  lam = -INFINITY;
  finite = true;
  bool lam_nan = false;
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    const double r = q[i][0], mx = q[i][1], my = q[i][2], en = q[i][3];
    const double p = node_pressure<R>(q[i][0], q[i][1], q[i][2], q[i][3], gm1, POSITIVITY_FLOOR);
    rmin = fmin(rmin, r);
    pmin = fmin(pmin, p);
    // time_integration.py:39-40: |u| + c
    const double s = wave_speed<R>(q[i][0], q[i][1], q[i][2], q[i][3], gamma);
    lam_nan |= (s != s);
    lam = fmax(lam, s);
#pragma unroll
    for (int c = 0; c < 4; ++c) finite &= finite_(q[i][c]);
  }
  if (lam_nan) lam = NAN;
}


// One face node of the surface term: exterior state, interface flux, lifted
// jump, boundary-flux contribution (dg.py:153-164, boundary: dg.py:119-137).
template <typename R, int FLUX>
__device__ __forceinline__ void face_node_flux(const CfdMesh& m, const R* __restrict__ src, int e, int ld, R gamma,
                                               int n, int kind, int nb, int pn, R nx, R ny, R fs, double bw,
                                               R jump[4], Red& red) {
  R qm[4], qp[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) qm[c] = src[(c * NP + n) * ld + e];
  if (kind == CFD_FACE_INTERIOR) {
#pragma unroll
    for (int c = 0; c < 4; ++c) qp[c] = src[(c * NP + pn) * ld + nb];
  } else if (kind == CFD_FACE_SLIP_WALL) {
    const R mn = qm[1] * nx + qm[2] * ny;
    qp[0] = qm[0];
    qp[1] = qm[1] - R(2) * mn * nx;
    qp[2] = qm[2] - R(2) * mn * ny;
    qp[3] = qm[3];
  } else {
#pragma unroll
    for (int c = 0; c < 4; ++c) qp[c] = (R)m.bc_states[nb * 4 + c];
  }
  R fhat[4], fm[4];
  trace_flux<R, FLUX>(qm, qp, nx, ny, gamma, fhat, fm);
#pragma unroll
  for (int c = 0; c < 4; ++c) jump[c] = fs * (fm[c] - fhat[c]);
  if (kind != CFD_FACE_INTERIOR) {
#pragma unroll
    for (int c = 0; c < 4; ++c) red.b[c] += bw * (double)fhat[c];
  }
}

// ----------------------------------------------------------- stage kernel ---
struct StageParams {
  CfdMesh m;
  const CfdControl* ctl;
  const void* x0;
  const void* x1;
  void* stage;
  int stage_idx;  // 1..3; 0 = rhs only
  double gamma;
  double* avg;
  double* aux;
  CfdStageAcc* acc;
  const void* q_in;  // MODE_RHS
  void* q_out;       // MODE_RHS
  double* bflux_out; // MODE_RHS, [instances][4]
  void* tape_src;    // optional: copy of the stage input written here (tiled kernels)
  void* tape_dst;    // optional: second copy of the stage result (before limiting)
};

template <typename R>
__device__ __forceinline__ void select_buffers(const StageParams& P, int par, const R*& src, const R*& base, R*& dst) {
  const R* cur = (const R*)(par ? P.x1 : P.x0);
  R* nxt = (R*)(par ? P.x0 : P.x1);
  if (P.stage_idx == 1) {
    src = cur;
    base = nullptr;
    dst = nxt;
  } else if (P.stage_idx == 2) {
    src = nxt;
    base = cur;
    dst = (R*)P.stage;
  } else {
    src = (const R*)P.stage;
    base = cur;
    dst = nxt;
  }
}

// SSP-RK3 third stage q = q_n / 3 + 2 (q_2 + dt L(q_2)) / 3 with v = q_2 +
// dt L(q_2) (time_integration.py:64-66). The plain form evaluates it as the
// reference does. In single precision float(1/3) + float(2/3) = 1 + 3e-8,
// which would scale the whole state by that factor every step (a steady
// drift of mass and energy), so the FP32 form uses q_n + (2/3)(v - q_n),
// whose weights sum to one exactly.
template <typename R>
__device__ __forceinline__ R stage3_combine(R b, R v) {
  if (sizeof(R) == 8) return b * (R)(1.0 / 3.0) + (R)(2.0 / 3.0) * v;
  return fma((R)(2.0 / 3.0), v - b, b);
}

#include "stage_pair.cuh"
#include "stage_tile.cuh"
#include "limiter.cuh"
#include "control.cuh"
#include "batch.cuh"

inline unsigned blocks_for(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// Records `msg` as the calling thread's last error (cfd_last_error) and
// returns `code`; defined in kernels.cu.
int cfd_fail(int code, const char* msg);

// ---------------------------------------------------- stage-kernel launches ---
template <typename R, int FLUX, int MODE>
void launch_stage_bs(const StageParams& p, int bs, cudaStream_t st) {
  const unsigned g = blocks_for(p.m.num_elements, bs / 2);  // two threads per element
  if (bs == 64) stage_pair_kernel<R, FLUX, MODE, 64><<<g, 64, 0, st>>>(p);
  else if (bs == 256) stage_pair_kernel<R, FLUX, MODE, 256><<<g, 256, 0, st>>>(p);
  else stage_pair_kernel<R, FLUX, MODE, 128><<<g, 128, 0, st>>>(p);
}
template <typename R, int MODE>
void launch_stage_flux(const StageParams& p, int flux, int bs, cudaStream_t st) {
  if (flux == 0) launch_stage_bs<R, 0, MODE>(p, bs, st);
  else if (flux == 1) launch_stage_bs<R, 1, MODE>(p, bs, st);
  else launch_stage_bs<R, 2, MODE>(p, bs, st);
}
template <typename R, int FLUX, int MODE, int EPB, bool SB, int MINB = (sizeof(R) == 4 ? 512 : 384) / (2 * EPB),
          bool UF = true, bool PK = true, bool CF = false, bool FJ = false, bool VR = false>
void launch_tile(const StageParams& p, cudaStream_t st) {
  using L = TileLayout<R, EPB, SB, FJ>;
  constexpr bool PACK = PK && sizeof(R) == 4;  // FP64 shares the unpacked instantiation
  constexpr bool CALL = CF && sizeof(R) == 4;
  // opt in to > 48 KB of dynamic shared memory, once per instantiation and
  // device (the attribute belongs to the device's context); setting it twice
  // is harmless, so concurrent first calls need no lock
  constexpr int MAX_DEV = 64;
  static bool configured[MAX_DEV] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= MAX_DEV || !configured[dev]) {
    cudaFuncSetAttribute(stage_tile_kernel<R, FLUX, MODE, EPB, SB, MINB, UF, PACK, CALL, FJ, VR>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, L::BYTES);
    if (dev >= 0 && dev < MAX_DEV) configured[dev] = true;
  }
  const unsigned g = blocks_for(p.m.num_elements, EPB);
  stage_tile_kernel<R, FLUX, MODE, EPB, SB, MINB, UF, PACK, CALL, FJ, VR><<<g, 2 * EPB, L::BYTES, st>>>(p);
}
template <typename R, int FLUX, int MODE>
void launch_stage_variant(const StageParams& p, int variant, int bs, cudaStream_t st) {
  if (variant == 2) launch_stage_bs<R, FLUX, MODE>(p, bs, st);
  else if (variant == 1) launch_tile<R, FLUX, MODE, 32, true>(p, st);
  else if (variant == 3) launch_tile<R, FLUX, MODE, 64, false>(p, st);
  else if (variant == 4) launch_tile<R, FLUX, MODE, 32, false, sizeof(R) == 4 ? 10 : 8>(p, st);
  else if (variant == 5) launch_tile<R, FLUX, MODE, 64, false, (sizeof(R) == 4 ? 512 : 384) / 128, false>(p, st);
  // 6 / 7: variants 3 / 5 with scalar FMAs in the contractions (the bitwise reference of the packed form)
  else if (variant == 6) launch_tile<R, FLUX, MODE, 64, false, (sizeof(R) == 4 ? 512 : 384) / 128, true, false>(p, st);
  else if (variant == 7) launch_tile<R, FLUX, MODE, 64, false, (sizeof(R) == 4 ? 512 : 384) / 128, false, false>(p, st);
  else if (variant == 8) launch_tile<R, FLUX, MODE, 64, true>(p, st);
  else if (variant == 9) launch_tile<R, FLUX, MODE, 64, true, (sizeof(R) == 4 ? 512 : 384) / 128, true, true, true>(p, st);
  // 10 / 11: the face-job form (each face's flux once for both sides), without / with staged base rows
  else if (variant == 10)
    launch_tile<R, FLUX, MODE, 64, false, (sizeof(R) == 4 ? 512 : 384) / 128, true, true, true, true>(p, st);
  else if (variant == 11) launch_tile<R, FLUX, MODE, 64, true, sizeof(R) == 4 ? 3 : 2, true, true, true, true>(p, st);
  // 12 / 13: variant 9 with the volume node loop kept rolled, with unrolled / rolled face rounds;
  // 14: variant 5 with the volume node loop kept rolled (smaller code)
  else if (variant == 12)
    launch_tile<R, FLUX, MODE, 64, true, (sizeof(R) == 4 ? 512 : 384) / 128, true, true, true, false, true>(p, st);
  else if (variant == 13)
    launch_tile<R, FLUX, MODE, 64, true, (sizeof(R) == 4 ? 512 : 384) / 128, false, true, true, false, true>(p, st);
  else if (variant == 14)
    launch_tile<R, FLUX, MODE, 64, false, (sizeof(R) == 4 ? 512 : 384) / 128, false, true, false, false, true>(p, st);
  else launch_tile<R, FLUX, MODE, 32, false>(p, st);
}
// One precision and mode of the stage kernels, every flux and shape; each
// combination is instantiated in its own object (stage_inst.cu).
template <typename R, int MODE>
void launch_stage_part(const StageParams& p, int flux, int variant, int bs, cudaStream_t st) {
  if (flux == 0) launch_stage_variant<R, 0, MODE>(p, variant, bs, st);
  else if (flux == 1) launch_stage_variant<R, 1, MODE>(p, variant, bs, st);
  else launch_stage_variant<R, 2, MODE>(p, variant, bs, st);
}
#define CFD_DECLARE_STAGE_PART(R, MODE) \
  extern template void launch_stage_part<R, MODE>(const StageParams&, int, int, int, cudaStream_t);
CFD_DECLARE_STAGE_PART(double, MODE_RHS)
CFD_DECLARE_STAGE_PART(double, MODE_LIMITED)
CFD_DECLARE_STAGE_PART(double, MODE_UNLIMITED)
CFD_DECLARE_STAGE_PART(float, MODE_RHS)
CFD_DECLARE_STAGE_PART(float, MODE_LIMITED)
CFD_DECLARE_STAGE_PART(float, MODE_UNLIMITED)

}  // namespace cfd
