// physics.cuh — pointwise Euler physics shared by every kernel (device code).
//
// Formulas follow CFD-demo (paths relative to its project root):
//   conserved_to_primitive / normal_flux   src/cfd_demo/euler.py:21-61
//   rusanov / roe / hllc                   src/cfd_demo/fluxes.py:28-143
//   phi(r) limiter functions               src/cfd_demo/limiters.py:16-39
// Templated on the arithmetic type R (double for the plain form, float for the
// mixed form). jmin/jmax propagate NaN like jax.numpy.minimum/maximum (CUDA's
// fmin/fmax would drop it), so the non-finite cases take the same branches as
// the reference. 1/rho is formed once and multiplied (the reference divides
// twice): results differ from the reference by at most an ulp or two.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace cfd {

template <typename R> __device__ __forceinline__ R jmax(R a, R b) {
  return (a != a || b != b) ? (a + b) : (a > b ? a : b);
}
template <typename R> __device__ __forceinline__ R jmin(R a, R b) {
  return (a != a || b != b) ? (a + b) : (a < b ? a : b);
}
template <typename R> __device__ __forceinline__ R rcp(R x);
template <> __device__ __forceinline__ double rcp<double>(double x) { return __drcp_rn(x); }
// FP32-mixed form: the SFU's approximate reciprocal / square root (PTX
// rcp.approx.ftz.f32 / sqrt.approx.ftz.f32, about 1 ulp) instead of the
// correctly rounded sequences; the plain FP64 form keeps IEEE operations.
template <> __device__ __forceinline__ float rcp<float>(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
template <typename R> __device__ __forceinline__ R sqrt_(R x);
template <> __device__ __forceinline__ double sqrt_<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float sqrt_<float>(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
template <typename R> __device__ __forceinline__ R div_(R a, R b) { return a / b; }
template <> __device__ __forceinline__ float div_<float>(float a, float b) { return a * rcp<float>(b); }
template <typename R> __device__ __forceinline__ R abs_(R x) { return x < R(0) ? -x : (x == R(0) ? R(0) : x); }
template <> __device__ __forceinline__ double abs_<double>(double x) { return fabs(x); }
template <> __device__ __forceinline__ float abs_<float>(float x) { return fabsf(x); }
// Unfused, correctly rounded arithmetic in the reference's (NumPy's) operation
// order, for the limiter decisions and the positivity scaling whose outcome can
// hinge on the last bit (an FMA would round once instead of twice).
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdiv_rn(a, b); }

// fluxes.py:24-25 — replace an exact zero by the smallest normal number.
template <typename R> __device__ __forceinline__ R nonzero(R x);
template <> __device__ __forceinline__ double nonzero<double>(double x) { return x == 0.0 ? 2.2250738585072014e-308 : x; }
template <> __device__ __forceinline__ float nonzero<float>(float x) { return x == 0.0f ? 1.17549435e-38f : x; }

template <typename R> struct Prim {
  R rho, u, v, p, inv_rho;
};

// euler.py:21-27
template <typename R>
__device__ __forceinline__ Prim<R> primitive(const R q[4], R gm1) {
  Prim<R> w;
  w.rho = q[0];
  w.inv_rho = rcp(q[0]);
  w.u = q[1] * w.inv_rho;
  w.v = q[2] * w.inv_rho;
  w.p = gm1 * (q[3] - R(0.5) * (q[1] * w.u + q[2] * w.v));
  return w;
}

template <typename R>
__device__ __forceinline__ R pressure(const R q[4], R gm1) {
  const R ir = rcp(q[0]);
  return gm1 * (q[3] - R(0.5) * (q[1] * (q[1] * ir) + q[2] * (q[2] * ir)));
}

// euler.py:35-37
template <typename R>
__device__ __forceinline__ R sound_speed(const Prim<R>& w, R gamma) {
  return sqrt_(gamma * w.p * w.inv_rho);
}

// euler.py:40-46 — Cartesian fluxes F (x) and G (y).
template <typename R>
__device__ __forceinline__ void cartesian(const R q[4], const Prim<R>& w, R f[4], R g[4]) {
  const R ep = q[3] + w.p;
  f[0] = q[1];
  f[1] = q[1] * w.u + w.p;
  f[2] = q[2] * w.u;
  f[3] = ep * w.u;
  g[0] = q[2];
  g[1] = q[1] * w.v;
  g[2] = q[2] * w.v + w.p;
  g[3] = ep * w.v;
}

// euler.py:49-61
template <typename R>
__device__ __forceinline__ void normal_flux(const R q[4], const Prim<R>& w, R nx, R ny, R f[4]) {
  const R un = w.u * nx + w.v * ny;
  f[0] = w.rho * un;
  f[1] = q[1] * un + w.p * nx;
  f[2] = q[2] * un + w.p * ny;
  f[3] = (q[3] + w.p) * un;
}

enum { FLUX_RUSANOV = 0, FLUX_ROE = 1, FLUX_HLLC = 2 };

// fluxes.py:28-37
template <typename R>
__device__ __forceinline__ void rusanov(const R qm[4], const R qp[4], const Prim<R>& wm, const Prim<R>& wp,
                                        R nx, R ny, R gamma, const R fm[4], const R fp[4], R out[4]) {
  const R sm = abs_(wm.u * nx + wm.v * ny) + sound_speed(wm, gamma);
  const R sp = abs_(wp.u * nx + wp.v * ny) + sound_speed(wp, gamma);
  const R a = jmax(sm, sp);
#pragma unroll
  for (int c = 0; c < 4; ++c) out[c] = R(0.5) * (fm[c] + fp[c]) - R(0.5) * a * (qp[c] - qm[c]);
}

// fluxes.py:40-51 — Roe averages (sqrt(rho_m rho_p), u, v, H, c).
template <typename R>
__device__ __forceinline__ void roe_mean(const R qm[4], const R qp[4], const Prim<R>& wm, const Prim<R>& wp, R gm1,
                                         R& rho, R& u, R& v, R& h, R& c) {
  const R hm = (qm[3] + wm.p) * wm.inv_rho;
  const R hp = (qp[3] + wp.p) * wp.inv_rho;
  const R sm = sqrt_(wm.rho), sp = sqrt_(wp.rho);
  const R is = rcp(sm + sp);
  u = (sm * wm.u + sp * wp.u) * is;
  v = (sm * wm.v + sp * wp.v) * is;
  h = (sm * hm + sp * hp) * is;
  c = sqrt_(gm1 * (h - R(0.5) * (u * u + v * v)));
  rho = sm * sp;
}

// fluxes.py:54-98 — Roe flux with Harten's entropy fix on the acoustic waves.
template <typename R>
__device__ __forceinline__ void roe(const R qm[4], const R qp[4], const Prim<R>& wm, const Prim<R>& wp,
                                    R nx, R ny, R gamma, const R fm[4], const R fp[4], R out[4]) {
  R rho, u, v, h, c;
  roe_mean(qm, qp, wm, wp, gamma - R(1), rho, u, v, h, c);
  const R un = u * nx + v * ny;
  const R ut = -u * ny + v * nx;
  const R drho = wp.rho - wm.rho;
  const R dp = wp.p - wm.p;
  const R dun = (wp.u * nx + wp.v * ny) - (wm.u * nx + wm.v * ny);
  const R dut = (-wp.u * ny + wp.v * nx) - (-wm.u * ny + wm.v * nx);
  const R c2 = c * c;
  const R ic2 = rcp(c2);
  const R i2c2 = R(0.5) * ic2;  // = rcp(2 c2): exact in FP64 (a power-of-two scaling commutes with
                                 // the correctly rounded reciprocal), one reciprocal fewer per flux
  const R a_m = (dp - rho * c * dun) * i2c2;
  const R a_e = drho - dp * ic2;
  const R a_s = rho * dut;
  const R a_p = (dp + rho * c * dun) * i2c2;
  const R delta = R(0.1) * (abs_(un) + c);
  const R i2d = rcp(R(2) * delta);
  auto fixed = [&](R lam) {
    const R mag = abs_(lam);
    return mag < delta ? (lam * lam + delta * delta) * i2d : mag;
  };
  const R l_m = fixed(un - c), l_p = fixed(un + c), l_0 = abs_(un);
  const R wmn = l_m * a_m, we = l_0 * a_e, ws = l_0 * a_s, wpl = l_p * a_p;
  const R d0 = wmn + we + wpl;
  const R d1 = wmn * (u - c * nx) + we * u + ws * (-ny) + wpl * (u + c * nx);
  const R d2 = wmn * (v - c * ny) + we * v + ws * nx + wpl * (v + c * ny);
  const R d3 = wmn * (h - c * un) + we * (R(0.5) * (u * u + v * v)) + ws * ut + wpl * (h + c * un);
  out[0] = R(0.5) * (fm[0] + fp[0]) - R(0.5) * d0;
  out[1] = R(0.5) * (fm[1] + fp[1]) - R(0.5) * d1;
  out[2] = R(0.5) * (fm[2] + fp[2]) - R(0.5) * d2;
  out[3] = R(0.5) * (fm[3] + fp[3]) - R(0.5) * d3;
}

// fluxes.py:101-143 — Toro's HLLC with Einfeldt (Roe-average) wave speeds.
template <typename R>
__device__ __forceinline__ void hllc(const R qm[4], const R qp[4], const Prim<R>& wm, const Prim<R>& wp,
                                     R nx, R ny, R gamma, const R fm[4], const R fp[4], R out[4]) {
  const R unm = wm.u * nx + wm.v * ny;
  const R unp = wp.u * nx + wp.v * ny;
  const R cm = sound_speed(wm, gamma), cp = sound_speed(wp, gamma);
  R rho, u, v, h, c;
  roe_mean(qm, qp, wm, wp, gamma - R(1), rho, u, v, h, c);
  const R un = u * nx + v * ny;
  const R s_m = jmin(unm - cm, un - c);
  const R s_p = jmax(unp + cp, un + c);
  const R mass_m = wm.rho * (s_m - unm);
  const R mass_p = wp.rho * (s_p - unp);
  const R s_star = div_(wp.p - wm.p + mass_m * unm - mass_p * unp, nonzero(mass_m - mass_p));
  if (s_m >= R(0)) {
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = fm[k];
  } else if (s_star >= R(0)) {
    const R fac = div_(mass_m, nonzero(s_m - s_star));
    const R sh = s_star - unm;
    const R st[4] = {fac, fac * (wm.u + sh * nx), fac * (wm.v + sh * ny),
                     fac * (qm[3] * wm.inv_rho + sh * (s_star + div_(wm.p, nonzero(mass_m))))};
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = fm[k] + s_m * (st[k] - qm[k]);
  } else if (s_p > R(0)) {
    const R fac = div_(mass_p, nonzero(s_p - s_star));
    const R sh = s_star - unp;
    const R st[4] = {fac, fac * (wp.u + sh * nx), fac * (wp.v + sh * ny),
                     fac * (qp[3] * wp.inv_rho + sh * (s_star + div_(wp.p, nonzero(mass_p))))};
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = fp[k] + s_p * (st[k] - qp[k]);
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) out[k] = fp[k];
  }
  // NaN wave speeds: every jnp.where test is false, so the reference returns fp.
}

// Interface flux Fhat(q-, q+, n) and the normal flux F(q-).n of the interior trace.
template <typename R, int FLUX>
__device__ __forceinline__ void interface_flux(const R qm[4], const R qp[4], R nx, R ny, R gamma, R fhat[4], R fm[4]) {
  const R gm1 = gamma - R(1);
  const Prim<R> wm = primitive(qm, gm1);
  const Prim<R> wp = primitive(qp, gm1);
  R fp[4];
  normal_flux(qm, wm, nx, ny, fm);
  normal_flux(qp, wp, nx, ny, fp);
  if (FLUX == FLUX_RUSANOV) rusanov(qm, qp, wm, wp, nx, ny, gamma, fm, fp, fhat);
  else if (FLUX == FLUX_ROE) roe(qm, qp, wm, wp, nx, ny, gamma, fm, fp, fhat);
  else hllc(qm, qp, wm, wp, nx, ny, gamma, fm, fp, fhat);
}

// Interface flux of a face node as the stage kernels use it. The FP32-mixed
// form returns F(q-).n exactly when the two traces are equal, so a uniform
// state has no surface term (HLLC's star state would otherwise carry
// single-precision rounding into every face of a uniform region).
template <typename R, int FLUX>
__device__ __forceinline__ void trace_flux(const R qm[4], const R qp[4], R nx, R ny, R gamma, R fhat[4], R fm[4]) {
  interface_flux<R, FLUX>(qm, qp, nx, ny, gamma, fhat, fm);
  if (sizeof(R) == 4 && qm[0] == qp[0] && qm[1] == qp[1] && qm[2] == qp[2] && qm[3] == qp[3]) {
#pragma unroll
    for (int c = 0; c < 4; ++c) fhat[c] = fm[c];
  }
}

// The same, also returning the normal flux F(q+).n of the exterior trace
// (with the interior normal): the face-job form lifts the neighbour's side
// from it.
template <typename R, int FLUX>
__device__ __forceinline__ void trace_flux3(const R qm[4], const R qp[4], R nx, R ny, R gamma, R fhat[4], R fm[4],
                                            R fp[4]) {
  const R gm1 = gamma - R(1);
  const Prim<R> wm = primitive(qm, gm1);
  const Prim<R> wp = primitive(qp, gm1);
  normal_flux(qm, wm, nx, ny, fm);
  normal_flux(qp, wp, nx, ny, fp);
  if (FLUX == FLUX_RUSANOV) rusanov(qm, qp, wm, wp, nx, ny, gamma, fm, fp, fhat);
  else if (FLUX == FLUX_ROE) roe(qm, qp, wm, wp, nx, ny, gamma, fm, fp, fhat);
  else hllc(qm, qp, wm, wp, nx, ny, gamma, fm, fp, fhat);
  if (sizeof(R) == 4 && qm[0] == qp[0] && qm[1] == qp[1] && qm[2] == qp[2] && qm[3] == qp[3]) {
#pragma unroll
    for (int c = 0; c < 4; ++c) fhat[c] = fm[c];
  }
}

enum { LIM_MINMOD = 0, LIM_MC = 1, LIM_VAN_LEER = 2, LIM_SUPERBEE = 3, LIM_UNLIMITED = 4 };

// limiters.py:16-39
template <typename R, int PHI>
__device__ __forceinline__ R phi(R r) {
  if (PHI == LIM_MINMOD) return jmax(R(0), jmin(R(1), r));
  if (PHI == LIM_MC) return jmax(R(0), jmin(jmin(xmul(R(2), r), xmul(R(0.5), xadd(R(1), r))), R(2)));
  if (PHI == LIM_VAN_LEER) return xdiv(xadd(r, abs_(r)), xadd(R(1), abs_(r)));
  if (PHI == LIM_SUPERBEE) return jmax(R(0), jmax(jmin(xmul(R(2), r), R(1)), jmin(r, R(2))));
  return R(1);
}

// limiting.py:124-125 — minmod of two values.
template <typename R>
__device__ __forceinline__ R minmod2(R a, R b) {
  if (xmul(a, b) > R(0)) {
    const R m = jmin(abs_(a), abs_(b));
    return a > R(0) ? m : -m;
  }
  return R(0);
}

}  // namespace cfd
