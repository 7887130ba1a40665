// adjoint.cuh — hand-written discrete adjoint (vector-Jacobian products) of
// one fixed-size SSP-RK3 step: stage combine, limiters and the DG right-hand
// side. Included by kernels.cu inside namespace cfd.
//
// For a stage  q' = Lambda(qt),  qt = a q_n + b (q_s + dt L(q_s))  and the
// adjoint g of q', the backward pass computes
//   qt_bar = Lambda'(qt)^T g                (limiter branches replayed from qt)
//   q_n_bar += a qt_bar,   q_s_bar = b qt_bar + b dt L'(q_s)^T qt_bar.
// dt is a constant of the step: CFD-demo's run loop converts it to a host
// float (solver.py:181), so a gradient taken through it carries no dt term.
//   L'(q)^T v, volume (dg.py:148-151, Ft = rx F + ry G, Gt = sx F + sy G):
//     Ft_bar = -Dr^T v, Gt_bar = -Ds^T v, F_bar = rx Ft_bar + sx Gt_bar,
//     G_bar = ry Ft_bar + sy Gt_bar, q_bar_j = (dF/dq)^T F_bar + (dG/dq)^T G_bar.
//   surface (dg.py:153-164): w = Fscale LIFT^T v at the 15 face nodes, then
//     q_bar += (d(F.n)/dq)^T w_own + (dFhat/dq-)^T (w_nbr - w_own):
//   the neighbour evaluates Fhat(q_nbr, q_own, -n) = -Fhat(q_own, q_nbr, n), so
//   its share is gathered from its w at the matching node instead of being
//   scattered (no atomics). Slip walls chain through the mirror state; fixed
//   exterior states feed the adjoint of the boundary state.
//   Lambda'^T replays the forward decisions from the taped pre-limiting state,
//   cell averages and nodal minima, so every branch is the one the forward
//   step took: troubled flag, phi piece, min(1, phi), the +/- rescaling case
//   (limiting.py:136-163); the density scaling theta with its min routed to
//   the argmin node (limiting.py:170-181). The pressure-scaling theta is found
//   by bisection (limiting.py:183-200), piecewise constant in q: jax.grad
//   gives it a zero derivative (hold_theta), while the root it approximates
//   to 2^-60 moves with q; by default its implicit derivative is used, which
//   is what a finite difference of the forward step sees.
// Rusanov Jacobians are analytic; Roe and HLLC use forward-mode dual numbers
// through the same device flux code as the forward kernels.
#pragma once

// ---- forward-mode dual numbers -----------------------------------------------
template <typename T>
struct Dual {
  T v, d;
  __device__ __forceinline__ Dual() {}
  __device__ __forceinline__ Dual(T x) : v(x), d(T(0)) {}
  __device__ __forceinline__ Dual(T x, T dx) : v(x), d(dx) {}
};
template <typename T> __device__ __forceinline__ Dual<T> operator+(Dual<T> a, Dual<T> b) { return Dual<T>(a.v + b.v, a.d + b.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator-(Dual<T> a, Dual<T> b) { return Dual<T>(a.v - b.v, a.d - b.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator-(Dual<T> a) { return Dual<T>(-a.v, -a.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator*(Dual<T> a, Dual<T> b) { return Dual<T>(a.v * b.v, a.d * b.v + a.v * b.d); }
template <typename T> __device__ __forceinline__ Dual<T> operator/(Dual<T> a, Dual<T> b) {
  const T q = a.v / b.v;
  return Dual<T>(q, (a.d - q * b.d) / b.v);
}
template <typename T> __device__ __forceinline__ bool operator<(Dual<T> a, Dual<T> b) { return a.v < b.v; }
template <typename T> __device__ __forceinline__ bool operator>(Dual<T> a, Dual<T> b) { return a.v > b.v; }
template <typename T> __device__ __forceinline__ bool operator<=(Dual<T> a, Dual<T> b) { return a.v <= b.v; }
template <typename T> __device__ __forceinline__ bool operator>=(Dual<T> a, Dual<T> b) { return a.v >= b.v; }
template <typename T> __device__ __forceinline__ bool operator==(Dual<T> a, Dual<T> b) { return a.v == b.v; }
template <typename T> __device__ __forceinline__ bool operator!=(Dual<T> a, Dual<T> b) { return a.v != b.v; }
template <typename T> __device__ __forceinline__ Dual<T> rcp(Dual<T> x) {
  const T r = rcp(x.v);
  return Dual<T>(r, -x.d * r * r);
}
template <typename T> __device__ __forceinline__ Dual<T> sqrt_(Dual<T> x) {
  const T s = sqrt_(x.v);
  return Dual<T>(s, x.d * T(0.5) / s);
}
// |x| with derivative sign(x) dx, sign(0) = 0 (jax.numpy.abs; a central
// difference across the kink sees 0 as well)
template <typename T> __device__ __forceinline__ Dual<T> abs_(Dual<T> x) {
  return Dual<T>(x.v < T(0) ? -x.v : x.v, x.v < T(0) ? -x.d : (x.v > T(0) ? x.d : T(0)));
}
template <typename T> __device__ __forceinline__ Dual<T> nonzero(Dual<T> x) { return Dual<T>(nonzero(x.v), x.d); }
template <typename T> __device__ __forceinline__ Dual<T> div_(Dual<T> a, Dual<T> b) { return a / b; }

// (dFhat/dq_side)^T w of the interface flux by four forward-mode evaluations
// seeded on q- (side 0) or q+ (side 1).
template <typename R, int FLUX>
__device__ __forceinline__ void flux_vjp_dual(const R qm[4], const R qp[4], R nx, R ny, R gamma, const R w[4],
                                              int side, R out[4]) {
#pragma unroll 1
  for (int k = 0; k < 4; ++k) {
    Dual<R> a[4], b[4], fh[4], fm[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      a[c] = Dual<R>(qm[c], (side == 0 && c == k) ? R(1) : R(0));
      b[c] = Dual<R>(qp[c], (side == 1 && c == k) ? R(1) : R(0));
    }
    interface_flux<Dual<R>, FLUX>(a, b, Dual<R>(nx), Dual<R>(ny), Dual<R>(gamma), fh, fm);
    R s = R(0);
#pragma unroll
    for (int c = 0; c < 4; ++c) s += fh[c].d * w[c];
    out[k] = s;
  }
}

// (d(F(q).n)/dq)^T w for the Euler normal flux (euler.py:49-61), analytic.
template <typename R>
__device__ __forceinline__ void normal_flux_vjp(const R q[4], R nx, R ny, R gm1, const R w[4], R out[4]) {
  const R ir = R(1) / q[0];
  const R u = q[1] * ir, v = q[2] * ir;
  const R un = u * nx + v * ny;
  const R p = gm1 * (q[3] - R(0.5) * (q[1] * u + q[2] * v));
  const R wun = w[1] * q[1] + w[2] * q[2] + w[3] * (q[3] + p);  // weight of d(un)
  const R wp = w[1] * nx + w[2] * ny + w[3] * un;               // weight of d(p)
  // d(un) = (-un, nx, ny, 0) / rho ;  d(p) = gm1 (|u|^2 / 2, -u, -v, 1)
  out[0] = -wun * un * ir + wp * gm1 * R(0.5) * (u * u + v * v);
  out[1] = w[0] * nx + wun * nx * ir - wp * gm1 * u + un * w[1];
  out[2] = w[0] * ny + wun * ny * ir - wp * gm1 * v + un * w[2];
  out[3] = wp * gm1 + un * w[3];
}

// s = |u.n| + c and its gradient with respect to q (Rusanov's wave speed)
template <typename R>
__device__ __forceinline__ void speed_grad(const R q[4], R nx, R ny, R gamma, R& s, R g[4]) {
  const R gm1 = gamma - R(1);
  const R ir = R(1) / q[0];
  const R u = q[1] * ir, v = q[2] * ir;
  const R un = u * nx + v * ny;
  const R p = gm1 * (q[3] - R(0.5) * (q[1] * u + q[2] * v));
  const R c = sqrt_(gamma * p * ir);
  s = abs_(un) + c;
  const R sg = un < R(0) ? R(-1) : (un > R(0) ? R(1) : R(0));  // d|un|, sign(0) = 0
  const R kc = gamma * ir / (R(2) * c);  // dc = kc (dp - (p / rho) d rho)
  g[0] = sg * (-un * ir) + kc * (gm1 * R(0.5) * (u * u + v * v) - p * ir);
  g[1] = sg * nx * ir + kc * (-gm1 * u);
  g[2] = sg * ny * ir + kc * (-gm1 * v);
  g[3] = kc * gm1;
}

// Rusanov (fluxes.py:28-37): (dFhat/dq-)^T w (side 0) or (dFhat/dq+)^T w (side 1).
template <typename R>
__device__ __forceinline__ void rusanov_vjp(const R qm[4], const R qp[4], R nx, R ny, R gamma, const R w[4], int side,
                                            R out[4]) {
  R sm, sp, gm[4], gp[4];
  speed_grad(qm, nx, ny, gamma, sm, gm);
  speed_grad(qp, nx, ny, gamma, sp, gp);
  const bool minus_max = sm > sp;  // alpha = max(sm, sp) as the forward flux picks it
  const R alpha = minus_max ? sm : sp;
  R jf[4];
  normal_flux_vjp(side == 0 ? qm : qp, nx, ny, gamma - R(1), w, jf);
  R wdq = R(0);
#pragma unroll
  for (int c = 0; c < 4; ++c) wdq += w[c] * (qp[c] - qm[c]);
  const bool alpha_here = side == 0 ? minus_max : !minus_max;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const R ga = alpha_here ? (side == 0 ? gm[c] : gp[c]) : R(0);
    out[c] = R(0.5) * jf[c] + (side == 0 ? R(0.5) : R(-0.5)) * alpha * w[c] - R(0.5) * wdq * ga;
  }
}

template <typename R, int FLUX>
__device__ __forceinline__ void iflux_vjp(const R qm[4], const R qp[4], R nx, R ny, R gamma, const R w[4], int side,
                                          R out[4]) {
  if (FLUX == FLUX_RUSANOV) rusanov_vjp(qm, qp, nx, ny, gamma, w, side, out);
  else flux_vjp_dual<R, FLUX>(qm, qp, nx, ny, gamma, w, side, out);
}

struct AdjParams {
  CfdMesh m;
  double gamma;
  const double* dt;    // per-instance step size
  const void* qt;      // pre-limiting stage state (tape)
  const double* avg;   // its cell averages [4][ld] (tape)
  const double* aux;   // its nodal density / pressure minima [2][ld] (tape)
  const double* pos;   // the positivity limiter's pressure theta and critical node [2][ld] (tape)
  const void* qs;      // stage input state
  const void* g;       // adjoint of the limited stage state
  void* qtb;           // adjoint of qt (out)
  void* w;             // face-node adjoints [60][ld]
  void* nab;           // adjoints of the neighbour averages [12][ld]
  void* src_bar;       // adjoint of q_s (written or accumulated)
  void* base_bar;      // adjoint of q_n (accumulated; null when a = 0)
  double* bc_bar;      // [rows][4] adjoint of the fixed exterior states (accumulated; may be null)
  double a, b;         // stage coefficients
  int accumulate_src;  // 1: src_bar += ..., 0: src_bar = ...
  int limited;         // troubled-cell limiter active
  int hold_theta;      // 1: pressure-scaling theta constant (jax.grad semantics)
  int* list;           // elements that need the full limiter replay [ld]
  int* count;          // their number
  uint8_t* listed;     // per element: 1 if listed (qtb holds its adjoint), 0 if qt_bar = g [ld]
};

__device__ __forceinline__ int element_instance(const CfdMesh& m, int e) { return m.instance ? m.instance[e] : 0; }

// ---- limiter adjoint ------------------------------------------------------------
// phi'(r) on the piece the forward value lies on (limiters.py:16-39)
template <typename R, int PHI>
__device__ __forceinline__ R phi_grad(R r) {
  if (PHI == LIM_MINMOD) return (r > R(0) && r < R(1)) ? R(1) : R(0);
  if (PHI == LIM_MC) {
    if (!(r > R(0))) return R(0);
    const R a = R(2) * r, b = R(0.5) * (R(1) + r);
    const R m = a < b ? a : b;
    if (!(m < R(2))) return R(0);
    return a < b ? R(2) : R(0.5);
  }
  if (PHI == LIM_VAN_LEER) return r > R(0) ? R(2) / ((R(1) + r) * (R(1) + r)) : R(0);
  if (PHI == LIM_SUPERBEE) {
    if (!(r > R(0))) return R(0);
    const R a = (R(2) * r < R(1)) ? R(2) * r : R(1);
    const R b = (r < R(2)) ? r : R(2);
    if (a >= b) return R(2) * r < R(1) ? R(2) : R(0);
    return r < R(2) ? R(1) : R(0);
  }
  return R(0);
}

// Replays limit_kernel's decisions for element e (limiting.py:128-151):
// the averages a, the positivity target, the scaled neighbour differences and
// whether the element was troubled or needed the positivity limiter.
template <typename R, int PHI>
__device__ __forceinline__ void adj_limit_decide(const AdjParams& P, int e, double a[4], double& eps, double& pt,
                                                 R scaled[3][4], bool& troubled, bool& need_pos) {
  const CfdMesh& m = P.m;
  const int ld = m.ld;
  const R* __restrict__ qt = (const R*)P.qt;
  const double gm1 = P.gamma - 1.0;
#pragma unroll
  for (int c = 0; c < 4; ++c) a[c] = P.avg[c * ld + e];
  const double pa = pressure_x(a[0], a[1], a[2], a[3], gm1);
  eps = jmin(POSITIVITY_FLOOR, jmin(a[0], pa));
  pt = pressure_target<R>(eps, pa, a[3], gm1);
  const int finfo = m.face_info[e];
  troubled = false;
  if (PHI != LIM_UNLIMITED) {
    const double det_tol = sizeof(R) == 8 ? DETECTION_TOLERANCE : DETECTION_TOLERANCE_FP32;
    R dif[3][4];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const int kind = (finfo >> (8 * f)) & 3;
      double na[4];
      if (kind == CFD_FACE_INTERIOR) {
        const int nb = m.neighbor[f * ld + e];
#pragma unroll
        for (int c = 0; c < 4; ++c) na[c] = P.avg[c * ld + nb];
      } else if (kind == CFD_FACE_SLIP_WALL) {
        const double nx = m.face_geo[(3 * f) * ld + e], ny = m.face_geo[(3 * f + 1) * ld + e];
        const double mn = xadd(xmul(a[1], nx), xmul(a[2], ny));
        na[0] = a[0];
        na[1] = xsub(a[1], xmul(xmul(2.0, mn), nx));
        na[2] = xsub(a[2], xmul(xmul(2.0, mn), ny));
        na[3] = a[3];
      } else {
        const int row = m.neighbor[f * ld + e] + (kind == CFD_FACE_EXACT_STATE ? NFP : 0);
#pragma unroll
        for (int c = 0; c < 4; ++c) na[c] = m.bc_states[row * 4 + c];
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) dif[f][c] = (R)xsub(na[c], a[c]);
    }
    const R* __restrict__ cs = GeoPtr<R>::cs(m);
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const int pf = (finfo >> (8 * f + 4)) & 3;
      const R al = cs[f * ld + e], be = cs[(3 + f) * ld + e];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const R pd = pf == 0 ? dif[0][c] : (pf == 1 ? dif[1][c] : dif[2][c]);
        scaled[f][c] = xmul((R)NEIGHBOR_FACTOR, xadd(xmul(al, dif[f][c]), xmul(be, pd)));
      }
    }
#pragma unroll
    for (int f = 0; f < 3; ++f)
#pragma unroll
      for (int cc = 0; cc < 2; ++cc) {
        const int c = cc == 0 ? 0 : 3;
        const R tr = xsub(qt[(c * NP + tab::MID_NODES[f]) * ld + e], (R)a[c]);
        const R ex = abs_(xsub(minmod2(tr, scaled[f][c]), tr));
        troubled |= (double)ex > xmul(det_tol, fabs(a[c]));
      }
  }
  need_pos = (P.aux[e] < eps) || (P.aux[ld + e] < pt);
}

// Light pass over every element: where the limiters left the element as it
// was, qt_bar = g and the neighbour-average adjoints are zero (adj_lift_kernel
// reads g and the listed flags instead of a copy); the
// others (troubled or positivity-scaled, a small minority) are flagged and
// listed for adj_limit_heavy_kernel.
template <typename R, int PHI>
__global__ void __launch_bounds__(128) adj_limit_scan_kernel(const AdjParams P) {
  const CfdMesh& m = P.m;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = e < m.num_elements && element_instance(m, e) >= 0;
  bool listed = false;
  if (live) {
    double a[4], eps, pt;
    R scaled[3][4];
    bool troubled, need_pos;
    adj_limit_decide<R, PHI>(P, e, a, eps, pt, scaled, troubled, need_pos);
    listed = troubled || need_pos;
  }
  warp_list_append(P.list, P.count, listed, e);  // every lane of the warp takes part
  if (e < m.ld) P.listed[e] = listed ? 1 : 0;
}

// qt_bar = Lambda'(qt)^T g for one listed element, plus the adjoints of the
// three neighbour / ghost averages it read (gathered by adj_lift_kernel).
// Four lanes of a warp share the element, lane c (= lane % 4) owning
// conserved variable c: the troubled-cell reconstruction and its reverse are
// separate per variable; the positivity scalings couple the variables through
// the density minimum, the scaling thetas and the pressure gradient at the
// critical node, which the quad exchanges with shuffles under its own mask
// (the four lanes always take the same branches: every decision is made from
// values they share).
template <typename R, int PHI>
__device__ __forceinline__ void adj_limit_quad(const AdjParams& P, int e, int c, unsigned qmask, int base) {
  const CfdMesh& m = P.m;
  const int ld = m.ld;
  const R* __restrict__ qt = (const R*)P.qt;
  const R* __restrict__ g = (const R*)P.g;
  R* __restrict__ qtb = (R*)P.qtb;
  R* __restrict__ nab = (R*)P.nab;
  const double gm1 = P.gamma - 1.0;
  const int finfo = m.face_info[e];
  double a[4], eps, pt;
  R scaled[3][4];
  bool troubled, need_pos;
  adj_limit_decide<R, PHI>(P, e, a, eps, pt, scaled, troubled, need_pos);
  const double ac_d = c == 0 ? a[0] : (c == 1 ? a[1] : (c == 2 ? a[2] : a[3]));
  R sc[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) sc[f] = c == 0 ? scaled[f][0] : (c == 1 ? scaled[f][1] : (c == 2 ? scaled[f][2] : scaled[f][3]));

  R s[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) s[i] = qt[(c * NP + i) * ld + e];
  // --- forward troubled-cell reconstruction of variable c, keeping what the reverse needs
  R proj[3], mfac[3], del[3], thp = R(0), thn = R(0), pos = R(0), neg = R(0);
  if (troubled) {
    const R ac = (R)ac_d;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      R pr = xmul((R)tab::P1MID[f][0], s[0]);
#pragma unroll
      for (int i = 1; i < NP; ++i) pr = xadd(pr, xmul((R)tab::P1MID[f][i], s[i]));
      pr = xsub(pr, ac);
      proj[f] = pr;
      R d = R(0), mf = R(0);
      if (pr != R(0)) {
        mf = jmin(R(1), phi<R, PHI>(xdiv(sc[f], pr)));
        d = xmul(pr, mf);
      }
      mfac[f] = mf;
      del[f] = d;
      pos = f == 0 ? jmax(d, R(0)) : xadd(pos, jmax(d, R(0)));
      neg = f == 0 ? jmax(-d, R(0)) : xadd(neg, jmax(-d, R(0)));
    }
    thp = pos > R(0) ? jmin(R(1), xdiv(neg, pos)) : R(0);
    thn = neg > R(0) ? jmin(R(1), xdiv(pos, neg)) : R(0);
    R dl[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) dl[f] = xsub(xmul(thp, jmax(del[f], R(0))), xmul(thn, jmax(-del[f], R(0))));
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      R v = xmul((R)tab::LINBASIS[i][0], dl[0]);
      v = xadd(v, xmul((R)tab::LINBASIS[i][1], dl[1]));
      v = xadd(v, xmul((R)tab::LINBASIS[i][2], dl[2]));
      s[i] = xadd(ac, v);
    }
  }
  // --- forward positivity decisions (the order of positivity() in kernels.cu);
  // the density minimum comes from lane 0 of the quad
  int imin = 0;
  double rmin = (double)s[0];
#pragma unroll
  for (int i = 1; i < NP; ++i) {
    const double r = (double)s[i];
    imin = r < rmin ? i : imin;
    rmin = jmin(rmin, r);
  }
  rmin = __shfl_sync(qmask, rmin, base);
  double th1 = 1.0;
  bool dens = false, dclip = true;
  if (rmin < eps) {
    dens = true;
    const double raw = xdiv(xsub(a[0], eps), xsub(a[0], rmin));
    th1 = jmin(jmax(raw, 0.0), 1.0);
    dclip = !(raw > 0.0 && raw < 1.0);
#pragma unroll
    for (int i = 0; i < NP; ++i) s[i] = (R)xadd(ac_d, xmul(th1, xsub((double)s[i], ac_d)));
  }
  // the pressure-scaling theta and its critical node, as the forward
  // bisection found them (limit_kernel records them in the tape)
  double th2 = P.pos[e];
  const int i2 = (int)P.pos[ld + e];
  if (!(th2 < 1.0)) th2 = 1.0;

  // --- reverse pass; y is the running adjoint of the nodal values of
  // variable c, abar that of its cell average (an AVG_W-weighted sum of qt)
  R y[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) y[i] = g[(c * NP + i) * ld + e];
  R abar = R(0);
  // pressure scaling out = a + th2 (in - a). th2 is the bisection root of
  // p(a + th (in_i2 - a)) = pt at the critical node i2: held constant (the
  // derivative of the bisection itself), or differentiated implicitly,
  //   d th2 = -grad p(z) . ((1 - th2) da + th2 d in_i2) / (grad p(z) . (in_i2 - a)),
  // z = a + th2 (in_i2 - a), which follows the root the bisection resolves to
  // 2^-60 (pt held constant, like eps).
  if (th2 < 1.0) {
    R part = R(0), sum = R(0);
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      part += (R)((double)s[i] - ac_d) * y[i];
      sum += y[i];
      y[i] *= (R)th2;
    }
    abar += (R)(1.0 - th2) * sum;
    part += __shfl_xor_sync(qmask, part, 1);
    const R thbar = part + __shfl_xor_sync(qmask, part, 2);
    if (!P.hold_theta && i2 >= 0) {
      double dc = 0.0;
#pragma unroll
      for (int j = 0; j < NP; ++j) dc = (j == i2) ? (double)s[j] : dc;
      dc -= ac_d;
      double d[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) d[k] = __shfl_sync(qmask, dc, base + k);
      const double z0 = a[0] + th2 * d[0], u = (a[1] + th2 * d[1]) / z0, v = (a[2] + th2 * d[2]) / z0;
      const double gp[4] = {gm1 * 0.5 * (u * u + v * v), -gm1 * u, -gm1 * v, gm1};  // grad p(z)
      const double den = gp[0] * d[0] + gp[1] * d[1] + gp[2] * d[2] + gp[3] * d[3];
      if (den != 0.0) {
        const double k = -(double)thbar / den;
        const double gpc = c == 0 ? gp[0] : (c == 1 ? gp[1] : (c == 2 ? gp[2] : gp[3]));
        abar += (R)(k * (1.0 - th2) * gpc);
#pragma unroll
        for (int i = 0; i < NP; ++i)
          if (i == i2) y[i] += (R)(k * th2 * gpc);
      }
    }
  }
  // density scaling out = a + th1 (in - a), th1 = (a_rho - eps) / (a_rho - min_i rho_i)
  if (dens) {
    R part = R(0), sum = R(0);
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const R din = th1 > 0.0 ? (R)(((double)s[i] - ac_d) / th1) : R(0);  // in - a
      part += din * y[i];
      sum += y[i];
      y[i] *= (R)th1;
    }
    abar += (R)(1.0 - th1) * sum;
    part += __shfl_xor_sync(qmask, part, 1);
    const R thbar = part + __shfl_xor_sync(qmask, part, 2);
    if (!dclip && c == 0) {
      const double span = a[0] - rmin;
      abar += thbar * (R)((eps - rmin) / (span * span));
      const R dth_dmin = (R)((a[0] - eps) / (span * span));
#pragma unroll
      for (int i = 0; i < NP; ++i)
        if (i == imin) y[i] += thbar * dth_dmin;
    }
  }
  // troubled-cell reconstruction
  R nabar[3] = {R(0), R(0), R(0)};
  if (troubled) {
    const R* __restrict__ cs = GeoPtr<R>::cs(m);
    R ab = R(0), dpb[3] = {R(0), R(0), R(0)};
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      ab += y[i];
#pragma unroll
      for (int f = 0; f < 3; ++f) dpb[f] += (R)tab::LINBASIS[i][f] * y[i];
      y[i] = R(0);  // a rebuilt element depends on its nodes only through the P1 projections
    }
    R thpb = R(0), thnb = R(0), pb[3], nb_[3];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      pb[f] = thp * dpb[f];
      nb_[f] = -thn * dpb[f];
      thpb += jmax(del[f], R(0)) * dpb[f];
      thnb -= jmax(-del[f], R(0)) * dpb[f];
    }
    R posb = R(0), negb = R(0);
    if (pos > R(0) && neg < pos) {  // thp = neg / pos below the cap
      negb += thpb / pos;
      posb -= thpb * neg / (pos * pos);
    }
    if (neg > R(0) && pos < neg) {  // thn = pos / neg below the cap
      posb += thnb / neg;
      negb -= thnb * pos / (neg * neg);
    }
    R difb[3] = {R(0), R(0), R(0)};
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const R d = del[f];
      const R delb = d > R(0) ? pb[f] + posb : (d < R(0) ? -(nb_[f] + negb) : R(0));
      R projb = R(0), scb = R(0);
      const R pr = proj[f];
      if (pr != R(0)) {
        projb = mfac[f] * delb;
        const R r = sc[f] / pr;
        const R rb = phi<R, PHI>(r) < R(1) ? phi_grad<R, PHI>(r) * pr * delb : R(0);
        scb = rb / pr;
        projb -= rb * sc[f] / (pr * pr);
      }
      // proj_f = P1MID_f . q - a ; scaled_f = 1.5 (alpha_f dif_f + beta_f dif_pf), dif = na - a
      ab -= projb;
#pragma unroll
      for (int i = 0; i < NP; ++i) y[i] += (R)tab::P1MID[f][i] * projb;
      const int pf = (finfo >> (8 * f + 4)) & 3;
      const R al = cs[f * ld + e], be = cs[(3 + f) * ld + e];
      difb[f] += (R)NEIGHBOR_FACTOR * al * scb;
      const R t = (R)NEIGHBOR_FACTOR * be * scb;
      if (pf == 0) difb[0] += t;
      else if (pf == 1) difb[1] += t;
      else difb[2] += t;
    }
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      nabar[f] = difb[f];
      ab -= difb[f];
    }
    abar += ab;
    // ghost averages: a slip wall mirrors this element's average (the
    // mirror couples the momentum lanes); a fixed exterior state is a
    // boundary parameter
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const int kind = (finfo >> (8 * f)) & 3;
      if (kind == CFD_FACE_SLIP_WALL) {
        const R nx = (R)m.face_geo[(3 * f) * ld + e], ny = (R)m.face_geo[(3 * f + 1) * ld + e];
        const R n1 = __shfl_sync(qmask, nabar[f], base + 1), n2 = __shfl_sync(qmask, nabar[f], base + 2);
        const R dm = n1 * nx + n2 * ny;
        abar += c == 1 ? nabar[f] - R(2) * dm * nx : (c == 2 ? nabar[f] - R(2) * dm * ny : nabar[f]);
      } else if (kind >= CFD_FACE_FIXED_STATE && P.bc_bar) {  // fixed or exact state: its ghost row
        const int row = m.neighbor[f * ld + e] + (kind == CFD_FACE_EXACT_STATE ? NFP : 0);
        if (nabar[f] != R(0)) atomicAdd(&P.bc_bar[row * 4 + c], (double)nabar[f]);
      }
      if (kind != CFD_FACE_INTERIOR) nabar[f] = R(0);
    }
  }
#pragma unroll
  for (int i = 0; i < NP; ++i) qtb[(c * NP + i) * ld + e] = y[i] + (R)tab::AVG_W[i] * abar;
  if (PHI != LIM_UNLIMITED) {
#pragma unroll
    for (int f = 0; f < 3; ++f) nab[(f * 4 + c) * ld + e] = nabar[f];
  }
}

// the listed elements, grid-stride, four lanes per element
template <typename R, int PHI>
__global__ void __launch_bounds__(64) adj_limit_heavy_kernel(const AdjParams P) {
  const int n = *P.count;
  const int lane = threadIdx.x & 31, c = lane & 3, base = lane & ~3;
  const unsigned qmask = 0xfu << base;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 2; t < n; t += (gridDim.x * blockDim.x) >> 2)
    adj_limit_quad<R, PHI>(P, P.list[t], c, qmask, base);
}

// surface pass A: w = b dt Fscale LIFT^T qt_bar at the 15 face nodes; one
// thread per (element, conserved variable). With the troubled-cell limiter it
// first gathers the neighbours' adjoints of the element's average into
// qt_bar (the adjoints the heavy limiter pass wrote for its neighbour faces).
template <typename R>
__global__ void __launch_bounds__(128) adj_lift_kernel(const AdjParams P) {
  const CfdMesh& m = P.m;
  const int ld = m.ld;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (e >= m.num_elements) return;
  const int inst = element_instance(m, e);
  if (inst < 0) return;
  R* __restrict__ v = (R*)P.qtb;
  R* __restrict__ w = (R*)P.w;
  const R scale = (R)(P.b * P.dt[inst]);
  R fs[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) fs[f] = scale * (R)m.face_geo[(3 * f + 2) * ld + e];
  const bool own = P.listed[e] != 0;
  const R* __restrict__ src = own ? v : (const R*)P.g;
  R vi[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) vi[i] = src[(c * NP + i) * ld + e];
  if (P.limited) {
    // the listed neighbours' adjoints of this element's average (they read
    // it in their troubled-cell tests): qt_bar += AVG_W * sum
    const int finfo = m.face_info[e];
    const R* __restrict__ nab = (const R*)P.nab;
    R ab = R(0);
    bool nb_listed = false;
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const int info = (finfo >> (8 * f)) & 0xff;
      if ((info & 3) != CFD_FACE_INTERIOR) continue;
      const int nb = m.neighbor[f * ld + e];
      if (!P.listed[nb]) continue;
      nb_listed = true;
      ab += nab[(((info >> 2) & 3) * 4 + c) * ld + nb];
    }
    if (nb_listed) {
#pragma unroll
      for (int i = 0; i < NP; ++i) vi[i] += (R)tab::AVG_W[i] * ab;
    }
  }
  // the node pass reads qt_bar from qtb for every element (the pass-through
  // elements' g is copied here, where it is in registers anyway)
#pragma unroll
  for (int i = 0; i < NP; ++i) v[(c * NP + i) * ld + e] = vi[i];
#pragma unroll
  for (int col = 0; col < 3 * NFP; ++col) {
    R t = R(0);
#pragma unroll
    for (int i = 0; i < NP; ++i) t = fma((R)tab::LIFT[i][col], vi[i], t);
    w[(c * NP + col) * ld + e] = fs[col / NFP] * t;
  }
}

// pass B: the adjoints of the stage input (volume + surface) and of the base
// state. One thread per (element, node j): a block covers ADJ_EPB elements x
// 15 nodes (threadIdx.x = element, threadIdx.y = node, so a warp holds one
// node of 32 elements: coalesced, and uniform in the node). The block's
// qt_bar tile is staged in shared memory. Node j's thread owns every output
// at node j: the volume term at j and the surface terms of the face slots
// that meet at j (corner nodes lie on two faces).
// For each node j, the face slots (f * NFP + k) whose face node is j: none
// (interior nodes), one, or two (the corners lie on two faces), packed as
// slot + 1 in 6-bit fields.
struct NodeSlotTable {
  int v[NP];
};
constexpr NodeSlotTable make_node_slots() {
  NodeSlotTable t{};
  for (int j = 0; j < NP; ++j) {
    int n = 0, packed = 0;
    for (int sl = 0; sl < 3 * NFP; ++sl)
      if ((int)((FN_PACK >> (4 * sl)) & 15ull) == j) packed |= (sl + 1) << (6 * n++);
    t.v[j] = packed;
  }
  return t;
}
__device__ constexpr NodeSlotTable NODE_SLOTS = make_node_slots();

constexpr int ADJ_EPB = 32;
constexpr int ADJ_NODE_MINB = 1;  // resident blocks per SM the register budget is sized for

template <typename R, int FLUX>
__global__ void __launch_bounds__(ADJ_EPB * NP, ADJ_NODE_MINB) adj_rhs_node_kernel(const AdjParams P) {
  __shared__ R s_v[4 * NP][ADJ_EPB];
  const CfdMesh& m = P.m;
  const int ld = m.ld;
  const int lane = threadIdx.x, j = threadIdx.y;
  const int e = blockIdx.x * ADJ_EPB + lane;
  const bool in = e < m.num_elements;
  const R* __restrict__ qtb = (const R*)P.qtb;
  const R* __restrict__ qs = (const R*)P.qs;
  // this node's state and the element's metric, loaded ahead of the staging
  // barrier so that their latency overlaps it
  R q[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) q[c] = in ? qs[(c * NP + j) * ld + e] : R(1);
  const R rx = in ? (R)m.metric[e] : R(0), ry = in ? (R)m.metric[ld + e] : R(0);
  const R sx = in ? (R)m.metric[2 * ld + e] : R(0), sy = in ? (R)m.metric[3 * ld + e] : R(0);
  const int finfo = in ? m.face_info[e] : 0;
#pragma unroll
  for (int r = j; r < 4 * NP; r += NP) s_v[r][lane] = in ? qtb[r * ld + e] : R(0);
  __syncthreads();
  if (!in) return;
  const int inst = element_instance(m, e);
  if (inst < 0) return;
  const R* __restrict__ w = (const R*)P.w;
  R* __restrict__ sb = (R*)P.src_bar;
  R* __restrict__ bb = (R*)P.base_bar;
  const R gamma = (R)P.gamma, gm1 = gamma - R(1);
  const R scale = (R)(P.b * P.dt[inst]);
  if (bb) {
#pragma unroll
    for (int c = 0; c < 4; ++c) bb[(c * NP + j) * ld + e] += (R)P.a * s_v[c * NP + j][lane];
  }
  // volume at node j: Ft_bar_j = -sum_i Dr[i][j] v_i, Gt_bar_j likewise
  R acc[4];
  {
    R fb[4], gb[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      R sf = R(0), sg = R(0);
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        const R vi = s_v[c * NP + i][lane];
        sf = fma((R)ctab::DR[i][j], vi, sf);
        sg = fma((R)ctab::DS[i][j], vi, sg);
      }
      const R ftb = -scale * sf, gtb = -scale * sg;
      fb[c] = rx * ftb + sx * gtb;
      gb[c] = ry * ftb + sy * gtb;
    }
    R jf[4], jg[4];
    normal_flux_vjp(q, R(1), R(0), gm1, fb, jf);
    normal_flux_vjp(q, R(0), R(1), gm1, gb, jg);
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[c] = (R)P.b * s_v[c * NP + j][lane] + jf[c] + jg[c];
  }
  // surface: the face slots (f, k) whose node is j
  const int slots = NODE_SLOTS.v[j];  // warp-uniform
#pragma unroll 1
  for (int u = 0; u < 2; ++u) {
    const int sl = ((slots >> (6 * u)) & 63) - 1;
    if (sl < 0) break;
    const int f = sl / NFP, k = sl - f * NFP;
    const int info = (finfo >> (8 * f)) & 0xff;
    const int kind = info & 3;
    const R nx = (R)m.face_geo[(3 * f) * ld + e], ny = (R)m.face_geo[(3 * f + 1) * ld + e];
    R qp[4], wo[4], jfm[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) wo[c] = w[(c * NP + sl) * ld + e];
    normal_flux_vjp(q, nx, ny, gm1, wo, jfm);
    if (kind == CFD_FACE_INTERIOR) {
      const int nb = m.neighbor[f * ld + e];
      const int nf = (info >> 2) & 3;
      const int kk = ((f == 2) == (nf == 2)) ? NFP - 1 - k : k;
      const int pn = face_node_rt(nf, kk);
      R wd[4], jm[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        qp[c] = qs[(c * NP + pn) * ld + nb];
        wd[c] = w[(c * NP + nf * NFP + kk) * ld + nb] - wo[c];
      }
      iflux_vjp<R, FLUX>(q, qp, nx, ny, gamma, wd, 0, jm);
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[c] += jfm[c] + jm[c];
    } else if (kind == CFD_FACE_SLIP_WALL) {
      const R mn = q[1] * nx + q[2] * ny;
      qp[0] = q[0];
      qp[1] = q[1] - R(2) * mn * nx;
      qp[2] = q[2] - R(2) * mn * ny;
      qp[3] = q[3];
      R jm[4], jp[4];
      iflux_vjp<R, FLUX>(q, qp, nx, ny, gamma, wo, 0, jm);
      iflux_vjp<R, FLUX>(q, qp, nx, ny, gamma, wo, 1, jp);
      // q+ = M q- with M = M^T (the normal momentum reversed)
      const R dm = jp[1] * nx + jp[2] * ny;
      acc[0] += jfm[0] - jm[0] - jp[0];
      acc[1] += jfm[1] - jm[1] - (jp[1] - R(2) * dm * nx);
      acc[2] += jfm[2] - jm[2] - (jp[2] - R(2) * dm * ny);
      acc[3] += jfm[3] - jm[3] - jp[3];
    } else {
      const int row = m.neighbor[f * ld + e] + (kind == CFD_FACE_EXACT_STATE ? k : 0);
#pragma unroll
      for (int c = 0; c < 4; ++c) qp[c] = (R)m.bc_states[row * 4 + c];
      R jm[4];
      iflux_vjp<R, FLUX>(q, qp, nx, ny, gamma, wo, 0, jm);
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[c] += jfm[c] - jm[c];
      if (P.bc_bar) {
        R jp[4];
        iflux_vjp<R, FLUX>(q, qp, nx, ny, gamma, wo, 1, jp);
#pragma unroll
        for (int c = 0; c < 4; ++c) atomicAdd(&P.bc_bar[row * 4 + c], -(double)jp[c]);
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int idx = (c * NP + j) * ld + e;
    sb[idx] = P.accumulate_src ? sb[idx] + acc[c] : acc[c];
  }
}
