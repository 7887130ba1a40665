// limiter.cuh — the Cockburn-Shu troubled-cell limiter and the Zhang-Shu
// positivity limiter of a stage state (limiting.py:136-216 of CFD-demo), as
// per-element bodies and the one-pass / two-pass kernels that run them.
// Included by common.cuh inside namespace cfd.
#pragma once

// ----------------------------------------------------------- limit kernel ---
struct LimitParams {
  CfdMesh m;
  const CfdControl* ctl;  // null: always active (cfd_limit)
  const void* x0;
  const void* x1;
  void* stage;
  int stage_idx;          // 1..3, or 0 with q = q_io (cfd_limit)
  void* q_io;
  double gamma;
  const double* avg;
  const double* aux;
  CfdStageAcc* acc;       // stage mode
  int32_t* troubled_out;  // cfd_limit mode
  double* pos_out;        // optional [2][ld]: pressure-scaling theta and its critical node
  int* list;              // two-pass form: elements for the rewrite pass, and
  int* count;             // their number (zeroed before the scan)
  uint8_t* flags;         // optional [ld]: troubled-cell indicator per element
};

// Troubled-cell detection of element e (limiting.py:128-151): the scaled
// neighbour differences (Cockburn-Shu coefficients, neighbour or ghost
// averages) and whether a density or energy trace at a face midpoint leaves
// its minmod bound. q is the stage state (element-major rows).
template <typename R, int PHI>
__device__ __forceinline__ bool limit_detect(const LimitParams& P, int e, const R* __restrict__ q, const double a[4],
                                             int finfo, double det_tol, R (&scaled)[3][4]) {
  const CfdMesh& m = P.m;
  const int ld = m.ld;
  bool troubled = false;
  {
      // neighbour / ghost averages (limiting.py:128-133), unfused as in NumPy
      R diff[3][4];
      const double* fgd = m.face_geo;
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        const int kind = (finfo >> (8 * f)) & 3;
        double na[4];
        if (kind == CFD_FACE_INTERIOR) {
          const int nb = m.neighbor[f * ld + e];
#pragma unroll
          for (int c = 0; c < 4; ++c) na[c] = P.avg[c * ld + nb];
        } else if (kind == CFD_FACE_SLIP_WALL) {
          const double nx = fgd[(3 * f) * ld + e], ny = fgd[(3 * f + 1) * ld + e];
          const double mn = xadd(xmul(a[1], nx), xmul(a[2], ny));
          na[0] = a[0];
          na[1] = xsub(a[1], xmul(xmul(2.0, mn), nx));
          na[2] = xsub(a[2], xmul(xmul(2.0, mn), ny));
          na[3] = a[3];
        } else {
          // the ghost average: the fixed state, or the exact state's row after its node rows
          const int row = m.neighbor[f * ld + e] + (kind == CFD_FACE_EXACT_STATE ? NFP : 0);
#pragma unroll
          for (int c = 0; c < 4; ++c) na[c] = m.bc_states[row * 4 + c];
        }
#pragma unroll
        for (int c = 0; c < 4; ++c) diff[f][c] = (R)xsub(na[c], a[c]);
      }
      const R* __restrict__ cs = GeoPtr<R>::cs(m);
#pragma unroll
      for (int f = 0; f < 3; ++f) {
        const int pf = (finfo >> (8 * f + 4)) & 3;
        const R al = cs[f * ld + e], be = cs[(3 + f) * ld + e];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const R pd = pf == 0 ? diff[0][c] : (pf == 1 ? diff[1][c] : diff[2][c]);
          scaled[f][c] = xmul((R)NEIGHBOR_FACTOR, xadd(xmul(al, diff[f][c]), xmul(be, pd)));
        }
      }
      // detection on rho and E at the three face midpoints (limiting.py:147-151)
#pragma unroll
      for (int f = 0; f < 3; ++f) {
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int c = cc == 0 ? 0 : 3;
          const R tr = xsub(q[(c * NP + tab::MID_NODES[f]) * ld + e], (R)a[c]);
          const R ex = abs_(xsub(minmod2(tr, scaled[f][c]), tr));
          troubled |= (double)ex > xmul(det_tol, fabs(a[c]));
        }
      }
      }
  return troubled;
}

// Cockburn-Shu troubled-cell limiter (limiting.py:136-163) followed by the
// positivity limiter (limiting.py:166-200), in place on the stage state, for
// element e of instance inst. PART 0: everything in one pass; PART 1 (scan):
// elements the limiters leave as they are contribute their minima, the others
// are only marked `listed`; PART 2: the rewrite of a listed element.
template <typename R, int PHI, int PART>
__device__ __forceinline__ void limit_body(const LimitParams& P, int e, int par, Red& red, bool& listed) {
  const CfdMesh& m = P.m;
  const int ld = m.ld;
  {
    R* __restrict__ q;
    if (P.stage_idx == 0) {
      q = (R*)P.q_io;
    } else if (P.stage_idx == 2) {
      q = (R*)P.stage;
    } else {
      q = (R*)(par ? P.x0 : P.x1);
    }
    const double gm1 = P.gamma - 1.0;
    double a[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) a[c] = P.avg[c * ld + e];
    const double pa = pressure_x(a[0], a[1], a[2], a[3], gm1);
    const double eps = jmin(POSITIVITY_FLOOR, jmin(a[0], pa));
    const double pt = pressure_target<R>(eps, pa, a[3], gm1);
    const double det_tol = sizeof(R) == 8 ? DETECTION_TOLERANCE : DETECTION_TOLERANCE_FP32;
    const int finfo = m.face_info[e];
    bool troubled = false;
    R scaled[3][4];
    if (PHI != LIM_UNLIMITED) troubled = limit_detect<R, PHI>(P, e, q, a, finfo, det_tol, scaled);
    if (PART != 2 && P.flags) P.flags[e] = troubled ? 1 : 0;
    const double rmin0 = P.aux[e], pmin0 = P.aux[ld + e];
    const bool need_pos = (rmin0 < eps) || (pmin0 < pt);
    if (!troubled && !need_pos) {
      red.kr = dkey(rmin0);
      red.kp = dkey(pmin0);
      if (P.stage_idx == 3) {
        const double d = m.dt_geo[e] / P.aux[2 * ld + e];
        red.kd = dkey(d);
        if (d != d) red.fl |= FLAG_NAN_DT;
      }
    } else {
      if (PART == 1) {  // the scan pass lists the element for the rewrite pass
        listed = true;
        return;
      }
      R s[NP][4];
#pragma unroll
      for (int i = 0; i < NP; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) s[i][c] = q[(c * NP + i) * ld + e];
      if (troubled) {
        // P1 midpoint values, phi-limited deltas, +/- rescaling, linear rebuild
        // (limiting.py:153-162), in NumPy's operation order
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const R ac = (R)a[c];
          R deltas[3];
          R pos = R(0), neg = R(0);
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            R pr = xmul((R)tab::P1MID[f][0], s[0][c]);
#pragma unroll
            for (int i = 1; i < NP; ++i) pr = xadd(pr, xmul((R)tab::P1MID[f][i], s[i][c]));
            pr = xsub(pr, ac);
            R d = R(0);
            if (pr != R(0)) d = xmul(pr, jmin(R(1), phi<R, PHI>(xdiv(scaled[f][c], pr))));
            deltas[f] = d;
            pos = f == 0 ? jmax(d, R(0)) : xadd(pos, jmax(d, R(0)));
            neg = f == 0 ? jmax(-d, R(0)) : xadd(neg, jmax(-d, R(0)));
          }
          const R thp = pos > R(0) ? jmin(R(1), xdiv(neg, pos)) : R(0);
          const R thn = neg > R(0) ? jmin(R(1), xdiv(pos, neg)) : R(0);
#pragma unroll
          for (int f = 0; f < 3; ++f)
            deltas[f] = xsub(xmul(thp, jmax(deltas[f], R(0))), xmul(thn, jmax(-deltas[f], R(0))));
#pragma unroll
          for (int i = 0; i < NP; ++i) {
            R v = xmul((R)tab::LINBASIS[i][0], deltas[0]);
            v = xadd(v, xmul((R)tab::LINBASIS[i][1], deltas[1]));
            v = xadd(v, xmul((R)tab::LINBASIS[i][2], deltas[2]));
            s[i][c] = xadd(ac, v);
          }
        }
        red.tr = 1;
      }
      if (P.pos_out) {
        double th;
        int node;
        positivity<R>(s, a, gm1, &th, &node);
        P.pos_out[e] = th;
        P.pos_out[ld + e] = (double)node;
      } else {
        positivity<R>(s, a, gm1);
      }
#pragma unroll
      for (int i = 0; i < NP; ++i)
#pragma unroll
        for (int c = 0; c < 4; ++c) q[(c * NP + i) * ld + e] = s[i][c];
      double rmin, pmin, lam;
      bool finite;
      element_stats<R>(s, gm1, P.gamma, rmin, pmin, lam, finite);
      if (!finite) red.fl |= FLAG_NONFINITE;
      red.kr = dkey(rmin);
      red.kp = dkey(pmin);
      if (P.stage_idx == 3) {
        const double d = m.dt_geo[e] / lam;
        red.kd = dkey(d);
        if (d != d) red.fl |= FLAG_NAN_DT;
      }
    }
    }
}

template <typename R, int PHI, int BS>
__global__ void __launch_bounds__(BS) limit_kernel(const LimitParams P) {
  const CfdMesh& m = P.m;
  const int e = blockIdx.x * BS + threadIdx.x;
  bool live = e < m.num_elements;
  int inst = 0;
  if (live && m.instance) inst = m.instance[e];
  if (inst < 0) {  // padding between instances
    live = false;
    inst = 0;
  }
  int par = 0;
  if (live && P.ctl) {
    live = P.ctl[inst].status == CFD_RUN_ACTIVE;
    par = P.ctl[inst].parity;
  }
  Red red;
  red.init();
  bool listed = false;
  if (live) limit_body<R, PHI, 0>(P, e, par, red, listed);
  if (P.stage_idx == 0) {
    if (live && red.tr) atomicAdd(&P.troubled_out[inst], red.tr);
  } else {
    block_commit<BS>(red, live, inst, P.acc, 3, P.stage_idx - 1);
  }
}

// The same limiter in two passes. The scan runs the detection for every
// element with few registers, commits the minima (and CFL step) of the
// elements the limiters leave as they are, and lists the others (troubled,
// or below the positivity floor: a small minority); the rewrite pass then
// runs the full reconstruction and positivity scaling on the listed
// elements only, committing their minima one element at a time. Same
// arithmetic, same results as limit_kernel.
// The scan of the elements e0 .. e0 + BS - 1 by a block of BS threads.
template <typename R, int PHI, int BS>
__device__ __forceinline__ void limit_scan_body(const LimitParams& P, const int e0) {
  const CfdMesh& m = P.m;
  const int e = e0 + threadIdx.x;
  bool live = e < m.num_elements;
  int inst = 0;
  if (live && m.instance) inst = m.instance[e];
  if (inst < 0) {
    live = false;
    inst = 0;
  }
  int par = 0;
  if (live && P.ctl) {
    live = P.ctl[inst].status == CFD_RUN_ACTIVE;
    par = P.ctl[inst].parity;
  }
  Red red;
  red.init();
  bool listed = false;
  if (live) limit_body<R, PHI, 1>(P, e, par, red, listed);
  warp_list_append(P.list, P.count, listed, e);
  if (listed) red.init();
  if (P.stage_idx == 0) {
    if (live && red.tr) atomicAdd(&P.troubled_out[inst], red.tr);
  } else {
    block_commit<BS>(red, live && !listed, inst, P.acc, 3, P.stage_idx - 1);
  }
}

template <typename R, int PHI, int BS>
__global__ void __launch_bounds__(BS) limit_scan_kernel(const LimitParams P) {
  limit_scan_body<R, PHI, BS>(P, blockIdx.x * BS);
}

// The rewrite of one listed element by the four lanes base .. base + 3 of a
// warp, lane c owning conserved variable c; the same results, bit for bit,
// as limit_body's rewrite (PART 2). The detection and the troubled-cell
// reconstruction run per variable in limit_body's operation order. The
// positivity limiter and the element statistics deal node i out to lane
// i % 4 (each lane gathers the node's four values by shuffles): the node
// tests and the 60-step bisections then run four at a time, and their
// results are combined by order-independent reductions (min / max, and for
// the critical node the smallest index attaining the minimum theta, as the
// sequential loop finds it). The element's reductions end in lane c = 0.
template <typename R, int PHI>
__device__ __forceinline__ void limit_rewrite_quad(const LimitParams& P, int e, int par, int c, unsigned qmask,
                                                   int base, Red& red) {
  const CfdMesh& m = P.m;
  const int ld = m.ld;
  R* __restrict__ q;
  if (P.stage_idx == 0) {
    q = (R*)P.q_io;
  } else if (P.stage_idx == 2) {
    q = (R*)P.stage;
  } else {
    q = (R*)(par ? P.x0 : P.x1);
  }
  const double gm1 = P.gamma - 1.0;
  double a[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) a[k] = P.avg[k * ld + e];
  const double pa = pressure_x(a[0], a[1], a[2], a[3], gm1);
  const double eps = jmin(POSITIVITY_FLOOR, jmin(a[0], pa));
  const double pt = pressure_target<R>(eps, pa, a[3], gm1);
  const double det_tol = sizeof(R) == 8 ? DETECTION_TOLERANCE : DETECTION_TOLERANCE_FP32;
  const int finfo = m.face_info[e];
  bool troubled = false;
  R scaled[3][4];
  if (PHI != LIM_UNLIMITED) troubled = limit_detect<R, PHI>(P, e, q, a, finfo, det_tol, scaled);
  const double rmin0 = P.aux[e], pmin0 = P.aux[ld + e];
  const bool need_pos = (rmin0 < eps) || (pmin0 < pt);
  if (!troubled && !need_pos) {  // (the scan lists no such element)
    if (c == 0) {
      red.kr = dkey(rmin0);
      red.kp = dkey(pmin0);
      if (P.stage_idx == 3) {
        const double d = m.dt_geo[e] / P.aux[2 * ld + e];
        red.kd = dkey(d);
        if (d != d) red.fl |= FLAG_NAN_DT;
      }
    }
    return;
  }
  const double ac_d = c == 0 ? a[0] : (c == 1 ? a[1] : (c == 2 ? a[2] : a[3]));
  R s[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) s[i] = q[(c * NP + i) * ld + e];
  if (troubled) {
    // P1 midpoint values, phi-limited deltas, +/- rescaling, linear rebuild
    // (limiting.py:153-162), in NumPy's operation order, for variable c
    const R ac = (R)ac_d;
    R deltas[3];
    R pos = R(0), neg = R(0);
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const R sc = c == 0 ? scaled[f][0] : (c == 1 ? scaled[f][1] : (c == 2 ? scaled[f][2] : scaled[f][3]));
      R pr = xmul((R)tab::P1MID[f][0], s[0]);
#pragma unroll
      for (int i = 1; i < NP; ++i) pr = xadd(pr, xmul((R)tab::P1MID[f][i], s[i]));
      pr = xsub(pr, ac);
      R d = R(0);
      if (pr != R(0)) d = xmul(pr, jmin(R(1), phi<R, PHI>(xdiv(sc, pr))));
      deltas[f] = d;
      pos = f == 0 ? jmax(d, R(0)) : xadd(pos, jmax(d, R(0)));
      neg = f == 0 ? jmax(-d, R(0)) : xadd(neg, jmax(-d, R(0)));
    }
    const R thp = pos > R(0) ? jmin(R(1), xdiv(neg, pos)) : R(0);
    const R thn = neg > R(0) ? jmin(R(1), xdiv(pos, neg)) : R(0);
#pragma unroll
    for (int f = 0; f < 3; ++f) deltas[f] = xsub(xmul(thp, jmax(deltas[f], R(0))), xmul(thn, jmax(-deltas[f], R(0))));
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      R v = xmul((R)tab::LINBASIS[i][0], deltas[0]);
      v = xadd(v, xmul((R)tab::LINBASIS[i][1], deltas[1]));
      v = xadd(v, xmul((R)tab::LINBASIS[i][2], deltas[2]));
      s[i] = xadd(ac, v);
    }
    red.tr = c == 0 ? 1 : 0;
  }
  // ---- positivity (positivity() in common.cuh): density scaling
  double rmin = (double)s[0];
#pragma unroll
  for (int i = 1; i < NP; ++i) rmin = jmin(rmin, (double)s[i]);
  rmin = __shfl_sync(qmask, rmin, base);  // lane 0 holds the density
  if (rmin < eps) {
    const double span = xsub(a[0], rmin);
    const double theta = jmin(jmax(xdiv(xsub(a[0], eps), span), 0.0), 1.0);
#pragma unroll
    for (int i = 0; i < NP; ++i) s[i] = (R)xadd(ac_d, xmul(theta, xsub((double)s[i], ac_d)));
  }
  // node tests: lane i % 4 tests node i and keeps its four values for the bisection
  R keep[4][4];
  unsigned need = 0;
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    R v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = __shfl_sync(qmask, s[i], base + k);
    if ((i & 3) == c) {
#pragma unroll
      for (int k = 0; k < 4; ++k) keep[i >> 2][k] = v[k];
      if (pressure_near(v[0], v[1], v[2], v[3], gm1, pt) < pt) need |= 1u << i;
    }
  }
  need |= __shfl_xor_sync(qmask, need, 1);
  need |= __shfl_xor_sync(qmask, need, 2);
  double th = 1.0;
  int node = -1;
  if (need) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int i = 4 * k + c;
      if (i >= NP || !((need >> i) & 1u)) continue;
      const double d0 = xsub((double)keep[k][0], a[0]), d1 = xsub((double)keep[k][1], a[1]);
      const double d2 = xsub((double)keep[k][2], a[2]), d3 = xsub((double)keep[k][3], a[3]);
      double lo = 0.0, hi = 1.0;
#pragma unroll 1
      for (int it = 0; it < BISECTION_STEPS; ++it) {
        const double mid = xmul(0.5, xadd(lo, hi));
        const bool ok = pressure_x(xadd(a[0], xmul(mid, d0)), xadd(a[1], xmul(mid, d1)), xadd(a[2], xmul(mid, d2)),
                                   xadd(a[3], xmul(mid, d3)), gm1) >= pt;
        lo = ok ? mid : lo;
        hi = ok ? hi : mid;
      }
      if (lo < th) {  // ascending i within the lane: the smallest index of a tie stays
        th = lo;
        node = i;
      }
    }
#pragma unroll
    for (int off = 1; off <= 2; off <<= 1) {
      const double oth = __shfl_xor_sync(qmask, th, off);
      const int onode = __shfl_xor_sync(qmask, node, off);
      if (oth < th || (oth == th && onode >= 0 && (node < 0 || onode < node))) {
        th = oth;
        node = onode;
      }
    }
    if (th < 1.0) {
#pragma unroll
      for (int i = 0; i < NP; ++i) s[i] = (R)xadd(ac_d, xmul(th, xsub((double)s[i], ac_d)));
    }
  }
  if (P.pos_out && c == 0) {
    P.pos_out[e] = th;
    P.pos_out[ld + e] = (double)node;
  }
#pragma unroll
  for (int i = 0; i < NP; ++i) q[(c * NP + i) * ld + e] = s[i];
  // ---- element statistics (element_stats in common.cuh), node i in lane i % 4
  double rmn = INFINITY, pmn = INFINITY, lam = -INFINITY;
  bool finite = true, lam_nan = false;
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    R v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = __shfl_sync(qmask, s[i], base + k);
    if ((i & 3) == c) {
      const double p = node_pressure<R>(v[0], v[1], v[2], v[3], gm1, POSITIVITY_FLOOR);
      rmn = fmin(rmn, (double)v[0]);
      pmn = fmin(pmn, p);
      const double sp = wave_speed<R>(v[0], v[1], v[2], v[3], P.gamma);
      lam_nan |= (sp != sp);
      lam = fmax(lam, sp);
#pragma unroll
      for (int k = 0; k < 4; ++k) finite &= finite_(v[k]);
    }
  }
  unsigned bits = (finite ? 1u : 0u) | (lam_nan ? 2u : 0u);
#pragma unroll
  for (int off = 1; off <= 2; off <<= 1) {
    rmn = fmin(rmn, __shfl_xor_sync(qmask, rmn, off));
    pmn = fmin(pmn, __shfl_xor_sync(qmask, pmn, off));
    lam = fmax(lam, __shfl_xor_sync(qmask, lam, off));
    const unsigned ob = __shfl_xor_sync(qmask, bits, off);
    bits = ((bits & ob) & 1u) | ((bits | ob) & 2u);
  }
  if (bits & 2u) lam = NAN;
  if (c == 0) {
    if (!(bits & 1u)) red.fl |= FLAG_NONFINITE;
    red.kr = dkey(rmn);
    red.kp = dkey(pmn);
    if (P.stage_idx == 3) {
      const double d = m.dt_geo[e] / lam;
      red.kd = dkey(d);
      if (d != d) red.fl |= FLAG_NAN_DT;
    }
  }
}

// The rewrite of the listed elements, four lanes per element, spread over
// every thread of the grid (the block size is a multiple of 4, so the four
// lanes of an element are always in one warp and take the same trips).
template <typename R, int PHI>
__device__ __forceinline__ void limit_rewrite_body(const LimitParams& P) {
  const CfdMesh& m = P.m;
  const int n = *(volatile int*)P.count;
  const int lane = threadIdx.x & 31, c = lane & 3, base = lane & ~3;
  const unsigned qmask = 0xfu << base;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 2; t < n; t += (gridDim.x * blockDim.x) >> 2) {
    const int e = P.list[t];
    const int inst = m.instance ? m.instance[e] : 0;
    const int par = P.ctl ? P.ctl[inst].parity : 0;
    Red red;
    red.init();
    limit_rewrite_quad<R, PHI>(P, e, par, c, qmask, base, red);
    if (c != 0) continue;
    if (P.stage_idx == 0) {
      if (red.tr) atomicAdd(&P.troubled_out[inst], red.tr);
    } else {
      commit_one(red, P.acc + 3 * inst + (P.stage_idx - 1));
    }
  }
}

template <typename R, int PHI>
__global__ void __launch_bounds__(64) limit_rewrite_kernel(const LimitParams P) {
  limit_rewrite_body<R, PHI>(P);
}
