// stage_pair.cuh — the fused DG stage kernel, two threads per element.
//
// Thread pair (lanes 2t, 2t+1 of a warp) = one element. The even lane owns
// conserved variables {rho, rho u}, the odd lane {rho v, E}; each keeps a
// 15x2 register tile of the right-hand side, half of the element's 15x4.
//   volume  (dg.py:148-151): both lanes form the node's primitives, each its
//           two rows of the contravariant fluxes, and accumulates
//           -(Dr Ft + Ds Gt) for its two variables. [Dr|Ds] columns are
//           warp-uniform constant-bank reads.
//   surface (dg.py:153-164): the 15 face nodes are dealt out in 8 rounds
//           (even lane: node 2r, odd lane: node 2r+1); each lane evaluates the
//           full interface flux of its node, the pair swaps the two jump
//           components the other lane owns (one shfl.xor per value), and both
//           lift the round's two columns into their tiles.
//   epilogue: SSP-RK3 stage combine (time_integration.py:61-66), cell
//           averages in double (limiting.py:209), the node states completed
//           by one exchange per node for the minima / wave speed / positivity
//           tests; the rare positivity repair (limiting.py:166-200) runs on a
//           shared-memory copy of the element so it adds no registers.
#pragma once
// Included by kernels.cu inside namespace cfd.

template <typename R>
__device__ __forceinline__ R shfl_pair(R v) {
  return __shfl_xor_sync(0xffffffffu, v, 1);
}

// Positivity limiter on one element held in shared memory as s[c*15 + i]
// (same arithmetic as `positivity`, node by node, no register tile).
template <typename R>
__device__ __noinline__ void positivity_smem(R* s, const double* a, double gm1) {
  const double pa = pressure_x(a[0], a[1], a[2], a[3], gm1);
  const double eps = jmin(POSITIVITY_FLOOR, jmin(a[0], pa));
  const double pt = pressure_target<R>(eps, pa, a[3], gm1);
  double rmin = (double)s[0];
#pragma unroll 1
  for (int i = 1; i < NP; ++i) rmin = jmin(rmin, (double)s[i]);
  if (rmin < eps) {
    const double theta = jmin(jmax(xdiv(xsub(a[0], eps), xsub(a[0], rmin)), 0.0), 1.0);
#pragma unroll 1
    for (int k = 0; k < 4 * NP; ++k) s[k] = (R)xadd(a[k / NP], xmul(theta, xsub((double)s[k], a[k / NP])));
  }
  double theta = 1.0;
#pragma unroll 1
  for (int i = 0; i < NP; ++i) {
    const double q0 = s[i], q1 = s[NP + i], q2 = s[2 * NP + i], q3 = s[3 * NP + i];
    if (!(pressure_near(q0, q1, q2, q3, gm1, pt) < pt)) continue;
    const double d0 = xsub(q0, a[0]), d1 = xsub(q1, a[1]), d2 = xsub(q2, a[2]), d3 = xsub(q3, a[3]);
    double lo = 0.0, hi = 1.0;
#pragma unroll 1
    for (int it = 0; it < BISECTION_STEPS; ++it) {
      const double mid = xmul(0.5, xadd(lo, hi));
      const bool ok = pressure_x(xadd(a[0], xmul(mid, d0)), xadd(a[1], xmul(mid, d1)), xadd(a[2], xmul(mid, d2)),
                                 xadd(a[3], xmul(mid, d3)), gm1) >= pt;
      lo = ok ? mid : lo;
      hi = ok ? hi : mid;
    }
    theta = jmin(theta, lo);
  }
  if (theta < 1.0) {
#pragma unroll 1
    for (int k = 0; k < 4 * NP; ++k) s[k] = (R)xadd(a[k / NP], xmul(theta, xsub((double)s[k], a[k / NP])));
  }
}

template <typename R, int FLUX, int MODE, int BS>
__global__ void __launch_bounds__(BS, (sizeof(R) == 4 ? 512 : 384) / BS) stage_pair_kernel(const StageParams P) {
  constexpr int EPB = BS / 2;  // elements per block
  __shared__ R s_rep[BS / 32][4 * NP];  // one element per warp for the rare positivity repair
  const CfdMesh& m = P.m;
  const int ld = m.ld;
  const int half = threadIdx.x & 1;
  const int slot = threadIdx.x >> 1;
  const int e_raw = blockIdx.x * EPB + slot;
  bool live = e_raw < m.num_elements;
  const int e = live ? e_raw : m.num_elements - 1;  // dead lanes still take part in the shuffles
  int inst = 0;
  if (m.instance) inst = m.instance[e];
  if (inst < 0) {  // padding between instances
    live = false;
    inst = 0;
  }
  double dt = 0.0;
  int par = 0;
  if (MODE != MODE_RHS) {
    const CfdControl* c = P.ctl + inst;
    live = live && c->status == CFD_RUN_ACTIVE;
    dt = c->dt;
    par = c->parity;
  }
  Red red;
  red.init();
  const bool warp_live = __any_sync(0xffffffffu, live);
  if (warp_live) {
    const R* src_;
    const R* base_;
    R* dst_;
    if (MODE == MODE_RHS) {
      src_ = (const R*)P.q_in;
      base_ = nullptr;
      dst_ = (R*)P.q_out;
    } else {
      select_buffers<R>(P, par, src_, base_, dst_);
    }
    const R* __restrict__ src = src_;
    const R* __restrict__ base = base_;
    R* __restrict__ dst = dst_;
    const R gamma = (R)P.gamma;
    const R gm1 = gamma - R(1);
    const int c0 = 2 * half;  // first owned variable
    const R* __restrict__ mg = GeoPtr<R>::metric(m);
    const R rx = mg[e], ry = mg[ld + e], sx = mg[2 * ld + e], sy = mg[3 * ld + e];

    R acc[NP][2];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i][0] = acc[i][1] = R(0);

    // ---- volume term (node loop fully unrolled: the [Dr|Ds] entries are
    // compile-time operands; the FP32 form skips the round-off zeros)
    {
      const R* __restrict__ pj = src + e;
      R qn[4];
      R f0a = R(0), f0b = R(0), g0a = R(0), g0b = R(0);
#pragma unroll
      for (int c = 0; c < 4; ++c) qn[c] = pj[(c * NP) * ld];
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        R q[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) q[c] = qn[c];
        if (j + 1 < NP) {  // prefetch the next node
#pragma unroll
          for (int c = 0; c < 4; ++c) qn[c] = pj[(c * NP + j + 1) * ld];
        }
        const Prim<R> w = primitive(q, gm1);
        // rows c0, c0+1 of F = (mx, mx u + p, my u, (E+p) u), G = (my, mx v, my v + p, (E+p) v)
        const R ep = q[3] + w.p;
        const R fa = half ? q[2] * w.u : q[1];
        const R fb = half ? ep * w.u : q[1] * w.u + w.p;
        const R ga = half ? q[2] * w.v + w.p : q[2];
        const R gb = half ? ep * w.v : q[1] * w.v;
        R fta = rx * fa + ry * ga, ftb = rx * fb + ry * gb;
        R gta = sx * fa + sy * ga, gtb = sx * fb + sy * gb;
        if (sizeof(R) == 4) {
          // FP32 form: differentiate F~ - F~(node 0) ([Dr|Ds] annihilate constants),
          // so that a uniform state's volume term is exactly zero; with the
          // rounded tables and metric it would leave a source of one sign in every
          // element of a uniform region, and mass and energy would drift
          if (j == 0) {
            f0a = fta, f0b = ftb, g0a = gta, g0b = gtb;
            continue;
          }
          fta -= f0a, ftb -= f0b, gta -= g0a, gtb -= g0b;
        }
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          if (keep_entry<R>(tab::DR[i][j])) {
            acc[i][0] = fma((R)(-tab::DR[i][j]), fta, acc[i][0]);
            acc[i][1] = fma((R)(-tab::DR[i][j]), ftb, acc[i][1]);
          }
          if (keep_entry<R>(tab::DS[i][j])) {
            acc[i][0] = fma((R)(-tab::DS[i][j]), gta, acc[i][0]);
            acc[i][1] = fma((R)(-tab::DS[i][j]), gtb, acc[i][1]);
          }
        }
      }
    }

    // ---- surface term
    const R* __restrict__ fg = GeoPtr<R>::face(m);
    const int finfo = m.face_info[e];
#pragma unroll 1
    for (int r = 0; r < 8; ++r) {
      const int sl = 2 * r + half;  // this lane's face node slot (15 = none)
      R jump[4] = {R(0), R(0), R(0), R(0)};
      if (sl < 3 * NFP) {
        const int f = sl / NFP, k = sl - NFP * (sl / NFP);
        const int info = (finfo >> (8 * f)) & 0xff;
        const int kind = info & 3;
        const int nf = (info >> 2) & 3;
        const R nx = fg[(3 * f) * ld + e], ny = fg[(3 * f + 1) * ld + e], fs = fg[(3 * f + 2) * ld + e];
        // interior: the neighbour; fixed state: the face's row; exact state: the node's row
        const int nb = (kind != CFD_FACE_SLIP_WALL) ? m.neighbor[f * ld + e] + (kind == CFD_FACE_EXACT_STATE ? k : 0) : 0;
        const double bw = (kind != CFD_FACE_INTERIOR) ? ctab::FACE_W[k] * m.face_hlen[f * ld + e] : 0.0;
        const bool same_order = (f == 2) != (nf == 2);
        const int pn = face_node_rt(nf, same_order ? k : NFP - 1 - k);
        face_node_flux<R, FLUX>(m, src, e, ld, gamma, face_node_rt(f, k), kind, nb, pn, nx, ny, fs, bw, jump, red);
      }
      // swap: the even lane needs jump[0..1] of node 2r+1, the odd lane jump[2..3] of node 2r
      const R s0 = shfl_pair(half ? jump[0] : jump[2]);
      const R s1 = shfl_pair(half ? jump[1] : jump[3]);
      const R ja0 = half ? s0 : jump[0], ja1 = half ? s1 : jump[1];  // node 2r, owned variables
      const R jb0 = half ? jump[2] : s0, jb1 = half ? jump[3] : s1;  // node 2r+1
      const int col = 2 * r;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        const R la = tabv<R>::lift(i, col);
        const R lb = col + 1 < 3 * NFP ? tabv<R>::lift(i, col + 1) : R(0);
        acc[i][0] = fma(lb, jb0, fma(la, ja0, acc[i][0]));
        acc[i][1] = fma(lb, jb1, fma(la, ja1, acc[i][1]));
      }
    }

    if (MODE == MODE_RHS) {
      if (live) {
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          dst[(c0 * NP + i) * ld + e] = acc[i][0];
          dst[((c0 + 1) * NP + i) * ld + e] = acc[i][1];
        }
      }
    } else {
      // ---- SSP-RK3 stage combine
      const R rdt = (R)dt;
#pragma unroll
      for (int i = 0; i < NP; ++i)
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int idx = ((c0 + cc) * NP + i) * ld + e;
          const R v = src[idx] + rdt * acc[i][cc];
          if (P.stage_idx == 1) acc[i][cc] = v;
          else if (P.stage_idx == 2) acc[i][cc] = R(0.75) * base[idx] + R(0.25) * v;
          else acc[i][cc] = stage3_combine(base[idx], v);
        }
#include "stage_epilogue.inc"
    }
  }
  if (!live) red.init();
  if (MODE == MODE_RHS) {
    if (live) {
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (red.b[c] != 0.0) atomicAdd(&P.bflux_out[inst * 4 + c], red.b[c]);
    }
  } else {
    block_commit<BS>(red, live, inst, P.acc, 3, P.stage_idx - 1);
  }
}
