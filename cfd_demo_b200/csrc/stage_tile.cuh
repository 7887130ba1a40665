// stage_tile.cuh — the fused DG stage kernel with shared-memory element tiles.
//
// Same arithmetic as stage_pair_kernel (two threads per element, the even lane
// owning {rho, rho u}, the odd lane {rho v, E}), but every block first stages
// its EPB elements into shared memory with asynchronous copies so that the
// long-latency global loads are all in flight at once instead of trickling
// through the dependent arithmetic:
//   group A  own state rows [60][EPB] and geometry rows (16-byte cp.async)
//   group B  the neighbours' face traces (4/8-byte cp.async, one per value)
//            and, from stage 2 on, the stage base rows; these complete while
//            the volume term runs from shared memory
// then the surface rounds, the RK combine and the epilogue read shared memory
// and only the stage result is stored to global memory (coalesced).
// Blocks are instance-uniform: several meshes are laid out with every
// instance starting at a multiple of 64 elements (operators.py).
#pragma once
// Included by kernels.cu inside namespace cfd.

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_small(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(N) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Shared-memory layout of one block (all offsets in elements of R, 16-byte
// aligned). With FACE_JOBS the neighbour-trace region holds the traces of the
// owned out-of-tile faces by face (TRC, [3 EPB][NFP][4]) and a jump region
// (JMP, [EPB][3 NFP][4]) and the owned-face list follow.
template <typename R, int EPB, bool STAGE_BASE, bool FACE_JOBS = false>
struct TileLayout {
  // row stride of the [60][.] state tiles: 30 rows apart (the two lanes'
  // variables) must fall 16 banks apart, and rows must stay 16-byte aligned
  static constexpr int S = sizeof(R) == 4 ? EPB + 8 : EPB + 4;
  static constexpr int OWN = 0;
  static constexpr int BASE = OWN + 60 * S;
  // base rows unpadded; the odd lane's rows (30..59) sit 16 words further on,
  // so the two lanes of a warp still read different banks (saves the padding:
  // four 64-element FP32 blocks with base rows fit an SM's shared memory)
  static __device__ __forceinline__ int base_at(int row, int col) { return row * EPB + (row >= 30 ? 16 : 0) + col; }
  static constexpr int NBR = BASE + (STAGE_BASE ? 60 * EPB + 16 : 0);  // [8 rounds][4 vars][EPB][2 lanes]
  static constexpr int JMP = NBR + (FACE_JOBS ? 3 * EPB * NFP * 4 : 64 * EPB);
  static constexpr int GEO = JMP + (FACE_JOBS ? EPB * 3 * NFP * 4 : 0);  // [13][S]: rx ry sx sy, (nx ny fs) x 3
  static constexpr int INT_BYTES_OFF = (GEO + 13 * S) * (int)sizeof(R);  // int rows [4][EPB]
  static constexpr int FACES_BYTES_OFF = INT_BYTES_OFF + 4 * EPB * 4;    // owned faces [3 EPB] + count
  static constexpr int BYTES = FACES_BYTES_OFF + (FACE_JOBS ? 3 * EPB * 4 + 16 : 0);
};

// FACE_JOBS: the owner of a face computes its flux once for both sides. The
// block lists the faces it owns (every boundary or out-of-tile face of its
// elements, and each in-tile interior face once, by its lower-numbered
// element), deals their face nodes out to all threads as jobs, and writes the
// lifted-jump inputs of both elements into the jump region; a face F-hat of
// the neighbour's side is -F-hat with its own normal, so the neighbour's
// input is fs_nb (F-hat - F(q+).n).
template <typename R> struct NodeFlux3 { R fhat[4], fm[4], fp[4]; };
template <typename R, int FLUX>
__device__ __noinline__ NodeFlux3<R> trace_flux3_call(R m0, R m1, R m2, R m3, R p0, R p1, R p2, R p3, R nx, R ny,
                                                      R gamma) {
  const R qm[4] = {m0, m1, m2, m3}, qp[4] = {p0, p1, p2, p3};
  NodeFlux3<R> o;
  trace_flux3<R, FLUX>(qm, qp, nx, ny, gamma, o.fhat, o.fm, o.fp);
  return o;
}

// y0 += a x0, y1 += a x1. With PACK in the FP32 form: one packed
// fma.rn.f32x2 (sm_100), each lane rounded exactly like a scalar fmaf, so the
// results are bitwise those of the two scalar FMAs in one issue slot.
template <typename R, bool PACK>
__device__ __forceinline__ void fma_pair(R a, R x0, R x1, R& y0, R& y1) {
  if constexpr (PACK && sizeof(R) == 4) {
    const float2 r = __ffma2_rn(make_float2(a, a), make_float2(x0, x1), make_float2(y0, y1));
    y0 = r.x;
    y1 = r.y;
  } else {
    y0 = fma(a, x0, y0);
    y1 = fma(a, x1, y1);
  }
}

// (y0, y1) = a (f0, f1) + b (g0, g1): a contravariant flux pair. The FP32 form
// fixes the rounding as fma(b, g, a f), one packed FMUL2 + FFMA2 with PACK
// (bitwise the scalar pair); FP64 keeps the plain expression.
template <typename R, bool PACK>
__device__ __forceinline__ void lin_pair(R a, R b, R f0, R f1, R g0, R g1, R& y0, R& y1) {
  if constexpr (sizeof(R) == 4) {
    if constexpr (PACK) {
      const float2 r = __ffma2_rn(make_float2(b, b), make_float2(g0, g1),
                                  __fmul2_rn(make_float2(a, a), make_float2(f0, f1)));
      y0 = r.x;
      y1 = r.y;
    } else {
      y0 = fmaf(b, g0, a * f0);
      y1 = fmaf(b, g1, a * f1);
    }
  } else {
    y0 = a * f0 + b * g0;
    y1 = a * f1 + b * g1;
  }
}
// (y0, y1) -= (d0, d1), one packed FADD2 of the negated pair with PACK.
template <typename R, bool PACK>
__device__ __forceinline__ void sub_pair(R& y0, R& y1, R d0, R d1) {
  if constexpr (PACK && sizeof(R) == 4) {
    const float2 r = __fadd2_rn(make_float2(y0, y1), make_float2(-d0, -d1));
    y0 = r.x;
    y1 = r.y;
  } else {
    y0 -= d0;
    y1 -= d1;
  }
}

// SSP-RK3 stage combine of a lane's pair of values: v = own + dt acc, then
// stage 1: v; stage 2: 3/4 b + 1/4 v; stage 3: b + 2/3 (v - b). The FP32 form
// fixes the roundings (fma(dt, acc, own), fma(1/4, v, 3/4 b), fma(2/3, v - b,
// b)), as packed FP32x2 operations with PACK (bitwise the scalar pair); FP64
// keeps the reference's expressions.
template <typename R, bool PACK>
__device__ __forceinline__ void combine_pair(int stage, R rdt, R o0, R o1, R b0, R b1, R& a0, R& a1) {
  if constexpr (sizeof(R) == 4) {
    if constexpr (PACK) {
      const float2 v = __ffma2_rn(make_float2(rdt, rdt), make_float2(a0, a1), make_float2(o0, o1));
      float2 r = v;
      if (stage == 2)
        r = __ffma2_rn(make_float2(0.25f, 0.25f), v, __fmul2_rn(make_float2(0.75f, 0.75f), make_float2(b0, b1)));
      else if (stage == 3)
        r = __ffma2_rn(make_float2(2.0f / 3.0f, 2.0f / 3.0f), __fadd2_rn(v, make_float2(-b0, -b1)),
                       make_float2(b0, b1));
      a0 = r.x;
      a1 = r.y;
    } else {
      const float v0 = fmaf(rdt, a0, o0), v1 = fmaf(rdt, a1, o1);
      if (stage == 1) a0 = v0, a1 = v1;
      else if (stage == 2) a0 = fmaf(0.25f, v0, 0.75f * b0), a1 = fmaf(0.25f, v1, 0.75f * b1);
      else a0 = fmaf(2.0f / 3.0f, v0 - b0, b0), a1 = fmaf(2.0f / 3.0f, v1 - b1, b1);
    }
  } else {
    const R v0 = o0 + rdt * a0, v1 = o1 + rdt * a1;
    if (stage == 1) a0 = v0, a1 = v1;
    else if (stage == 2) a0 = R(0.75) * b0 + R(0.25) * v0, a1 = R(0.75) * b1 + R(0.25) * v1;
    else a0 = stage3_combine(b0, v0), a1 = stage3_combine(b1, v1);
  }
}
// (j0, j1) = s ((m0, m1) - (h0, h1)), packed with PACK (bitwise the scalar pair).
template <typename R, bool PACK>
__device__ __forceinline__ void jump_pair(R s, R m0, R m1, R h0, R h1, R& j0, R& j1) {
  if constexpr (PACK && sizeof(R) == 4) {
    const float2 r = __fmul2_rn(make_float2(s, s), __fadd2_rn(make_float2(m0, m1), make_float2(-h0, -h1)));
    j0 = r.x;
    j1 = r.y;
  } else {
    j0 = s * (m0 - h0);
    j1 = s * (m1 - h1);
  }
}

// The interface flux of one face node as an out-of-line call (CALL_FLUX):
// the eight unrolled face rounds then share one copy of the flux code, which
// keeps the kernel's instruction footprint small, while the LIFT columns stay
// immediates.
template <typename R> struct NodeFlux { R fhat[4], fm[4]; };
template <typename R, int FLUX>
__device__ __noinline__ NodeFlux<R> trace_flux_call(R m0, R m1, R m2, R m3, R p0, R p1, R p2, R p3, R nx, R ny,
                                                    R gamma) {
  const R qm[4] = {m0, m1, m2, m3}, qp[4] = {p0, p1, p2, p3};
  NodeFlux<R> o;
  trace_flux<R, FLUX>(qm, qp, nx, ny, gamma, o.fhat, o.fm);
  return o;
}

// MINB: resident blocks per SM the register allocation must allow (the
// default shapes: 512 / 384 threads per SM for FP32 / FP64; the autotuner
// also tries a denser one, trading registers for occupancy). UNROLL_FACES:
// the FP32 form unrolls the 8 face rounds so the LIFT columns are immediates
// (more code: 8 inlined flux evaluations); without it the rounds stay rolled
// and LIFT comes from the constant bank, as in the FP64 form. PACK: the
// [Dr|Ds] and LIFT contractions of the FP32 form as packed FP32x2 FMAs over
// the lane's two variables (no effect in FP64); every launched FP32 shape
// packs except the scalar reference shapes. CALL_FLUX: the face-node flux
// as a call instead of eight inlined copies (FP32 form).
// The stage work of one tile (EPB consecutive elements) by one block of
// 2 EPB threads: the body of stage_tile_kernel, and of the persistent batch
// kernel, whose blocks loop over tiles.
template <typename R, int FLUX, int MODE, int EPB, bool STAGE_BASE, bool UNROLL_FACES = true, bool PACK = false,
          bool CALL_FLUX = false, bool FACE_JOBS = false, bool VROLL = false>
__device__ __forceinline__ void stage_tile_body(const StageParams& P, const int tile) {
  constexpr int BS = 2 * EPB;
  using L = TileLayout<R, EPB, STAGE_BASE, FACE_JOBS>;
  constexpr int S = L::S;
  constexpr int VEC = 16 / (int)sizeof(R);  // elements per 16-byte chunk
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* t_own = reinterpret_cast<R*>(smem_raw) + L::OWN;
  R* t_base = reinterpret_cast<R*>(smem_raw) + L::BASE;
  R* t_nbr = reinterpret_cast<R*>(smem_raw) + L::NBR;
  R* t_geo = reinterpret_cast<R*>(smem_raw) + L::GEO;
  int* t_int = reinterpret_cast<int*>(smem_raw + L::INT_BYTES_OFF);
  R* t_jmp = reinterpret_cast<R*>(smem_raw) + L::JMP;  // FACE_JOBS: [EPB][3 NFP][4]
  int* t_faces = reinterpret_cast<int*>(smem_raw + L::FACES_BYTES_OFF);  // FACE_JOBS: owned faces, count last
  __shared__ R s_rep[BS / 32][4 * NP];  // one element per warp for the rare positivity repair

  const CfdMesh& m = P.m;
  const int ld = m.ld;
  const int K = m.num_elements;
  const int tid = threadIdx.x;
  const int half = tid & 1;
  const int slot = tid >> 1;
  const int e0 = tile * EPB;
  const int e = e0 + slot;
  // block-uniform instance and loop state
  const int inst_raw = m.instance ? m.instance[e0] : 0;
  bool block_live = inst_raw >= 0;  // a block of padding between instances does nothing
  const int inst = block_live ? inst_raw : 0;
  double dt = 0.0;
  int par = 0;
  if (MODE != MODE_RHS && block_live) {
    const CfdControl* c = P.ctl + inst;
    block_live = c->status == CFD_RUN_ACTIVE;
    dt = c->dt;
    par = c->parity;
  }
  const bool live = block_live && e < K && (m.instance == nullptr || m.instance[e] == inst);
  Red red;
  red.init();

  if (block_live) {
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
    const bool has_base = MODE != MODE_RHS && P.stage_idx >= 2;

    // ---- group A: own state rows and geometry rows
    {
      constexpr int CPR = EPB / VEC;  // chunks per row
      for (int ch = tid; ch < 60 * CPR; ch += BS) {
        const int row = ch / CPR, col = (ch - row * CPR) * VEC;
        cp_async16(&t_own[row * S + col], src + (size_t)row * ld + e0 + col);
      }
      const R* mg = GeoPtr<R>::metric(m);
      const R* fg = GeoPtr<R>::face(m);
      for (int ch = tid; ch < 13 * CPR; ch += BS) {
        const int row = ch / CPR, col = (ch - row * CPR) * VEC;
        const R* g = row < 4 ? mg + (size_t)row * ld : fg + (size_t)(row - 4) * ld;
        cp_async16(&t_geo[row * S + col], g + e0 + col);
      }
      constexpr int ICPR = EPB / 4;
      for (int ch = tid; ch < 4 * ICPR; ch += BS) {
        const int row = ch / ICPR, col = (ch - row * ICPR) * 4;
        const int* g = row == 0 ? m.face_info : m.neighbor + (size_t)(row - 1) * ld;
        cp_async16(&t_int[row * EPB + col], g + e0 + col);
      }
      cp_async_commit();
      if (!STAGE_BASE && MODE != MODE_RHS && P.stage_idx >= 2) {
        // the stage base rows are read in the combine, long after this point:
        // bring the block's rows into L2 now (one 128-byte line per request)
        constexpr int LPR = (EPB * (int)sizeof(R) + 127) / 128;  // lines per row
        for (int i = tid; i < 60 * LPR; i += BS) {
          const int row = i / LPR, ln = i - row * LPR;
          prefetch_l2(reinterpret_cast<const char*>(base + (size_t)row * ld + e0) + 128 * ln);
        }
      }
      cp_async_wait<0>();
      __syncthreads();
      if (MODE == MODE_LIMITED && P.tape_src) {  // adjoint tape: the stage input, coalesced
        R* __restrict__ ts = (R*)P.tape_src;
        for (int i = tid; i < 60 * EPB; i += BS) {
          const int row = i / EPB, col = i - row * EPB;
          if (e0 + col < K) ts[(size_t)row * ld + e0 + col] = t_own[row * S + col];
        }
      }
    }
    // ---- group B: neighbour face traces (this lane's two variables) and the base rows
    const int finfo = t_int[slot];
    int nfaces = 0;
    if constexpr (FACE_JOBS) {
      // the owned faces, in a fixed order: lanes of element slot s test faces
      // {0, 1} (even lane) and {2} (odd lane); warp prefix sums give the slots
      unsigned own = 0;
      if (live) {
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const int f = half ? 2 : q;
          if (half && q == 1) break;
          const int info = (finfo >> (8 * f)) & 0xff;
          bool mine = true;
          if ((info & 3) == CFD_FACE_INTERIOR) {
            const int nb = t_int[(1 + f) * EPB + slot];
            mine = nb - e0 < 0 || nb - e0 >= EPB || nb > e;
          }
          if (mine) own |= 1u << q;
        }
      }
      const int cnt = __popc(own);
      const int lane = tid & 31, warp = tid >> 5;
      int pre = cnt;  // inclusive warp prefix
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, pre, o);
        if (lane >= o) pre += v;
      }
      __shared__ int s_wsum[BS / 32];
      if (lane == 31) s_wsum[warp] = pre;
      __syncthreads();
      int off = pre - cnt;
      for (int w = 0; w < warp; ++w) off += s_wsum[w];
      for (int q = 0; q < 2; ++q)
        if ((own >> q) & 1u) t_faces[off++] = slot | ((half ? 2 : q) << 8);
      nfaces = 0;
      for (int w = 0; w < BS / 32; ++w) nfaces += s_wsum[w];
      __syncthreads();
      // traces of the owned out-of-tile faces: TRC[face][k][c]
      for (int i = tid; i < nfaces * NFP * 4; i += BS) {
        const int fi = i / (NFP * 4), kc = i - fi * (NFP * 4), k = kc >> 2, c = kc & 3;
        const int fe = t_faces[fi], os = fe & 0xff, f = fe >> 8;
        const int info = (t_int[os] >> (8 * f)) & 0xff;
        if ((info & 3) != CFD_FACE_INTERIOR) continue;
        const int nb = t_int[(1 + f) * EPB + os];
        if (nb - e0 >= 0 && nb - e0 < EPB) continue;
        const int nf = (info >> 2) & 3;
        const bool same_order = (f == 2) != (nf == 2);
        const int pn = face_node_rt(nf, same_order ? k : NFP - 1 - k);
        cp_async_small<sizeof(R)>(&t_nbr[i], src + (size_t)(c * NP + pn) * ld + nb);
      }
    } else if (live) {
#pragma unroll
      for (int sl = 0; sl < 3 * NFP; ++sl) {
        const int f = sl / NFP, k = sl % NFP;
        const int info = (finfo >> (8 * f)) & 0xff;
        if ((info & 3) != CFD_FACE_INTERIOR) continue;
        const int nf = (info >> 2) & 3;
        const int nb = t_int[(1 + f) * EPB + slot];
        const bool same_order = (f == 2) != (nf == 2);
        const int pn = face_node_rt(nf, same_order ? k : NFP - 1 - k);
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int c = 2 * half + cc;
          cp_async_small<sizeof(R)>(&t_nbr[(((sl >> 1) * 4 + c) * EPB + slot) * 2 + (sl & 1)],
                                    src + (size_t)(c * NP + pn) * ld + nb);
        }
      }
    }
    if (STAGE_BASE && has_base) {
      constexpr int CPR = EPB / VEC;
      for (int ch = tid; ch < 60 * CPR; ch += BS) {
        const int row = ch / CPR, col = (ch - row * CPR) * VEC;
        cp_async16(&t_base[L::base_at(row, col)], base + (size_t)row * ld + e0 + col);
      }
    }
    cp_async_commit();

    const R gamma = (R)P.gamma;
    const R gm1 = gamma - R(1);
    const int c0 = 2 * half;
    const R rx = t_geo[0 * S + slot], ry = t_geo[1 * S + slot], sx = t_geo[2 * S + slot], sy = t_geo[3 * S + slot];
    R acc[NP][2];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i][0] = acc[i][1] = R(0);

    // ---- volume term from the own tile (dg.py:148-151)
    // the contravariant fluxes F~, G~ of this lane's two variables at node j
    auto node_flux = [&](int j, R& fta, R& ftb, R& gta, R& gtb) {
      R q[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) q[c] = t_own[(c * NP + j) * S + slot];
      const Prim<R> w = primitive(q, gm1);
      const R ep = q[3] + w.p;
      const R fa = half ? q[2] * w.u : q[1];
      const R fb = half ? ep * w.u : q[1] * w.u + w.p;
      const R ga = half ? q[2] * w.v + w.p : q[2];
      const R gb = half ? ep * w.v : q[1] * w.v;
      lin_pair<R, PACK>(rx, ry, fa, fb, ga, gb, fta, ftb);
      lin_pair<R, PACK>(sx, sy, fa, fb, ga, gb, gta, gtb);
    };
    R f0a = R(0), f0b = R(0), g0a = R(0), g0b = R(0);
    if constexpr (VROLL) {
      // the node loop kept rolled: [Dr|Ds] columns from the constant bank at a
      // warp-uniform index, every entry taken (a fifteenth of the unrolled
      // loop's code, for 130 more packed FMAs per lane in the FP32 form)
      if (sizeof(R) == 4) node_flux(0, f0a, f0b, g0a, g0b);
#pragma unroll 1
      for (int j = sizeof(R) == 4 ? 1 : 0; j < NP; ++j) {
        R fta, ftb, gta, gtb;
        node_flux(j, fta, ftb, gta, gtb);
        if (sizeof(R) == 4) {
          sub_pair<R, PACK>(fta, ftb, f0a, f0b);
          sub_pair<R, PACK>(gta, gtb, g0a, g0b);
        }
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          fma_pair<R, PACK>(-tabv<R>::dr(i, j), fta, ftb, acc[i][0], acc[i][1]);
          fma_pair<R, PACK>(-tabv<R>::ds(i, j), gta, gtb, acc[i][0], acc[i][1]);
        }
      }
    } else {
#pragma unroll
      for (int j = 0; j < NP; ++j) {
        R fta, ftb, gta, gtb;
        node_flux(j, fta, ftb, gta, gtb);
        if (sizeof(R) == 4) {
          // FP32 form: differentiate F~ - F~(node 0) ([Dr|Ds] annihilate constants),
          // so that a uniform state's volume term is exactly zero; with the
          // rounded tables and metric it would leave a source of one sign in every
          // element of a uniform region, and mass and energy would drift
          if (j == 0) {
            f0a = fta, f0b = ftb, g0a = gta, g0b = gtb;
            continue;
          }
          sub_pair<R, PACK>(fta, ftb, f0a, f0b);
          sub_pair<R, PACK>(gta, gtb, g0a, g0b);
        }
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          if (keep_entry<R>(tab::DR[i][j])) fma_pair<R, PACK>((R)(-tab::DR[i][j]), fta, ftb, acc[i][0], acc[i][1]);
          if (keep_entry<R>(tab::DS[i][j])) fma_pair<R, PACK>((R)(-tab::DS[i][j]), gta, gtb, acc[i][0], acc[i][1]);
        }
      }
    }

    cp_async_wait<0>();
    __syncthreads();

    if constexpr (FACE_JOBS) {
      // ---- surface term (dg.py:153-164) by face-node jobs: each owned face's
      // nodes once, writing the lifted-jump inputs of both sides
      for (int j = tid; j < nfaces * NFP; j += BS) {
        const int fi = j / NFP, k = j - fi * NFP;
        const int fe = t_faces[fi], os = fe & 0xff, f = fe >> 8;
        const int info = (t_int[os] >> (8 * f)) & 0xff;
        const int kind = info & 3;
        const R nx = t_geo[(4 + 3 * f) * S + os], ny = t_geo[(5 + 3 * f) * S + os];
        const R fs = t_geo[(6 + 3 * f) * S + os];
        const int n = face_node_rt(f, k);
        R qm[4], qp[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) qm[c] = t_own[(c * NP + n) * S + os];
        int ns = -1, nslot = 0;  // in-tile neighbour: its slot and jump slot
        if (kind == CFD_FACE_INTERIOR) {
          const int nb = t_int[(1 + f) * EPB + os];
          const int nf = (info >> 2) & 3;
          const bool same_order = (f == 2) != (nf == 2);
          const int kk = same_order ? k : NFP - 1 - k;
          if (nb - e0 >= 0 && nb - e0 < EPB) {
            ns = nb - e0;
            nslot = nf * NFP + kk;
            const int pn = face_node_rt(nf, kk);
#pragma unroll
            for (int c = 0; c < 4; ++c) qp[c] = t_own[(c * NP + pn) * S + ns];
          } else {
#pragma unroll
            for (int c = 0; c < 4; ++c) qp[c] = t_nbr[j * 4 + c];
          }
        } else if (kind == CFD_FACE_SLIP_WALL) {  // dg.py:119-126
          const R mn = qm[1] * nx + qm[2] * ny;
          qp[0] = qm[0];
          qp[1] = qm[1] - R(2) * mn * nx;
          qp[2] = qm[2] - R(2) * mn * ny;
          qp[3] = qm[3];
        } else {
          // fixed state: one row per face; exact state: one row per face node
          const int row = t_int[(1 + f) * EPB + os] + (kind == CFD_FACE_EXACT_STATE ? k : 0);
#pragma unroll
          for (int c = 0; c < 4; ++c) qp[c] = (R)m.bc_states[row * 4 + c];
        }
        const NodeFlux3<R> o = trace_flux3_call<R, FLUX>(qm[0], qm[1], qm[2], qm[3], qp[0], qp[1], qp[2], qp[3], nx,
                                                         ny, gamma);
        R jm[4];
        jump_pair<R, PACK>(fs, o.fm[0], o.fm[1], o.fhat[0], o.fhat[1], jm[0], jm[1]);
        jump_pair<R, PACK>(fs, o.fm[2], o.fm[3], o.fhat[2], o.fhat[3], jm[2], jm[3]);
#pragma unroll
        for (int c = 0; c < 4; ++c) t_jmp[(os * 3 * NFP + f * NFP + k) * 4 + c] = jm[c];
        if (ns >= 0) {
          const int nf = nslot / NFP;
          const R fsn = t_geo[(6 + 3 * nf) * S + ns];
          R jn[4];
          jump_pair<R, PACK>(fsn, o.fhat[0], o.fhat[1], o.fp[0], o.fp[1], jn[0], jn[1]);
          jump_pair<R, PACK>(fsn, o.fhat[2], o.fhat[3], o.fp[2], o.fp[3], jn[2], jn[3]);
#pragma unroll
          for (int c = 0; c < 4; ++c) t_jmp[(ns * 3 * NFP + nslot) * 4 + c] = jn[c];
        }
        if (kind != CFD_FACE_INTERIOR) {
          const double bw = ctab::FACE_W[k] * m.face_hlen[(size_t)f * ld + e0 + os];
#pragma unroll
          for (int c = 0; c < 4; ++c) red.b[c] += bw * (double)o.fhat[c];
        }
      }
      __syncthreads();
      // ---- LIFT of the element's 15 jump inputs (this lane's two variables)
#pragma unroll
      for (int sl = 0; sl < 3 * NFP; ++sl) {
        const R ja0 = t_jmp[(slot * 3 * NFP + sl) * 4 + c0], ja1 = t_jmp[(slot * 3 * NFP + sl) * 4 + c0 + 1];
#pragma unroll
        for (int i = 0; i < NP; ++i) fma_pair<R, PACK>((R)tab::LIFT[i][sl], ja0, ja1, acc[i][0], acc[i][1]);
      }
    }

    // ---- surface term (dg.py:153-164): 8 rounds, the lanes take nodes 2r and 2r+1;
    // unrolled in the FP32 form so the LIFT columns are compile-time operands
    // (the FP64 form keeps the loop rolled: fewer live registers)
#pragma unroll((sizeof(R) == 4 && UNROLL_FACES) ? 8 : 1)
    for (int r = 0; r < (FACE_JOBS ? 0 : 8); ++r) {
      const int sl = 2 * r + half;
      R jump[4] = {R(0), R(0), R(0), R(0)};
      if (sl < 3 * NFP) {
        const int f = sl / NFP, k = sl - NFP * f;
        const int kind = (finfo >> (8 * f)) & 3;
        const R nx = t_geo[(4 + 3 * f) * S + slot], ny = t_geo[(5 + 3 * f) * S + slot];
        const R fs = t_geo[(6 + 3 * f) * S + slot];
        const int n = face_node_rt(f, k);
        R qm[4], qp[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) qm[c] = t_own[(c * NP + n) * S + slot];
        if (kind == CFD_FACE_INTERIOR) {
#pragma unroll
          for (int c = 0; c < 4; ++c) qp[c] = t_nbr[((r * 4 + c) * EPB + slot) * 2 + half];
        } else if (kind == CFD_FACE_SLIP_WALL) {  // dg.py:119-126
          const R mn = qm[1] * nx + qm[2] * ny;
          qp[0] = qm[0];
          qp[1] = qm[1] - R(2) * mn * nx;
          qp[2] = qm[2] - R(2) * mn * ny;
          qp[3] = qm[3];
        } else {
          // fixed state: one row per face; exact state: one row per face node
          const int row = t_int[(1 + f) * EPB + slot] + (kind == CFD_FACE_EXACT_STATE ? k : 0);
#pragma unroll
          for (int c = 0; c < 4; ++c) qp[c] = (R)m.bc_states[row * 4 + c];
        }
        R fhat[4], fm[4];
        if constexpr (CALL_FLUX) {
          const NodeFlux<R> o = trace_flux_call<R, FLUX>(qm[0], qm[1], qm[2], qm[3], qp[0], qp[1], qp[2], qp[3], nx,
                                                         ny, gamma);
#pragma unroll
          for (int c = 0; c < 4; ++c) fhat[c] = o.fhat[c], fm[c] = o.fm[c];
        } else {
          trace_flux<R, FLUX>(qm, qp, nx, ny, gamma, fhat, fm);
        }
        jump_pair<R, PACK>(fs, fm[0], fm[1], fhat[0], fhat[1], jump[0], jump[1]);
        jump_pair<R, PACK>(fs, fm[2], fm[3], fhat[2], fhat[3], jump[2], jump[3]);
        if (kind != CFD_FACE_INTERIOR) {
          const double bw = ctab::FACE_W[k] * m.face_hlen[(size_t)f * ld + e];
#pragma unroll
          for (int c = 0; c < 4; ++c) red.b[c] += bw * (double)fhat[c];
        }
      }
      const R s0 = shfl_pair(half ? jump[0] : jump[2]);
      const R s1 = shfl_pair(half ? jump[1] : jump[3]);
      const R ja0 = half ? s0 : jump[0], ja1 = half ? s1 : jump[1];
      const R jb0 = half ? jump[2] : s0, jb1 = half ? jump[3] : s1;
      const int col = 2 * r;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        const R la = (sizeof(R) == 4 && UNROLL_FACES) ? (R)tab::LIFT[i][col] : tabv<R>::lift(i, col);
        fma_pair<R, PACK>(la, ja0, ja1, acc[i][0], acc[i][1]);
        if (col + 1 < 3 * NFP) {
          const int c1 = col + 1 < 3 * NFP ? col + 1 : col;
          const R lb = (sizeof(R) == 4 && UNROLL_FACES) ? (R)tab::LIFT[i][c1] : tabv<R>::lift(i, c1);
          fma_pair<R, PACK>(lb, jb0, jb1, acc[i][0], acc[i][1]);
        }
      }
    }

    if (MODE == MODE_RHS) {
      if (live) {
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          dst[(size_t)(c0 * NP + i) * ld + e] = acc[i][0];
          dst[(size_t)((c0 + 1) * NP + i) * ld + e] = acc[i][1];
        }
      }
    } else {
      // ---- SSP-RK3 stage combine (time_integration.py:61-66)
      const R rdt = (R)dt;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        R o[2], b[2];
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
          const int row = (c0 + cc) * NP + i;
          o[cc] = t_own[row * S + slot];
          b[cc] = !has_base ? R(0) : (STAGE_BASE ? t_base[L::base_at(row, slot)] : base[(size_t)row * ld + e]);
        }
        combine_pair<R, PACK>(P.stage_idx, rdt, o[0], o[1], b[0], b[1], acc[i][0], acc[i][1]);
      }
#include "stage_epilogue.inc"
    }
  }
  if (!live) {  // a face-job thread may hold boundary-flux terms of live elements
    double b[4] = {red.b[0], red.b[1], red.b[2], red.b[3]};
    red.init();
    if (FACE_JOBS && block_live)
      for (int c = 0; c < 4; ++c) red.b[c] = b[c];
  }
  if (MODE == MODE_RHS) {
    if (live || FACE_JOBS) {
#pragma unroll
      for (int c = 0; c < 4; ++c)
        if (red.b[c] != 0.0) atomicAdd(&P.bflux_out[inst * 4 + c], red.b[c]);
    }
  } else {
    block_commit<BS>(red, live, inst, P.acc, 3, P.stage_idx - 1);
  }
}

template <typename R, int FLUX, int MODE, int EPB, bool STAGE_BASE, int MINB, bool UNROLL_FACES = true,
          bool PACK = false, bool CALL_FLUX = false, bool FACE_JOBS = false, bool VROLL = false>
__global__ void __launch_bounds__(2 * EPB, MINB) stage_tile_kernel(const StageParams P) {
  stage_tile_body<R, FLUX, MODE, EPB, STAGE_BASE, UNROLL_FACES, PACK, CALL_FLUX, FACE_JOBS, VROLL>(P, blockIdx.x);
}
