// setup.cu — the mesh tables of the kernels built on the GPU from the vertex
// and element arrays (the host builders mesh.py:135-251 and limiting.py:51-94
// of CFD-demo build the same quantities in NumPy):
//   geometry_kernel      per element: Jacobian, inverse-map derivatives,
//                        outward normals, edge lengths, centroid, face
//                        midpoints (mesh.py:216-243) and the kernels' metric,
//                        face_geo, face_hlen, dt_geo and jacobian rows
//   face_insert_kernel   every face's vertex-pair code into an open-addressing
//   edge_insert_kernel   hash table, every tagged boundary edge into a second
//   face_match_kernel    one; then each face finds its partner face or its tag
//                        (mesh.py:135-185)
//   cs_kernel            the Cockburn-Shu coefficients and partner faces
//                        (limiting.py:51-94) and the packed face_info and
//                        neighbor rows
//   pairing_kernel       face node k of face f meets node k or 4-k of the
//                        neighbour's face (the rule the stage kernels use),
//                        checked by coordinates (mesh.py:254-291)
// Every floating-point expression is evaluated unfused in NumPy's operation
// order, so the tables equal the host builder's bit for bit. Errors of the
// input (a non-conforming mesh, an untagged or doubly tagged boundary edge, an
// element without nonnegative coefficients, face nodes that do not meet) set
// bits of a status word; the host then reports them with the host builder's
// messages.
#include "common.cuh"

namespace cfd {
namespace {

constexpr unsigned long long HASH_EMPTY = ~0ull;

__device__ __forceinline__ unsigned long long edge_code(long long a, long long b, long long nv) {
  const long long lo = a < b ? a : b, hi = a < b ? b : a;
  return (unsigned long long)(lo * nv + hi);
}
__device__ __forceinline__ unsigned hash_slot(unsigned long long k, unsigned mask) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdull;
  k ^= k >> 33;
  return (unsigned)k & mask;
}

struct SetupArgs {
  CfdMeshBuild in;
  // outputs (device, leading dimension ld)
  double* metric;
  double* face_geo;
  double* face_hlen;
  double* dt_geo;
  double* jacobian;
  double* cs_coef;
  int32_t* neighbor;
  int32_t* face_info;
  // work
  double* cen;        // [2][K]
  double* mid;        // [6][K]  face midpoints x, y per face
  double* nrm;        // [6][K]  normals x, y per face
  double* len;        // [3][K]
  unsigned long long* fkey;  // [T] face table
  int* fcnt;                 // [T]
  int* fid;                  // [2 T]
  unsigned long long* bkey;  // [Tb] boundary-edge table
  int* bcnt;                 // [Tb]
  int* btag;                 // [Tb]
  int* nb_e;                 // [3K] neighbour element (-1 boundary)
  int* nb_f;                 // [3K] neighbour face or boundary tag
  unsigned mask, bmask;
  int* status;
};

__device__ __forceinline__ double m_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double a_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double s_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double d_(double a, double b) { return __ddiv_rn(a, b); }

__global__ void geometry_kernel(const SetupArgs A) {
  const int K = A.in.num_elements, ld = A.in.ld;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= K) return;
  double cx[3], cy[3];
  for (int v = 0; v < 3; ++v) {
    const long long id = A.in.elements[3 * (long long)e + v];
    cx[v] = A.in.vertices[2 * id];
    cy[v] = A.in.vertices[2 * id + 1];
  }
  const double xr = m_(0.5, s_(cx[1], cx[0])), xs = m_(0.5, s_(cx[2], cx[0]));
  const double yr = m_(0.5, s_(cy[1], cy[0])), ys = m_(0.5, s_(cy[2], cy[0]));
  const double jac = s_(m_(xr, ys), m_(xs, yr));
  A.metric[e] = d_(ys, jac);
  A.metric[ld + e] = d_(-xs, jac);
  A.metric[2 * ld + e] = d_(-yr, jac);
  A.metric[3 * ld + e] = d_(xr, jac);
  A.jacobian[e] = jac;
  const double area = m_(2.0, jac);
  double dtg = 0.0;
  for (int f = 0; f < 3; ++f) {
    const int g = f == 2 ? 0 : f + 1;
    const double dx = s_(cx[g], cx[f]), dy = s_(cy[g], cy[f]);
    const double l = sqrt(a_(m_(dx, dx), m_(dy, dy)));
    const double nx = d_(dy, l), ny = d_(-dx, l);
    A.face_geo[(3 * f) * ld + e] = nx;
    A.face_geo[(3 * f + 1) * ld + e] = ny;
    A.face_geo[(3 * f + 2) * ld + e] = d_(m_(0.5, l), jac);  // Fscale = sJ / J (dg.py:99)
    A.face_hlen[f * ld + e] = m_(0.5, l);
    const double dtf = d_(m_(2.0, area), m_(25.0, l));      // 2|K| / ((N+1)^2 |e|)
    dtg = f == 0 ? dtf : (dtf < dtg ? dtf : dtg);
    A.len[f * K + e] = l;
    A.nrm[(2 * f) * K + e] = nx;
    A.nrm[(2 * f + 1) * K + e] = ny;
    A.mid[(2 * f) * K + e] = m_(0.5, a_(cx[f], cx[g]));
    A.mid[(2 * f + 1) * K + e] = m_(0.5, a_(cy[f], cy[g]));
  }
  A.dt_geo[e] = dtg;
  A.cen[e] = d_(a_(a_(cx[0], cx[1]), cx[2]), 3.0);
  A.cen[K + e] = d_(a_(a_(cy[0], cy[1]), cy[2]), 3.0);
}

// Bounded linear probing: a full table is reported, never looped on.
__device__ __forceinline__ int probe_insert(unsigned long long* keys, unsigned mask, unsigned long long code) {
  unsigned h = hash_slot(code, mask);
  for (unsigned i = 0; i <= mask; ++i) {
    const unsigned long long prev = atomicCAS(keys + h, HASH_EMPTY, code);
    if (prev == HASH_EMPTY || prev == code) return (int)h;
    h = (h + 1) & mask;
  }
  return -1;
}
__device__ __forceinline__ int probe_find(const unsigned long long* keys, unsigned mask, unsigned long long code) {
  unsigned h = hash_slot(code, mask);
  for (unsigned i = 0; i <= mask; ++i) {
    const unsigned long long k = keys[h];
    if (k == code) return (int)h;
    if (k == HASH_EMPTY) return -1;
    h = (h + 1) & mask;
  }
  return -1;
}

__global__ void face_insert_kernel(const SetupArgs A) {
  const int K = A.in.num_elements;
  const long long nv = A.in.num_vertices;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * K) return;
  const int e = t / 3, f = t - 3 * e;
  const long long a = A.in.elements[3 * (long long)e + f], b = A.in.elements[3 * (long long)e + (f == 2 ? 0 : f + 1)];
  const int h = probe_insert(A.fkey, A.mask, edge_code(a, b, nv));
  if (h < 0) {
    atomicOr(A.status, CFD_SETUP_TABLE_FULL);
    return;
  }
  const int i = atomicAdd(A.fcnt + h, 1);
  if (i < 2) A.fid[2 * h + i] = t;
  else atomicOr(A.status, CFD_SETUP_NONCONFORMING);
}

__global__ void edge_insert_kernel(const SetupArgs A) {
  const long long nv = A.in.num_vertices;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.in.num_boundary_edges) return;
  const long long a = A.in.boundary_edges[2 * (long long)t], b = A.in.boundary_edges[2 * (long long)t + 1];
  const int tag = A.in.boundary_tag[t];
  if (tag < 0 || tag >= A.in.num_tags) {
    atomicOr(A.status, CFD_SETUP_UNTAGGED);
    return;
  }
  const int h = probe_insert(A.bkey, A.bmask, edge_code(a, b, nv));
  if (h < 0) {
    atomicOr(A.status, CFD_SETUP_TABLE_FULL);
    return;
  }
  if (atomicAdd(A.bcnt + h, 1) > 0) atomicOr(A.status, CFD_SETUP_DOUBLE_TAG);
  A.btag[h] = tag;
}

__global__ void face_match_kernel(const SetupArgs A) {
  const int K = A.in.num_elements;
  const long long nv = A.in.num_vertices;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * K) return;
  const int e = t / 3, f = t - 3 * e;
  const unsigned long long code =
      edge_code(A.in.elements[3 * (long long)e + f], A.in.elements[3 * (long long)e + (f == 2 ? 0 : f + 1)], nv);
  const int h = probe_find(A.fkey, A.mask, code);
  if (h < 0) {  // every face was inserted: only a full table gets here
    atomicOr(A.status, CFD_SETUP_TABLE_FULL);
    A.nb_e[t] = -1;
    A.nb_f[t] = -1;
    return;
  }
  if (A.fcnt[h] == 2) {
    const int other = A.fid[2 * h] == t ? A.fid[2 * h + 1] : A.fid[2 * h];
    A.nb_e[t] = other / 3;
    A.nb_f[t] = other % 3;
  } else {
    A.nb_e[t] = -1;
    const int b = probe_find(A.bkey, A.bmask, code);
    if (b < 0) atomicOr(A.status, CFD_SETUP_UNTAGGED);
    A.nb_f[t] = b < 0 ? -1 : A.btag[b];
  }
}

// every tagged edge must be a boundary face
__global__ void edge_check_kernel(const SetupArgs A) {
  const long long nv = A.in.num_vertices;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= A.in.num_boundary_edges) return;
  const unsigned long long code =
      edge_code(A.in.boundary_edges[2 * (long long)t], A.in.boundary_edges[2 * (long long)t + 1], nv);
  const int h = probe_find(A.fkey, A.mask, code);
  if (h < 0 || A.fcnt[h] != 1) atomicOr(A.status, CFD_SETUP_TAG_NOT_BOUNDARY);
}

// Cockburn-Shu coefficients (limiting.py:51-94) and the packed face tables.
__global__ void cs_kernel(const SetupArgs A) {
  const int K = A.in.num_elements, ld = A.in.ld;
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= K) return;
  const double cx = A.cen[e], cy = A.cen[K + e];
  double dx[3], dy[3], tx[3], ty[3];
  for (int f = 0; f < 3; ++f) {
    const double mx = A.mid[(2 * f) * K + e], my = A.mid[(2 * f + 1) * K + e];
    const double nx = A.nrm[(2 * f) * K + e], ny = A.nrm[(2 * f + 1) * K + e];
    const int nb = A.nb_e[3 * e + f];
    double ncx, ncy;
    if (nb >= 0) {
      ncx = A.cen[nb];
      ncy = A.cen[K + nb];
    } else {  // the centroid reflected across the face
      const double off = a_(m_(s_(mx, cx), nx), m_(s_(my, cy), ny));
      ncx = a_(cx, m_(m_(2.0, off), nx));
      ncy = a_(cy, m_(m_(2.0, off), ny));
    }
    dx[f] = s_(ncx, cx);
    dy[f] = s_(ncy, cy);
    tx[f] = s_(mx, cx);
    ty[f] = s_(my, cy);
  }
  int info = 0;
  bool ok = true;
  for (int f = 0; f < 3; ++f) {
    double alpha = 0.0, beta = 0.0;
    int partner = -1;
    for (int shift = 1; shift <= 2 && partner < 0; ++shift) {
      const int o = (f + shift) % 3;
      const double det = s_(m_(dx[f], dy[o]), m_(dy[f], dx[o]));
      const double safe = det == 0.0 ? 1.0 : det;
      const double a = d_(s_(m_(tx[f], dy[o]), m_(ty[f], dx[o])), safe);
      const double b = d_(s_(m_(dx[f], ty[f]), m_(dy[f], tx[f])), safe);
      if (det != 0.0 && a >= -1e-12 && b >= -1e-12) {
        alpha = a > 0.0 ? a : 0.0;
        beta = b > 0.0 ? b : 0.0;
        partner = o;
      }
    }
    if (partner < 0) ok = false;
    A.cs_coef[f * ld + e] = alpha;
    A.cs_coef[(3 + f) * ld + e] = beta;
    const int nb = A.nb_e[3 * e + f];
    int kind, nbr, nface = 0;
    if (nb >= 0) {
      kind = CFD_FACE_INTERIOR;
      nbr = nb;
      nface = A.nb_f[3 * e + f];
    } else {
      const int tag = A.nb_f[3 * e + f];  // -1: untagged (reported in the status)
      const bool known = tag >= 0 && tag < A.in.num_tags;
      kind = known ? A.in.tag_kind[tag] : CFD_FACE_SLIP_WALL;
      if (kind != CFD_FACE_SLIP_WALL && kind != CFD_FACE_FIXED_STATE) {
        atomicOr(A.status, CFD_SETUP_UNSUPPORTED_KIND);
        kind = CFD_FACE_SLIP_WALL;
      }
      nbr = known && kind == CFD_FACE_FIXED_STATE ? A.in.tag_row[tag] : 0;
    }
    A.neighbor[f * ld + e] = nbr;
    info |= (kind | (nface << 2) | ((partner < 0 ? 0 : partner) << 4)) << (8 * f);
  }
  A.face_info[e] = info;
  if (!ok) atomicOr(A.status, CFD_SETUP_NO_COEFFICIENTS);
}

// Face node k of face f at barycentric weights of the reference face nodes;
// the neighbour's node is k or 4 - k (the stage kernels' pairing rule).
__global__ void pairing_kernel(const SetupArgs A, const double* bary, double rtol) {
  const int K = A.in.num_elements;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * K) return;
  const int e = t / 3, f = t - 3 * e;
  const int nb = A.nb_e[t];
  if (nb < 0) return;
  const int g = A.nb_f[t];
  const bool same_order = (f == 2) != (g == 2);
  double ex[3], ey[3], nx_[3], ny_[3];
  for (int v = 0; v < 3; ++v) {
    const long long a = A.in.elements[3 * (long long)e + v], b = A.in.elements[3 * (long long)nb + v];
    ex[v] = A.in.vertices[2 * a];
    ey[v] = A.in.vertices[2 * a + 1];
    nx_[v] = A.in.vertices[2 * b];
    ny_[v] = A.in.vertices[2 * b + 1];
  }
  const double tol = rtol * A.len[f * K + e];
  for (int k = 0; k < NFP; ++k) {
    const int kk = same_order ? k : NFP - 1 - k;
    const double* wo = bary + (f * NFP + k) * 3;
    const double* wn = bary + (g * NFP + kk) * 3;
    const double ox = wo[0] * ex[0] + wo[1] * ex[1] + wo[2] * ex[2], oy = wo[0] * ey[0] + wo[1] * ey[1] + wo[2] * ey[2];
    const double px = wn[0] * nx_[0] + wn[1] * nx_[1] + wn[2] * nx_[2];
    const double py = wn[0] * ny_[0] + wn[1] * ny_[1] + wn[2] * ny_[2];
    if (hypot(ox - px, oy - py) > tol) atomicOr(A.status, CFD_SETUP_NOT_CONFORMING_NODES);
  }
}

unsigned table_mask(long long n) {
  unsigned long long t = 64;
  while (t < 2ull * (unsigned long long)n) t <<= 1;
  return (unsigned)(t - 1);
}

}  // namespace
}  // namespace cfd

using namespace cfd;

extern "C" int64_t cfd_mesh_build_work_bytes(int32_t num_elements, int32_t num_boundary_edges) {
  if (num_elements <= 0 || num_boundary_edges < 0) return -1;
  const long long K = num_elements;
  const long long T = (long long)table_mask(3 * K) + 1, Tb = (long long)table_mask(num_boundary_edges) + 1;
  const long long doubles = 2 * K + 6 * K + 6 * K + 3 * K;
  return (int64_t)(doubles * 8 + T * (8 + 4 + 8) + Tb * (8 + 4 + 4) + 6 * K * 4 + 16 * 256);
}

extern "C" int cfd_mesh_build(const CfdMeshBuild* in, const CfdMesh* out, const double* face_node_bary,
                              double pairing_rtol, void* work, int64_t work_bytes, int32_t* status, void* stream) {
  if (!in || !out || !face_node_bary || !work || !status || !in->vertices || !in->elements)
    return cfd_fail(CFD_E_ARG, "cfd_mesh_build: null pointer");
  const int K = in->num_elements;
  if (K <= 0 || in->ld < K || in->num_vertices <= 0 || in->num_boundary_edges < 0 || out->ld != in->ld ||
      out->num_elements != K)
    return cfd_fail(CFD_E_ARG, "cfd_mesh_build: bad sizes");
  if (in->num_tags < 0 || (in->num_boundary_edges > 0 && (!in->boundary_edges || !in->boundary_tag)) ||
      (in->num_tags > 0 && (!in->tag_kind || !in->tag_row)))
    return cfd_fail(CFD_E_ARG, "cfd_mesh_build: boundary tables missing");
  if (!out->metric || !out->face_geo || !out->face_hlen || !out->dt_geo || !out->jacobian || !out->cs_coef ||
      !out->neighbor || !out->face_info)
    return cfd_fail(CFD_E_ARG, "cfd_mesh_build: output table pointer is null");
  if (work_bytes < cfd_mesh_build_work_bytes(K, in->num_boundary_edges))
    return cfd_fail(CFD_E_ARG, "cfd_mesh_build: work buffer too small");
  cudaStream_t st = (cudaStream_t)stream;
  SetupArgs A;
  memset(&A, 0, sizeof(A));
  A.in = *in;
  A.metric = const_cast<double*>(out->metric);
  A.face_geo = const_cast<double*>(out->face_geo);
  A.face_hlen = const_cast<double*>(out->face_hlen);
  A.dt_geo = const_cast<double*>(out->dt_geo);
  A.jacobian = const_cast<double*>(out->jacobian);
  A.cs_coef = const_cast<double*>(out->cs_coef);
  A.neighbor = const_cast<int32_t*>(out->neighbor);
  A.face_info = const_cast<int32_t*>(out->face_info);
  A.mask = table_mask(3LL * K);
  A.bmask = table_mask(in->num_boundary_edges);
  const long long T = (long long)A.mask + 1, Tb = (long long)A.bmask + 1;
  char* w = (char*)work;
  auto take = [&](size_t bytes) {
    char* p = w;
    w += (bytes + 255) / 256 * 256;
    return (void*)p;
  };
  A.cen = (double*)take(sizeof(double) * 2 * K);
  A.mid = (double*)take(sizeof(double) * 6 * K);
  A.nrm = (double*)take(sizeof(double) * 6 * K);
  A.len = (double*)take(sizeof(double) * 3 * K);
  A.fkey = (unsigned long long*)take(8 * T);
  A.fcnt = (int*)take(4 * T);
  A.fid = (int*)take(8 * T);
  A.bkey = (unsigned long long*)take(8 * Tb);
  A.bcnt = (int*)take(4 * Tb);
  A.btag = (int*)take(4 * Tb);
  A.nb_e = (int*)take(4 * 3 * (size_t)K);
  A.nb_f = (int*)take(4 * 3 * (size_t)K);
  A.status = status;
  if ((long long)(w - (char*)work) > work_bytes) return cfd_fail(CFD_E_ARG, "cfd_mesh_build: work buffer too small");
  if (cudaMemsetAsync(status, 0, sizeof(int32_t), st) != cudaSuccess ||
      cudaMemsetAsync(A.fkey, 0xff, 8 * T, st) != cudaSuccess || cudaMemsetAsync(A.fcnt, 0, 4 * T, st) != cudaSuccess ||
      cudaMemsetAsync(A.bkey, 0xff, 8 * Tb, st) != cudaSuccess || cudaMemsetAsync(A.bcnt, 0, 4 * Tb, st) != cudaSuccess)
    return cfd_fail(CFD_E_CUDA, "cfd_mesh_build: memset failed");
  const int bs = 128;
  geometry_kernel<<<blocks_for(K, bs), bs, 0, st>>>(A);
  face_insert_kernel<<<blocks_for(3LL * K, bs), bs, 0, st>>>(A);
  if (in->num_boundary_edges > 0) edge_insert_kernel<<<blocks_for(in->num_boundary_edges, bs), bs, 0, st>>>(A);
  face_match_kernel<<<blocks_for(3LL * K, bs), bs, 0, st>>>(A);
  if (in->num_boundary_edges > 0) edge_check_kernel<<<blocks_for(in->num_boundary_edges, bs), bs, 0, st>>>(A);
  cs_kernel<<<blocks_for(K, bs), bs, 0, st>>>(A);
  pairing_kernel<<<blocks_for(3LL * K, bs), bs, 0, st>>>(A, face_node_bary, pairing_rtol);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CFD_OK : cfd_fail(CFD_E_CUDA, cudaGetErrorString(e));
}
