// Device FEM topology and assembly: replaces prepare_mesh + gen_fwdmat
// (DOGPUP/dMesh.m:945-1235), which assembles on the GPU page by page but then
// builds the sparse matrices on the CPU with sparse() (:1123-1124, :1181).
//
// Here everything stays on the device:
//   * boundary nodes = nodes of faces owned by exactly one tet (:964-980),
//     found with one radix sort of packed face keys;
//   * the Robin face set of :1129-1140 (all 4 faces of tets with 4 boundary
//     nodes, the boundary face of tets with 3), compacted with a scan;
//   * the symmetric CSR pattern and a contribution list per CSR slot, from a
//     stable radix sort of (row, col) keys of every element and face entry;
//   * assembly = element kernel (4x4 K_e, M_e and 3x3 Robin blocks with the
//     reference's Keast / 3-point rules) + one thread per CSR slot summing its
//     contributions in element order: deterministic, no atomics, and
//     bitwise-symmetric K and M.
#include <cub/cub.cuh>

#include "dgp_common.cuh"
#include "dgp_internal.h"

namespace dgp {

namespace {

constexpr double kCVac = 2.99792458e11;  // mm/s, dMesh.m:42

// Keast 5-point rule (dMesh.m:1204-1207) and the 3-point triangle rule (:1225-1227)
__constant__ double c_tq[4][5];  // basis values N_l(x_q), l = 0..3
__constant__ double c_tw[5];
__constant__ double c_fq[3][3];  // triangle basis values N_l(x_q)
__constant__ double c_fw[3];

struct Geo {
  double vol;
  double g[4][3];  // gradients of the 4 basis functions
};

__device__ inline Geo tet_geometry(const double *__restrict__ node, const int32_t *e, int *bad) {
  double p[4][3];
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int d = 0; d < 3; ++d) p[v][d] = node[3 * (int64_t)e[v] + d];
  // B = [p1-p0, p2-p0, p3-p0] as columns (dMesh.m:1017-1019)
  double B[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = 0; d < 3; ++d) B[d][c] = p[c + 1][d] - p[0][d];
  // det(B) = dot(cross(a, b), c) with a, b, c the columns (vol, :952-955)
  double cx = B[1][0] * B[2][1] - B[2][0] * B[1][1];
  double cy = B[2][0] * B[0][1] - B[0][0] * B[2][1];
  double cz = B[0][0] * B[1][1] - B[1][0] * B[0][1];
  double det = cx * B[0][2] + cy * B[1][2] + cz * B[2][2];
  Geo G;
  G.vol = fabs(det / 6.0);
  if (!(G.vol > 0.0) && bad) atomicOr(bad, 1);
  // inv(B^T) = cof(B) / det(B): (B^-T)_{ij} = cofactor_{ij}(B) / det
  double cof[3][3];
  cof[0][0] = B[1][1] * B[2][2] - B[1][2] * B[2][1];
  cof[0][1] = B[1][2] * B[2][0] - B[1][0] * B[2][2];
  cof[0][2] = B[1][0] * B[2][1] - B[1][1] * B[2][0];
  cof[1][0] = B[0][2] * B[2][1] - B[0][1] * B[2][2];
  cof[1][1] = B[0][0] * B[2][2] - B[0][2] * B[2][0];
  cof[1][2] = B[0][1] * B[2][0] - B[0][0] * B[2][1];
  cof[2][0] = B[0][1] * B[1][2] - B[0][2] * B[1][1];
  cof[2][1] = B[0][2] * B[1][0] - B[0][0] * B[1][2];
  cof[2][2] = B[0][0] * B[1][1] - B[0][1] * B[1][0];
  double inv = 1.0 / det;
  // reference-element gradients (:1061): N0 = (-1,-1,-1), N1..3 = unit vectors
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double g1 = cof[d][0] * inv, g2 = cof[d][1] * inv, g3 = cof[d][2] * inv;
    G.g[1][d] = g1;
    G.g[2][d] = g2;
    G.g[3][d] = g3;
    G.g[0][d] = -g1 - g2 - g3;
  }
  return G;
}

__global__ void k_check_elems(const double *__restrict__ node, const int32_t *__restrict__ elem,
                              int64_t ne, int64_t nn, int *bad) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int32_t v[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    v[l] = elem[4 * e + l];
    if (v[l] < 0 || v[l] >= nn) { atomicOr(bad, 2); return; }
  }
  tet_geometry(node, v, bad);
}

// 21 bits per id (nn < 2^21) packs a sorted face triple into 63 bits
__device__ inline uint64_t face_key(int32_t a, int32_t b, int32_t c) {
  return ((uint64_t)a << 42) | ((uint64_t)b << 21) | (uint64_t)c;
}

__device__ inline void sort4(int32_t *s) {
#define SW(i, j) if (s[i] > s[j]) { int32_t t = s[i]; s[i] = s[j]; s[j] = t; }
  SW(0, 1) SW(2, 3) SW(0, 2) SW(1, 3) SW(1, 2)
#undef SW
}

__global__ void k_face_keys(const int32_t *__restrict__ elem, int64_t ne, uint64_t *keys) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int32_t s[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) s[l] = elem[4 * e + l];
  sort4(s);
  keys[4 * e + 0] = face_key(s[0], s[1], s[2]);
  keys[4 * e + 1] = face_key(s[0], s[1], s[3]);
  keys[4 * e + 2] = face_key(s[0], s[2], s[3]);
  keys[4 * e + 3] = face_key(s[1], s[2], s[3]);
}

__global__ void k_mark_boundary(const uint64_t *__restrict__ keys, int64_t nk, int32_t *bnd) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= nk) return;
  uint64_t k = keys[p];
  bool once = (p == 0 || keys[p - 1] != k) && (p == nk - 1 || keys[p + 1] != k);
  if (!once) return;
  const uint64_t m = (1ull << 21) - 1;
  bnd[(k >> 42) & m] = 1;
  bnd[(k >> 21) & m] = 1;
  bnd[k & m] = 1;
}

__global__ void k_robin_count(const int32_t *__restrict__ elem, const int32_t *__restrict__ bnd,
                              int64_t ne, int32_t *cnt) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int c = 0;
#pragma unroll
  for (int l = 0; l < 4; ++l) c += bnd[elem[4 * e + l]] != 0;
  cnt[e] = c == 4 ? 4 : (c == 3 ? 1 : 0);
}

__global__ void k_robin_fill(const int32_t *__restrict__ elem, const int32_t *__restrict__ bnd,
                             const int32_t *__restrict__ off, int64_t ne, int32_t *faces) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int32_t s[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) s[l] = elem[4 * e + l];
  sort4(s);  // dMesh.m:1129 sorts each tet's node ids
  int f = off[e];
  int fl[4], c = 0;
#pragma unroll
  for (int l = 0; l < 4; ++l) { fl[l] = bnd[s[l]] != 0; c += fl[l]; }
  if (c == 4) {  // :1134-1136
    const int tri[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    for (int t = 0; t < 4; ++t)
      for (int q = 0; q < 3; ++q) faces[3 * (int64_t)(f + t) + q] = s[tri[t][q]];
  } else if (c == 3) {  // :1138-1139, the 3 flagged ids in ascending order
    int q = 0;
    for (int l = 0; l < 4; ++l)
      if (fl[l]) faces[3 * (int64_t)f + (q++)] = s[l];
  }
}

// (row, col) keys of every element entry (16 per tet) and every Robin face
// entry (9 per face); payload = position in the element / face value buffers.
__global__ void k_pair_keys(const int32_t *__restrict__ elem, int64_t ne,
                            const int32_t *__restrict__ faces, int64_t nf,
                            uint64_t *keys, int32_t *payload) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t ntot = 16 * ne + 9 * nf;
  if (t >= ntot) return;
  int32_t i, j;
  if (t < 16 * ne) {
    int64_t e = t >> 4;
    int a = (t >> 2) & 3, b = t & 3;
    i = elem[4 * e + a];
    j = elem[4 * e + b];
  } else {
    int64_t u = t - 16 * ne;
    int64_t f = u / 9;
    int r = u % 9;
    i = faces[3 * f + r / 3];
    j = faces[3 * f + r % 3];
  }
  keys[t] = ((uint64_t)(uint32_t)i << 32) | (uint32_t)j;
  payload[t] = (int32_t)t;
}

__global__ void k_slot_heads(const uint64_t *__restrict__ keys, int64_t nk, int32_t *head) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= nk) return;
  head[p] = (p == 0 || keys[p - 1] != keys[p]) ? 1 : 0;
}

// slot ids (inclusive scan of heads, minus one) -> columns, contribution
// start offsets, and row pointers.
__global__ void k_build_csr(const uint64_t *__restrict__ keys, const int32_t *__restrict__ slot_incl,
                            int64_t nk, int64_t nn, int32_t *col, int32_t *cstart, int32_t *rowptr) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= nk) return;
  bool head = (p == 0 || keys[p - 1] != keys[p]);
  if (!head) return;
  int32_t u = slot_incl[p] - 1;
  int32_t r = (int32_t)(keys[p] >> 32);
  col[u] = (int32_t)(keys[p] & 0xffffffffu);
  cstart[u] = (int32_t)p;
  int32_t rprev = (u == 0) ? -1 : (int32_t)(keys[p - 1] >> 32);
  for (int32_t rr = rprev + 1; rr <= r; ++rr) rowptr[rr] = u;
}

__global__ void k_close_rows(const uint64_t *__restrict__ keys, int64_t nk, int64_t nn, int32_t nnz,
                             int32_t *rowptr) {
  int32_t rlast = (int32_t)(keys[nk - 1] >> 32);
  for (int64_t r = rlast + 1 + threadIdx.x; r <= nn; r += blockDim.x) rowptr[r] = nnz;
}

// 4x4 element blocks (dMesh.m:1080-1121), 3x3 Robin blocks (:1142-1179).
__global__ void k_element_blocks(const double *__restrict__ node, const int32_t *__restrict__ elem,
                                 int64_t ne, const double *__restrict__ mua,
                                 const double *__restrict__ musp, double *Ke, double *Me, int *bad) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int32_t v[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) v[l] = elem[4 * e + l];
  Geo G = tet_geometry(node, v, bad);
  double kap[4], mu[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    double a = mua[v[l]];
    mu[l] = a;
    kap[l] = 1.0 / (3.0 * (a + musp[v[l]]));  // dMesh.m:74, :85
  }
  // property values at the quadrature points times the weights (:1083-1087)
  double kq[5], mq[5], ksum = 0.0;
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    double kk = 0.0, mm = 0.0;
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      kk += c_tq[l][q] * kap[l];
      mm += c_tq[l][q] * mu[l];
    }
    kq[q] = c_tw[q] * kk;
    mq[q] = c_tw[q] * mm;
  }
#pragma unroll
  for (int q = 0; q < 5; ++q) ksum += kq[q];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      double gg = G.g[i][0] * G.g[j][0] + G.g[i][1] * G.g[j][1] + G.g[i][2] * G.g[j][2];
      double stiff = (G.vol * gg) * ksum;                       // :1107-1110
      double ab = 0.0, ms = 0.0;
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        ab += mq[q] * c_tq[i][q] * c_tq[j][q];                  // :1113
        ms += c_tw[q] * c_tq[i][q] * c_tq[j][q];                // :1118
      }
      Ke[16 * e + 4 * i + j] = stiff + G.vol * ab;              // :1115
      Me[16 * e + 4 * i + j] = G.vol * ms;                      // :1119
    }
  }
}

__global__ void k_face_blocks(const double *__restrict__ node, const int32_t *__restrict__ faces,
                              int64_t nf, const int32_t *__restrict__ bnd, double rfac, double *Be) {
  int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (f >= nf) return;
  double p[3][3];
  double R[3];
#pragma unroll
  for (int l = 0; l < 3; ++l) {
    int32_t v = faces[3 * f + l];
    R[l] = rfac * (double)bnd[v];  // R = bnd/(2A), :1011
#pragma unroll
    for (int d = 0; d < 3; ++d) p[l][d] = node[3 * (int64_t)v + d];
  }
  double a[3], b[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) { a[d] = p[1][d] - p[0][d]; b[d] = p[2][d] - p[0][d]; }
  double nx = a[1] * b[2] - a[2] * b[1], ny = a[2] * b[0] - a[0] * b[2], nz = a[0] * b[1] - a[1] * b[0];
  double area = sqrt(nx * nx + ny * ny + nz * nz) * 0.5;      // :1143-1146
  double rq[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double r = 0.0;
#pragma unroll
    for (int l = 0; l < 3; ++l) r += c_fq[l][q] * R[l];
    rq[q] = c_fw[q] * r;                                       // :1159-1163
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < 3; ++q) s += rq[q] * c_fq[i][q] * c_fq[j][q];
      Be[9 * f + 3 * i + j] = area * s;                        // :1176
    }
}

// one thread per CSR slot: K = (sum of element entries) + (sum of Robin
// entries), M = sum of element entries, each in ascending element order.
// A slot (r, c) below the diagonal takes the transposed local entry of each
// contribution, i.e. exactly the value of slot (c, r): the reference keeps
// triu(K), triu(M) and mirrors them (dMesh.m:1189-1190, :1242), so A is
// bitwise symmetric there as well.
__global__ void k_gather_slots(const int32_t *__restrict__ cstart, const int32_t *__restrict__ payload,
                               int32_t nnz, int64_t nk, int64_t ne16, const int32_t *__restrict__ elem,
                               const int32_t *__restrict__ faces, const double *__restrict__ Ke,
                               const double *__restrict__ Me, const double *__restrict__ Be, double *K,
                               double *M) {
  int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (u >= nnz) return;
  int64_t b = cstart[u];
  int64_t e = (u + 1 < nnz) ? cstart[u + 1] : nk;
  double kv = 0.0, mv = 0.0, kb = 0.0;
  for (int64_t p = b; p < e; ++p) {
    int64_t t = payload[p];
    if (t < ne16) {
      int64_t el = t >> 4;
      int a = (t >> 2) & 3, c = t & 3;
      if (elem[4 * el + a] > elem[4 * el + c]) t = (el << 4) | (c << 2) | a;
      kv += Ke[t];
      mv += Me[t];
    } else {
      int64_t q = t - ne16;
      int64_t f = q / 9;
      int a = (int)(q % 9) / 3, c = (int)(q % 9) % 3;
      if (faces[3 * f + a] > faces[3 * f + c]) q = 9 * f + 3 * c + a;
      kb += Be[q];
    }
  }
  K[u] = kv + kb;
  M[u] = mv;
}

// Adjoint gradient of a real functional L(phi(mua, musp)) for every node:
//   dL/dmua_v = -Re sum_{s,k} lam^T (dA_k/dmua_v) phi,  dL/dmusp_v likewise,
// with dA/dp differentiated through exactly the element quadrature above:
// absorption block vol sum_q w_q N_v N_i N_j, and the stiffness block
// vol (grad N_i . grad N_j) d(ksum)/dp with ksum = sum_q w_q sum_l N_l kappa_l,
// d(ksum)/dmua_v = d(ksum)/dmusp_v = -3 kappa_v^2 sum_q w_q N_v(x_q)
// (kappa = 1/(3(mua + musp)), dMesh.m:74, :85).  One warp per element, lanes
// over sources, all harmonics; the per-vertex sums leave by one FP64 atomic
// per vertex and output.  Robin and M blocks do not depend on mua or musp.
__global__ void __launch_bounds__(256) k_elem_grad(const double *__restrict__ node, const int32_t *__restrict__ elem,
                                                   int64_t ne, const double2 *__restrict__ phi,
                                                   const double2 *__restrict__ lam, int64_t n, int nf, int ns,
                                                   const double *__restrict__ mua, const double *__restrict__ musp,
                                                   double *gmua, double *gmusp) {
  const int lane = threadIdx.x & 31;
  const int64_t e = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  if (e >= ne) return;
  int32_t v[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) v[l] = elem[4 * e + l];
  Geo G = tet_geometry(node, v, nullptr);
  double dk[4];
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    double cv = 0.0;
#pragma unroll
    for (int q = 0; q < 5; ++q) cv += c_tw[q] * c_tq[l][q];
    double kap = 1.0 / (3.0 * (mua[v[l]] + musp[v[l]]));
    dk[l] = -3.0 * kap * kap * cv * G.vol;
  }
  double acc_a[4] = {0, 0, 0, 0}, acc_k = 0.0;
  for (int k = 0; k < nf; ++k) {
    const int64_t base = (int64_t)k * n;
    for (int s = lane; s < ns; s += 32) {
      double2 f[4], a[4];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        f[l] = phi[(base + v[l]) * ns + s];
        a[l] = lam[(base + v[l]) * ns + s];
      }
      // absorption: sum_q w_q N_v(x_q) Re(lam(x_q) phi(x_q))
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        double fr = 0, fi = 0, ar = 0, ai = 0;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          fr += c_tq[l][q] * f[l].x;
          fi += c_tq[l][q] * f[l].y;
          ar += c_tq[l][q] * a[l].x;
          ai += c_tq[l][q] * a[l].y;
        }
        const double pr = c_tw[q] * (ar * fr - ai * fi);
#pragma unroll
        for (int l = 0; l < 4; ++l) acc_a[l] += c_tq[l][q] * pr;
      }
      // stiffness: Re(grad lam . grad phi), shared by all four vertices
      double dot = 0.0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double lr = 0, li = 0, pr = 0, pi = 0;
#pragma unroll
        for (int l = 0; l < 4; ++l) {
          lr += G.g[l][d] * a[l].x;
          li += G.g[l][d] * a[l].y;
          pr += G.g[l][d] * f[l].x;
          pi += G.g[l][d] * f[l].y;
        }
        dot += lr * pr - li * pi;
      }
      acc_k += dot;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
    for (int l = 0; l < 4; ++l) acc_a[l] += __shfl_xor_sync(0xffffffffu, acc_a[l], off);
    acc_k += __shfl_xor_sync(0xffffffffu, acc_k, off);
  }
  if (lane == 0) {
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const double stiff = acc_k * dk[l];
      atomicAdd(gmua + v[l], -(G.vol * acc_a[l] + stiff));
      if (gmusp) atomicAdd(gmusp + v[l], -stiff);
    }
  }
}

double robin_factor(double nr) {
  double r0 = (nr - 1.0) * (nr - 1.0) / ((nr + 1.0) * (nr + 1.0));
  double ct = fabs(cos(asin(1.0 / nr)));
  double a = (2.0 / (1.0 - r0) - 1.0 + ct * ct * ct) / (1.0 - ct * ct);
  return 1.0 / (2.0 * a);
}

int upload_quadrature() {
  static bool done[64] = {false};
  int dev = 0;
  DGP_CUDA(cudaGetDevice(&dev));
  if (dev < 64 && done[dev]) return DGP_OK;
  const double xa[5] = {1. / 4, 1. / 2, 1. / 6, 1. / 6, 1. / 6};
  const double ya[5] = {1. / 4, 1. / 6, 1. / 6, 1. / 6, 1. / 2};
  const double za[5] = {1. / 4, 1. / 6, 1. / 6, 1. / 2, 1. / 6};
  const double wt[5] = {-0.8, 0.45, 0.45, 0.45, 0.45};
  double tq[4][5];
  for (int q = 0; q < 5; ++q) {
    tq[0][q] = 1 - xa[q] - ya[q] - za[q];
    tq[1][q] = xa[q];
    tq[2][q] = ya[q];
    tq[3][q] = za[q];
  }
  const double fx[3] = {2. / 3, 1. / 6, 1. / 6};
  const double fy[3] = {1. / 6, 2. / 3, 1. / 6};
  const double fw[3] = {1. / 3, 1. / 3, 1. / 3};
  double fq[3][3];
  for (int q = 0; q < 3; ++q) {
    fq[0][q] = 1 - fx[q] - fy[q];
    fq[1][q] = fx[q];
    fq[2][q] = fy[q];
  }
  DGP_CUDA(cudaMemcpyToSymbol(c_tq, tq, sizeof(tq)));
  DGP_CUDA(cudaMemcpyToSymbol(c_tw, wt, sizeof(wt)));
  DGP_CUDA(cudaMemcpyToSymbol(c_fq, fq, sizeof(fq)));
  DGP_CUDA(cudaMemcpyToSymbol(c_fw, fw, sizeof(fw)));
  if (dev < 64) done[dev] = true;
  return DGP_OK;
}

inline unsigned grid1(int64_t n, int bs) { return (unsigned)ceil_div(n, bs); }

}  // namespace

int fem_create(FemPlan *F, const double *d_node, const int32_t *d_elem, int64_t nn, int64_t ne,
               double nr, cudaStream_t st) {
  DGP_REQUIRE(nn > 0 && ne > 0, "fem: empty mesh");
  DGP_REQUIRE(nn < (1 << 21), "fem: more than 2^21 - 1 nodes is not supported by the face-key packing");
  DGP_REQUIRE(16 * ne + 36 * ne < (int64_t)INT32_MAX, "fem: too many elements for int32 slot payloads");
  DGP_REQUIRE(nr > 1.0, "fem: refractive index must exceed 1");
  DGP_TRY(upload_quadrature());
  F->nn = nn;
  F->ne = ne;
  F->nr = nr;
  F->c = kCVac / nr;
  F->rfac = robin_factor(nr);
  DGP_TRY(F->node.alloc(sizeof(double) * 3 * nn));
  DGP_TRY(F->elem.alloc(sizeof(int32_t) * 4 * ne));
  DGP_CUDA(cudaMemcpyAsync(F->node.p, d_node, sizeof(double) * 3 * nn, cudaMemcpyDeviceToDevice, st));
  DGP_CUDA(cudaMemcpyAsync(F->elem.p, d_elem, sizeof(int32_t) * 4 * ne, cudaMemcpyDeviceToDevice, st));
  const int bs = 256;
  DevBuf flag;
  DGP_TRY(flag.alloc(sizeof(int)));
  DGP_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
  k_check_elems<<<grid1(ne, bs), bs, 0, st>>>(F->node.as<double>(), F->elem.as<int32_t>(), ne, nn,
                                             flag.as<int>());
  DGP_CHECK_LAUNCH();
  int hbad = 0;
  DGP_CUDA(cudaMemcpyAsync(&hbad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  if (hbad & 2) return fail(DGP_ERR_MESH, "fem: element node id out of range");
  if (hbad & 1) return fail(DGP_ERR_MESH, "fem: degenerate (zero-volume) tetrahedron");

  // ---- boundary nodes: faces owned by one tet
  {
    int64_t nk = 4 * ne;
    DevBuf k0, k1, tmp;
    DGP_TRY(k0.alloc(sizeof(uint64_t) * nk));
    DGP_TRY(k1.alloc(sizeof(uint64_t) * nk));
    k_face_keys<<<grid1(ne, bs), bs, 0, st>>>(F->elem.as<int32_t>(), ne, k0.as<uint64_t>());
    DGP_CHECK_LAUNCH();
    size_t tb = 0;
    DGP_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, k0.as<uint64_t>(), k1.as<uint64_t>(), (int)nk, 0, 63, st));
    DGP_TRY(tmp.alloc(tb));
    DGP_CUDA(cub::DeviceRadixSort::SortKeys(tmp.p, tb, k0.as<uint64_t>(), k1.as<uint64_t>(), (int)nk, 0, 63, st));
    DGP_TRY(F->bnd.alloc(sizeof(int32_t) * nn));
    DGP_CUDA(cudaMemsetAsync(F->bnd.p, 0, sizeof(int32_t) * nn, st));
    k_mark_boundary<<<grid1(nk, bs), bs, 0, st>>>(k1.as<uint64_t>(), nk, F->bnd.as<int32_t>());
    DGP_CHECK_LAUNCH();
  }
  // ---- Robin face set
  {
    DevBuf cnt, off, tmp;
    DGP_TRY(cnt.alloc(sizeof(int32_t) * (ne + 1)));
    DGP_TRY(off.alloc(sizeof(int32_t) * (ne + 1)));
    DGP_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * (ne + 1), st));
    k_robin_count<<<grid1(ne, bs), bs, 0, st>>>(F->elem.as<int32_t>(), F->bnd.as<int32_t>(), ne,
                                               cnt.as<int32_t>());
    DGP_CHECK_LAUNCH();
    size_t tb = 0;
    DGP_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<int32_t>(), off.as<int32_t>(), (int)(ne + 1), st));
    DGP_TRY(tmp.alloc(tb));
    DGP_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.as<int32_t>(), off.as<int32_t>(), (int)(ne + 1), st));
    int32_t hnf = 0;
    DGP_CUDA(cudaMemcpyAsync(&hnf, off.as<int32_t>() + ne, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaStreamSynchronize(st));
    F->nfaces = hnf;
    DGP_TRY(F->faces.alloc(sizeof(int32_t) * 3 * (hnf > 0 ? hnf : 1)));
    if (hnf > 0) {
      k_robin_fill<<<grid1(ne, bs), bs, 0, st>>>(F->elem.as<int32_t>(), F->bnd.as<int32_t>(),
                                                off.as<int32_t>(), ne, F->faces.as<int32_t>());
      DGP_CHECK_LAUNCH();
    }
  }
  // ---- CSR pattern + per-slot contribution lists
  {
    int64_t nk = 16 * ne + 9 * F->nfaces;
    F->nk = nk;
    DevBuf k0, k1, p0, tmp, head, incl;
    DGP_TRY(k0.alloc(sizeof(uint64_t) * nk));
    DGP_TRY(k1.alloc(sizeof(uint64_t) * nk));
    DGP_TRY(p0.alloc(sizeof(int32_t) * nk));
    DGP_TRY(F->payload.alloc(sizeof(int32_t) * nk));
    k_pair_keys<<<grid1(nk, bs), bs, 0, st>>>(F->elem.as<int32_t>(), ne, F->faces.as<int32_t>(), F->nfaces,
                                             k0.as<uint64_t>(), p0.as<int32_t>());
    DGP_CHECK_LAUNCH();
    int endbit = 32;
    while ((1ll << (endbit - 32)) <= nn && endbit < 64) ++endbit;
    size_t tb = 0;
    DGP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, k0.as<uint64_t>(), k1.as<uint64_t>(), p0.as<int32_t>(),
                                             F->payload.as<int32_t>(), (int)nk, 0, endbit, st));
    DGP_TRY(tmp.alloc(tb));
    DGP_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, k0.as<uint64_t>(), k1.as<uint64_t>(), p0.as<int32_t>(),
                                             F->payload.as<int32_t>(), (int)nk, 0, endbit, st));
    DGP_TRY(head.alloc(sizeof(int32_t) * nk));
    DGP_TRY(incl.alloc(sizeof(int32_t) * nk));
    k_slot_heads<<<grid1(nk, bs), bs, 0, st>>>(k1.as<uint64_t>(), nk, head.as<int32_t>());
    DGP_CHECK_LAUNCH();
    size_t tb2 = 0;
    DGP_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb2, head.as<int32_t>(), incl.as<int32_t>(), (int)nk, st));
    DevBuf tmp2;
    DGP_TRY(tmp2.alloc(tb2));
    DGP_CUDA(cub::DeviceScan::InclusiveSum(tmp2.p, tb2, head.as<int32_t>(), incl.as<int32_t>(), (int)nk, st));
    int32_t hnnz = 0;
    DGP_CUDA(cudaMemcpyAsync(&hnnz, incl.as<int32_t>() + nk - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaStreamSynchronize(st));
    F->nnz = hnnz;
    DGP_TRY(F->rowptr.alloc(sizeof(int32_t) * (nn + 1)));
    DGP_TRY(F->col.alloc(sizeof(int32_t) * hnnz));
    DGP_TRY(F->cstart.alloc(sizeof(int32_t) * hnnz));
    k_build_csr<<<grid1(nk, bs), bs, 0, st>>>(k1.as<uint64_t>(), incl.as<int32_t>(), nk, nn, F->col.as<int32_t>(),
                                             F->cstart.as<int32_t>(), F->rowptr.as<int32_t>());
    DGP_CHECK_LAUNCH();
    k_close_rows<<<1, 256, 0, st>>>(k1.as<uint64_t>(), nk, nn, hnnz, F->rowptr.as<int32_t>());
    DGP_CHECK_LAUNCH();
  }
  // element / face block buffers used by every assembly
  DGP_TRY(F->Ke.alloc(sizeof(double) * 16 * ne));
  DGP_TRY(F->Me.alloc(sizeof(double) * 16 * ne));
  DGP_TRY(F->Be.alloc(sizeof(double) * 9 * (F->nfaces > 0 ? F->nfaces : 1)));
  int64_t hb = 0;
  {
    DevBuf d;
    DGP_TRY(d.alloc(sizeof(int64_t)));
    size_t tb = 0;
    DGP_CUDA(cub::DeviceReduce::Sum(nullptr, tb, F->bnd.as<int32_t>(), d.as<int64_t>(), (int)nn, st));
    DevBuf tmp;
    DGP_TRY(tmp.alloc(tb));
    DGP_CUDA(cub::DeviceReduce::Sum(tmp.p, tb, F->bnd.as<int32_t>(), d.as<int64_t>(), (int)nn, st));
    DGP_CUDA(cudaMemcpyAsync(&hb, d.p, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaStreamSynchronize(st));
  }
  F->nbnd = hb;
  return DGP_OK;
}

int fem_assemble(FemPlan *F, const double *d_mua, const double *d_musp, double *d_K, double *d_M,
                 cudaStream_t st) {
  DGP_REQUIRE(d_mua && d_musp && d_K && d_M, "fem_assemble: null pointer");
  const int bs = 128;
  if (!F->flag.p) DGP_TRY(F->flag.alloc(sizeof(int)));
  DGP_CUDA(cudaMemsetAsync(F->flag.p, 0, sizeof(int), st));
  k_element_blocks<<<grid1(F->ne, bs), bs, 0, st>>>(F->node.as<double>(), F->elem.as<int32_t>(), F->ne, d_mua,
                                                   d_musp, F->Ke.as<double>(), F->Me.as<double>(), F->flag.as<int>());
  DGP_CHECK_LAUNCH();
  if (F->nfaces > 0) {
    k_face_blocks<<<grid1(F->nfaces, bs), bs, 0, st>>>(F->node.as<double>(), F->faces.as<int32_t>(), F->nfaces,
                                                      F->bnd.as<int32_t>(), F->rfac, F->Be.as<double>());
    DGP_CHECK_LAUNCH();
  }
  k_gather_slots<<<grid1(F->nnz, 256), 256, 0, st>>>(F->cstart.as<int32_t>(), F->payload.as<int32_t>(), F->nnz,
                                                    F->nk, 16 * F->ne, F->elem.as<int32_t>(),
                                                    F->faces.as<int32_t>(), F->Ke.as<double>(), F->Me.as<double>(),
                                                    F->Be.as<double>(), d_K, d_M);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

int fem_adjoint_grad(FemPlan *F, const double *d_mua, const double *d_musp, const double *d_phi,
                     const double *d_lam, int32_t nf, int32_t ns, double *d_gmua, double *d_gmusp,
                     cudaStream_t st) {
  DGP_REQUIRE(d_mua && d_musp && d_phi && d_lam && d_gmua, "fem_adjoint_grad: null pointer");
  DGP_REQUIRE(nf > 0 && ns > 0, "fem_adjoint_grad: nf and ns must be positive");
  DGP_TRY(upload_quadrature());
  DGP_CUDA(cudaMemsetAsync(d_gmua, 0, sizeof(double) * F->nn, st));
  if (d_gmusp) DGP_CUDA(cudaMemsetAsync(d_gmusp, 0, sizeof(double) * F->nn, st));
  k_elem_grad<<<grid1(F->ne * 32, 256), 256, 0, st>>>(F->node.as<double>(), F->elem.as<int32_t>(), F->ne,
                                                      (const double2 *)d_phi, (const double2 *)d_lam, F->nn, nf, ns,
                                                      d_mua, d_musp, d_gmua, d_gmusp);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

}  // namespace dgp
