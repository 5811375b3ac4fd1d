// Point location on the device: the containing tetrahedron and barycentric
// weights of many points (voxel centres of the Jacobian's grid basis).
//
// Replaces the point location inside mesh2grid (DOGPUP/dMesh.m:286-380; the
// reference calls MATLAB's pointLocation on the host).  Elements are binned
// into a uniform grid of cells by their bounding boxes (count, scan, fill);
// each point tests the elements of its cell and keeps the one whose smallest
// barycentric weight is largest (ties: lower element id), accepted when that
// weight is >= -eps -- the same rule as the host locator, independent of the
// order in which the bins were filled.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "dgp_common.cuh"
#include "dgp_internal.h"

namespace dgp {

namespace {

struct Bins {
  double lo[3];
  double inv[3];  // cells per unit length
  int n[3];
  __device__ int clampi(int v, int d) const { return v < 0 ? 0 : (v >= n[d] ? n[d] - 1 : v); }
  __device__ int cell_of(double x, int d) const { return clampi((int)floor((x - lo[d]) * inv[d]), d); }
};

__device__ inline void elem_box(const double *__restrict__ node, const int32_t *__restrict__ elem, int64_t e,
                                const Bins &B, int c0[3], int c1[3]) {
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
#pragma unroll
  for (int l = 0; l < 4; ++l) {
    const int64_t v = elem[4 * e + l];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double x = node[3 * v + d];
      mn[d] = fmin(mn[d], x);
      mx[d] = fmax(mx[d], x);
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    c0[d] = B.cell_of(mn[d], d);
    c1[d] = B.cell_of(mx[d], d);
  }
}

__global__ void k_bin_count(const double *__restrict__ node, const int32_t *__restrict__ elem, int64_t ne, Bins B,
                            int32_t *count) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int c0[3], c1[3];
  elem_box(node, elem, e, B, c0, c1);
  for (int k = c0[2]; k <= c1[2]; ++k)
    for (int j = c0[1]; j <= c1[1]; ++j)
      for (int i = c0[0]; i <= c1[0]; ++i) atomicAdd(count + ((int64_t)k * B.n[1] + j) * B.n[0] + i, 1);
}

__global__ void k_bin_fill(const double *__restrict__ node, const int32_t *__restrict__ elem, int64_t ne, Bins B,
                           const int32_t *__restrict__ start, int32_t *cursor, int32_t *items) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ne) return;
  int c0[3], c1[3];
  elem_box(node, elem, e, B, c0, c1);
  for (int k = c0[2]; k <= c1[2]; ++k)
    for (int j = c0[1]; j <= c1[1]; ++j)
      for (int i = c0[0]; i <= c1[0]; ++i) {
        const int64_t c = ((int64_t)k * B.n[1] + j) * B.n[0] + i;
        items[start[c] + atomicAdd(cursor + c, 1)] = (int32_t)e;
      }
}

// barycentric weights of p in element e (weights of vertices 0..3)
__device__ inline void bary(const double *__restrict__ node, const int32_t *__restrict__ elem, int64_t e,
                            const double p[3], double w[4]) {
  double v[4][3];
#pragma unroll
  for (int l = 0; l < 4; ++l)
#pragma unroll
    for (int d = 0; d < 3; ++d) v[l][d] = node[3 * (int64_t)elem[4 * e + l] + d];
  // columns a = v1 - v0, b = v2 - v0, c = v3 - v0; solve [a b c] l = p - v0 by Cramer's rule
  double a[3], b[3], c[3], q[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    a[d] = v[1][d] - v[0][d];
    b[d] = v[2][d] - v[0][d];
    c[d] = v[3][d] - v[0][d];
    q[d] = p[d] - v[0][d];
  }
  auto det3 = [](const double x[3], const double y[3], const double z[3]) {
    return x[0] * (y[1] * z[2] - y[2] * z[1]) - y[0] * (x[1] * z[2] - x[2] * z[1]) + z[0] * (x[1] * y[2] - x[2] * y[1]);
  };
  const double D = det3(a, b, c);
  const double l1 = det3(q, b, c) / D, l2 = det3(a, q, c) / D, l3 = det3(a, b, q) / D;
  w[0] = 1.0 - l1 - l2 - l3;
  w[1] = l1;
  w[2] = l2;
  w[3] = l3;
}

__global__ void k_locate(const double *__restrict__ node, const int32_t *__restrict__ elem, Bins B,
                         const int32_t *__restrict__ start, const int32_t *__restrict__ items,
                         const double *__restrict__ pts, int64_t np, double eps, int32_t *eid, double *wout) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= np) return;
  const double p[3] = {pts[3 * t], pts[3 * t + 1], pts[3 * t + 2]};
  bool inside = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double f = (p[d] - B.lo[d]) * B.inv[d];
    if (f < -1e-9 || f > B.n[d] + 1e-9) inside = false;
  }
  int32_t best = -1;
  double bs = -1e300, bw[4] = {0, 0, 0, 0};
  if (inside) {
    const int64_t c = ((int64_t)B.cell_of(p[2], 2) * B.n[1] + B.cell_of(p[1], 1)) * B.n[0] + B.cell_of(p[0], 0);
    for (int q = start[c]; q < start[c + 1]; ++q) {
      const int32_t e = items[q];
      double w[4];
      bary(node, elem, e, p, w);
      const double s = fmin(fmin(w[0], w[1]), fmin(w[2], w[3]));
      if (s > bs || (s == bs && e < best)) {
        bs = s;
        best = e;
#pragma unroll
        for (int l = 0; l < 4; ++l) bw[l] = w[l];
      }
    }
  }
  const bool ok = best >= 0 && bs >= -eps;
  eid[t] = ok ? best : -1;
#pragma unroll
  for (int l = 0; l < 4; ++l) wout[4 * t + l] = ok ? bw[l] : 0.0;
}

}  // namespace

int locate_points(const double *d_node, const int32_t *d_elem, int64_t nn, int64_t ne, const double *d_pts,
                  int64_t np, double eps, int32_t *d_eid, double *d_w, cudaStream_t st) {
  DGP_REQUIRE(d_node && d_elem, "locate_points: null mesh pointer");
  DGP_REQUIRE(nn > 0 && ne > 0 && np >= 0, "locate_points: bad sizes");
  if (np == 0) return DGP_OK;
  DGP_REQUIRE(d_pts && d_eid && d_w, "locate_points: null point pointer");
  DGP_TRY(ids_in_range(d_elem, 4 * ne, nn, "locate_points", st));
  // bins: bounding box of the nodes, cells of about two mean element edges
  std::vector<double> h((size_t)3 * nn);
  DGP_CUDA(cudaMemcpyAsync(h.data(), d_node, sizeof(double) * 3 * nn, cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int64_t i = 0; i < nn; ++i)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], h[3 * i + d]);
      hi[d] = std::max(hi[d], h[3 * i + d]);
    }
  const double vol = std::max(1e-300, (hi[0] - lo[0]) * (hi[1] - lo[1]) * (hi[2] - lo[2]));
  const double cell = 2.0 * std::cbrt(vol / (double)ne * 6.0);
  Bins B;
  int64_t ncell = 1;
  for (int d = 0; d < 3; ++d) {
    const double ext = std::max(hi[d] - lo[d], 1e-12);
    B.n[d] = (int)std::min<double>(512.0, std::max(1.0, std::ceil(ext / std::max(cell, 1e-300))));
    B.lo[d] = lo[d];
    B.inv[d] = B.n[d] / ext;
    ncell *= B.n[d];
  }
  DevBuf cnt, start, cursor, items, tmp;
  DGP_TRY(cnt.alloc(sizeof(int32_t) * (ncell + 1)));
  DGP_TRY(start.alloc(sizeof(int32_t) * (ncell + 1)));
  DGP_TRY(cursor.alloc(sizeof(int32_t) * ncell));
  DGP_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * (ncell + 1), st));
  DGP_CUDA(cudaMemsetAsync(cursor.p, 0, sizeof(int32_t) * ncell, st));
  const unsigned ge = (unsigned)ceil_div(ne, 256);
  k_bin_count<<<ge, 256, 0, st>>>(d_node, d_elem, ne, B, cnt.as<int32_t>());
  DGP_CHECK_LAUNCH();
  size_t tb = 0;
  DGP_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<int32_t>(), start.as<int32_t>(), (int)(ncell + 1), st));
  DGP_TRY(tmp.alloc(tb));
  DGP_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.as<int32_t>(), start.as<int32_t>(), (int)(ncell + 1), st));
  int32_t total = 0;
  DGP_CUDA(cudaMemcpyAsync(&total, start.as<int32_t>() + ncell, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  DGP_TRY(items.alloc(sizeof(int32_t) * std::max(1, total)));
  k_bin_fill<<<ge, 256, 0, st>>>(d_node, d_elem, ne, B, start.as<int32_t>(), cursor.as<int32_t>(),
                                 items.as<int32_t>());
  DGP_CHECK_LAUNCH();
  k_locate<<<(unsigned)ceil_div(np, 128), 128, 0, st>>>(d_node, d_elem, B, start.as<int32_t>(), items.as<int32_t>(),
                                                       d_pts, np, eps, d_eid, d_w);
  DGP_CHECK_LAUNCH();
  DGP_CUDA(cudaStreamSynchronize(st));
  return DGP_OK;
}


// ---------------------------------------------------------------------------
// Grid-to-mesh interpolation g2m [nn x nv] (dMesh.m:330-373).
//
// The reference triangulates the voxel centres (delaunay), locates every node
// in that triangulation and keeps the barycentric weights of in-mesh voxels;
// a node none of whose four voxels is in the mesh takes its nearest in-mesh
// voxel with weight 1; rows are normalised to sum 1 (rows summing to 0 stay
// 0).  The Delaunay triangulation of a rectilinear lattice is not unique
// (the eight corners of a cell are cospherical); the Kuhn split is used:
// cell corner c, fractional offsets sorted t_a >= t_b >= t_c (ties by axis
// order) give the simplex c, c+e_a, c+e_a+e_b, c+1 with weights 1-t_a,
// t_a-t_b, t_b-t_c, t_c.  No search is needed for the simplex; the nearest
// in-mesh voxel is found by expanding shells around the nearest lattice point.
// ---------------------------------------------------------------------------
namespace {

struct Lattice {
  double o[3], d[3];
  int n[3];
  __device__ int64_t index(int i, int j, int k) const { return ((int64_t)k * n[1] + j) * n[0] + i; }
};

__device__ inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// nearest in-mesh voxel of p (ties: lower voxel index); -1 if the grid has none
__device__ int64_t nearest_inmesh(const Lattice &L, const uint8_t *__restrict__ inmesh, const double p[3]) {
  double f[3];
  int c[3];
  double e = 0.0, dmin = 1e300;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    f[d] = (p[d] - L.o[d]) / L.d[d];
    const double r = rint(fmin(fmax(f[d], -1.0), (double)L.n[d]));
    c[d] = clampi((int)r, 0, L.n[d] - 1);
    e = fmax(e, fabs(f[d] - c[d]));
    dmin = fmin(dmin, fabs(L.d[d]));
  }
  const int rmax = max(L.n[0], max(L.n[1], L.n[2]));
  int64_t best = -1;
  double bd = 1e300;
  for (int r = 0; r <= rmax; ++r) {
    // every voxel of shell r is at least dmin * (r - e) away
    if (best >= 0 && (r - e) * dmin > sqrt(bd)) break;
    const int k0 = max(c[2] - r, 0), k1 = min(c[2] + r, L.n[2] - 1);
    const int j0 = max(c[1] - r, 0), j1 = min(c[1] + r, L.n[1] - 1);
    for (int k = k0; k <= k1; ++k)
      for (int j = j0; j <= j1; ++j) {
        const bool face = abs(k - c[2]) == r || abs(j - c[1]) == r;
        const int step = face ? 1 : 2 * r;
        for (int i = c[0] - r; i <= c[0] + r; i += (r == 0 ? 1 : step)) {
          if (i < 0 || i >= L.n[0]) continue;
          const int64_t v = L.index(i, j, k);
          if (!inmesh[v]) continue;
          // voxel centre o + i*d and squared distance rounded step by step (no contraction),
          // so that equal distances compare equal whatever the compiler fuses
          const double dx = p[0] - __dadd_rn(L.o[0], __dmul_rn((double)i, L.d[0]));
          const double dy = p[1] - __dadd_rn(L.o[1], __dmul_rn((double)j, L.d[1]));
          const double dz = p[2] - __dadd_rn(L.o[2], __dmul_rn((double)k, L.d[2]));
          const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
          if (d2 < bd || (d2 == bd && v < best)) {
            bd = d2;
            best = v;
          }
        }
      }
  }
  return best;
}

__global__ void k_grid_to_mesh(const double *__restrict__ node, int64_t nn, Lattice L,
                               const uint8_t *__restrict__ inmesh, int32_t *__restrict__ col,
                               double *__restrict__ val) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nn) return;
  const double p[3] = {node[3 * t], node[3 * t + 1], node[3 * t + 2]};
  int32_t vc[4] = {-1, -1, -1, -1};
  double vw[4] = {0, 0, 0, 0};
  bool in_grid = true;
  int cell[3];
  double fr[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double f = (p[d] - L.o[d]) / L.d[d];
    if (!(f >= 0.0 && f <= (double)(L.n[d] - 1))) in_grid = false;   // also NaN
    const int hi = max(L.n[d] - 2, 0);
    cell[d] = in_grid ? clampi((int)floor(f), 0, hi) : 0;
    fr[d] = in_grid ? f - cell[d] : 0.0;
    if (L.n[d] == 1) fr[d] = 0.0;                                     // flat axis: stay on the plane
  }
  int kept = 0;
  if (in_grid) {
    // axis order by descending fraction (stable in x, y, z)
    int a = 0, b = 1, c = 2;
    if (fr[b] > fr[a]) { int s = a; a = b; b = s; }
    if (fr[c] > fr[b]) { int s = b; b = c; c = s; }
    if (fr[b] > fr[a]) { int s = a; a = b; b = s; }
    const double w[4] = {1.0 - fr[a], fr[a] - fr[b], fr[b] - fr[c], fr[c]};
    int v[3] = {cell[0], cell[1], cell[2]};
    const int ax[3] = {a, b, c};
    double sum = 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (q > 0) v[ax[q - 1]] = min(v[ax[q - 1]] + 1, L.n[ax[q - 1]] - 1);
      const int64_t vox = L.index(v[0], v[1], v[2]);
      if (inmesh[vox]) {
        ++kept;
        if (w[q] != 0.0) {
          vc[q] = (int32_t)vox;
          vw[q] = w[q];
          sum += w[q];
        }
      }
    }
    if (kept > 0 && sum != 0.0) {
#pragma unroll
      for (int q = 0; q < 4; ++q) vw[q] = vw[q] / sum;
    }
  }
  if (kept == 0) {
    const int64_t v = nearest_inmesh(L, inmesh, p);
    if (v >= 0) {
      vc[0] = (int32_t)v;
      vw[0] = 1.0;
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    col[4 * t + q] = vc[q];
    val[4 * t + q] = vw[q];
  }
}

}  // namespace

int grid_to_mesh(const double *d_node, int64_t nn, const double origin[3], const double spacing[3], const int32_t n[3],
                 const uint8_t *d_inmesh, int32_t *d_col, double *d_val, cudaStream_t st) {
  DGP_REQUIRE(d_node && d_inmesh && d_col && d_val, "grid_to_mesh: null pointer");
  DGP_REQUIRE(nn > 0, "grid_to_mesh: no nodes");
  Lattice L;
  int64_t nv = 1;
  for (int d = 0; d < 3; ++d) {
    DGP_REQUIRE(n[d] >= 1 && spacing[d] != 0.0 && std::isfinite(spacing[d]) && std::isfinite(origin[d]),
                "grid_to_mesh: bad lattice");
    L.o[d] = origin[d];
    L.d[d] = spacing[d];
    L.n[d] = n[d];
    nv *= n[d];
  }
  DGP_REQUIRE(nv < (int64_t)INT32_MAX, "grid_to_mesh: more than 2^31-1 voxels");
  k_grid_to_mesh<<<(unsigned)ceil_div(nn, 128), 128, 0, st>>>(d_node, nn, L, d_inmesh, d_col, d_val);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

// ---------------------------------------------------------------------------
// Optode snapping (snap_pos, dOptode.m:155-190): nearest boundary node
// (dsearchn), then the closest point on the surface triangles that contain
// that node (ties: lower face index) and the face's normal -cross(b-a, c-a)
// normalised.  One block per optode; both searches are block-wide argmins.
// ---------------------------------------------------------------------------
namespace {

struct D3 {
  double x, y, z;
};
__device__ inline D3 ld3(const double *p, int64_t i) { return D3{p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }
__device__ inline D3 sub3(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ inline D3 axpy3(double s, D3 a, D3 b) { return D3{b.x + s * a.x, b.y + s * a.y, b.z + s * a.z}; }
__device__ inline double dot3(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// closest point of triangle abc to p: Voronoi-region walk over the vertices, edges and the
// face (Ericson, Real-Time Collision Detection, sec. 5.1.5)
__device__ D3 closest_on_triangle(D3 p, D3 a, D3 b, D3 c) {
  const D3 ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
  const double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0 && d2 <= 0) return a;
  const D3 bp = sub3(p, b);
  const double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0 && d4 <= d3) return b;
  const double vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) return axpy3(d1 / (d1 - d3), ab, a);
  const D3 cp = sub3(p, c);
  const double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0 && d5 <= d6) return c;
  const double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) return axpy3(d2 / (d2 - d6), ac, a);
  const double va = d3 * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0)
    return axpy3((d4 - d3) / ((d4 - d3) + (d5 - d6)), sub3(c, b), b);
  const double den = 1.0 / (va + vb + vc);
  return axpy3(vc * den, ac, axpy3(vb * den, ab, a));
}

// block argmin of (value, index): smaller value, then smaller index; result in thread 0's return
template <int NT>
__device__ void block_argmin(double &v, int64_t &i) {
  __shared__ double sv[NT];
  __shared__ int64_t si[NT];
  sv[threadIdx.x] = v;
  si[threadIdx.x] = i;
  __syncthreads();
  for (int o = NT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      const double w = sv[threadIdx.x + o];
      const int64_t j = si[threadIdx.x + o];
      if (w < sv[threadIdx.x] || (w == sv[threadIdx.x] && j >= 0 && (si[threadIdx.x] < 0 || j < si[threadIdx.x]))) {
        sv[threadIdx.x] = w;
        si[threadIdx.x] = j;
      }
    }
    __syncthreads();
  }
  v = sv[0];
  i = si[0];
  __syncthreads();
}

constexpr int SNAP_NT = 256;

__global__ void __launch_bounds__(SNAP_NT) k_snap(const double *__restrict__ node, int64_t nn,
                                                  const int32_t *__restrict__ bnd, const int32_t *__restrict__ face,
                                                  int64_t nface, const double *__restrict__ pos,
                                                  double *__restrict__ out_pos, double *__restrict__ out_dir,
                                                  int32_t *__restrict__ out_face) {
  const int64_t o = blockIdx.x;
  const D3 p = ld3(pos, o);
  // nearest boundary node
  double bd = INFINITY;
  int64_t bi = -1;
  for (int64_t i = threadIdx.x; i < nn; i += SNAP_NT) {
    if (!bnd[i]) continue;
    const D3 d = sub3(ld3(node, i), p);
    const double d2 = dot3(d, d);
    if (d2 < bd) {  // ascending i per thread: the first minimum is kept
      bd = d2;
      bi = i;
    }
  }
  block_argmin<SNAP_NT>(bd, bi);
  // closest point over the faces that contain that node
  double fd = INFINITY;
  int64_t fi = -1;
  if (bi >= 0) {
    for (int64_t f = threadIdx.x; f < nface; f += SNAP_NT) {
      const int32_t v0 = face[3 * f], v1 = face[3 * f + 1], v2 = face[3 * f + 2];
      if (v0 != bi && v1 != bi && v2 != bi) continue;
      const D3 q = closest_on_triangle(p, ld3(node, v0), ld3(node, v1), ld3(node, v2));
      const D3 d = sub3(q, p);
      const double dist = sqrt(dot3(d, d));
      if (dist < fd) {
        fd = dist;
        fi = f;
      }
    }
  }
  block_argmin<SNAP_NT>(fd, fi);
  if (threadIdx.x != 0) return;
  out_face[o] = (int32_t)fi;
  if (fi < 0) {
    for (int d = 0; d < 3; ++d) out_pos[3 * o + d] = out_dir[3 * o + d] = NAN;
    return;
  }
  const D3 a = ld3(node, face[3 * fi]), b = ld3(node, face[3 * fi + 1]), c = ld3(node, face[3 * fi + 2]);
  const D3 q = closest_on_triangle(p, a, b, c);
  const D3 u = sub3(b, a), w = sub3(c, a);
  D3 nv{-(u.y * w.z - u.z * w.y), -(u.z * w.x - u.x * w.z), -(u.x * w.y - u.y * w.x)};
  const double len = sqrt(dot3(nv, nv));
  out_pos[3 * o] = q.x;
  out_pos[3 * o + 1] = q.y;
  out_pos[3 * o + 2] = q.z;
  out_dir[3 * o] = nv.x / len;
  out_dir[3 * o + 1] = nv.y / len;
  out_dir[3 * o + 2] = nv.z / len;
}

}  // namespace

int snap_to_surface(const double *d_node, int64_t nn, const int32_t *d_bnd, const int32_t *d_face, int64_t nface,
                    const double *d_pos, int64_t n, double *d_out_pos, double *d_out_dir, int32_t *d_out_face,
                    cudaStream_t st) {
  DGP_REQUIRE(nn > 0 && nface > 0 && n >= 0, "snap_to_surface: bad sizes");
  if (n == 0) return DGP_OK;
  DGP_REQUIRE(d_node && d_bnd && d_face && d_pos && d_out_pos && d_out_dir && d_out_face,
              "snap_to_surface: null pointer");
  DGP_REQUIRE(n <= INT32_MAX, "snap_to_surface: too many optodes");
  DGP_TRY(ids_in_range(d_face, 3 * nface, nn, "snap_to_surface", st));
  k_snap<<<(unsigned)n, SNAP_NT, 0, st>>>(d_node, nn, d_bnd, d_face, nface, d_pos, d_out_pos, d_out_dir, d_out_face);
  DGP_CHECK_LAUNCH();
  std::vector<int32_t> hf((size_t)n);
  DGP_CUDA(cudaMemcpyAsync(hf.data(), d_out_face, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  for (int64_t i = 0; i < n; ++i)
    if (hf[i] < 0) return fail(DGP_ERR_ARG, "snap_to_surface: no boundary node or no face on it");
  return DGP_OK;
}

}  // namespace dgp
