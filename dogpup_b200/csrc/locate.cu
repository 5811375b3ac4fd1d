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

}  // namespace dgp
