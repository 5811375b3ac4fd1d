// Fourier-series transforms and detector read-out on the device.
//
//   td2fc  DOGPUP/td2fc.m:26-32  c_k = dt/t_end * sum_t exp(-i f_k t) x(t)
//   fc2td  DOGPUP/fc2td.m:24-31  x(t) = 2 Re sum_k exp(i f_k t) c~_k, c~_0 = c_0/2
//   fc2tg  DOGPUP/fc2tg.m:25-32  y_g = Nt * 2 Re sum_k conj(gate_gk) c~_k
//   meas   DOGPUP/dMesh.m:144-171 data[m,k] = sum_l w_dl phi[k, node_dl, s_m]
//   csr    y = A x for a real FP64 CSR A: the voxel-basis maps of the LM update,
//          G = m2g * mua and d_mu = g2m * x (wghtd_LM_recon.m:105, :133)
//
// These act on detector-sized data (NM x NF); the large Jacobian-sized
// fc2tg is fused into the Jacobian kernels.  One thread per output element,
// FP64 throughout, angles f_k * t formed as the reference forms them.
#include "dgp_common.cuh"
#include "dgp_internal.h"

namespace dgp {

namespace {

__global__ void k_td2fc(const double *__restrict__ x, int64_t nr, int nt, const double *__restrict__ t,
                        const double *__restrict__ f, int nf, double2 *__restrict__ c) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= nr * nf) return;
  int64_t r = e / nf;
  int k = (int)(e % nf);
  const double dt = t[1] - t[0], P = t[nt - 1];
  double sr = 0.0, si = 0.0;
  for (int q = 0; q < nt; ++q) {
    double s, co;
    sincos(t[q] * f[k], &s, &co);
    double v = x[r * nt + q];
    sr += co * v;
    si -= s * v;
  }
  c[e] = make_double2(dt * sr / P, dt * si / P);
}

__global__ void k_fc2td(const double2 *__restrict__ c, int64_t nr, int nf, const double *__restrict__ f,
                        const double *__restrict__ t, int nt, double *__restrict__ x) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= nr * nt) return;
  int64_t r = e / nt;
  int q = (int)(e % nt);
  double acc = 0.0;
  for (int k = 0; k < nf; ++k) {
    double2 v = c[r * nf + k];
    if (k == 0) { v.x *= 0.5; v.y *= 0.5; }
    double s, co;
    sincos(f[k] * t[q], &s, &co);
    acc += co * v.x - s * v.y;
  }
  x[e] = 2.0 * acc;
}

__global__ void k_fc2tg(const double2 *__restrict__ c, int64_t nr, int nf, const double2 *__restrict__ gate, int ng,
                        int nt, double *__restrict__ y) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= nr * ng) return;
  int64_t r = e / ng;
  int g = (int)(e % ng);
  double acc = 0.0;
  for (int k = 0; k < nf; ++k) {
    double2 v = c[r * nf + k];
    if (k == 0) { v.x *= 0.5; v.y *= 0.5; }
    double2 gk = gate[(int64_t)g * nf + k];
    acc += gk.x * v.x + gk.y * v.y;  // Re(conj(gate) * c)
  }
  y[e] = (double)nt * 2.0 * acc;
}

__global__ void k_meas(const int32_t *__restrict__ dn, const double *__restrict__ dw, int nd,
                       const int32_t *__restrict__ link, int nm, const double2 *__restrict__ phi, int64_t n, int nf, int ns, double2 *__restrict__ data,
                       int *bad) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)nm * nf) return;
  int m = (int)(e / nf), k = (int)(e % nf);
  int s = link[2 * m], d = link[2 * m + 1];
  if (s < 0 || s >= ns || d < 0 || d >= nd) { atomicOr(bad, 1); return; }
  double2 acc = make_double2(0, 0);
  for (int l = 0; l < 4; ++l) {
    double w = dw[4 * d + l];
    int32_t node = dn[4 * d + l];
    if (!(w > 0.0)) continue;  // the reference keeps strictly positive weights only (dMesh.m:157-160)
    if (node < 0 || node >= n) { atomicOr(bad, 2); continue; }
    double2 p = phi[((int64_t)k * n + node) * ns + s];
    acc.x += w * p.x;
    acc.y += w * p.y;
  }
  data[e] = acc;
}

// one thread per row (the basis maps hold <= 8 entries per row); entries whose column
// lies outside [0, ncols) are skipped, so a malformed matrix cannot read past x
__global__ void k_csr_spmv(const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                           const double *__restrict__ val, int64_t nrows, int64_t ncols, const double *__restrict__ x,
                           double *__restrict__ y) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nrows) return;
  double acc = 0.0;
  for (int p = rowptr[i], e = rowptr[i + 1]; p < e; ++p) {
    const int j = col[p];
    if (j >= 0 && j < ncols) acc = fma(val[p], x[j], acc);
  }
  y[i] = acc;
}

inline unsigned g1(int64_t n, int bs) { return (unsigned)ceil_div(n, bs); }

}  // namespace

int td2fc_run(const double *x, int64_t nr, int nt, const double *t, const double *f, int nf, double *c,
              cudaStream_t st) {
  DGP_REQUIRE(x && t && f && c, "td2fc: null pointer");
  DGP_REQUIRE(nr > 0 && nt >= 2 && nf > 0, "td2fc: need nr > 0, nt >= 2, nf > 0");
  k_td2fc<<<g1(nr * nf, 128), 128, 0, st>>>(x, nr, nt, t, f, nf, (double2 *)c);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

int fc2td_run(const double *c, int64_t nr, int nf, const double *f, const double *t, int nt, double *x,
              cudaStream_t st) {
  DGP_REQUIRE(x && t && f && c, "fc2td: null pointer");
  DGP_REQUIRE(nr > 0 && nt > 0 && nf > 0, "fc2td: sizes must be positive");
  k_fc2td<<<g1(nr * nt, 128), 128, 0, st>>>((const double2 *)c, nr, nf, f, t, nt, x);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

int fc2tg_run(const double *c, int64_t nr, int nf, const double *gate, int ng, int nt, double *y, cudaStream_t st) {
  DGP_REQUIRE(c && gate && y, "fc2tg: null pointer");
  DGP_REQUIRE(nr > 0 && ng > 0 && nf > 0, "fc2tg: sizes must be positive");
  k_fc2tg<<<g1(nr * ng, 128), 128, 0, st>>>((const double2 *)c, nr, nf, (const double2 *)gate, ng, nt, y);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

int csr_spmv_run(const int32_t *rowptr, const int32_t *col, const double *val, int64_t nrows, int64_t ncols,
                 const double *x, double *y, cudaStream_t st) {
  DGP_REQUIRE(rowptr && col && val && x && y, "csr_spmv: null pointer");
  DGP_REQUIRE(nrows > 0 && ncols > 0, "csr_spmv: sizes must be positive");
  k_csr_spmv<<<g1(nrows, 256), 256, 0, st>>>(rowptr, col, val, nrows, ncols, x, y);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

int meas_run(const int32_t *dn, const double *dw, int nd, const int32_t *link, int nm, const double *phi, int64_t n, int nf,
             int ns, double *data, cudaStream_t st) {
  DGP_REQUIRE(dn && dw && link && phi && data, "meas: null pointer");
  DGP_REQUIRE(nm > 0 && n > 0 && nf > 0 && ns > 0, "meas: sizes must be positive");
  DevBuf flag;
  DGP_TRY(flag.alloc(sizeof(int)));
  DGP_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
  k_meas<<<g1((int64_t)nm * nf, 128), 128, 0, st>>>(dn, dw, nd, link, nm, (const double2 *)phi, n, nf, ns,
                                                     (double2 *)data, flag.as<int>());
  DGP_CHECK_LAUNCH();
  int h = 0;
  DGP_CUDA(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  if (h & 1) return fail(DGP_ERR_ARG, "meas: link source or detector index out of range");
  if (h & 2) return fail(DGP_ERR_ARG, "meas: detector node index out of range");
  return DGP_OK;
}

}  // namespace dgp
