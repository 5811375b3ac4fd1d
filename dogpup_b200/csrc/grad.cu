// Adjoint right-hand sides for the gradient of time-gated detector data.
//
// The reference differentiates its forward model through the explicit
// absorption Jacobian (J_complex, DOGPUP/dMesh.m:206-247, then fc2tg); the
// reverse-mode path here needs no J.  For a real functional
//   L = sum_{m,g} g[m][g] y[m][g],   y = fc2tg(meas(phi))     (fc2tg.m:25-32)
// the chain rule through fc2tg and meas_flu (dMesh.m:144-171) gives
//   c[m][k]   = 2 Nt h_k sum_g g[m][g] conj(gate[g][k])       (h_0 = 1/2, else 1)
//   B[k][:,s] = sum_{m = (s, d)} c[m][k] D_d                  (D_d: detector d's weights)
// and lam = A_k^-1 B (A_k^T = A_k) is one solve per source x harmonic, the
// same batch shape as the forward solve.  The element kernel in fem.cu turns
// (phi, lam) into dL/dmua and dL/dmusp.
#include <vector>

#include "dgp_common.cuh"
#include "dgp_internal.h"

namespace dgp {

namespace {

// c[m][k] = 2 Nt h_k sum_g g[m][g] conj(gate[g][k])
__global__ void k_tg_coef(const double *__restrict__ g, const double2 *__restrict__ gate, int nm, int ng, int nf,
                          int nt, double2 *c) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)nm * nf) return;
  const int m = (int)(t / nf), k = (int)(t % nf);
  double re = 0.0, im = 0.0;
  for (int q = 0; q < ng; ++q) {
    const double w = g[(int64_t)m * ng + q];
    const double2 gk = gate[(int64_t)q * nf + k];
    re += w * gk.x;
    im -= w * gk.y;
  }
  const double s = 2.0 * nt * (k == 0 ? 0.5 : 1.0);
  c[t] = make_double2(s * re, s * im);
}

// one thread per (source, harmonic): the source's links in ascending order,
// so every right-hand-side entry is summed in a fixed order (no atomics)
__global__ void k_adjoint_rhs(const int32_t *__restrict__ dn, const double *__restrict__ dw,
                              const int32_t *__restrict__ lrow, const int32_t *__restrict__ lidx,
                              const int32_t *__restrict__ link, const double2 *__restrict__ c, int64_t n, int nf,
                              int ns, double2 *B, int *bad) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)ns * nf) return;
  const int k = (int)(t / ns), s = (int)(t % ns);
  double2 *col = B + (int64_t)k * n * ns + s;
  for (int p = lrow[s]; p < lrow[s + 1]; ++p) {
    const int m = lidx[p];
    const int d = link[2 * m + 1];
    const double2 cm = c[(int64_t)m * nf + k];
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      const double w = dw[4 * d + l];
      if (!(w > 0.0)) continue;  // detector weights as meas_flu uses them (dMesh.m:157-160)
      const int32_t node = dn[4 * d + l];
      if (node < 0 || node >= n) { atomicOr(bad, 2); continue; }
      double2 *dst = col + (int64_t)node * ns;
      dst->x += w * cm.x;
      dst->y += w * cm.y;
    }
  }
}

}  // namespace

int tg_adjoint_rhs(const int32_t *d_det_nodes, const double *d_det_w, int32_t nd, const int32_t *d_link, int32_t nm,
                   const double *d_gate_fc, int32_t ng, int32_t nt, const double *d_g, int64_t n, int32_t nf,
                   int32_t ns, double *d_B, cudaStream_t st) {
  DGP_REQUIRE(d_det_nodes && d_det_w && d_link && d_gate_fc && d_g && d_B, "tg_adjoint_rhs: null pointer");
  DGP_REQUIRE(nd > 0 && nm > 0 && ng > 0 && nt > 0 && n > 0 && nf > 0 && ns > 0, "tg_adjoint_rhs: bad sizes");
  // links grouped by source on the host: nm is small (sources x detectors)
  std::vector<int32_t> hl(2 * (size_t)nm);
  DGP_CUDA(cudaMemcpyAsync(hl.data(), d_link, sizeof(int32_t) * 2 * nm, cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  std::vector<int32_t> rowp(ns + 1, 0), idx(nm);
  for (int m = 0; m < nm; ++m) {
    const int s = hl[2 * m], d = hl[2 * m + 1];
    if (s < 0 || s >= ns || d < 0 || d >= nd) return fail(DGP_ERR_ARG, "tg_adjoint_rhs: link index out of range");
    rowp[s + 1]++;
  }
  for (int s = 0; s < ns; ++s) rowp[s + 1] += rowp[s];
  {
    std::vector<int32_t> fill(rowp.begin(), rowp.end() - 1);
    for (int m = 0; m < nm; ++m) idx[fill[hl[2 * m]]++] = m;
  }
  DevBuf ws;
  const size_t coef_bytes = sizeof(double2) * (size_t)nm * nf;
  const size_t meta = sizeof(int32_t) * ((size_t)ns + 1 + nm) + sizeof(int);
  DGP_TRY(ws.alloc(coef_bytes + meta));
  double2 *c = ws.as<double2>();
  int32_t *d_rowp = (int32_t *)((char *)ws.p + coef_bytes);
  int32_t *d_idx = d_rowp + ns + 1;
  int *bad = (int *)(d_idx + nm);
  DGP_CUDA(cudaMemcpyAsync(d_rowp, rowp.data(), sizeof(int32_t) * (ns + 1), cudaMemcpyHostToDevice, st));
  DGP_CUDA(cudaMemcpyAsync(d_idx, idx.data(), sizeof(int32_t) * nm, cudaMemcpyHostToDevice, st));
  DGP_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), st));
  DGP_CUDA(cudaMemsetAsync(d_B, 0, sizeof(double2) * (size_t)nf * n * ns, st));
  k_tg_coef<<<(unsigned)ceil_div((int64_t)nm * nf, 256), 256, 0, st>>>(d_g, (const double2 *)d_gate_fc, nm, ng, nf,
                                                                        nt, c);
  DGP_CHECK_LAUNCH();
  k_adjoint_rhs<<<(unsigned)ceil_div((int64_t)ns * nf, 128), 128, 0, st>>>(d_det_nodes, d_det_w, d_rowp, d_idx,
                                                                            d_link, c, n, nf, ns, (double2 *)d_B, bad);
  DGP_CHECK_LAUNCH();
  int h = 0;
  DGP_CUDA(cudaMemcpyAsync(&h, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  if (h) return fail(DGP_ERR_ARG, "tg_adjoint_rhs: detector node index out of range");
  return DGP_OK;
}

}  // namespace dgp
