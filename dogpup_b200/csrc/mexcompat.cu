// Drop-ins for the three host functions of the reference mex sources, on the
// reference's own layouts: split real/imag planes, column-major
// [nrows x ncols x nfreqs] (element (row, col, f) at f*ncols*nrows +
// col*nrows + row), 0-based int32 CSR.
//
//   smv_call    cuda_lib/mex_sources/smvMex.hpp:4-15,    smv_CUDA.cu:8-82
//   FSAImv_call cuda_lib/mex_sources/FSAImvMex.hpp:4-15, FSAImv_CUDA.cu:8-81
//   FSAIP_call  cuda_lib/mex_sources/FSAIP.hpp:4-13,     FSAIP_CUDA.cu:92-180
//
// The reference launches one thread per output element and re-reads the CSR
// row for every (column, frequency).  Here a thread owns one row and CPT
// (column, frequency) pairs: the row's indices and values are loaded once and
// applied to all of them; consecutive threads own consecutive rows, so the
// plane loads and stores stay coalesced.
#include "dgp_common.cuh"
#include "dgp_internal.h"

namespace dgp {

namespace {

constexpr int CPT = 8;

// MODE 0: smv (coefficient ReA + i*fAxis[f]*ImA); MODE 1: FSAImv (G values per f).
// ES = 1: split real / imaginary planes (the reference's host functions);
// ES = 2: interleaved complex, *_im = *_re + 1 (MATLAB's interleaved-complex API).
template <int MODE, int ES>
__global__ void __launch_bounds__(128) k_mexlayout_spmv(double *__restrict__ out_re, double *__restrict__ out_im,
                                                        const double *__restrict__ x_re,
                                                        const double *__restrict__ x_im,
                                                        const double *__restrict__ fAxis,
                                                        const double *__restrict__ v_re,
                                                        const double *__restrict__ v_im, const int *__restrict__ rPtr,
                                                        const int *__restrict__ cPtr, int64_t nnz, int nrows,
                                                        int ncols, int nfreqs) {
  const int64_t row = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t ncol_tot = (int64_t)ncols * nfreqs;
  const int64_t c0 = (int64_t)blockIdx.y * CPT;
  if (row >= nrows) return;
  const int64_t plane = (int64_t)nrows;
  double yr[CPT], yi[CPT], fs[CPT];
  int64_t voff[CPT];
  int nc = 0;
#pragma unroll
  for (int q = 0; q < CPT; ++q) {
    yr[q] = yi[q] = 0.0;
    int64_t c = c0 + q;
    if (c < ncol_tot) nc = q + 1;
    int64_t f = c < ncol_tot ? c / ncols : 0;
    fs[q] = MODE == 0 ? (c < ncol_tot ? fAxis[f] : 0.0) : 0.0;
    voff[q] = MODE == 1 ? nnz * f : 0;
  }
  const int b = rPtr[row], e = rPtr[row + 1];
  for (int p = b; p < e; ++p) {
    const int64_t j = cPtr[p];
    const double ar = v_re[ES * (int64_t)p], ai = v_im[ES * (int64_t)p];
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      if (q >= nc) break;
      double cr, ci;
      if (MODE == 0) {
        cr = ar;
        ci = fs[q] * ai;
      } else {
        cr = v_re[ES * (voff[q] + p)];
        ci = v_im[ES * (voff[q] + p)];
      }
      const int64_t xi = ES * ((c0 + q) * plane + j);
      const double xr = x_re[xi], xim = x_im[xi];
      yr[q] += cr * xr - ci * xim;
      yi[q] += cr * xim + ci * xr;
    }
  }
#pragma unroll
  for (int q = 0; q < CPT; ++q) {
    if (q >= nc) break;
    const int64_t o = ES * ((c0 + q) * plane + row);
    out_re[o] = yr[q];
    out_im[o] = yi[q];
  }
}

__global__ void k_rowmax(const int *__restrict__ rptr, int n, int *m) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicMax(m, rptr[i + 1] - rptr[i]);
}

__global__ void k_split(const double2 *__restrict__ in, int64_t n, double *re, double *im) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < n) {
    re[t] = in[t].x;
    im[t] = in[t].y;
  }
}

// out(k, c, r) = in(k, r, c) for every slice k, 32 x 32 tiles through shared
// memory; in(k, r, c) = in[k*ski + r*sri + c], out(k, c, r) = out[k*sko + c*sco + r]
__global__ void k_transpose_slices(const double2 *__restrict__ in, double2 *__restrict__ out, int64_t R, int64_t C,
                                   int64_t ski, int64_t sri, int64_t sko, int64_t sco) {
  __shared__ double2 tile[32][33];
  const int64_t k = blockIdx.z;
  const int64_t r0 = (int64_t)blockIdx.y * 32, c0 = (int64_t)blockIdx.x * 32;
  const double2 *src = in + k * ski;
  double2 *dst = out + k * sko;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int64_t r = r0 + dy, c = c0 + threadIdx.x;
    if (r < R && c < C) tile[dy][threadIdx.x] = src[r * sri + c];
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int64_t c = c0 + dy, r = r0 + threadIdx.x;
    if (r < R && c < C) dst[c * sco + r] = tile[threadIdx.x][dy];
  }
}

int transpose_slices(const double2 *in, double2 *out, int64_t nk, int64_t R, int64_t C, int64_t ski, int64_t sri,
                     int64_t sko, int64_t sco, cudaStream_t st) {
  DGP_REQUIRE(nk <= 65535 && ceil_div(R, 32) <= 65535, "transpose: too many slices or rows");
  dim3 grid((unsigned)ceil_div(C, 32), (unsigned)ceil_div(R, 32), (unsigned)nk);
  k_transpose_slices<<<grid, dim3(32, 8), 0, st>>>(in, out, R, C, ski, sri, sko, sco);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

}  // namespace

// The whole gpuBicstab_FSAIP contract (dMesh.m:1247-1348) on MATLAB's
// layouts, interleaved complex, column-major:
//   layout 0: [N x NS x NF], element (i, s, k) at i + N*(s + NS*k) (smv_mex's x)
//   layout 1: [N x NF x NS], element (i, k, s) at i + N*(k + NF*s) (fluGPU's Q, phi)
// The batched solver works on [NF][N][NS]; both sides are transposed on the
// device around the solve (two passes against the solve's ~28 per iteration).
int solve_mexlayout(SolverPlan *S, const double *d_Q, double *d_X, int32_t ns, int32_t layout,
                    const dgp_solve_opts *opts, dgp_solve_report *rep, cudaStream_t st) {
  DGP_REQUIRE(d_Q && d_X, "solve_mex: null pointer");
  DGP_REQUIRE(ns >= 1 && ns <= S->ns_max, "solve_mex: 1 <= ns <= ns_max");
  DGP_REQUIRE(layout == 0 || layout == 1, "solve_mex: layout must be 0 ([N x NS x NF]) or 1 ([N x NF x NS])");
  const int64_t n = S->n, nf = S->nf, cnt = nf * n * ns;
  // slice k, row s, column i of the MATLAB array: offsets of (k, s) steps
  const int64_t sk = layout == 0 ? (int64_t)ns * n : n;
  const int64_t ss = layout == 0 ? n : nf * n;
  DevBuf B, X;
  DGP_TRY(B.alloc(sizeof(double2) * cnt));
  DGP_TRY(X.alloc(sizeof(double2) * cnt));
  DGP_TRY(transpose_slices((const double2 *)d_Q, B.as<double2>(), nf, ns, n, sk, ss, n * ns, ns, st));
  const int rc = solver_solve(S, B.as<double>(), nullptr, nullptr, nullptr, X.as<double>(), ns, opts, rep, st);
  if (rc != DGP_OK && rc != DGP_ERR_NOT_CONVERGED) return rc;
  DGP_TRY(transpose_slices(X.as<double2>(), (double2 *)d_X, nf, n, ns, n * ns, ns, sk, ss, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  return rc;
}

int mex_spmv(int mode, double *out_re, double *out_im, const double *x_re, const double *x_im, const double *fAxis,
             const double *v_re, const double *v_im, const int *rPtr, const int *cPtr, int64_t nnz, int nrows,
             int ncols, int nfreqs, cudaStream_t st, int es) {
  DGP_REQUIRE(nrows > 0 && ncols > 0 && nfreqs > 0, "mex spmv: sizes must be positive");
  DGP_REQUIRE(out_re && out_im && x_re && x_im && v_re && v_im && rPtr && cPtr, "mex spmv: null pointer");
  DGP_REQUIRE(mode == 1 || fAxis, "smv: null fAxis");
  int64_t cols = (int64_t)ncols * nfreqs;
  DGP_REQUIRE(ceil_div(cols, CPT) <= 65535, "mex spmv: ncols*nfreqs too large for one launch");
  dim3 grid((unsigned)ceil_div(nrows, 128), (unsigned)ceil_div(cols, CPT));
  DGP_REQUIRE(es == 1 || es == 2, "mex spmv: element stride must be 1 (split) or 2 (interleaved)");
  auto *kern = mode == 0 ? (es == 1 ? k_mexlayout_spmv<0, 1> : k_mexlayout_spmv<0, 2>)
                         : (es == 1 ? k_mexlayout_spmv<1, 1> : k_mexlayout_spmv<1, 2>);
  kern<<<grid, 128, 0, st>>>(out_re, out_im, x_re, x_im, fAxis, v_re, v_im, rPtr, cPtr, nnz, nrows, ncols, nfreqs);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

int mex_fsaip(double *out_re, double *out_im, const double *A_re, const double *A_im, const int *rPtrA,
              const int *cPtrA, const int *rPtrG, const int *cPtrG, int nfreqs, int nrows, cudaStream_t st,
              int es) {
  DGP_REQUIRE(nrows > 0 && nfreqs > 0, "FSAIP: sizes must be positive");
  DGP_REQUIRE(es == 1 || es == 2, "FSAIP: element stride must be 1 (split) or 2 (interleaved)");
  DevBuf m, g, planes;
  DGP_TRY(m.alloc(sizeof(int)));
  DGP_CUDA(cudaMemsetAsync(m.p, 0, sizeof(int), st));
  k_rowmax<<<(unsigned)ceil_div(nrows, 256), 256, 0, st>>>(rPtrG, nrows, m.as<int>());
  DGP_CHECK_LAUNCH();
  int mmax = 0, nnzG = 0;
  DGP_CUDA(cudaMemcpyAsync(&mmax, m.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaMemcpyAsync(&nnzG, rPtrG + nrows, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  DGP_REQUIRE(mmax >= 1 && mmax <= 32, "FSAIP: pattern rows must hold 1..32 entries (the reference caps them at 30)");
  int64_t tot = (int64_t)nnzG * nfreqs;
  if (es == 2) {
    // interleaved tril(A) values -> planes; G is written interleaved straight into the output
    int nnzA = 0;
    DGP_CUDA(cudaMemcpyAsync(&nnzA, rPtrA + nrows, sizeof(int), cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaStreamSynchronize(st));
    DGP_TRY(planes.alloc(sizeof(double) * 2 * (size_t)(nnzA > 0 ? nnzA : 1)));
    double *pre = planes.as<double>(), *pim = pre + nnzA;
    k_split<<<(unsigned)ceil_div(nnzA, 256) + 1, 256, 0, st>>>((const double2 *)A_re, nnzA, pre, pim);
    DGP_CHECK_LAUNCH();
    DGP_TRY(fsai_factor_run(rPtrA, cPtrA, pre, pim, nrows, rPtrG, cPtrG, mmax, nfreqs, (double2 *)out_re, nfreqs, 1,
                            st));
    DGP_CUDA(cudaStreamSynchronize(st));
    return DGP_OK;
  }
  DGP_TRY(g.alloc(sizeof(double2) * tot));
  // output [nnzG][NF] with the harmonic fastest, as the reference writes it (FSAIP_CUDA.cu:112,156)
  DGP_TRY(fsai_factor_run(rPtrA, cPtrA, A_re, A_im, nrows, rPtrG, cPtrG, mmax, nfreqs, g.as<double2>(), nfreqs, 1,
                          st));
  k_split<<<(unsigned)ceil_div(tot, 256), 256, 0, st>>>(g.as<double2>(), tot, out_re, out_im);
  DGP_CHECK_LAUNCH();
  DGP_CUDA(cudaStreamSynchronize(st));
  return DGP_OK;
}

}  // namespace dgp
