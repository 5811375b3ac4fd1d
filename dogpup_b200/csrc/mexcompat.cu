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

// MODE 0: smv (coefficient ReA + i*fAxis[f]*ImA); MODE 1: FSAImv (G values per f)
template <int MODE>
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
    const double ar = v_re[p], ai = v_im[p];
#pragma unroll
    for (int q = 0; q < CPT; ++q) {
      if (q >= nc) break;
      double cr, ci;
      if (MODE == 0) {
        cr = ar;
        ci = fs[q] * ai;
      } else {
        cr = v_re[voff[q] + p];
        ci = v_im[voff[q] + p];
      }
      const int64_t xi = (c0 + q) * plane + j;
      const double xr = x_re[xi], xim = x_im[xi];
      yr[q] += cr * xr - ci * xim;
      yi[q] += cr * xim + ci * xr;
    }
  }
#pragma unroll
  for (int q = 0; q < CPT; ++q) {
    if (q >= nc) break;
    const int64_t o = (c0 + q) * plane + row;
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

}  // namespace

int mex_spmv(int mode, double *out_re, double *out_im, const double *x_re, const double *x_im, const double *fAxis,
             const double *v_re, const double *v_im, const int *rPtr, const int *cPtr, int64_t nnz, int nrows,
             int ncols, int nfreqs, cudaStream_t st) {
  DGP_REQUIRE(nrows > 0 && ncols > 0 && nfreqs > 0, "mex spmv: sizes must be positive");
  DGP_REQUIRE(out_re && out_im && x_re && x_im && v_re && v_im && rPtr && cPtr, "mex spmv: null pointer");
  DGP_REQUIRE(mode == 1 || fAxis, "smv: null fAxis");
  int64_t cols = (int64_t)ncols * nfreqs;
  DGP_REQUIRE(ceil_div(cols, CPT) <= 65535, "mex spmv: ncols*nfreqs too large for one launch");
  dim3 grid((unsigned)ceil_div(nrows, 128), (unsigned)ceil_div(cols, CPT));
  if (mode == 0)
    k_mexlayout_spmv<0><<<grid, 128, 0, st>>>(out_re, out_im, x_re, x_im, fAxis, v_re, v_im, rPtr, cPtr, nnz, nrows,
                                              ncols, nfreqs);
  else
    k_mexlayout_spmv<1><<<grid, 128, 0, st>>>(out_re, out_im, x_re, x_im, fAxis, v_re, v_im, rPtr, cPtr, nnz, nrows,
                                              ncols, nfreqs);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

int mex_fsaip(double *out_re, double *out_im, const double *A_re, const double *A_im, const int *rPtrA,
              const int *cPtrA, const int *rPtrG, const int *cPtrG, int nfreqs, int nrows, cudaStream_t st) {
  DGP_REQUIRE(nrows > 0 && nfreqs > 0, "FSAIP: sizes must be positive");
  DevBuf m, g;
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
