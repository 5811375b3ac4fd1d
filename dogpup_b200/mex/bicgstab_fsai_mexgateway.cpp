// [phi, iters, relres, nbad] = bicgstab_fsai_mex(Q, K, M, dfc [, tol, maxit, precision])
//
// The whole of fluGPU + gpuBicstab_FSAIP (DOGPUP/dMesh.m:1238-1348) in one
// call, for the one-line change in fluGPU:
//
//   phi = bicgstab_fsai_mex(Q, mesh.K, mesh.M, mesh.optode.df./mesh.c, 1e-12, 1e3);
//
// Q       [N x NF x NS] complex double (host or gpuArray), as fluGPU gets it
// K, M    N x N real sparse (host), the triu matrices gen_fwdmat returns
//         (dMesh.m:1189-1190) or their full symmetric form
// dfc     df / c; harmonic k solves (K + i*k*dfc*M) phi = Q(:, k+1, :)
// tol     relative residual target, default 1e-12; maxit default 1000
// precision 'fp64' (reference arithmetic, default) or 'mixed' (complex FP32
//         inner iterations with FP64 residual refinement to tol)
// phi     [N x NF x NS] complex double, a gpuArray if Q is one, else a host
//         array (fluGPU's gather() is then a no-op); iters, relres: total
//         iterations and the largest final relative residual; nbad: columns
//         that missed tol (a warning is raised when nbad > 0, where the
//         reference stops silently at maxit).
// No reference counterpart: the reference drives smv_mex / FSAImv_mex from
// a MATLAB loop with host synchronisation after each call.
#include <algorithm>
#include <string>

#include "dgp_mex.hpp"

namespace {

const char *GW = "bicgstab_fsai_mex";

struct DevArr {
  void *p = nullptr;
  ~DevArr() {
    if (p) cudaFree(p);
  }
  void *get(size_t bytes) {
    if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) dgp_mex::fail(GW, "cuda", "device allocation failed");
    return p;
  }
};

struct Csr {
  std::vector<int32_t> rowptr, col;
  std::vector<double> K, M;
};

// union pattern of K and M as full symmetric CSR (int32, sorted columns);
// a triu input is mirrored, a full one is taken as it is
Csr symmetric_csr(const mxArray *K, const mxArray *M, mwSize n) {
  struct E {
    mwIndex r, c;
    double k, m;
  };
  std::vector<E> e;
  bool lower = false;
  for (int which = 0; which < 2; ++which) {
    const mxArray *S = which ? M : K;
    const mwIndex *jc = mxGetJc(S), *ir = mxGetIr(S);
    const double *v = mxGetDoubles(S);
    for (mwIndex c = 0; c < n; ++c)
      for (mwIndex p = jc[c]; p < jc[c + 1]; ++p) {
        const mwIndex r = ir[p];
        if (r > c) lower = true;
        e.push_back(E{r, c, which ? 0.0 : v[p], which ? v[p] : 0.0});
      }
  }
  if (!lower) {  // triu: add the mirrored strict upper part
    const size_t m = e.size();
    for (size_t q = 0; q < m; ++q)
      if (e[q].r != e[q].c) e.push_back(E{e[q].c, e[q].r, e[q].k, e[q].m});
  }
  std::sort(e.begin(), e.end(), [](const E &a, const E &b) { return a.r != b.r ? a.r < b.r : a.c < b.c; });
  Csr o;
  o.rowptr.assign(n + 1, 0);
  for (size_t q = 0; q < e.size();) {
    size_t t = q;
    double k = 0, m = 0;
    for (; t < e.size() && e[t].r == e[q].r && e[t].c == e[q].c; ++t) {
      k += e[t].k;
      m += e[t].m;
    }
    o.col.push_back((int32_t)e[q].c);
    o.K.push_back(k);
    o.M.push_back(m);
    o.rowptr[e[q].r + 1]++;
    q = t;
  }
  for (mwSize i = 0; i < n; ++i) o.rowptr[i + 1] += o.rowptr[i];
  return o;
}

}  // namespace

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  if (nrhs < 4 || nrhs > 7) dgp_mex::fail(GW, "nrhs", "usage: bicgstab_fsai_mex(Q, K, M, dfc [, tol, maxit, precision])");
  if (nlhs > 4) dgp_mex::fail(GW, "nlhs", "at most 4 outputs");
  mxInitGPU();
  const mxArray *K = prhs[1], *M = prhs[2];
  if (!mxIsSparse(K) || !mxIsSparse(M) || mxIsComplex(K) || mxIsComplex(M) || mxIsGPUArray(K) || mxIsGPUArray(M))
    dgp_mex::fail(GW, "type", "K and M must be real sparse host matrices");
  const mwSize n = mxGetM(K);
  if (mxGetN(K) != n || mxGetM(M) != n || mxGetN(M) != n) dgp_mex::fail(GW, "dims", "K and M must be N x N");
  const double dfc = dgp_mex::scalar(GW, "dfc must be a real scalar", prhs[3]);
  dgp_solve_opts o;
  dgp_solve_opts_default(&o);
  if (nrhs > 4) o.tol = dgp_mex::scalar(GW, "tol must be a real scalar", prhs[4]);
  if (nrhs > 5) o.maxit = (int32_t)dgp_mex::scalar(GW, "maxit must be a real scalar", prhs[5]);
  if (nrhs > 6) {
    const mxArray *p = prhs[6];
    if (mxIsChar(p)) {
      char buf[16] = {0};
      mxGetString(p, buf, sizeof(buf));
      const std::string s(buf);
      if (s == "fp64") o.precision = DGP_PREC_FP64;
      else if (s == "mixed") o.precision = DGP_PREC_MIXED;
      else if (s == "mixed_bicgstab") o.precision = DGP_PREC_MIXED_BICGSTAB;
      else dgp_mex::fail(GW, "precision", "precision must be 'fp64', 'mixed' or 'mixed_bicgstab'");
    } else {
      o.precision = (int32_t)dgp_mex::scalar(GW, "precision must be 'fp64', 'mixed' or 'mixed_bicgstab'", p);
    }
  }
  dgp_mex::Handles H;
  const double *q = dgp_mex::complex_data(GW, "Q must be double", prhs[0], H);
  mwSize dims[3];
  dgp_mex::dims_of(H.held.back(), dims, 3);
  if (dims[0] != n) dgp_mex::fail(GW, "dims", "Q must be [N x NF x NS] with N = size(K, 1)");
  const mwSize nf = dims[1], ns = dims[2];

  Csr A = symmetric_csr(K, M, n);
  const size_t nnz = A.col.size();
  DevArr drp, dcl, dK, dM;
  int32_t *rp = (int32_t *)drp.get(sizeof(int32_t) * (n + 1));
  int32_t *cl = (int32_t *)dcl.get(sizeof(int32_t) * nnz);
  double *kv = (double *)dK.get(sizeof(double) * nnz);
  double *mv = (double *)dM.get(sizeof(double) * nnz);
  if (cudaMemcpy(rp, A.rowptr.data(), sizeof(int32_t) * (n + 1), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(cl, A.col.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(kv, A.K.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(mv, A.M.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice) != cudaSuccess)
    dgp_mex::fail(GW, "cuda", "copying K and M to the device failed");

  dgp_solver_t S = nullptr;
  dgp_mex::check(GW, dgp_solver_create(&S, rp, cl, (int64_t)n, (int64_t)nnz, kv, mv, dfc, (int32_t)nf, (int32_t)ns,
                                       &o, nullptr));
  mxGPUArray *x = H.keep(mxGPUCreateGPUArray(3, dims, mxDOUBLE_CLASS, mxCOMPLEX, MX_GPU_DO_NOT_INITIALIZE));
  dgp_solve_report rep;
  memset(&rep, 0, sizeof(rep));
  const int rc = dgp_solve_mex(S, q, (double *)mxGPUGetData(x), (int32_t)ns, DGP_LAYOUT_N_NF_NS, &o, &rep, nullptr);
  dgp_solver_destroy(S);
  if (rc != DGP_OK && rc != DGP_ERR_NOT_CONVERGED) dgp_mex::check(GW, rc);
  if (rep.n_not_converged > 0)
    mexWarnMsgIdAndTxt("dogpup_b200:bicgstab_fsai_mex:maxit", "%d right-hand sides did not reach tol %g",
                       rep.n_not_converged, o.tol);
  plhs[0] = mxIsGPUArray(prhs[0]) ? mxGPUCreateMxArrayOnGPU(x) : mxGPUCreateMxArrayOnCPU(x);
  if (nlhs > 1) plhs[1] = mxCreateDoubleScalar(rep.iterations);
  if (nlhs > 2) plhs[2] = mxCreateDoubleScalar(rep.max_rel_residual);
  if (nlhs > 3) plhs[3] = mxCreateDoubleScalar(rep.n_not_converged);
}
