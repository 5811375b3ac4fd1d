// y = smv_mex(x, f, A, rPtrA, cPtrA)        (call sites: DOGPUP/dMesh.m:1284,1301,1319)
//
// Drop-in for the reference gateway of the same name (cuda_lib/mex_sources/
// smv_mexgateway.cpp:8-100): y(:,s,k) = (Re A + i*f(k)*Im A) * x(:,s,k) for a
// complex x of size [N x NS x NF] (trailing singleton dimensions may be
// dropped), f [1 x NF] double, A complex [nnzA] (CSR values), rPtrA int32
// [N+1], cPtrA int32 [nnzA] (0-based).  Inputs may be gpuArrays or host
// arrays; y is a complex gpuArray [N x NS x NF], as in the reference.
#include "dgp_mex.hpp"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  static const char *G = "smv_mex";
  if (nrhs != 5) dgp_mex::fail(G, "nrhs", "5 inputs required: x, f, A, rPtrA, cPtrA");
  if (nlhs > 1) dgp_mex::fail(G, "nlhs", "one output");
  mxInitGPU();
  dgp_mex::Handles H;
  const double *x = dgp_mex::complex_data(G, "x must be double", prhs[0], H);
  mwSize dims[3];
  dgp_mex::dims_of(H.held.back(), dims, 3);
  if (dims[0] == 0) dgp_mex::fail(G, "dims", "x must be [N x NS x NF]");
  mwSize nf_f = 0, nnz = 0, nr = 0, nc = 0;
  const double *f = dgp_mex::real_data(G, "f must be real double", prhs[1], H, &nf_f);
  const double *A = dgp_mex::complex_data(G, "A must be double", prhs[2], H);
  const int *rp = dgp_mex::int32_data(G, "rPtrA must be int32", prhs[3], H, &nr);
  const int *cp = dgp_mex::int32_data(G, "cPtrA must be int32", prhs[4], H, &nc);
  nnz = mxGetNumberOfElements(prhs[2]);
  if (nf_f != dims[2]) dgp_mex::fail(G, "dims", "numel(f) must equal size(x, 3)");
  if (nr != dims[0] + 1) dgp_mex::fail(G, "dims", "numel(rPtrA) must be size(x, 1) + 1");
  if (nc != nnz) dgp_mex::fail(G, "dims", "numel(cPtrA) must equal numel(A)");
  mxGPUArray *y = H.keep(mxGPUCreateGPUArray(3, dims, mxDOUBLE_CLASS, mxCOMPLEX, MX_GPU_DO_NOT_INITIALIZE));
  dgp_mex::check(G, dgp_smv_mex_ic((double *)mxGPUGetData(y), x, f, A, rp, cp, (int)dims[0], (int)dims[1],
                                   (int)dims[2], nullptr));
  plhs[0] = mxGPUCreateMxArrayOnGPU(y);
}
