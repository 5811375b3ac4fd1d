// y = FSAImv_mex(x, G, rPtrG, cPtrG)        (call sites: DOGPUP/dMesh.m:1295-1296,1315-1316,1322)
//
// Drop-in for the reference gateway of the same name (cuda_lib/mex_sources/
// FSAImv_mexgateway.cpp:8-99): y(:,s,k) = G_k * x(:,s,k) with G [nnzG x NF]
// complex (column k = the values of G_k on the CSR pattern rPtrG / cPtrG,
// int32, 0-based).  x complex [N x NS x NF]; y a complex gpuArray of the
// same size.
#include "dgp_mex.hpp"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  static const char *GW = "FSAImv_mex";
  if (nrhs != 4) dgp_mex::fail(GW, "nrhs", "4 inputs required: x, G, rPtrG, cPtrG");
  if (nlhs > 1) dgp_mex::fail(GW, "nlhs", "one output");
  mxInitGPU();
  dgp_mex::Handles H;
  const double *x = dgp_mex::complex_data(GW, "x must be double", prhs[0], H);
  mwSize dims[3];
  dgp_mex::dims_of(H.held.back(), dims, 3);
  if (dims[0] == 0) dgp_mex::fail(GW, "dims", "x must be [N x NS x NF]");
  const double *G = dgp_mex::complex_data(GW, "G must be double", prhs[1], H);
  mwSize nr = 0, nnz = 0;
  const int *rp = dgp_mex::int32_data(GW, "rPtrG must be int32", prhs[2], H, &nr);
  const int *cp = dgp_mex::int32_data(GW, "cPtrG must be int32", prhs[3], H, &nnz);
  if (nr != dims[0] + 1) dgp_mex::fail(GW, "dims", "numel(rPtrG) must be size(x, 1) + 1");
  if (mxGetNumberOfElements(prhs[1]) != nnz * dims[2]) dgp_mex::fail(GW, "dims", "G must be [numel(cPtrG) x NF]");
  mxGPUArray *y = H.keep(mxGPUCreateGPUArray(3, dims, mxDOUBLE_CLASS, mxCOMPLEX, MX_GPU_DO_NOT_INITIALIZE));
  dgp_mex::check(GW, dgp_fsaimv_mex_ic((double *)mxGPUGetData(y), x, G, rp, cp, (int)nnz, (int)dims[0],
                                       (int)dims[1], (int)dims[2], nullptr));
  plhs[0] = mxGPUCreateMxArrayOnGPU(y);
}
