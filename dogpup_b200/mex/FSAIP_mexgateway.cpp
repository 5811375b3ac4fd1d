// G = FSAIP_gen_mex(valA, rPtrA, cPtrA, rPtrG, cPtrG, int32(NF))   (call site: DOGPUP/dMesh.m:1384)
//
// Drop-in for the reference gateway of the same name (cuda_lib/mex_sources/
// FSAIP_mexgateway.cpp:8-85): the FSAI factor of tril(A_k) = Re A + i*k*Im A
// for k = 0 .. NF-1 on the pattern rPtrG / cPtrG.  valA complex values of
// tril(A) on the CSR rPtrA / cPtrA (int32, 0-based).  G is a HOST complex
// array [NF x nnzG] (harmonic fastest), as the reference returns it.
#include "dgp_mex.hpp"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]) {
  static const char *GW = "FSAIP_gen_mex";
  if (nrhs != 6) dgp_mex::fail(GW, "nrhs", "6 inputs required: valA, rPtrA, cPtrA, rPtrG, cPtrG, NF");
  if (nlhs > 1) dgp_mex::fail(GW, "nlhs", "one output");
  mxInitGPU();
  dgp_mex::Handles H;
  const double *valA = dgp_mex::complex_data(GW, "valA must be double", prhs[0], H);
  mwSize nrA = 0, ncA = 0, nrG = 0, nnzG = 0;
  const int *rpA = dgp_mex::int32_data(GW, "rPtrA must be int32", prhs[1], H, &nrA);
  const int *cpA = dgp_mex::int32_data(GW, "cPtrA must be int32", prhs[2], H, &ncA);
  const int *rpG = dgp_mex::int32_data(GW, "rPtrG must be int32", prhs[3], H, &nrG);
  const int *cpG = dgp_mex::int32_data(GW, "cPtrG must be int32", prhs[4], H, &nnzG);
  const double nfd = dgp_mex::scalar(GW, "NF must be a real scalar", prhs[5]);
  if (!(nfd >= 1 && nfd <= 2147483647.0)) dgp_mex::fail(GW, "NF", "NF must be a positive integer");
  if (nrA != nrG || nrG < 2) dgp_mex::fail(GW, "dims", "rPtrA and rPtrG must both hold N+1 entries");
  if (mxGetNumberOfElements(prhs[0]) != ncA) dgp_mex::fail(GW, "dims", "numel(valA) must equal numel(cPtrA)");
  mwSize dims[2] = {(mwSize)nfd, nnzG};
  mxGPUArray *g = H.keep(mxGPUCreateGPUArray(2, dims, mxDOUBLE_CLASS, mxCOMPLEX, MX_GPU_DO_NOT_INITIALIZE));
  dgp_mex::check(GW, dgp_fsaip_mex_ic((double *)mxGPUGetData(g), valA, rpA, cpA, rpG, cpG, (int)nfd, (int)(nrG - 1),
                                      nullptr));
  plhs[0] = mxGPUCreateMxArrayOnCPU(g);
}
