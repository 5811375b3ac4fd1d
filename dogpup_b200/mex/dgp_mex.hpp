// Shared helpers of the MATLAB gateways (smv_mex, FSAImv_mex, FSAIP_gen_mex,
// bicgstab_fsai_mex) over libdogpup_b200.  Written against MATLAB's documented
// C mex API and gpuArray API (mex.h, gpu/mxGPUArray.h) with the
// interleaved-complex data model (build with `mexcuda -R2018a`), so every
// complex array reaches the library as one pointer to (re, im) pairs.
//
// Error behaviour: argument and library errors raise a MATLAB error through
// mexErrMsgIdAndTxt with the id "dogpup_b200:<gateway>:<what>" and, for a
// library failure, dgp_last_error()'s text.  The reference gateways only
// check the argument count (e.g. FSAIP_mexgateway.cpp:11-16).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <vector>

#include "dogpup_b200.h"
#include "gpu/mxGPUArray.h"
#include "mex.h"

namespace dgp_mex {

// mxGPUArray handles destroyed when the gateway returns (or raises)
struct Handles {
  std::vector<const mxGPUArray *> held;
  ~Handles() {
    for (const mxGPUArray *g : held) mxGPUDestroyGPUArray(g);
  }
  const mxGPUArray *keep(const mxGPUArray *g) {
    held.push_back(g);
    return g;
  }
  mxGPUArray *keep(mxGPUArray *g) {
    held.push_back(g);
    return g;
  }
};

inline void fail(const char *gateway, const char *what, const char *msg) {
  char id[128];
  snprintf(id, sizeof(id), "dogpup_b200:%s:%s", gateway, what);
  mexErrMsgIdAndTxt(id, "%s", msg);
}

inline void check(const char *gateway, int rc) {
  if (rc != DGP_OK) fail(gateway, "library", dgp_last_error());
}

// dims of an mxGPUArray padded with trailing singletons to n entries
inline void dims_of(const mxGPUArray *g, mwSize *out, int n) {
  const mwSize nd = mxGPUGetNumberOfDimensions(g);
  const mwSize *d = mxGPUGetDimensions(g);
  for (int i = 0; i < n; ++i) out[i] = (mwSize)i < nd ? d[i] : 1;
  for (mwSize i = (mwSize)n; i < nd; ++i)
    if (d[i] != 1) {
      mxFree((void *)d);
      out[0] = 0;  // more non-singleton dimensions than the gateway accepts
      return;
    }
  mxFree((void *)d);
}

// A double array as complex on the device: a complex input is used in place;
// a real one (MATLAB drops all-zero imaginary parts) is widened into a new
// complex array with zero imaginary parts.
inline const double *complex_data(const char *gateway, const char *name, const mxArray *a, Handles &H) {
  const mxGPUArray *g = H.keep(mxGPUCreateFromMxArray(a));
  if (mxGPUGetClassID(g) != mxDOUBLE_CLASS) fail(gateway, "type", name);
  if (mxGPUGetComplexity(g) == mxCOMPLEX) return (const double *)mxGPUGetDataReadOnly(g);
  const mwSize nd = mxGPUGetNumberOfDimensions(g);
  const mwSize *d = mxGPUGetDimensions(g);
  mxGPUArray *c = H.keep(mxGPUCreateGPUArray(nd, d, mxDOUBLE_CLASS, mxCOMPLEX, MX_GPU_INITIALIZE_VALUES));
  mxFree((void *)d);
  const size_t n = (size_t)mxGPUGetNumberOfElements(g);
  if (n > 0 &&
      cudaMemcpy2D(mxGPUGetData(c), 2 * sizeof(double), mxGPUGetDataReadOnly(g), sizeof(double), sizeof(double), n,
                   cudaMemcpyDeviceToDevice) != cudaSuccess)
    fail(gateway, "cuda", "widening a real array to complex failed");
  return (const double *)mxGPUGetDataReadOnly(c);
}

inline const int *int32_data(const char *gateway, const char *name, const mxArray *a, Handles &H, mwSize *count) {
  const mxGPUArray *g = H.keep(mxGPUCreateFromMxArray(a));
  if (mxGPUGetClassID(g) != mxINT32_CLASS || mxGPUGetComplexity(g) != mxREAL) fail(gateway, "type", name);
  *count = mxGPUGetNumberOfElements(g);
  return (const int *)mxGPUGetDataReadOnly(g);
}

inline const double *real_data(const char *gateway, const char *name, const mxArray *a, Handles &H, mwSize *count) {
  const mxGPUArray *g = H.keep(mxGPUCreateFromMxArray(a));
  if (mxGPUGetClassID(g) != mxDOUBLE_CLASS || mxGPUGetComplexity(g) != mxREAL) fail(gateway, "type", name);
  *count = mxGPUGetNumberOfElements(g);
  return (const double *)mxGPUGetDataReadOnly(g);
}

// a scalar argument, host or gpuArray
inline double scalar(const char *gateway, const char *name, const mxArray *a) {
  if (!mxIsGPUArray(a)) {
    if (mxGetNumberOfElements(a) != 1 || mxIsComplex(a)) fail(gateway, "type", name);
    return mxGetScalar(a);
  }
  const mxGPUArray *g = mxGPUCreateFromMxArray(a);
  double v = 0.0;
  const mxClassID c = mxGPUGetClassID(g);
  bool ok = mxGPUGetNumberOfElements(g) == 1 && mxGPUGetComplexity(g) == mxREAL;
  if (ok && c == mxDOUBLE_CLASS) {
    ok = cudaMemcpy(&v, mxGPUGetDataReadOnly(g), sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess;
  } else if (ok && c == mxINT32_CLASS) {
    int32_t i = 0;
    ok = cudaMemcpy(&i, mxGPUGetDataReadOnly(g), sizeof(int32_t), cudaMemcpyDeviceToHost) == cudaSuccess;
    v = i;
  } else {
    ok = false;
  }
  mxGPUDestroyGPUArray(g);
  if (!ok) fail(gateway, "type", name);
  return v;
}

}  // namespace dgp_mex
