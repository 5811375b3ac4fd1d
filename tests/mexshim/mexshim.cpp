// Test double of the MATLAB mex / gpuArray runtime used to drive
// dogpup_b200's gateways from pytest (TEST INFRASTRUCTURE ONLY).
//
// mxArray: host arrays (dense numeric, char, sparse double) and gpuArrays
// (device memory shared with the mxGPUArray handles made from them).
// mexErrMsgIdAndTxt throws; shim_call catches it and returns the message, so
// a gateway error surfaces in Python as a failed call with MATLAB's id/text.
// The extern "C" shim_* functions are the harness Python calls through ctypes.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpu/mxGPUArray.h"
#include "mex.h"

namespace {

struct MexError : std::runtime_error {
  std::string id;
  MexError(const std::string &i, const std::string &m) : std::runtime_error(m), id(i) {}
};

size_t elem_size(mxClassID c) {
  switch (c) {
    case mxDOUBLE_CLASS: return 8;
    case mxSINGLE_CLASS: return 4;
    case mxINT32_CLASS: return 4;
    case mxCHAR_CLASS: return 2;
    default: return 0;
  }
}

std::shared_ptr<void> dev_alloc(size_t bytes) {
  void *p = nullptr;
  if (cudaMalloc(&p, bytes ? bytes : 1) != cudaSuccess) throw MexError("shim:cuda", "cudaMalloc failed");
  return std::shared_ptr<void>(p, [](void *q) { cudaFree(q); });
}

size_t count(const std::vector<mwSize> &d) {
  size_t n = 1;
  for (mwSize x : d) n *= x;
  return n;
}

std::string g_warnings;

}  // namespace

struct mxGPUArray_tag {
  mxClassID cls;
  mxComplexity cx;
  std::vector<mwSize> dims;
  std::shared_ptr<void> dev;
  size_t bytes() const { return count(dims) * elem_size(cls) * (cx == mxCOMPLEX ? 2 : 1); }
};

struct mxArray_tag {
  mxClassID cls = mxDOUBLE_CLASS;
  mxComplexity cx = mxREAL;
  bool sparse = false;
  std::vector<mwSize> dims;
  std::vector<unsigned char> host;   // dense data (interleaved when complex) or sparse values
  std::vector<mwIndex> jc, ir;       // sparse structure
  std::shared_ptr<mxGPUArray_tag> gpu;  // gpuArray payload
  size_t bytes() const { return count(dims) * elem_size(cls) * (cx == mxCOMPLEX ? 2 : 1); }
};

extern "C" {

void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw MexError(id, buf);
}

void mexWarnMsgIdAndTxt(const char *id, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_warnings += std::string(id) + ": " + buf + "\n";
}

void mxFree(void *p) { free(p); }

int mxIsComplex(const mxArray *a) { return a->cx == mxCOMPLEX; }
int mxIsSparse(const mxArray *a) { return a->sparse; }
int mxIsChar(const mxArray *a) { return a->cls == mxCHAR_CLASS; }
size_t mxGetM(const mxArray *a) { return a->dims.empty() ? 0 : a->dims[0]; }
size_t mxGetN(const mxArray *a) {
  size_t n = 1;
  for (size_t i = 1; i < a->dims.size(); ++i) n *= a->dims[i];
  return n;
}
size_t mxGetNumberOfElements(const mxArray *a) { return count(a->dims); }
double mxGetScalar(const mxArray *a) {
  if (a->gpu) throw MexError("shim:scalar", "mxGetScalar on a gpuArray");
  if (a->host.empty()) return 0.0;
  switch (a->cls) {
    case mxDOUBLE_CLASS: return *(const double *)a->host.data();
    case mxSINGLE_CLASS: return *(const float *)a->host.data();
    case mxINT32_CLASS: return *(const int32_t *)a->host.data();
    default: return 0.0;
  }
}
double *mxGetDoubles(const mxArray *a) {
  return (a->cls == mxDOUBLE_CLASS && a->cx == mxREAL && !a->gpu) ? (double *)a->host.data() : nullptr;
}
mxComplexDouble *mxGetComplexDoubles(const mxArray *a) {
  return (a->cls == mxDOUBLE_CLASS && a->cx == mxCOMPLEX && !a->gpu) ? (mxComplexDouble *)a->host.data() : nullptr;
}
mwIndex *mxGetJc(const mxArray *a) { return a->sparse ? (mwIndex *)a->jc.data() : nullptr; }
mwIndex *mxGetIr(const mxArray *a) { return a->sparse ? (mwIndex *)a->ir.data() : nullptr; }
int mxGetString(const mxArray *a, char *buf, mwSize len) {
  if (a->cls != mxCHAR_CLASS || len == 0) return 1;
  const size_t n = count(a->dims);
  const uint16_t *c = (const uint16_t *)a->host.data();
  size_t i = 0;
  for (; i < n && i + 1 < len; ++i) buf[i] = (char)c[i];
  buf[i] = 0;
  return i < n ? 1 : 0;
}
mxArray *mxCreateDoubleScalar(double v) {
  mxArray *a = new mxArray_tag();
  a->dims = {1, 1};
  a->host.resize(8);
  memcpy(a->host.data(), &v, 8);
  return a;
}

int mxInitGPU(void) { return cudaFree(nullptr) == cudaSuccess ? MX_GPU_SUCCESS : MX_GPU_FAILURE; }
int mxIsGPUArray(const mxArray *a) { return a->gpu != nullptr; }

const mxGPUArray *mxGPUCreateFromMxArray(const mxArray *a) {
  if (a->sparse) throw MexError("shim:sparse", "sparse arrays cannot become gpuArrays here");
  auto *g = new mxGPUArray_tag();
  if (a->gpu) {
    *g = *a->gpu;  // shares the device data
    return g;
  }
  g->cls = a->cls;
  g->cx = a->cx;
  g->dims = a->dims;
  g->dev = dev_alloc(g->bytes());
  if (g->bytes() && cudaMemcpy(g->dev.get(), a->host.data(), g->bytes(), cudaMemcpyHostToDevice) != cudaSuccess)
    throw MexError("shim:cuda", "host to device copy failed");
  return g;
}

mxGPUArray *mxGPUCreateGPUArray(mwSize ndims, const mwSize *dims, mxClassID cid, mxComplexity cx,
                                mxGPUInitialize init) {
  auto *g = new mxGPUArray_tag();
  g->cls = cid;
  g->cx = cx;
  g->dims.assign(dims, dims + ndims);
  g->dev = dev_alloc(g->bytes());
  if (init == MX_GPU_INITIALIZE_VALUES) cudaMemset(g->dev.get(), 0, g->bytes());
  return g;
}

const void *mxGPUGetDataReadOnly(const mxGPUArray *g) { return g->dev.get(); }
void *mxGPUGetData(mxGPUArray *g) { return g->dev.get(); }
mwSize mxGPUGetNumberOfDimensions(const mxGPUArray *g) { return g->dims.size(); }
const mwSize *mxGPUGetDimensions(const mxGPUArray *g) {
  mwSize *d = (mwSize *)malloc(sizeof(mwSize) * (g->dims.size() + 1));
  for (size_t i = 0; i < g->dims.size(); ++i) d[i] = g->dims[i];
  return d;
}
mwSize mxGPUGetNumberOfElements(const mxGPUArray *g) { return count(g->dims); }
mxClassID mxGPUGetClassID(const mxGPUArray *g) { return g->cls; }
mxComplexity mxGPUGetComplexity(const mxGPUArray *g) { return g->cx; }

mxArray *mxGPUCreateMxArrayOnGPU(const mxGPUArray *g) {
  mxArray *a = new mxArray_tag();
  a->cls = g->cls;
  a->cx = g->cx;
  a->dims = g->dims;
  a->gpu = std::make_shared<mxGPUArray_tag>(*g);
  return a;
}

mxArray *mxGPUCreateMxArrayOnCPU(const mxGPUArray *g) {
  mxArray *a = new mxArray_tag();
  a->cls = g->cls;
  a->cx = g->cx;
  a->dims = g->dims;
  a->host.resize(a->bytes());
  cudaDeviceSynchronize();
  if (a->bytes() && cudaMemcpy(a->host.data(), g->dev.get(), a->bytes(), cudaMemcpyDeviceToHost) != cudaSuccess)
    throw MexError("shim:cuda", "device to host copy failed");
  return a;
}

void mxGPUDestroyGPUArray(const mxGPUArray *g) { delete g; }

// ------------------------------------------------------------ the harness
typedef void (*mex_fn)(int, mxArray **, int, const mxArray **);

mxArray *shim_array(int cls, int complex, int on_gpu, int ndim, const size_t *dims, const void *data) {
  mxArray *a = new mxArray_tag();
  a->cls = (mxClassID)cls;
  a->cx = complex ? mxCOMPLEX : mxREAL;
  a->dims.assign(dims, dims + ndim);
  a->host.resize(a->bytes());
  if (a->bytes()) memcpy(a->host.data(), data, a->bytes());
  if (on_gpu) {
    const mxGPUArray *g = mxGPUCreateFromMxArray(a);
    a->gpu = std::make_shared<mxGPUArray_tag>(*g);
    delete g;
    a->host.clear();
  }
  return a;
}

mxArray *shim_sparse(size_t m, size_t n, const size_t *jc, const size_t *ir, const double *v) {
  mxArray *a = new mxArray_tag();
  a->sparse = true;
  a->dims = {m, n};
  a->jc.assign(jc, jc + n + 1);
  const size_t nnz = jc[n];
  a->ir.assign(ir, ir + nnz);
  a->host.resize(nnz * 8);
  if (nnz) memcpy(a->host.data(), v, nnz * 8);
  return a;
}

mxArray *shim_string(const char *s) {
  mxArray *a = new mxArray_tag();
  a->cls = mxCHAR_CLASS;
  const size_t n = strlen(s);
  a->dims = {1, n};
  a->host.resize(2 * n);
  for (size_t i = 0; i < n; ++i) ((uint16_t *)a->host.data())[i] = (uint16_t)s[i];
  return a;
}

// 0 on success; 1 with "id: message" in err when the gateway raised
int shim_call(void *fn, int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs, char *err, int errlen) {
  try {
    ((mex_fn)fn)(nlhs, plhs, nrhs, prhs);
    return 0;
  } catch (const MexError &e) {
    snprintf(err, errlen, "%s: %s", e.id.c_str(), e.what());
  } catch (const std::exception &e) {
    snprintf(err, errlen, "shim: %s", e.what());
  }
  return 1;
}

int shim_info(const mxArray *a, int *cls, int *complex, int *on_gpu, size_t *dims, int maxdims) {
  *cls = a->cls;
  *complex = a->cx == mxCOMPLEX;
  *on_gpu = a->gpu != nullptr;
  for (int i = 0; i < maxdims; ++i) dims[i] = i < (int)a->dims.size() ? a->dims[i] : 1;
  return (int)a->dims.size();
}

int shim_read(const mxArray *a, void *out) {
  const size_t b = a->bytes();
  if (a->gpu) {
    cudaDeviceSynchronize();
    return cudaMemcpy(out, a->gpu->dev.get(), b, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : 1;
  }
  if (b) memcpy(out, a->host.data(), b);
  return 0;
}

const char *shim_warnings(void) { return g_warnings.c_str(); }
void shim_clear_warnings(void) { g_warnings.clear(); }
void shim_destroy(mxArray *a) { delete a; }

}  // extern "C"
