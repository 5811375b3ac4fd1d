// Shared device/host helpers for the dogpup_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <string>

#include "dogpup_b200.h"

namespace dgp {

// ---------------------------------------------------------------- errors
void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define DGP_CUDA(call)                                                         \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) return ::dgp::cuda_fail(e_, #call, __FILE__, __LINE__); \
  } while (0)

// kernels launched by this library (graph-contained kernels included)
void count_launches(int64_t n);
int64_t launch_count();

#define DGP_CHECK_LAUNCH()                                                     \
  do {                                                                         \
    ::dgp::count_launches(1);                                                  \
    DGP_CUDA(cudaGetLastError());                                              \
  } while (0)

#define DGP_TRY(call)                                                          \
  do {                                                                         \
    int s_ = (call);                                                           \
    if (s_ != DGP_OK) return s_;                                               \
  } while (0)

#define DGP_REQUIRE(cond, msg)                                                 \
  do {                                                                         \
    if (!(cond)) return ::dgp::fail(DGP_ERR_ARG, msg);                         \
  } while (0)

// Number of SMs of the current device (cached per device).
int sm_count();

// Allow `kernel` a dynamic shared-memory size of `bytes` (DGP_ERR_ARG when above what the device
// gives one block beside the kernel's static shared memory).  The kernel's limit is always set to
// that device maximum, never to the size of this call: the attribute is process-wide per kernel,
// and a per-call size set by one host thread could lower the limit under another thread's larger
// launch of the same kernel.
int allow_dyn_smem_impl(const void *kernel, size_t bytes);
template <class K> inline int allow_dyn_smem(K *kernel, size_t bytes) {
  return allow_dyn_smem_impl(reinterpret_cast<const void *>(kernel), bytes);
}

// Device buffer owned by a plan; freed in the destructor.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  int alloc(size_t n);
  void release();
  template <class T> T *as() const { return static_cast<T *>(p); }
};

#ifdef __CUDACC__
// ------------------------------------------------------------- complex
template <class R> struct cplx;
template <> struct cplx<double> { using t = double2; };
template <> struct cplx<float> { using t = float2; };

__host__ __device__ inline double2 mk(double r, double i) { return make_double2(r, i); }
__host__ __device__ inline float2 mk(float r, float i) { return make_float2(r, i); }

template <class C> __host__ __device__ inline C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <class C> __host__ __device__ inline C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <class C> __host__ __device__ inline C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a + b*c
template <class C> __host__ __device__ inline C cfma(C b, C c, C a) {
  return mk(fma(b.x, c.x, fma(-b.y, c.y, a.x)), fma(b.x, c.y, fma(b.y, c.x, a.y)));
}
__device__ inline float2 cfmaf(float2 b, float2 c, float2 a) {
  return make_float2(fmaf(b.x, c.x, fmaf(-b.y, c.y, a.x)), fmaf(b.x, c.y, fmaf(b.y, c.x, a.y)));
}
// a / b, textbook formula (the reference's complexDivision, FSAIP_CUDA.cu:20-26)
__host__ __device__ inline double2 cdiv(double2 a, double2 b) {
  double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__host__ __device__ inline double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }

// principal square root, the branch rule of FSAIP_CUDA.cu:28-43
__device__ inline double2 csqrt_ref(double a, double b) {
  double z = sqrt(a * a + b * b);
  double re = sqrt((z + a) / 2);
  double im;
  if (b == 0) {
    if (a < 0) { re = 0; im = sqrt(-a); } else { im = 0; }
  } else {
    im = (b > 0 ? 1.0 : -1.0) * sqrt((z - a) / 2);
  }
  return make_double2(re, im);
}

#endif  // __CUDACC__

__host__ __device__ inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace dgp
