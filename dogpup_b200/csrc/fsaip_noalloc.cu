// dgp_fsaip_mex_noalloc: the FSAI factor on the reference's mex layout for
// callers that must not allocate device memory themselves.
//
// Who cannot allocate: a MATLAB mex gateway is expected to take all device
// memory from MATLAB's gpuArray pool (mxGPUCreateGPUArray); a cudaMalloc /
// cudaFree issued behind that pool's back fragments it and, because cudaFree
// synchronises the whole device, stalls every other gpuArray operation.  Host
// applications that hand the GPU to their own pooling allocator (and give a
// library only the final output buffers) are in the same position.  This
// entry point therefore uses no allocation of any kind: its only scratch is
// the fixed file-scope device array below.
//
// The scratch holds a 256-byte header (the longest pattern row, reset on every
// call) and a staging area of 2^20 complex128 values (16 MiB).  The factor of a
// block of rows is staged there as interleaved complex and then split into the
// caller's real / imaginary output planes; blocks are sized so that one block
// of rows x all harmonics fits.  Limit: nfreqs * (longest pattern row) must not
// exceed 2^20; larger requests are rejected with DGP_ERR_ARG.
//
// Every GPU that loads the library keeps this 16 MiB array until the process
// exits.  All calls share it, so two calls whose work overlaps on the GPU (on
// different streams, or from different host threads) race on it: serialise
// them.  The first call on a device looks up the array's device address
// (cudaGetSymbolAddress) with that device current; make that first call
// before any stream capture is started.
#include <algorithm>
#include <cstdint>
#include <mutex>

#include "dgp_common.cuh"
#include "dgp_internal.h"

namespace dgp {

namespace {

constexpr size_t kHeaderBytes = 256;
constexpr int64_t kStageSlots = int64_t(1) << 20;  // complex128 values
constexpr size_t kScratchBytes = kHeaderBytes + sizeof(double2) * (size_t)kStageSlots;

static __device__ __align__(256) unsigned char g_fsaip_scratch[kScratchBytes];

__global__ void k_noalloc_rowmax(const int *__restrict__ rptr, int n, int *m) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) atomicMax(m, rptr[i + 1] - rptr[i]);
}

__global__ void k_noalloc_split(const double2 *__restrict__ stage, int64_t count, double *__restrict__ re,
                                double *__restrict__ im) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t < count) {
    double2 v = stage[t];
    re[t] = v.x;
    im[t] = v.y;
  }
}

constexpr int kMaxDevices = 128;
std::mutex g_addr_mutex;
void *g_addr[kMaxDevices] = {};

// device address of the scratch array for the current device, looked up once
int scratch_address(void **out) {
  int dev = 0;
  DGP_CUDA(cudaGetDevice(&dev));
  DGP_REQUIRE(dev >= 0 && dev < kMaxDevices, "fsaip_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (!g_addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_fsaip_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_fsaip_scratch)", __FILE__, __LINE__);
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return DGP_OK;
}

}  // namespace

int fsaip_noalloc(double *out_re, double *out_im, const double *A_re, const double *A_im, const int *rPtrA,
                  const int *cPtrA, const int *rPtrG, const int *cPtrG, int nfreqs, int nrows, cudaStream_t st) {
  DGP_REQUIRE(out_re && out_im && A_re && A_im && rPtrA && cPtrA && rPtrG && cPtrG,
              "fsaip_noalloc: null pointer");
  DGP_REQUIRE(nrows > 0 && nfreqs > 0, "fsaip_noalloc: sizes must be positive");
  void *base = nullptr;
  DGP_TRY(scratch_address(&base));
  int *d_rowmax = static_cast<int *>(base);
  double2 *stage = reinterpret_cast<double2 *>(static_cast<char *>(base) + kHeaderBytes);
  // the array keeps the previous call's contents: the maximum must restart at zero
  DGP_CUDA(cudaMemsetAsync(d_rowmax, 0, sizeof(int), st));
  k_noalloc_rowmax<<<(unsigned)ceil_div(nrows, 256), 256, 0, st>>>(rPtrG, nrows, d_rowmax);
  DGP_CHECK_LAUNCH();
  int mmax = 0, nnzG = 0;
  DGP_CUDA(cudaMemcpyAsync(&mmax, d_rowmax, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaMemcpyAsync(&nnzG, rPtrG + nrows, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  DGP_REQUIRE(mmax >= 1 && mmax <= 32, "fsaip_noalloc: pattern rows must hold 1..32 entries");
  if ((int64_t)nfreqs * mmax > kStageSlots)
    return fail(DGP_ERR_ARG, "fsaip_noalloc: nfreqs * longest pattern row exceeds the 1048576-value "
                             "scratch array (use dgp_fsaip_mex, which allocates)");
  const int64_t rows_per_block = kStageSlots / ((int64_t)nfreqs * mmax);
  for (int64_t r0 = 0; r0 < nrows; r0 += rows_per_block) {
    const int64_t nr = std::min<int64_t>(rows_per_block, nrows - r0);
    int s0 = 0, s1 = 0;
    DGP_CUDA(cudaMemcpyAsync(&s0, rPtrG + r0, sizeof(int), cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaMemcpyAsync(&s1, rPtrG + r0 + nr, sizeof(int), cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaStreamSynchronize(st));
    // the factor kernel writes pattern slot p, harmonic k to base[p * nfreqs + k]; offset the
    // base by the block's first slot so the block lands at the start of the staging area
    double2 *shifted = reinterpret_cast<double2 *>(reinterpret_cast<uintptr_t>(stage) -
                                                   (uintptr_t)s0 * (uintptr_t)nfreqs * sizeof(double2));
    DGP_TRY(fsai_factor_run(rPtrA, cPtrA, A_re, A_im, nr, rPtrG + r0, cPtrG, mmax, nfreqs, shifted, nfreqs, 1, st));
    const int64_t count = (int64_t)(s1 - s0) * nfreqs;
    if (count > 0) {
      k_noalloc_split<<<(unsigned)ceil_div(count, 256), 256, 0, st>>>(stage, count, out_re + (int64_t)s0 * nfreqs,
                                                                        out_im + (int64_t)s0 * nfreqs);
      DGP_CHECK_LAUNCH();
    }
  }
  DGP_CUDA(cudaStreamSynchronize(st));
  return DGP_OK;
}

}  // namespace dgp

extern "C" int dgp_fsaip_mex_noalloc(double *d_out_real, double *d_out_imag, const double *d_valA_real,
                                     const double *d_valA_imag, const int *d_rPtrA, const int *d_cPtrA,
                                     const int *d_rPtrG, const int *d_cPtrG, int nfreqs, int nrows,
                                     dgp_stream_t stream) {
  try {
    return dgp::fsaip_noalloc(d_out_real, d_out_imag, d_valA_real, d_valA_imag, d_rPtrA, d_cPtrA, d_rPtrG, d_cPtrG,
                              nfreqs, nrows, (cudaStream_t)stream);
  } catch (...) {
    return dgp::fail(DGP_ERR_ARG, "fsaip_noalloc: unexpected exception");
  }
}
