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
// The scratch holds a 256-byte header (the longest pattern row and a flag for
// a malformed row pointer, both reset on every call) and a staging area of
// 2^20 complex128 values (16 MiB).  The factor of a block of rows is staged
// there as interleaved complex and then split into the caller's real /
// imaginary output planes; blocks are sized so that one block of rows x all
// harmonics fits.  Limit: nfreqs * (longest pattern row) must not exceed 2^20;
// larger requests are rejected with DGP_ERR_ARG.  A G row pointer that does
// not start at 0 or decreases is rejected with DGP_ERR_MESH before anything is
// staged (a decreasing pointer would place a block's rows outside the array).
//
// Every GPU that loads the library keeps this 16 MiB array until the process
// exits.  All calls share it, so two calls whose work overlaps on the GPU (on
// different streams, or from different host threads) race on it: serialise
// them.  The array's device address belongs to the CUDA context the library's
// module is loaded in: the first call in a context looks it up
// (cudaGetSymbolAddress, with that context's device current) and keeps it
// with the context's id, so a context created after a device reset (MATLAB's
// reset(gpuDevice) destroys the context) gets the address looked up again.
// Make the first call in each context before any stream capture is started.
#include <cuda.h>

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

// hdr[0] = longest row of the pattern, hdr[1] = 1 when the row pointer does not start
// at 0 or decreases somewhere
__global__ void k_noalloc_rowmax(const int *__restrict__ rptr, int n, int *hdr) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const int a = rptr[i], b = rptr[i + 1];
    if (b < a || (i == 0 && a != 0)) atomicOr(hdr + 1, 1);
    atomicMax(hdr, b - a);
  }
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

// Driver entry points for the current context and its id (cuCtxGetId: unique for the
// process's lifetime, also when a destroyed context's handle is reused), fetched
// through the runtime so the library needs no link against libcuda.
using PfnCtxGetCurrent = CUresult (*)(CUcontext *);
using PfnCtxGetId = CUresult (*)(CUcontext, unsigned long long *);
std::once_flag g_pfn_once;
PfnCtxGetCurrent g_ctx_current = nullptr;
PfnCtxGetId g_ctx_id = nullptr;

int current_context_id(unsigned long long *id) {
  std::call_once(g_pfn_once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_current = reinterpret_cast<PfnCtxGetCurrent>(p);
    p = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_id = reinterpret_cast<PfnCtxGetId>(p);
  });
  DGP_REQUIRE(g_ctx_current && g_ctx_id, "fsaip_noalloc: driver entry points cuCtxGetCurrent / cuCtxGetId unavailable");
  CUcontext ctx = nullptr;
  if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return fail(DGP_ERR_CUDA, "fsaip_noalloc: no current CUDA context");
  if (g_ctx_id(ctx, id) != CUDA_SUCCESS) return fail(DGP_ERR_CUDA, "fsaip_noalloc: cuCtxGetId failed");
  return DGP_OK;
}

constexpr int kMaxDevices = 128;
struct ScratchAddr {
  unsigned long long ctx_id = 0;  // context the address was looked up in (0: none yet)
  void *addr = nullptr;
};
std::mutex g_addr_mutex;
ScratchAddr g_addr[kMaxDevices];

// device address of the scratch array in the current context, looked up once per
// (device, context)
int scratch_address(void **out) {
  int dev = 0;
  DGP_CUDA(cudaGetDevice(&dev));
  DGP_REQUIRE(dev >= 0 && dev < kMaxDevices, "fsaip_noalloc: device ordinal out of range");
  void *p = nullptr;
  unsigned long long id = 0;
  std::lock_guard<std::mutex> lock(g_addr_mutex);
  if (current_context_id(&id) != DGP_OK) {
    // no context is current on this thread yet: the symbol lookup makes the device's
    // primary context current, after which its id can be read
    cudaError_t e = cudaGetSymbolAddress(&p, g_fsaip_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_fsaip_scratch)", __FILE__, __LINE__);
    DGP_TRY(current_context_id(&id));
    g_addr[dev] = ScratchAddr{id, p};
  } else if (g_addr[dev].ctx_id != id || !g_addr[dev].addr) {
    cudaError_t e = cudaGetSymbolAddress(&p, g_fsaip_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_fsaip_scratch)", __FILE__, __LINE__);
    g_addr[dev] = ScratchAddr{id, p};
  }
  *out = g_addr[dev].addr;
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
  int *d_hdr = static_cast<int *>(base);
  double2 *stage = reinterpret_cast<double2 *>(static_cast<char *>(base) + kHeaderBytes);
  // the array keeps the previous call's contents: the maximum and the flag restart at zero
  DGP_CUDA(cudaMemsetAsync(d_hdr, 0, 2 * sizeof(int), st));
  k_noalloc_rowmax<<<(unsigned)ceil_div(nrows, 256), 256, 0, st>>>(rPtrG, nrows, d_hdr);
  DGP_CHECK_LAUNCH();
  int hdr[2] = {0, 0};
  DGP_CUDA(cudaMemcpyAsync(hdr, d_hdr, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  if (hdr[1]) return fail(DGP_ERR_MESH, "fsaip_noalloc: G row pointer does not start at 0 or decreases");
  const int mmax = hdr[0];
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
