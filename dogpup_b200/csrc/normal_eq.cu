// Weighted Levenberg-Marquardt normal-equation step on the device.
//
// Replaces tik_inv (DOGPUP/reconstruction/tik_inv.m:1-20), which forms
// H = J'J on the CPU, adds lam * max_j sum_i J_ij^2 to the diagonal and
// solves H \ (J'y) with MATLAB's backslash (Cholesky for SPD H); here with
// a diagonal data weight W = 1/sigma^2:
//
//   H = J' W J                         split-BF16 tcgen05 SYRK, FP32 accumulate
//   H_ii += lam * max_j (J'WJ)_jj      (or lam * (J'WJ)_ii), FP64 exact diagonal
//   r = J' W y                         FP64
//   H = L L', solve L L' x = r         FP64 blocked Cholesky + triangular solves
//                                      (cholesky.cu: FP64 tensor-core GEMMs, no BLAS)
//
// Input J is given transposed, Jt [nv][nmeas] float32 row-major -- the layout
// the TG Jacobian kernel writes -- so both GEMM operands are K-major.
//
// Split BF16: Js = sqrt(W) * Jt = hi + lo with hi = bf16(Js), lo =
// bf16(Js - hi); H = hi hi' + hi lo' + lo hi' (the lo lo' term, ~2^-16
// relative, is dropped), three BF16 tensor-core products per K step into one
// FP32 accumulator in tensor memory.
//
// SYRK kernel: one CTA per 128 x 128 tile of the lower triangle of H.
//   warp 0 lane 0: TMA producer (4 tiles per stage: A hi/lo, B hi/lo, each
//                  128 rows x 64 K of bf16 with the 128-byte swizzle),
//   warp 1 lane 0: MMA issuer (tcgen05.mma kind::f16, M=128 N=128 K=16),
//   warps 0..3:    epilogue (tcgen05.ld 32x32b, FP32 -> FP64 stores).
// Three pipeline stages (192 KB of shared memory).  Every mbarrier wait is
// bounded; a timeout sets an error flag, skips the remaining work, waits
// (bounded) for copies in flight and always frees the tensor memory.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "dgp_common.cuh"
#include "dgp_internal.h"
#include "tc_common.cuh"

namespace dgp {

namespace {

constexpr int TM = 128, TN = 128, TK = 64, STAGES = 3;
constexpr int TILE_BYTES = TM * TK * 2;       // 16 KB: 128 rows x 64 bf16
constexpr int STAGE_BYTES = 4 * TILE_BYTES;   // A hi, A lo, B hi, B lo
constexpr int SYRK_SMEM = STAGES * STAGE_BYTES + 1024;  // + alignment slack

using tc::mbar_expect_tx;
using tc::mbar_init;
using tc::mbar_wait;
using tc::sdesc_k_sw128;
using tc::smem_u32;
using tc::tmem_ld32;
using tc::umma_commit;

__device__ inline void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// instruction descriptor, kind::f16: BF16 x BF16 -> F32, both K-major, M=128, N=128
constexpr uint32_t kIdesc = tc::idesc(1, 1, TM, TN);

__device__ inline void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accum) {
  tc::umma_bf16<kIdesc>(d_tmem, adesc, bdesc, accum);
}

__global__ void __launch_bounds__(128, 1) k_syrk_tc(const __grid_constant__ CUtensorMap map_hi,
                                                    const __grid_constant__ CUtensorMap map_lo, int nk, int64_t nv,
                                                    double *__restrict__ H, int64_t ldh, int *err) {
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  // 1024-byte aligned stage buffers (the 128-byte swizzle atom is 8 rows x 128 B)
  unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(sm_raw) + 1023) & ~uintptr_t(1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // lower-triangular tile (ti >= tj) of this block
  const int64_t b = blockIdx.x;
  int64_t ti = (int64_t)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
  while (ti * (ti + 1) / 2 > b) --ti;
  while ((ti + 1) * (ti + 2) / 2 <= b) ++ti;
  const int64_t tj = b - ti * (ti + 1) / 2;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&done, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TN)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer
    int issued = 0;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      const uint32_t ph = (uint32_t)(kb / STAGES) & 1u;
      if (!mbar_wait(&empty[s], ph ^ 1u)) { atomicOr(err, 1); abort_flag = 1; break; }
      if (*(volatile int *)&abort_flag) break;
      unsigned char *st = sm + (size_t)s * STAGE_BYTES;
      mbar_expect_tx(&full[s], STAGE_BYTES);
      const int x = kb * TK;
      tma_load_2d(st + 0 * TILE_BYTES, &map_hi, &full[s], x, (int)(ti * TM));
      tma_load_2d(st + 1 * TILE_BYTES, &map_lo, &full[s], x, (int)(ti * TM));
      tma_load_2d(st + 2 * TILE_BYTES, &map_hi, &full[s], x, (int)(tj * TN));
      tma_load_2d(st + 3 * TILE_BYTES, &map_lo, &full[s], x, (int)(tj * TN));
      issued = kb + 1;
    }
    // on an abort, wait (bounded) for the copies still in flight before teardown
    if (*(volatile int *)&abort_flag) {
      for (int kb = std::max(0, issued - STAGES); kb < issued; ++kb)
        mbar_wait(&full[kb % STAGES], (uint32_t)(kb / STAGES) & 1u);
    }
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer
    bool ok = true;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      const uint32_t ph = (uint32_t)(kb / STAGES) & 1u;
      if (!mbar_wait(&full[s], ph)) { atomicOr(err, 2); abort_flag = 1; ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t base = smem_u32(sm + (size_t)s * STAGE_BYTES);
#pragma unroll
      for (int k = 0; k < TK / 16; ++k) {
        const uint32_t off = (uint32_t)k * 32u;  // 16 bf16 along K inside the swizzle atom
        const uint64_t ahi = sdesc_k_sw128(base + 0 * TILE_BYTES + off);
        const uint64_t alo = sdesc_k_sw128(base + 1 * TILE_BYTES + off);
        const uint64_t bhi = sdesc_k_sw128(base + 2 * TILE_BYTES + off);
        const uint64_t blo = sdesc_k_sw128(base + 3 * TILE_BYTES + off);
        umma_bf16(tmem, ahi, bhi, (kb | k) ? 1u : 0u);
        umma_bf16(tmem, ahi, blo, 1u);
        umma_bf16(tmem, alo, bhi, 1u);
      }
      umma_commit(&empty[s]);  // frees the stage once these MMAs have read it
    }
    if (ok) umma_commit(&done);
  }
  __syncwarp();
  // ---------------- epilogue: TMEM -> registers -> H (FP64)
  bool have = !*(volatile int *)&abort_flag;
  if (have) have = mbar_wait(&done, 0);
  have = __all_sync(0xffffffffu, have);  // tcgen05.ld below is warp-collective
  if (!have && lane == 0) atomicOr(err, 4);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (have) {
    const int64_t row = ti * TM + warp * 32 + lane;
#pragma unroll 1
    for (int c = 0; c < TN; c += 32) {
      uint32_t r[32];
      tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, r);
      if (row < nv) {
        double *dst = H + row * ldh + tj * TN + c;
#pragma unroll
        for (int q = 0; q < 32; ++q)
          if (tj * TN + c + q < nv) dst[q] = (double)__uint_as_float(r[q]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN) : "memory");
}

// Js = sqrt(W) Jt split into bf16 hi + lo, zero-padded to [nvp][nmp]; exact
// FP64 diagonal d[v] = sum_m W_m Jt[v][m]^2
__global__ void k_split(const float *__restrict__ Jt, const double *__restrict__ W, int64_t nv, int64_t nm,
                        int64_t nvp, int64_t nmp, __nv_bfloat16 *hi, __nv_bfloat16 *lo) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nvp * nmp) return;
  int64_t v = t / nmp, m = t % nmp;
  float x = 0.f;
  if (v < nv && m < nm) x = Jt[v * nm + m] * (W ? (float)sqrt(W[m]) : 1.f);
  __nv_bfloat16 h = __float2bfloat16_rn(x);
  hi[t] = h;
  lo[t] = __float2bfloat16_rn(x - __bfloat162float(h));
}

__global__ void k_check_weights(const double *__restrict__ W, int64_t nm, int *err) {
  int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (m < nm && !(W[m] >= 0.0 && isfinite(W[m]))) atomicOr(err, 16);
}

__global__ void k_row_dots(const float *__restrict__ Jt, const double *__restrict__ W, const double *__restrict__ y,
                           int64_t nv, int64_t nm, double *diag, double *rhs) {
  __shared__ double sd[256], sr[256];
  for (int64_t v = blockIdx.x; v < nv; v += gridDim.x) {
    double d = 0, r = 0;
    for (int64_t m = threadIdx.x; m < nm; m += blockDim.x) {
      double j = Jt[v * nm + m], w = W ? W[m] : 1.0;
      d += w * j * j;
      if (y) r += j * w * y[m];
    }
    sd[threadIdx.x] = d;
    sr[threadIdx.x] = r;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (threadIdx.x < o) {
        sd[threadIdx.x] += sd[threadIdx.x + o];
        sr[threadIdx.x] += sr[threadIdx.x + o];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      diag[v] = sd[0];
      if (rhs) rhs[v] = sr[0];
    }
    __syncthreads();
  }
}

// H_ii = d_i + lam * (mode 0: max_j d_j, the tik_inv rule; mode 1: d_i; mode 2: 1)
__global__ void k_damp(double *H, int64_t ldh, const double *__restrict__ diag, int64_t nv, double lam, int mode) {
  __shared__ double smax;
  if (threadIdx.x == 0) {
    double m = 0;
    for (int64_t i = 0; i < nv; ++i) m = fmax(m, diag[i]);
    smax = m;
  }
  __syncthreads();
  for (int64_t i = threadIdx.x; i < nv; i += blockDim.x)
    H[i * ldh + i] = diag[i] + lam * (mode == 0 ? smax : mode == 1 ? diag[i] : 1.0);
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

int make_map(CUtensorMap *map, void *base, int64_t rows, int64_t cols) {
  auto enc = get_encode();
  if (!enc) return fail(DGP_ERR_CUDA, "normal_eq: cuTensorMapEncodeTiled is unavailable");
  cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
  cuuint32_t box[2] = {(cuuint32_t)TK, (cuuint32_t)TM};
  cuuint32_t es[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, es,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(DGP_ERR_CUDA, "normal_eq: tensor map encoding failed");
  return DGP_OK;
}

// DGP_ERR_ARG unless every data weight W[0..nm) is finite and non-negative; errb is a zeroed device int.
int check_weights(const double *W, int64_t nm, int *errb, const char *who, cudaStream_t st) {
  k_check_weights<<<(unsigned)ceil_div(nm, 256), 256, 0, st>>>(W, nm, errb);
  DGP_CHECK_LAUNCH();
  int werr = 0;
  DGP_CUDA(cudaMemcpyAsync(&werr, errb, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  if (werr) return fail(DGP_ERR_ARG, std::string(who) + ": data weights must be finite and non-negative");
  return DGP_OK;
}

}  // namespace

int normal_eq_run(const float *Jt, int64_t nv, int64_t nm, const double *W, const double *y, double lam, int mode,
                  double *H, int64_t ldh, double *rhs, cudaStream_t st) {
  DGP_REQUIRE(Jt && H, "normal_eq: null pointer");
  DGP_REQUIRE(nv > 0 && nm > 0 && ldh >= nv, "normal_eq: bad sizes");
  DGP_REQUIRE(mode == 0 || mode == 1 || mode == 2,
              "normal_eq: damping mode is 0 (lam*max diag), 1 (lam*diag) or 2 (lam)");
  const int64_t nvp = ceil_div(nv, TM) * TM, nmp = ceil_div(nm, TK) * TK;
  DGP_REQUIRE(nmp < (int64_t)INT32_MAX && nvp < (int64_t)INT32_MAX, "normal_eq: sizes exceed TMA coordinates");
  DevBuf hi, lo, diag, errb;
  DGP_TRY(hi.alloc(sizeof(__nv_bfloat16) * (size_t)nvp * nmp));
  DGP_TRY(lo.alloc(sizeof(__nv_bfloat16) * (size_t)nvp * nmp));
  DGP_TRY(diag.alloc(sizeof(double) * nv));
  DGP_TRY(errb.alloc(sizeof(int)));
  DGP_CUDA(cudaMemsetAsync(errb.p, 0, sizeof(int), st));
  if (W) DGP_TRY(check_weights(W, nm, errb.as<int>(), "normal_eq", st));
  k_split<<<(unsigned)ceil_div(nvp * nmp, 256), 256, 0, st>>>(Jt, W, nv, nm, nvp, nmp, hi.as<__nv_bfloat16>(),
                                                               lo.as<__nv_bfloat16>());
  DGP_CHECK_LAUNCH();
  k_row_dots<<<(unsigned)std::min<int64_t>(nv, 4096), 256, 0, st>>>(Jt, W, y, nv, nm, diag.as<double>(), rhs);
  DGP_CHECK_LAUNCH();
  CUtensorMap mhi, mlo;
  DGP_TRY(make_map(&mhi, hi.p, nvp, nmp));
  DGP_TRY(make_map(&mlo, lo.p, nvp, nmp));
  DGP_CUDA(cudaFuncSetAttribute(k_syrk_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, SYRK_SMEM));
  const int64_t T = nvp / TM;
  const int64_t tiles = T * (T + 1) / 2;
  k_syrk_tc<<<(unsigned)tiles, 128, SYRK_SMEM, st>>>(mhi, mlo, (int)(nmp / TK), nv, H, ldh, errb.as<int>());
  DGP_CHECK_LAUNCH();
  k_damp<<<1, 256, 0, st>>>(H, ldh, diag.as<double>(), nv, lam, mode);
  DGP_CHECK_LAUNCH();
  int herr = 0;
  DGP_CUDA(cudaMemcpyAsync(&herr, errb.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  if (herr) return fail(DGP_ERR_CUDA, "normal_eq: tensor-core pipeline wait timed out (error flags " +
                                          std::to_string(herr) + ")");
  return DGP_OK;
}

// ----------------------------------------------------- tik_inv update
namespace {

// Jw[m][v] = sqrt(W[m]) Jt[v][m]: 32 x 32 tiles through shared memory
__global__ void k_scale_transpose(const float *__restrict__ Jt, const double *__restrict__ W, int64_t nv, int64_t nm,
                                  float *__restrict__ Jw) {
  __shared__ float t[32][33];
  const int64_t v0 = (int64_t)blockIdx.y * 32, m0 = (int64_t)blockIdx.x * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t v = v0 + r, m = m0 + threadIdx.x;
    t[r][threadIdx.x] = (v < nv && m < nm) ? Jt[v * nm + m] : 0.f;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int64_t m = m0 + r, v = v0 + threadIdx.x;
    if (m < nm && v < nv) Jw[m * nv + v] = (W ? (float)sqrt(W[m]) : 1.f) * t[threadIdx.x][r];
  }
}

// out[m] = sqrt(W[m]) in[m]
__global__ void k_scale_sqrtw(const double *in, const double *__restrict__ W, int64_t nm, double *out) {
  const int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (m < nm) out[m] = (W ? sqrt(W[m]) : 1.0) * in[m];
}

}  // namespace

namespace {
// out[a][m] = sum_v A[a][v] Jt[v][m]: thread m of block (x, y) accumulates spots 8y .. 8y+7 in
// FP64; the A columns of a 256-voxel chunk are staged in shared memory, Jt is read once per
// 8 spots with consecutive threads on consecutive m (coalesced)
__global__ void __launch_bounds__(256) k_times_jt(const double *__restrict__ A, int64_t na, int64_t nv,
                                                  const float *__restrict__ Jt, int64_t nm, double *__restrict__ out) {
  __shared__ double As[8][256];
  const int64_t m = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t a0 = (int64_t)blockIdx.y * 8;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t v0 = 0; v0 < nv; v0 += 256) {
    __syncthreads();
    for (int q = 0; q < 8; ++q) {
      const int64_t v = v0 + threadIdx.x;
      As[q][threadIdx.x] = (a0 + q < na && v < nv) ? A[(a0 + q) * nv + v] : 0.0;
    }
    __syncthreads();
    if (m < nm) {
      const int64_t vend = min(nv - v0, (int64_t)256);
      for (int64_t j = 0; j < vend; ++j) {
        const double x = (double)Jt[(v0 + j) * nm + m];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] += As[q][j] * x;
      }
    }
  }
  if (m < nm)
    for (int q = 0; q < 8; ++q)
      if (a0 + q < na) out[(a0 + q) * nm + m] = acc[q];
}
}  // namespace

int times_jt_run(const double *A, int64_t na, int64_t nv, const float *Jt, int64_t nm, double *out, cudaStream_t st) {
  DGP_REQUIRE(A && Jt && out && na > 0 && nv > 0 && nm > 0, "times_jt: bad arguments");
  DGP_REQUIRE(ceil_div(na, 8) <= 65535, "times_jt: too many rows in A");
  dim3 grid((unsigned)ceil_div(nm, 256), (unsigned)ceil_div(na, 8));
  k_times_jt<<<grid, 256, 0, st>>>(A, na, nv, Jt, nm, out);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

int row_dots_run(const float *Jt, int64_t nv, int64_t nm, const double *W, const double *y, double *diag, double *rhs,
                 cudaStream_t st) {
  DGP_REQUIRE(Jt && diag && nv > 0 && nm > 0, "row_dots: bad arguments");
  k_row_dots<<<(unsigned)std::min<int64_t>(nv, 4096), 256, 0, st>>>(Jt, W, y, nv, nm, diag, rhs);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

// update = (J^T W J + lam max_i (J^T W J)_ii I)^-1 J^T W y  (tik_inv.m:13-20 with W).  With fewer
// measurements than unknowns the same update is J_w^T (J_w J_w^T + mu I)^-1 W^1/2 y with
// J_w = W^1/2 J and mu = lam max_i (J^T W J)_ii: the Gram matrix and the factorisation are
// nmeas x nmeas instead of nv x nv.
int lm_update_run(const float *Jt, int64_t nv, int64_t nm, const double *W, const double *y, double lam, double *x,
                  int32_t form, int32_t *form_used, cudaStream_t st) {
  DGP_REQUIRE(Jt && y && x && nv > 0 && nm > 0, "lm_update: bad arguments");
  DGP_REQUIRE(form >= 0 && form <= 2, "lm_update: form is 0 (auto), 1 (unknowns) or 2 (measurements)");
  const bool dual = form == 2 || (form == 0 && nm < nv);
  if (form_used) *form_used = dual ? 2 : 1;
  if (!dual) {
    // an even leading dimension keeps every row 16-byte aligned: the Cholesky's GEMMs then move
    // their operands with 16-byte copies
    const int64_t ldh = nv + (nv & 1);
    DevBuf H;
    DGP_TRY(H.alloc(sizeof(double) * (size_t)nv * ldh));
    DGP_TRY(normal_eq_run(Jt, nv, nm, W, y, lam, 0, H.as<double>(), ldh, x, st));
    return cholesky_solve_run(H.as<double>(), nv, ldh, x, st);
  }
  DevBuf diag, Jw, G, z, errb;
  if (W) {
    DGP_TRY(errb.alloc(sizeof(int)));
    DGP_CUDA(cudaMemsetAsync(errb.p, 0, sizeof(int), st));
    DGP_TRY(check_weights(W, nm, errb.as<int>(), "lm_update", st));
  }
  DGP_TRY(diag.alloc(sizeof(double) * nv));
  DGP_TRY(Jw.alloc(sizeof(float) * (size_t)nm * nv));
  const int64_t ldg = nm + (nm & 1);
  DGP_TRY(G.alloc(sizeof(double) * (size_t)nm * ldg));
  DGP_TRY(z.alloc(sizeof(double) * nm));
  DGP_TRY(row_dots_run(Jt, nv, nm, W, nullptr, diag.as<double>(), nullptr, st));
  std::vector<double> hd((size_t)nv);
  DGP_CUDA(cudaMemcpyAsync(hd.data(), diag.p, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  double dmax = 0.0;
  for (double d : hd) dmax = std::max(dmax, d);
  const double mu = lam * dmax;
  dim3 tb(32, 8), tg((unsigned)ceil_div(nm, 32), (unsigned)ceil_div(nv, 32));
  DGP_REQUIRE(tg.y <= 65535u, "lm_update: too many unknowns for the transpose grid");
  k_scale_transpose<<<tg, tb, 0, st>>>(Jt, W, nv, nm, Jw.as<float>());
  DGP_CHECK_LAUNCH();
  // G = J_w J_w^T + mu I: the split-BF16 Gram kernel on J_w (rows = measurements)
  DGP_TRY(normal_eq_run(Jw.as<float>(), nm, nv, nullptr, nullptr, mu, 2, G.as<double>(), ldg, nullptr, st));
  k_scale_sqrtw<<<(unsigned)ceil_div(nm, 256), 256, 0, st>>>(y, W, nm, z.as<double>());
  DGP_CHECK_LAUNCH();
  DGP_TRY(cholesky_solve_run(G.as<double>(), nm, ldg, z.as<double>(), st));
  k_scale_sqrtw<<<(unsigned)ceil_div(nm, 256), 256, 0, st>>>(z.as<double>(), W, nm, z.as<double>());
  DGP_CHECK_LAUNCH();
  // x = J^T (W^1/2 z)
  DGP_TRY(row_dots_run(Jt, nv, nm, nullptr, z.as<double>(), diag.as<double>(), x, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  return DGP_OK;
}

}  // namespace dgp
