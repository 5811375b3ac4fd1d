// FP64 Cholesky factorisation and solves of the damped LM normal matrix, on this library's own
// kernels (FP64 tensor cores through mma.sync m16n8k4 .f64, no BLAS library).
//
// Replaces MATLAB's backslash in tik_inv (DOGPUP/reconstruction/tik_inv.m:20: H \ J'y with H
// symmetric positive definite, i.e. a Cholesky factorisation and two triangular solves).
//
// H is row-major [n][ldh]; its lower triangle is read and overwritten by L (H = L L^T); the
// strict upper triangle is not touched.  Right-looking, 512-column outer panels of 128-column
// steps:
//
//   for each step k (columns [k0, k0 + 128)) of the outer panel [o0, o0 + 512):
//     k_potrf_tile   the 128 x 128 diagonal block: L_kk in place, and inv(L_kk) into a scratch
//                    table (one CTA, block in shared memory: 32-column steps, a warp factors the
//                    32 x 32 diagonal, all warps solve and update the rest; the inverse by
//                    32-blocks)
//     k_dgemm_nt     panel: L_ik = A_ik inv(L_kk)^T for the rows below (in place: a CTA owns
//                    whole 128-row strips of the panel)
//     k_dgemm_nt     update of the outer panel's remaining columns: A_il -= L_ik L_lk^T
//   k_dgemm_nt       trailing update of the rest, depth 512: A_il -= sum over the outer panel
//
// k_dgemm_nt: C = beta C + alpha A B^T with A, B row-major (K contiguous); 128 x 128 CTA tiles,
// 256 threads (8 warps of 64 x 32), K in stages of 16 doubles moved by cp.async through a
// 4-deep shared-memory ring (rows padded to 20 doubles: the fragment loads hit 32 distinct banks
// per half-warp), 16 mma.sync m16n8k4 .f64 per warp per 4 K.
//
// Solves: L y = b and L^T x = y by 128-row blocks with the stored diagonal inverses:
//   y_b = inv(L_bb) (b_b - sum_{c<b} L_bc y_c),   x_b = inv(L_bb)^T (y_b - sum_{c>b} L_cb^T x_c),
// each block one partial-sum kernel over the off-diagonal blocks (FP64, atomics into a 128 x nrhs
// accumulator) and one small kernel for the diagonal product.
#include <algorithm>
#include <cmath>
#include <vector>

#include "dgp_common.cuh"
#include "dgp_internal.h"

namespace dgp {

namespace {

constexpr int CB = 128;          // panel width = CTA tile
constexpr int GK = 16;           // K per pipeline stage (doubles)
constexpr int LDK = GK + 4;      // padded shared-memory row (doubles)
constexpr int GSTAGES = 4;
constexpr int GTHREADS = 256;
constexpr int GEMM_SMEM = GSTAGES * 2 * CB * LDK * (int)sizeof(double);   // 160 KB
static_assert(GEMM_SMEM >= CB * (CB + 1) * (int)sizeof(double), "the epilogue tile must fit the stage ring");
constexpr int GV = 256;          // k per CTA of the solves' off-diagonal partial sums
#ifndef DGP_CHOL_NBO
#define DGP_CHOL_NBO 512
#endif
constexpr int64_t NBO = DGP_CHOL_NBO;  // outer panel width: depth of the trailing update GEMM

__device__ inline uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// dst <- 16 (or 8) bytes at src; zero-filled when !pred (src must still be a valid address)
template <int BYTES>
__device__ inline void cp_async(void *dst, const void *src, bool pred) {
  const int n = pred ? BYTES : 0;
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(su32(dst)), "l"(src), "r"(n) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(su32(dst)), "l"(src), "r"(n) : "memory");
}
__device__ inline void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ inline void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// D = A B + D for one m16n8k4 FP64 tile: a = {A[g][t], A[g+8][t]}, b = B[t][g] (g = lane/4,
// t = lane%4); d = {D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1]}
__device__ inline void mma_f64(double (&d)[4], double a0, double a1, double b) {
  asm volatile("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
               : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
               : "d"(a0), "d"(a1), "d"(b));
}

struct Gemm {
  const double *A;
  int64_t lda;
  const double *B;
  int64_t ldb;
  double *C;
  int64_t ldc;
  int64_t M, N, K;     // C is M x N, A is M x K, B is N x K
  double alpha, beta;
  int lower;           // 1: tiles with tj <= ti only, and in diagonal tiles only entries c <= r
  int64_t tn;          // tiles along N (full mode)
};

// C = beta C + alpha A B^T on 128 x 128 tiles (see the file comment).  V: bytes per cp.async
// (16 when every row start and the base addresses are 16-byte aligned, else 8).
template <int V>
__global__ void __launch_bounds__(GTHREADS, 1) k_dgemm_nt(Gemm g) {
  extern __shared__ __align__(16) double gsm[];
  int64_t ti, tj;
  if (g.lower) {
    const int64_t b = blockIdx.x;
    ti = (int64_t)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while (ti * (ti + 1) / 2 > b) --ti;
    while ((ti + 1) * (ti + 2) / 2 <= b) ++ti;
    tj = b - ti * (ti + 1) / 2;
  } else {
    ti = blockIdx.x / g.tn;
    tj = blockIdx.x % g.tn;
  }
  const int64_t r0 = ti * CB, c0 = tj * CB;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = warp & 1, wn = warp >> 1;          // warp tile: rows wm*64.., cols wn*32..
  const int gid = lane >> 2, tig = lane & 3;
  double acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;

  const int nk = (int)((g.K + GK - 1) / GK);
  constexpr int E = V / 8;                          // doubles per copy
  constexpr int PER_ROW = GK / E;                   // copies per row per stage
  auto load_stage = [&](int kb, int slot) {
    double *As = gsm + (size_t)slot * 2 * CB * LDK, *Bs = As + CB * LDK;
    const int64_t kbase = (int64_t)kb * GK;
    for (int e = tid; e < 2 * CB * PER_ROW; e += GTHREADS) {
      const int which = e / (CB * PER_ROW), rem = e % (CB * PER_ROW), row = rem / PER_ROW, kc = (rem % PER_ROW) * E;
      const int64_t grow = (which ? c0 : r0) + row, gk = kbase + kc;
      const bool ok = grow < (which ? g.N : g.M) && gk + E <= g.K;
      const double *base = which ? g.B : g.A;
      const int64_t ld = which ? g.ldb : g.lda;
      const double *src = ok ? base + grow * ld + gk : base;
      cp_async<V>((which ? Bs : As) + row * LDK + kc, src, ok);
    }
  };
  // prologue: GSTAGES - 1 stages in flight
#pragma unroll
  for (int s = 0; s < GSTAGES - 1; ++s) {
    if (s < nk) load_stage(s, s);
    cp_commit();
  }
  for (int kb = 0; kb < nk; ++kb) {
    cp_wait<GSTAGES - 2>();
    __syncthreads();
    const int nxt = kb + GSTAGES - 1;
    if (nxt < nk) load_stage(nxt, nxt % GSTAGES);
    cp_commit();
    const double *As = gsm + (size_t)(kb % GSTAGES) * 2 * CB * LDK, *Bs = As + CB * LDK;
#pragma unroll
    for (int k4 = 0; k4 < GK; k4 += 4) {
      double a[4][2], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int row = wm * 64 + i * 16 + gid;
        a[i][0] = As[row * LDK + k4 + tig];
        a[i][1] = As[(row + 8) * LDK + k4 + tig];
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[(wn * 32 + j * 8 + gid) * LDK + k4 + tig];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) mma_f64(acc[i][j], a[i][0], a[i][1], b[j]);
    }
  }
  cp_wait<0>();
  __syncthreads();   // the stage ring is free: the epilogue goes through shared memory
  // epilogue: the accumulators are written to shared memory (a 128 x 129-double tile), then the
  // CTA reads and writes C row by row, coalesced, with every load of C in flight together
  // (C = beta C + alpha acc; in diagonal tiles of the lower mode only entries c <= r)
  double *T = gsm;
  constexpr int TLD = CB + 1;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = wm * 64 + i * 16 + gid + (q >> 1) * 8, c = wn * 32 + j * 8 + 2 * tig + (q & 1);
        T[r * TLD + c] = acc[i][j][q];
      }
  __syncthreads();
  const int64_t rows = min((int64_t)CB, g.M - r0), cols = min((int64_t)CB, g.N - c0);
  // batches of 16 entries per thread: all 16 loads of C are issued before any store (a store to
  // C between loads would otherwise keep the compiler from overlapping their latencies)
  constexpr int BATCH = 16;
  for (int e0 = tid; e0 < CB * CB; e0 += GTHREADS * BATCH) {
    double cv[BATCH];
    bool in[BATCH];
#pragma unroll
    for (int u = 0; u < BATCH; ++u) {
      const int e = e0 + u * GTHREADS, r = e / CB, c = e % CB;
      in[u] = e < CB * CB && r < rows && c < cols && (!g.lower || ti != tj || c <= r);
      cv[u] = (in[u] && g.beta != 0.0) ? g.C[(r0 + r) * g.ldc + c0 + c] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < BATCH; ++u) {
      const int e = e0 + u * GTHREADS, r = e / CB, c = e % CB;
      if (in[u]) g.C[(r0 + r) * g.ldc + c0 + c] = g.beta * cv[u] + g.alpha * T[r * TLD + c];
    }
  }
}

// Factor the nb x nb diagonal block at (k0, k0) in place (lower) and write inv(L) (row-major,
// nb x nb, zero above the diagonal) to Linv.  One CTA of 128 threads; the block sits in shared
// memory with rows padded to 129 doubles.  32-column steps: warp 0 factors the 32 x 32 diagonal
// (warp-synchronous, one column per step), then every thread solves its rows of the 32-column
// panel below and the trailing lower triangle is updated.  err |= 1 on a non-positive or
// non-finite pivot.
constexpr int PT = 128, PLD = 129;
constexpr size_t POT_SMEM = sizeof(double) * ((size_t)PT * PLD + 3 * 32 * 33);
__global__ void __launch_bounds__(128) k_potrf_tile(double *__restrict__ H, int64_t ldh, int64_t k0, int nb,
                                                   double *__restrict__ Linv, int *err) {
  extern __shared__ double L[];                      // [PT][PLD], then the [3][32][33] level products
  __shared__ int bad;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) bad = 0;
  for (int e = tid; e < nb * nb; e += blockDim.x) {
    const int r = e / nb, c = e % nb;
    L[r * PLD + c] = c <= r ? H[(k0 + r) * ldh + k0 + c] : 0.0;
  }
  __syncthreads();
  for (int j0 = 0; j0 < nb; j0 += 32) {
    const int jw = min(32, nb - j0);
    // 1. warp 0: factor the jw x jw diagonal block, one column per step
    if (warp == 0) {
      for (int j = 0; j < jw; ++j) {
        const int c = j0 + j;
        double d = L[c * PLD + c];
        if (!(d > 0.0) || !isfinite(d)) {
          if (lane == 0) bad = 1;
          d = 1.0;
        }
        d = sqrt(d);
        __syncwarp();
        const int r = j0 + lane;
        if (lane > j && lane < jw) L[r * PLD + c] /= d;
        if (lane == 0) L[c * PLD + c] = d;
        __syncwarp();
        // update the rest of the diagonal block's lower triangle: columns j+1 .. lane of row r
        if (lane > j && lane < jw) {
          const double lrc = L[r * PLD + c];
          for (int q = j + 1; q <= lane; ++q) L[r * PLD + j0 + q] -= lrc * L[(j0 + q) * PLD + c];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    // 2. panel rows below: row r solves x L_dd^T = a  (forward substitution over the jw columns)
    for (int r = j0 + jw + tid; r < nb; r += blockDim.x) {
      for (int j = 0; j < jw; ++j) {
        const int c = j0 + j;
        double s = L[r * PLD + c];
        for (int q = 0; q < j; ++q) s -= L[r * PLD + j0 + q] * L[c * PLD + j0 + q];
        L[r * PLD + c] = s / L[c * PLD + c];
      }
    }
    __syncthreads();
    // 3. trailing lower triangle: A[r][c] -= sum_q L[r][q] L[c][q] over the panel's columns
    const int t0 = j0 + jw, nt = nb - t0;
    for (int e = tid; e < nt * nt; e += blockDim.x) {
      const int r = t0 + e / nt, c = t0 + e % nt;
      if (c > r) continue;
      double s = 0.0;
      for (int q = j0; q < j0 + jw; ++q) s += L[r * PLD + q] * L[c * PLD + q];
      L[r * PLD + c] -= s;
    }
    __syncthreads();
  }
  if (bad && tid == 0) atomicOr(err, 1);
  // write L back
  for (int e = tid; e < nb * nb; e += blockDim.x) {
    const int r = e / nb, c = e % nb;
    if (c <= r) H[(k0 + r) * ldh + k0 + c] = L[r * PLD + c];
  }
  // inv(L) = X, blocked by 32 (entries X[i][c], i > c, kept in the strict upper triangle of the
  // shared tile at [c][i]; X[c][c] = 1 / L[c][c] in dinv):
  //   1. the diagonal 32-blocks: warp w, lane l solves column c = 32 w + l of inv(L_ww)
  //   2. the off-diagonal blocks by distance d = I - J = 1, 2, 3 below the diagonal:
  //      T = sum_{K = J .. I-1} L_IK X_KJ, then X_IJ = -X_II T
  __shared__ double dinv[PT];
  for (int c = tid; c < nb; c += blockDim.x) dinv[c] = 1.0 / L[c * PLD + c];
  __syncthreads();
  auto X = [&](int k, int c) -> double { return k < c ? 0.0 : (k == c ? dinv[c] : L[c * PLD + k]); };
  {
    const int c = 32 * warp + lane;
    if (c < nb) {
      const int iend = min(32 * (warp + 1), nb);
      for (int i = c + 1; i < iend; ++i) {
        double t = L[i * PLD + c] * dinv[c];
        for (int l = c + 1; l < i; ++l) t += L[i * PLD + l] * L[c * PLD + l];
        L[c * PLD + i] = -t * dinv[i];
      }
    }
  }
  __syncthreads();
  double *Tb = L + PT * PLD;                          // [3][32][33] products of one level
  for (int d = 1; d < 4; ++d) {
    const int nblk = 4 - d;
    for (int e = tid; e < nblk * 1024; e += blockDim.x) {
      const int J = e / 1024, I = J + d, i = 32 * I + (e % 1024) / 32, c = 32 * J + e % 32;
      double t = 0.0;
      if (i < nb && c < nb)
        for (int k = 32 * J; k < 32 * I; ++k) t += L[i * PLD + k] * X(k, c);
      Tb[(J * 32 + (e % 1024) / 32) * 33 + e % 32] = t;
    }
    __syncthreads();
    for (int e = tid; e < nblk * 1024; e += blockDim.x) {
      const int J = e / 1024, I = J + d, i = 32 * I + (e % 1024) / 32, c = 32 * J + e % 32;
      if (i >= nb || c >= nb) continue;
      double x = 0.0;
      for (int m = 32 * I; m <= i; ++m) x += X(i, m) * Tb[(J * 32 + m - 32 * I) * 33 + e % 32];
      L[c * PLD + i] = -x;
    }
    __syncthreads();
  }
  for (int e = tid; e < nb * nb; e += blockDim.x) {
    const int i = e / nb, c = e % nb;
    Linv[e] = X(i, c);
  }
}

// ---------------------------------------------------------------- solves
// forward:  acc[r][i] += sum_{k in [kb, ke)} H[base + i][k] X[r][k]     (L_bc y_c)
//   block (x, y, z): k chunk x of GV, rows 8y .. 8y + 7 (one warp each), right-hand side z;
//   lanes stride k, warp shuffle, one FP64 atomic per (row, chunk)
// backward: acc[r][i] += sum_{k in [kb, ke)} H[k][base + i] X[r][k]     (L_cb^T x_c)
//   block (x, -, z): rows k of chunk x (GVB of them), thread i = column i (consecutive threads
//   read consecutive columns of a row), one FP64 atomic per (column, chunk)
// X is row-major [nrhs][ldx].
constexpr int GVB = 32;
template <bool TRANS>
__global__ void k_block_gemv(const double *__restrict__ H, int64_t ldh, int64_t base, int nbi, int64_t kb,
                             int64_t ke, const double *__restrict__ X, int64_t ldx, double *acc) {
  const int r = blockIdx.z;
  const double *x = X + (int64_t)r * ldx;
  if (!TRANS) {
    const int64_t k_lo = kb + (int64_t)blockIdx.x * GV, k_hi = min(ke, k_lo + GV);
    const int i = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (i >= nbi || k_lo >= k_hi) return;
    const double *row = H + (base + i) * ldh;
    double s = 0.0;
    for (int64_t k = k_lo + (threadIdx.x & 31); k < k_hi; k += 32) s += row[k] * x[k];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc + (int64_t)r * CB + i, s);
  } else {
    const int64_t k_lo = kb + (int64_t)blockIdx.x * GVB, k_hi = min(ke, k_lo + GVB);
    const int i = threadIdx.x;
    if (i >= nbi || k_lo >= k_hi) return;
    double s = 0.0;
#pragma unroll 8
    for (int64_t k = k_lo; k < k_hi; ++k) s += H[k * ldh + base + i] * x[k];
    atomicAdd(acc + (int64_t)r * CB + i, s);
  }
}

// X[r][base + i] = sum_j Linv'[i][j] (X[r][base + j] - acc[r][j]), Linv' = inv(L_bb) (forward) or
// its transpose (backward); one warp per output entry (lanes stride j, coalesced along rows of
// Linv for the forward product); acc is cleared for the next block.
template <bool TRANS>
__global__ void k_block_diag(const double *__restrict__ Linv, int nbi, int64_t base, double *X, int64_t ldx,
                             double *acc) {
  __shared__ double rhs[CB];
  const int r = blockIdx.x;
  double *x = X + (int64_t)r * ldx + base;
  for (int j = threadIdx.x; j < nbi; j += blockDim.x) rhs[j] = x[j] - acc[(int64_t)r * CB + j];
  __syncthreads();
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int i = threadIdx.x >> 5; i < nbi; i += nw) {
    double s = 0.0;
    if (!TRANS) {
      for (int j = lane; j <= i; j += 32) s += Linv[(int64_t)i * nbi + j] * rhs[j];
    } else {
      for (int j = i + lane; j < nbi; j += 32) s += Linv[(int64_t)j * nbi + i] * rhs[j];
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) {
      x[i] = s;
      acc[(int64_t)r * CB + i] = 0.0;
    }
  }
}

int gemm_nt(const Gemm &g0, cudaStream_t st) {
  Gemm g = g0;
  if (g.M <= 0 || g.N <= 0) return DGP_OK;
  const bool a16 = ((uintptr_t)g.A % 16 == 0) && ((uintptr_t)g.B % 16 == 0) && g.lda % 2 == 0 && g.ldb % 2 == 0 &&
                   g.K % 2 == 0;
  const int64_t tm = ceil_div(g.M, CB), tn = ceil_div(g.N, CB);
  g.tn = tn;
  const int64_t tiles = g.lower ? tm * (tm + 1) / 2 : tm * tn;
  DGP_REQUIRE(tiles <= INT32_MAX, "cholesky: too many tiles");
  if (a16) {
    DGP_CUDA(cudaFuncSetAttribute(k_dgemm_nt<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM));
    k_dgemm_nt<16><<<(unsigned)tiles, GTHREADS, GEMM_SMEM, st>>>(g);
  } else {
    DGP_CUDA(cudaFuncSetAttribute(k_dgemm_nt<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, GEMM_SMEM));
    k_dgemm_nt<8><<<(unsigned)tiles, GTHREADS, GEMM_SMEM, st>>>(g);
  }
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

}  // namespace

int cholesky_solve_many_run(double *H, int64_t n, int64_t ldh, double *x, int32_t nrhs, int64_t ldx,
                            cudaStream_t st) {
  DGP_REQUIRE(H && x && n > 0 && ldh >= n, "cholesky: bad arguments");
  DGP_REQUIRE(nrhs >= 1 && ldx >= n, "cholesky: need nrhs >= 1 and ldx >= n");
  DGP_REQUIRE(nrhs <= 65535, "cholesky: at most 65535 right-hand sides");
  DGP_REQUIRE(ceil_div(n, (int64_t)GVB) <= INT32_MAX, "cholesky: n too large for the solve grid");
  const int64_t nblk = ceil_div(n, CB);
  DevBuf linv, errb, acc;
  DGP_TRY(linv.alloc(sizeof(double) * (size_t)nblk * CB * CB));
  DGP_TRY(errb.alloc(sizeof(int)));
  DGP_TRY(acc.alloc(sizeof(double) * (size_t)CB * nrhs));
  DGP_CUDA(cudaMemsetAsync(errb.p, 0, sizeof(int), st));
  DGP_CUDA(cudaMemsetAsync(acc.p, 0, sizeof(double) * (size_t)CB * nrhs, st));
  const size_t pot_smem = POT_SMEM;
  DGP_CUDA(cudaFuncSetAttribute(k_potrf_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pot_smem));
  double *Li = linv.as<double>();
  int64_t launches = 0;
  // 512-column outer panels: inside one, 128-column steps update only the outer panel's own
  // columns (the rows below included); the rest of the matrix takes the outer panel's update in
  // one lower-triangle GEMM of depth 512
  for (int64_t o0 = 0; o0 < n; o0 += NBO) {
    const int64_t oend = std::min(n, o0 + NBO);
    bool last = false;
    for (int64_t k0 = o0; k0 < oend; k0 += CB) {
      const int64_t b = k0 / CB;
      const int nb = (int)std::min<int64_t>(CB, n - k0);
      double *Lb = Li + b * CB * CB;
      k_potrf_tile<<<1, 128, pot_smem, st>>>(H, ldh, k0, nb, Lb, errb.as<int>());
      DGP_CHECK_LAUNCH();
      ++launches;
      const int64_t kend = k0 + nb, rest = n - kend;
      if (rest <= 0) {
        last = true;
        break;
      }
      // L_ik = A_ik inv(L_kk)^T for every row below (in place, one CTA per 128-row strip)
      const Gemm p{H + kend * ldh + k0, ldh, Lb, nb, H + kend * ldh + k0, ldh, rest, nb, nb, 1.0, 0.0, 0, 0};
      DGP_TRY(gemm_nt(p, st));
      ++launches;
      const int64_t w = oend - kend;  // the outer panel's remaining columns
      if (w > 0) {
        const Gemm a{H + kend * ldh + k0, ldh, H + kend * ldh + k0, ldh, H + kend * ldh + kend, ldh, w, w, nb,
                     -1.0, 1.0, 1, 0};
        DGP_TRY(gemm_nt(a, st));
        ++launches;
        if (n > oend) {
          const Gemm r{H + oend * ldh + k0, ldh, H + kend * ldh + k0, ldh, H + oend * ldh + kend, ldh, n - oend, w,
                       nb, -1.0, 1.0, 0, 0};
          DGP_TRY(gemm_nt(r, st));
          ++launches;
        }
      }
    }
    if (last || n <= oend) break;
    // trailing lower triangle: rows/cols [oend, n) -= Q Q^T, Q = rows [oend, n) x cols [o0, oend)
    const Gemm t{H + oend * ldh + o0, ldh, H + oend * ldh + o0, ldh, H + oend * ldh + oend, ldh, n - oend, n - oend,
                 oend - o0, -1.0, 1.0, 1, 0};
    DGP_TRY(gemm_nt(t, st));
    ++launches;
  }
  // L y = b, then L^T x = y, by 128-row blocks
  for (int64_t b = 0; b < nblk; ++b) {
    const int64_t k0 = b * CB;
    const int nb = (int)std::min<int64_t>(CB, n - k0);
    if (k0 > 0) {
      dim3 gr((unsigned)ceil_div(k0, GV), (unsigned)ceil_div(nb, 8), (unsigned)nrhs);
      k_block_gemv<false><<<gr, 256, 0, st>>>(H, ldh, k0, nb, 0, k0, x, ldx, acc.as<double>());
      ++launches;
    }
    k_block_diag<false><<<(unsigned)nrhs, 256, 0, st>>>(Li + b * CB * CB, nb, k0, x, ldx, acc.as<double>());
    ++launches;
  }
  for (int64_t b = nblk - 1; b >= 0; --b) {
    const int64_t k0 = b * CB;
    const int nb = (int)std::min<int64_t>(CB, n - k0);
    const int64_t kend = k0 + nb;
    if (kend < n) {
      dim3 gr((unsigned)ceil_div(n - kend, GVB), 1, (unsigned)nrhs);
      k_block_gemv<true><<<gr, 128, 0, st>>>(H, ldh, k0, nb, kend, n, x, ldx, acc.as<double>());
      ++launches;
    }
    k_block_diag<true><<<(unsigned)nrhs, 256, 0, st>>>(Li + b * CB * CB, nb, k0, x, ldx, acc.as<double>());
    ++launches;
  }
  DGP_CHECK_LAUNCH();
  count_launches(launches);
  int herr = 0;
  DGP_CUDA(cudaMemcpyAsync(&herr, errb.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  if (herr) return fail(DGP_ERR_ARG, "cholesky: matrix is not positive definite");
  return DGP_OK;
}

int cholesky_solve_run(double *H, int64_t n, int64_t ldh, double *x, cudaStream_t st) {
  return cholesky_solve_many_run(H, n, ldh, x, 1, n, st);
}

}  // namespace dgp
