// FP64 Cholesky factorisation and solves of the damped LM normal matrix, on this library's own
// kernels (FP64 tensor cores through mma.sync m16n8k4 .f64, no BLAS library).
//
// Replaces MATLAB's backslash in tik_inv (DOGPUP/reconstruction/tik_inv.m:20: H \ J'y with H
// symmetric positive definite, i.e. a Cholesky factorisation and two triangular solves).
//
// H is row-major [n][ldh]; its lower triangle is read and overwritten by L (H = L L^T); the
// strict upper triangle is not touched.  Right-looking, 1536-column outer panels of 128-column
// steps:
//
//   for each step k (columns [k0, k0 + 128)) of the outer panel [o0, o0 + 1536):
//     k_potrf_tile   the 128 x 128 diagonal block: L_kk in place, and inv(L_kk) into a scratch
//                    table (one CTA, block in shared memory: 32-column steps, a warp factors the
//                    32 x 32 diagonal, all warps solve and update the rest; the inverse by
//                    32-blocks)
//     k_dgemm_nt     panel: L_ik = A_ik inv(L_kk)^T for the rows below (in place: a CTA owns
//                    whole 128-row strips of the panel)
//     k_dgemm_nt     update of the outer panel's remaining columns: A_il -= L_ik L_lk^T
//   k_dgemm_nt       trailing update of the rest, depth 1536: A_il -= sum over the outer panel
//
// k_dgemm_nt: C = beta C + alpha A B^T with A, B row-major (K contiguous); 128 x 64 CTA tiles,
// two CTAs per SM, 256 threads (8 warps of 32 x 32), K in stages of 16 doubles moved by cp.async
// through a 3-deep shared-memory ring (rows padded to 20 doubles: the fragment loads hit 32
// distinct banks per half-warp), 8 mma.sync m16n8k4 .f64 per warp per 4 K.  The updates of the
// factorisation (beta = 1, alpha = -1) start their accumulators from C in the fragments and
// store them back from registers.
//
// Solves: L y = b and L^T x = y by 128-row blocks with the stored diagonal inverses:
//   y_b = inv(L_bb) (b_b - sum_{c<b} L_bc y_c),   x_b = inv(L_bb)^T (y_b - sum_{c>b} L_cb^T x_c).
// One right-hand side: one cooperative launch per direction, a CTA per block, each block
// published by a flag that the later blocks wait for (k_trsv_chain).  Several right-hand sides
// (or more blocks than fit on the GPU at once): per block, one partial-sum kernel over the
// off-diagonal blocks (FP64, atomics into a 128 x nrhs accumulator) and one small kernel for the
// diagonal product.
#include <algorithm>
#include <cmath>
#include <vector>

#include "dgp_common.cuh"
#include "dgp_internal.h"

namespace dgp {

namespace {

constexpr int CB = 128;          // panel width = CTA tile
constexpr int GBM = 128;         // GEMM CTA tile rows; columns GBN = 64 (two CTAs per SM) or 128
constexpr int GK = 16;           // K per pipeline stage (doubles)
constexpr int LDK = GK + 4;      // padded shared-memory row (doubles)
constexpr int GSTAGES = 3;
constexpr int GTHREADS = 256;
// the stage ring, or the epilogue tile where that is larger: 90 KB (GBN = 64), 132 KB (GBN = 128)
constexpr int gemm_smem(int gbn) {
  return (int)sizeof(double) * (GSTAGES * (GBM + gbn) * LDK > GBM * (gbn + 1) ? GSTAGES * (GBM + gbn) * LDK
                                                                               : GBM * (gbn + 1));
}
constexpr int GV = 256;          // k per CTA of the solves' off-diagonal partial sums
#ifndef DGP_CHOL_NBO
#define DGP_CHOL_NBO 1536
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
  int lower;           // 1: only the tiles that meet the lower triangle, only entries c <= r
  int64_t tn;          // tiles along N (full mode)
  int cvec;            // C and ldc allow 16-byte accesses to column pairs (set by gemm_launch)
};

// C = beta C + alpha A B^T on 128 x GBN CTA tiles (see the file comment).  V: bytes per cp.async
// (16 when every row start and the base addresses are 16-byte aligned, else 8).  GBN = 128 when C
// is A itself (the in-place panel: a CTA must own whole rows of it).  Lower mode (GBN = 64): the
// tiles that meet the lower triangle, row ti holding tiles tj = 0 .. 2 ti + 1 (the last two
// straddle the diagonal; only entries c <= r are written).  REG (beta = 1, alpha = +-1): the
// accumulators start from C / alpha (exact) in the mma fragments, loaded before the main loop so
// that their latency hides behind the first stages, and C = alpha acc goes back from registers;
// otherwise the accumulators start at zero and C = beta C + alpha acc goes through shared memory.
template <int V, int GBN, bool REG>
__global__ void __launch_bounds__(GTHREADS, GBN == 64 ? 2 : 1) k_dgemm_nt(Gemm g) {
  constexpr int NJ = GBN / 16;                      // n8 fragments per warp (warp tile 32 x GBN / 2)
  extern __shared__ __align__(16) double gsm[];
  int64_t ti, tj;
  if (g.lower) {
    const int64_t b = blockIdx.x;                   // row ti starts at tile ti (ti + 1)
    ti = (int64_t)((sqrt(4.0 * (double)b + 1.0) - 1.0) * 0.5);
    while (ti * (ti + 1) > b) --ti;
    while ((ti + 1) * (ti + 2) <= b) ++ti;
    tj = b - ti * (ti + 1);
  } else {
    ti = blockIdx.x / g.tn;
    tj = blockIdx.x % g.tn;
  }
  const int64_t r0 = ti * GBM, c0 = tj * GBN;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = warp & 3, wn = warp >> 2;          // warp tile: rows wm*32.., cols wn*GBN/2..
  const int gid = lane >> 2, tig = lane & 3;
  double acc[2][NJ][4];
  // fragment entry (i, j, q) is C row wm*32 + i*16 + gid + 8*(q/2), column wn*GBN/2 + j*8 + 2*tig + q%2
  const int64_t rows = min((int64_t)GBM, g.M - r0), cols = min((int64_t)GBN, g.N - c0);
  // whole tile inside C and (lower mode) on or below the diagonal: column pairs as 16-byte accesses
  const bool whole = rows == GBM && cols == GBN && (!g.lower || c0 + GBN - 1 <= r0) && g.cvec;
  auto frag_in = [&](int r, int c) { return r < rows && c < cols && (!g.lower || c0 + c <= r0 + r); };
  if constexpr (REG) {
    const double sgn = g.alpha;                     // +-1: C / alpha = sgn C
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = wm * 32 + i * 16 + gid + 8 * h, c = wn * (GBN / 2) + j * 8 + 2 * tig;
          const double *cp = g.C + (r0 + r) * g.ldc + c0 + c;
          if (whole) {
            const double2 v = *reinterpret_cast<const double2 *>(cp);
            acc[i][j][2 * h] = sgn * v.x;
            acc[i][j][2 * h + 1] = sgn * v.y;
          } else {
            acc[i][j][2 * h] = frag_in(r, c) ? sgn * cp[0] : 0.0;
            acc[i][j][2 * h + 1] = frag_in(r, c + 1) ? sgn * cp[1] : 0.0;
          }
        }
  } else {
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][j][q] = 0.0;
  }

  const int nk = (int)((g.K + GK - 1) / GK);
  constexpr int E = V / 8;                          // doubles per copy
  constexpr int PER_ROW = GK / E;                   // copies per row per stage
  constexpr int COPIES = (GBM + GBN) * PER_ROW;
  auto load_stage = [&](int kb, int slot) {
    double *As = gsm + (size_t)slot * (GBM + GBN) * LDK, *Bs = As + GBM * LDK;
    const int64_t kbase = (int64_t)kb * GK;
#pragma unroll
    for (int e0 = 0; e0 < COPIES; e0 += GTHREADS) {
      const int e = e0 + tid;
      const bool isb = e >= GBM * PER_ROW;
      const int rem = isb ? e - GBM * PER_ROW : e, row = rem / PER_ROW, kc = (rem % PER_ROW) * E;
      const int64_t grow = (isb ? c0 : r0) + row, gk = kbase + kc;
      const bool ok = grow < (isb ? g.N : g.M) && gk + E <= g.K;
      const double *base = isb ? g.B : g.A;
      const int64_t ld = isb ? g.ldb : g.lda;
      const double *src = ok ? base + grow * ld + gk : base;
      cp_async<V>((isb ? Bs : As) + row * LDK + kc, src, ok);
    }
  };
  static_assert(COPIES % GTHREADS == 0, "whole copy rounds per stage");
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
    const double *As = gsm + (size_t)(kb % GSTAGES) * (GBM + GBN) * LDK, *Bs = As + GBM * LDK;
#pragma unroll
    for (int k4 = 0; k4 < GK; k4 += 4) {
      double a[2][2], b[NJ];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int row = wm * 32 + i * 16 + gid;
        a[i][0] = As[row * LDK + k4 + tig];
        a[i][1] = As[(row + 8) * LDK + k4 + tig];
      }
#pragma unroll
      for (int j = 0; j < NJ; ++j) b[j] = Bs[(wn * (GBN / 2) + j * 8 + gid) * LDK + k4 + tig];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) mma_f64(acc[i][j], a[i][0], a[i][1], b[j]);
    }
  }
  cp_wait<0>();
  if constexpr (REG) {
    const double sgn = g.alpha;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = wm * 32 + i * 16 + gid + 8 * h, c = wn * (GBN / 2) + j * 8 + 2 * tig;
          double *cp = g.C + (r0 + r) * g.ldc + c0 + c;
          if (whole) {
            *reinterpret_cast<double2 *>(cp) = make_double2(sgn * acc[i][j][2 * h], sgn * acc[i][j][2 * h + 1]);
          } else {
            if (frag_in(r, c)) cp[0] = sgn * acc[i][j][2 * h];
            if (frag_in(r, c + 1)) cp[1] = sgn * acc[i][j][2 * h + 1];
          }
        }
    return;
  }
  __syncthreads();   // the stage ring is free: the epilogue goes through shared memory
  // epilogue: the accumulators are written to shared memory (a 128 x (GBN + 1)-double tile), then the
  // CTA reads and writes C row by row, coalesced, with every load of C in flight together
  // (C = beta C + alpha acc; in the lower mode only entries c <= r)
  double *T = gsm;
  constexpr int TLD = GBN + 1;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int r = wm * 32 + i * 16 + gid + (q >> 1) * 8, c = wn * (GBN / 2) + j * 8 + 2 * tig + (q & 1);
        T[r * TLD + c] = acc[i][j][q];
      }
  __syncthreads();
  // batches of 16 entries per thread: all 16 loads of C are issued before any store (a store to
  // C between loads would otherwise keep the compiler from overlapping their latencies)
  constexpr int BATCH = 16;
  static_assert(GBM * GBN % (GTHREADS * BATCH) == 0, "whole epilogue batches");
#pragma unroll 1
  for (int e0 = tid; e0 < GBM * GBN; e0 += GTHREADS * BATCH) {
    double cv[BATCH];
    bool in[BATCH];
#pragma unroll
    for (int u = 0; u < BATCH; ++u) {
      const int e = e0 + u * GTHREADS, r = e / GBN, c = e % GBN;
      in[u] = r < rows && c < cols && (!g.lower || c0 + c <= r0 + r);
      cv[u] = (in[u] && g.beta != 0.0) ? g.C[(r0 + r) * g.ldc + c0 + c] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < BATCH; ++u) {
      const int e = e0 + u * GTHREADS, r = e / GBN, c = e % GBN;
      if (in[u]) g.C[(r0 + r) * g.ldc + c0 + c] = g.beta * cv[u] + g.alpha * T[r * TLD + c];
    }
  }
}

// Factor the nb x nb diagonal block at (k0, k0) in place (lower) and write inv(L) (row-major,
// nb x nb, zero above the diagonal) to Linv.  One CTA of 256 threads; the block sits in shared
// memory with rows padded to 129 doubles, rows and columns past nb set to the identity (which
// the factorisation leaves alone).  The strict upper triangle of the shared tile collects
// X = inv(L) transposed ([c][i] holds X[i][c]); dinv[c] = 1 / L[c][c].  Four 32-column steps:
//   1. warp 0 factors the 32 x 32 diagonal block D, one row per lane in registers (a column per
//      step: the pivot by shuffle, its reciprocal square root, the column scaled and passed
//      through shared memory, the rank-1 update of the lanes' rows)
//   2. the rows below by forward substitution, one row per thread: L_rD = A_rD L_D^-T
//   3. the trailing lower triangle: A -= L_rD L_cD^T in 4 x 4 register tiles
// then the four diagonal inverses X_II (a warp each, one column per lane) and the off-diagonal
// blocks of X by their distance d = I - J below the diagonal:
//   T = sum_{K = J .. I-1} L_IK X_KJ,   X_IJ = -X_II T   (a column of T per group of lanes).
// err |= 1 on a non-positive or non-finite pivot.
constexpr int PT = 128, PLD = 129, PTHREADS = 256;
// One level of the off-diagonal blocks of X = inv(L) in the shared tile of k_potrf_tile (X[i][c]
// kept at [c][i]), the 4 - D block pairs (J, I = J + D):
//   A. T = sum_{K=J}^{I-1} L_IK X_KJ, a TR x TC register tile per thread (rows i of block I,
//      columns c of block J), written where X_IJ goes ([c][32I + i], which nothing at this level
//      reads); X[k][c] is L[c][k] above c, dinv[c] on it, zero below
//   B. X_IJ = -X_II T, one column c per thread, T's column in registers and X_II[i][m] (at
//      [32I + m][32I + i]) read as a broadcast
template <int D, int TR, int TC>
__device__ inline void inv_level(double *L, const double *dinv) {
  constexpr int TPP = (32 / TR) * (32 / TC), NP = 4 - D;      // tiles per pair, pairs
  static_assert(NP * TPP <= PTHREADS, "one tile per thread");
  const int tid = threadIdx.x;
  if (tid < NP * TPP) {
    const int J = tid / TPP, rem = tid % TPP, I = J + D;
    const int i0 = 32 * I + (rem / (32 / TC)) * TR, c0 = 32 * J + (rem % (32 / TC)) * TC;
    double acc[TR][TC];
#pragma unroll
    for (int u = 0; u < TR; ++u)
#pragma unroll
      for (int v = 0; v < TC; ++v) acc[u][v] = 0.0;
#pragma unroll 4
    for (int k = 32 * J; k < 32 * I; ++k) {
      double lr[TR], xc[TC];
#pragma unroll
      for (int u = 0; u < TR; ++u) lr[u] = L[(i0 + u) * PLD + k];
#pragma unroll
      for (int v = 0; v < TC; ++v) {
        const int c = c0 + v;
        const double up = L[c * PLD + k];
        xc[v] = k > c ? up : (k == c ? dinv[c] : 0.0);
      }
#pragma unroll
      for (int u = 0; u < TR; ++u)
#pragma unroll
        for (int v = 0; v < TC; ++v) acc[u][v] += lr[u] * xc[v];
    }
#pragma unroll
    for (int u = 0; u < TR; ++u)
#pragma unroll
      for (int v = 0; v < TC; ++v) L[(c0 + v) * PLD + i0 + u] = acc[u][v];
  }
  __syncthreads();
  if (tid < NP * 32) {
    const int J = tid >> 5, I = J + D, c = 32 * J + (tid & 31), b = 32 * I;
    double t[32];
#pragma unroll
    for (int m = 0; m < 32; ++m) t[m] = L[c * PLD + b + m];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      double x0 = dinv[b + i] * t[i], x1 = 0.0;
#pragma unroll
      for (int m = 0; m + 1 < i; m += 2) {
        x0 += L[(b + m) * PLD + b + i] * t[m];
        x1 += L[(b + m + 1) * PLD + b + i] * t[m + 1];
      }
      if (i & 1) x0 += L[(b + i - 1) * PLD + b + i] * t[i - 1];
      L[c * PLD + b + i] = -(x0 + x1);
    }
  }
  __syncthreads();
}
constexpr size_t POT_SMEM = sizeof(double) * ((size_t)PT * PLD + PT);   // 130 KB: fits beside a GEMM CTA
__global__ void __launch_bounds__(PTHREADS, 1) k_potrf_tile(double *__restrict__ H, int64_t ldh, int64_t k0, int nb,
                                                           double *__restrict__ Linv, int *err) {
  extern __shared__ double L[];                      // [PT][PLD], then dinv[PT]
  double *dinv = L + PT * PLD;
  __shared__ __align__(16) double colj[32];
  __shared__ int bad;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr unsigned FULL = 0xffffffffu;
  if (tid == 0) bad = 0;
  // the lower triangle (16 loads in flight per thread); the identity past nb; zero above
  constexpr int PER = PT * PT / PTHREADS;
#pragma unroll 1
  for (int u0 = 0; u0 < PER; u0 += 16) {
    double v[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int e = tid + (u0 + u) * PTHREADS, r = e >> 7, c = e & (PT - 1);
      v[u] = (c <= r && r < nb) ? H[(k0 + r) * ldh + k0 + c] : (r == c ? 1.0 : 0.0);
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int e = tid + (u0 + u) * PTHREADS, r = e >> 7, c = e & (PT - 1);
      L[r * PLD + c] = v[u];
    }
  }
  __syncthreads();
  for (int j0 = 0; j0 < PT; j0 += 32) {
    // 1. D = L_D L_D^T with row lane of D in lane's registers (loops unrolled: every register
    //    index is a constant)
    if (warp == 0) {
      double a[32];
      double *row = L + (j0 + lane) * PLD + j0;            // row lane of D
#pragma unroll
      for (int q = 0; q < 32; ++q) a[q] = q <= lane ? row[q] : 0.0;
      bool lbad = false;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        double d = __shfl_sync(FULL, a[j], j);
        if (!(d > 0.0) || !isfinite(d)) {                  // the same d in every lane
          lbad = true;
          d = 1.0;
        }
        const double inv = rsqrt(d), s = d * inv;
        a[j] = lane == j ? s : (lane > j ? a[j] * inv : 0.0);
        if (lane == 0) dinv[j0 + j] = inv;
        const double aj = a[j];
        colj[lane] = aj;                                   // column j of L_D, read back as a broadcast
        __syncwarp();
#pragma unroll
        for (int q = j + 1; q < 32; ++q)
          if (lane >= q) a[q] -= aj * colj[q];             // colj[q] = L[q][j]
        __syncwarp();                                      // colj is rewritten at the next step
      }
#pragma unroll
      for (int q = 0; q < 32; ++q)
        if (q <= lane) row[q] = a[q];                      // L[lane][q]
      if (lbad && lane == 0) bad = 1;
      __syncwarp();
    }
    __syncthreads();
    const int t0 = j0 + 32, nr = PT - t0;
    if (nr == 0) break;
    // 2. rows below by substitution, one row per thread:
    //    L[r][j0 + c] = (A[r][j0 + c] - sum_{k<c} L[r][j0 + k] L[j0 + c][j0 + k]) / L[j0 + c][j0 + c]
    if (tid < nr) {
      const int r = t0 + tid;
      double a[32];
#pragma unroll
      for (int k = 0; k < 32; ++k) a[k] = L[r * PLD + j0 + k];
#pragma unroll
      for (int c = 0; c < 32; ++c) {
        const double l = a[c] * dinv[j0 + c];
        a[c] = l;
#pragma unroll
        for (int q = c + 1; q < 32; ++q) a[q] -= l * L[(j0 + q) * PLD + j0 + c];
      }
#pragma unroll
      for (int k = 0; k < 32; ++k) L[r * PLD + j0 + k] = a[k];
    }
    __syncthreads();
    // 3. trailing lower triangle of rows/columns [t0, PT): 4 x 4 tiles (ti >= tj)
    {
      const int T = nr / 4, ntile = T * (T + 1) / 2;
      for (int t = tid; t < ntile; t += PTHREADS) {
        int ti = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
        while (ti * (ti + 1) / 2 > t) --ti;
        while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
        const int tj = t - ti * (ti + 1) / 2;
        const int r0 = t0 + 4 * ti, c0 = t0 + 4 * tj;
        double acc[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[u][v] = 0.0;
#pragma unroll 8
        for (int q = 0; q < 32; ++q) {
          double lr[4], lc[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            lr[u] = L[(r0 + u) * PLD + j0 + q];
            lc[u] = L[(c0 + u) * PLD + j0 + q];
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] += lr[u] * lc[v];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v)
            if (c0 + v <= r0 + u) L[(r0 + u) * PLD + c0 + v] -= acc[u][v];
      }
    }
    __syncthreads();
  }
  // the four 32 x 32 diagonal inverses X_II, warp I each
  if (warp < 4) {
    const int j0 = 32 * warp;
    double *row = L + (j0 + lane) * PLD + j0;
    // column c = lane of X_D: X[i][c] = (delta_ic - sum_{m<i} L[i][m] X[m][c]) / L[i][i]
    // (X[m][c] = 0 for m < c; two partial sums halve the dependent chain), kept at [c][i]
    double x[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const double *li = L + (j0 + i) * PLD + j0;
      double t0 = i == lane ? 1.0 : 0.0, t1 = 0.0;
#pragma unroll
      for (int m = 0; m + 1 < i; m += 2) {
        t0 -= li[m] * x[m];
        t1 -= li[m + 1] * x[m + 1];
      }
      if (i & 1) t0 -= li[i - 1] * x[i - 1];
      x[i] = i >= lane ? (t0 + t1) * dinv[j0 + i] : 0.0;
    }
#pragma unroll
    for (int i = 0; i < 32; ++i)
      if (i > lane) row[i] = x[i];
  }
  __syncthreads();
  if (bad && tid == 0) atomicOr(err, 1);
  // the off-diagonal blocks of X by distance D = I - J (level D reads only the diagonal inverses
  // and the levels below it)
  inv_level<1, 4, 4>(L, dinv);
  inv_level<2, 4, 2>(L, dinv);
  inv_level<3, 2, 2>(L, dinv);
  // L back to H, inv(L) to Linv
#pragma unroll 16
  for (int u = 0; u < PER; ++u) {
    const int e = tid + u * PTHREADS, r = e >> 7, c = e & (PT - 1);
    if (r < nb && c <= r) H[(k0 + r) * ldh + k0 + c] = L[r * PLD + c];
  }
  if (nb == PT) {
#pragma unroll 16
    for (int u = 0; u < PER; ++u) {
      const int e = tid + u * PTHREADS, i = e >> 7, c = e & (PT - 1);
      Linv[e] = c > i ? 0.0 : (c == i ? dinv[i] : L[c * PLD + i]);
    }
  } else {
    for (int e = tid; e < nb * nb; e += PTHREADS) {
      const int i = e / nb, c = e % nb;
      Linv[e] = c > i ? 0.0 : (c == i ? dinv[i] : L[c * PLD + i]);
    }
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
// its transpose (backward), DRHS right-hand sides per CTA; acc is cleared for the next block.
//   forward:  warp w takes rows 8w .. 8w + 7 of Linv (all 32 of a lane's loads in flight
//             together, coalesced along the rows), then a warp sum per row
//   backward: thread (g, i) reads column i of Linv over rows 32g .. 32g + 31 (coalesced along
//             each row), and the four groups' partial sums meet in shared memory
constexpr int DTHREADS = 512, DRHS = 8;
template <bool TRANS>
__global__ void __launch_bounds__(DTHREADS) k_block_diag(const double *__restrict__ Linv, int nbi, int64_t base,
                                                        double *X, int64_t ldx, double *acc, int nrhs) {
  __shared__ double rhs[CB];
  __shared__ double part[4][CB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r_end = min(nrhs, (int)(blockIdx.x + 1) * DRHS);
  for (int r = blockIdx.x * DRHS; r < r_end; ++r) {
    double *x = X + (int64_t)r * ldx + base;
    __syncthreads();                                 // the previous right-hand side is done with rhs / part
    if (tid < CB) rhs[tid] = tid < nbi ? x[tid] - acc[(int64_t)r * CB + tid] : 0.0;
    __syncthreads();
    if (!TRANS) {
      double s[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const int i = warp * 8 + u;
        double t = 0.0;
#pragma unroll
        for (int q = 0; q < CB / 32; ++q) {
          const int j = lane + 32 * q;
          if (i < nbi && j < nbi) t += Linv[(int64_t)i * nbi + j] * rhs[j];
        }
        s[u] = t;
      }
#pragma unroll
      for (int u = 0; u < 8; ++u)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s[u] += __shfl_xor_sync(0xffffffffu, s[u], off);
      if (lane < 8) {
        double v = s[0];
#pragma unroll
        for (int u = 1; u < 8; ++u) v = lane == u ? s[u] : v;
        const int i = warp * 8 + lane;
        if (i < nbi) x[i] = v;
      }
    } else {
      const int i = tid & (CB - 1), g = tid / CB;
      double t = 0.0;
      if (i < nbi) {
#pragma unroll 8
        for (int jj = 0; jj < 32; ++jj) {
          const int j = 32 * g + jj;
          if (j < nbi) t += Linv[(int64_t)j * nbi + i] * rhs[j];
        }
      }
      part[g][i] = t;
      __syncthreads();
      if (tid < nbi) x[tid] = part[0][tid] + part[1][tid] + part[2][tid] + part[3][tid];
    }
    if (tid < nbi) acc[(int64_t)r * CB + tid] = 0.0;
  }
}

// ---------------------------------------------------------------- chained solves (one right-hand side)
// One cooperative launch per direction (every CTA resident at once): CTA b owns the 128-row
// block b of the solution and publishes it through flags[b] (release) once it is final; a CTA
// that needs block c waits for flags[c] (acquire; bounded: a wait that gives up sets err bit 2
// and goes on, so every CTA ends).
//   forward  (L y = b):   CTA b = blockIdx adds L_bc y_c for c = 0 .. b-1 as the flags come, then
//                         y_b = inv(L_bb) (b_b - sum)
//   backward (L^T x = y): CTA b = nblk-1-blockIdx adds L_cb^T x_c for c = nblk-1 .. b+1, then
//                         x_b = inv(L_bb)^T (y_b - sum)
// A 128 x 128 block M is read by rows: warp w takes rows 16w .. 16w + 15, lane l columns
// 4l .. 4l + 3 (each row one coalesced 1 KB read).  Forward sums over the lanes (a transpose
// through shared memory), backward over the warps.
constexpr int TS_THREADS = 256, TS_RLD = 33;
constexpr uint32_t TS_SPIN = 1u << 18;   // polls (~0.3 s) per wait; the whole chain takes about a millisecond

__device__ inline uint32_t ld_acquire_gpu(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ inline void st_release_gpu(uint32_t *p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// bounded wait for a published block; false when it gave up
__device__ inline bool wait_block(const uint32_t *f) {
  for (uint32_t it = 0; it < TS_SPIN; ++it) {
    if (ld_acquire_gpu(f)) return true;
    if (it > 64) __nanosleep(64);
  }
  return false;
}

// m <- entries col .. col + 3 of a row (p points at col), zero from ncol on; 16-byte loads when vec
// (p 16-byte aligned) and the four are inside
__device__ inline void ts_load4(const double *p, int col, int ncol, bool vec, double (&m)[4]) {
  if (vec && col + 3 < ncol) {
    const double2 a = __ldg(reinterpret_cast<const double2 *>(p)), b = __ldg(reinterpret_cast<const double2 *>(p + 2));
    m[0] = a.x;
    m[1] = a.y;
    m[2] = b.x;
    m[3] = b.y;
  } else {
#pragma unroll
    for (int e = 0; e < 4; ++e) m[e] = col + e < ncol ? __ldg(p + e) : 0.0;
  }
}

// Rows 16w .. 16w + 15 (below nrow) of M (row stride ld, ncol columns) times the lane's four
// entries of v:  forward  part[r] += sum_e M[16w + r][4l + e] v[4l + e]   (v4 = those four)
//                backward part[e] += sum_r M[16w + r][4l + e] v[16w + r]  (v16 = those sixteen)
template <bool TRANS>
__device__ inline void ts_block(const double *M, int64_t ld, int nrow, int ncol, bool vec, const double (&v4)[4],
                                const double (&v16)[16], double (&part)[16]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double *p0 = M + (int64_t)(16 * warp) * ld + 4 * lane;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    double m[8][4];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      if (16 * warp + 8 * h + r < nrow) {
        ts_load4(p0 + (int64_t)(8 * h + r) * ld, 4 * lane, ncol, vec, m[r]);
      } else {
#pragma unroll
        for (int e = 0; e < 4; ++e) m[r][e] = 0.0;
      }
    }
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        if (TRANS)
          part[e] += m[r][e] * v16[8 * h + r];
        else
          part[8 * h + r] += m[r][e] * v4[e];
      }
  }
}

// out[i] for i < 128 of the CTA's block: the per-thread partials summed over lanes (forward) or
// warps (backward); red is the shared scratch, valid for threads < 128 after the call
template <bool TRANS>
__device__ inline double ts_reduce(double *red, const double (&part)[16]) {
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  __syncthreads();                                   // red is free
  if (TRANS) {
#pragma unroll
    for (int e = 0; e < 4; ++e) red[warp * CB + 4 * lane + e] = part[e];
  } else {
#pragma unroll
    for (int r = 0; r < 16; ++r) red[(16 * warp + r) * TS_RLD + lane] = part[r];
  }
  __syncthreads();
  double s = 0.0;
  if (tid < CB) {
    if (TRANS) {
#pragma unroll
      for (int w = 0; w < TS_THREADS / 32; ++w) s += red[w * CB + tid];
    } else {
#pragma unroll 8
      for (int k = 0; k < 32; ++k) s += red[tid * TS_RLD + k];
    }
  }
  return s;
}

template <bool TRANS>
__global__ void __launch_bounds__(TS_THREADS, 2) k_trsv_chain(const double *__restrict__ H, int64_t ldh, int64_t n,
                                                             int nblk, const double *__restrict__ Linv, double *x,
                                                             uint32_t *flags, int *err, int vech) {
  __shared__ double red[CB * TS_RLD];
  __shared__ double rhs[CB];
  __shared__ int s_ready[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int b = TRANS ? nblk - 1 - (int)blockIdx.x : (int)blockIdx.x;
  const int64_t base = (int64_t)b * CB;
  const int nbi = (int)min((int64_t)CB, n - base);
  // forward: blocks [0, ready) are known final; backward: blocks [ready, nblk).  Every thread holds
  // the same value: thread 0 polls, writes slot (k & 1) before the k-th barrier, and each thread
  // reads that slot right after it; the slot is written again only after barrier k + 1, which
  // every thread reaches after its read.
  int ready = TRANS ? nblk : 0, nsync = 0;
  bool gave_up = false;
  double part[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) part[r] = 0.0;
  const int steps = TRANS ? nblk - 1 - b : b;
  for (int st = 0; st < steps; ++st) {
    const int c = TRANS ? nblk - 1 - st : st;
    if (TRANS ? c < ready : c >= ready) {
      if (tid == 0) {
        if (!wait_block(flags + c)) gave_up = true;
        int r = c;                                   // and every later block already published
        if (TRANS) {
          while (r - 1 > b && ld_acquire_gpu(flags + r - 1)) --r;
        } else {
          ++r;
          while (r < b && ld_acquire_gpu(flags + r)) ++r;
        }
        s_ready[nsync & 1] = r;
      }
      __syncthreads();
      ready = s_ready[nsync & 1];
      ++nsync;
    }
    const int64_t cb = (int64_t)c * CB;
    double v4[4], v16[16];
    if (TRANS) {
      const int nbc = (int)min((int64_t)CB, n - cb);
#pragma unroll
      for (int r = 0; r < 16; ++r) v16[r] = 16 * warp + r < nbc ? __ldcg(x + cb + 16 * warp + r) : 0.0;
      ts_block<true>(H + cb * ldh + base, ldh, nbc, CB, vech, v4, v16, part);
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) v4[e] = __ldcg(x + cb + 4 * lane + e);
      ts_block<false>(H + base * ldh + cb, ldh, nbi, CB, vech, v4, v16, part);
    }
  }
  // the block's right-hand side, then the product with inv(L_bb) (forward) or its transpose
  const double s = ts_reduce<TRANS>(red, part);
  if (tid < CB) rhs[tid] = tid < nbi ? x[base + tid] - s : 0.0;
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 16; ++r) part[r] = 0.0;
  {
    const double *Lb = Linv + base * CB;             // nbi x nbi, row-major
    const bool vl = nbi % 2 == 0;
    double v4[4], v16[16];
    if (TRANS) {
#pragma unroll
      for (int r = 0; r < 16; ++r) v16[r] = rhs[16 * warp + r];
    } else {
#pragma unroll
      for (int e = 0; e < 4; ++e) v4[e] = rhs[4 * lane + e];
    }
    ts_block<TRANS>(Lb, nbi, nbi, nbi, vl, v4, v16, part);
  }
  const double y = ts_reduce<TRANS>(red, part);
  if (tid < nbi) {
    x[base + tid] = y;
    __threadfence();
  }
  __syncthreads();
  if (tid == 0) {
    st_release_gpu(flags + b, 1u);
    if (gave_up) atomicOr(err, 2);
  }
}

// Both solves as two cooperative launches when every CTA fits on the GPU at once; false (nothing
// launched) when they do not, and the caller takes the per-block launches
bool trsv_chain(const double *H, int64_t ldh, int64_t n, const double *Linv, double *x, uint32_t *flags, int *err,
                cudaStream_t st, int *rc) {
  *rc = DGP_OK;
  const int nblk = (int)ceil_div(n, (int64_t)CB);
  int dev = 0, coop = 0, per_sm_f = 0, per_sm_b = 0;
  // a query that fails leaves the per-block path; its error is cleared so that the next launch
  // check does not report it
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_f, k_trsv_chain<false>, TS_THREADS, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_b, k_trsv_chain<true>, TS_THREADS, 0) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  if (!coop) return false;
  if ((int64_t)std::min(per_sm_f, per_sm_b) * sm_count() < nblk) return false;
  int vech = ((uintptr_t)H % 16 == 0) && ldh % 2 == 0;
  uint32_t *ff = flags, *fb = flags + nblk;
  void *af[] = {(void *)&H, (void *)&ldh, (void *)&n, (void *)&nblk, (void *)&Linv, (void *)&x, (void *)&ff,
                (void *)&err, (void *)&vech};
  void *ab[] = {(void *)&H, (void *)&ldh, (void *)&n, (void *)&nblk, (void *)&Linv, (void *)&x, (void *)&fb,
                (void *)&err, (void *)&vech};
  cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_trsv_chain<false>, dim3(nblk), dim3(TS_THREADS), af, 0, st);
  if (e == cudaSuccess)
    e = cudaLaunchCooperativeKernel((const void *)k_trsv_chain<true>, dim3(nblk), dim3(TS_THREADS), ab, 0, st);
  if (e != cudaSuccess) *rc = fail(DGP_ERR_CUDA, std::string("cholesky: chained solve launch: ") + cudaGetErrorString(e));
  return true;
}

template <int V, int GBN, bool REG>
int gemm_launch(Gemm g, cudaStream_t st) {
  constexpr int smem = gemm_smem(GBN);
  const int64_t tm = ceil_div(g.M, (int64_t)GBM), tn = ceil_div(g.N, (int64_t)GBN);
  g.tn = tn;
  g.cvec = ((uintptr_t)g.C % 16 == 0) && g.ldc % 2 == 0;
  // lower mode (M == N, GBN = 64): row ti of tiles holds tj = 0 .. 2 ti + 1; a tile past N (the
  // last one of a row when N is not a multiple of 128) writes nothing
  const int64_t tiles = g.lower ? tm * (tm + 1) : tm * tn;
  DGP_REQUIRE(tiles <= INT32_MAX, "cholesky: too many tiles");
  DGP_CUDA(cudaFuncSetAttribute(k_dgemm_nt<V, GBN, REG>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k_dgemm_nt<V, GBN, REG><<<(unsigned)tiles, GTHREADS, smem, st>>>(g);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

// C = beta C + alpha A B^T; 128-column tiles when C is A (in place), else 64-column tiles, with
// the accumulators started from C when beta = 1 and alpha = +-1 (every update of the factorisation)
int gemm_nt(const Gemm &g, cudaStream_t st) {
  if (g.M <= 0 || g.N <= 0) return DGP_OK;
  const bool a16 = ((uintptr_t)g.A % 16 == 0) && ((uintptr_t)g.B % 16 == 0) && g.lda % 2 == 0 && g.ldb % 2 == 0 &&
                   g.K % 2 == 0;
  const bool inplace = g.C == g.A;
  if (inplace) DGP_REQUIRE(!g.lower && g.N <= GBM, "cholesky: an in-place product must fit one 128-column tile");
  if (inplace) return a16 ? gemm_launch<16, 128, false>(g, st) : gemm_launch<8, 128, false>(g, st);
  const bool reg = g.beta == 1.0 && (g.alpha == 1.0 || g.alpha == -1.0);
  if (reg) return a16 ? gemm_launch<16, 64, true>(g, st) : gemm_launch<8, 64, true>(g, st);
  return a16 ? gemm_launch<16, 64, false>(g, st) : gemm_launch<8, 64, false>(g, st);
}

// The four streams and eight events of the lookahead; the destructor waits for every stream, so
// that an early error return never frees buffers that queued kernels still use.
struct LookaheadStreams {
  cudaStream_t f = nullptr, s = nullptr, b = nullptr, r = nullptr;
  cudaEvent_t fork = nullptr, panel = nullptr, rest = nullptr, join = nullptr, step = nullptr, side = nullptr,
              diag = nullptr, below = nullptr;
  int create() {
    int lo = 0, hi = 0;
    DGP_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    DGP_CUDA(cudaStreamCreateWithPriority(&f, cudaStreamNonBlocking, hi));
    DGP_CUDA(cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking, hi));
    DGP_CUDA(cudaStreamCreateWithPriority(&b, cudaStreamNonBlocking, hi));
    DGP_CUDA(cudaStreamCreateWithPriority(&r, cudaStreamNonBlocking, lo));
    for (cudaEvent_t *e : {&fork, &panel, &rest, &join, &step, &side, &diag, &below})
      DGP_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return DGP_OK;
  }
  ~LookaheadStreams() {
    for (cudaStream_t q : {f, s, b, r})
      if (q) cudaStreamSynchronize(q);
    for (cudaEvent_t e : {fork, panel, rest, join, step, side, diag, below})
      if (e) cudaEventDestroy(e);
    for (cudaStream_t q : {f, s, b, r})
      if (q) cudaStreamDestroy(q);
  }
};

}  // namespace

int cholesky_solve_many_run(double *H, int64_t n, int64_t ldh, double *x, int32_t nrhs, int64_t ldx,
                            cudaStream_t st) {
  DGP_REQUIRE(H && x && n > 0 && ldh >= n, "cholesky: bad arguments");
  DGP_REQUIRE(nrhs >= 1 && ldx >= n, "cholesky: need nrhs >= 1 and ldx >= n");
  DGP_REQUIRE(nrhs <= 65535, "cholesky: at most 65535 right-hand sides");
  DGP_REQUIRE(ceil_div(n, (int64_t)GVB) <= INT32_MAX, "cholesky: n too large for the solve grid");
  const int64_t nblk = ceil_div(n, CB);
  DevBuf linv, errb, acc, flags;
  DGP_TRY(linv.alloc(sizeof(double) * (size_t)nblk * CB * CB));
  DGP_TRY(errb.alloc(sizeof(int)));
  DGP_TRY(acc.alloc(sizeof(double) * (size_t)CB * nrhs));
  DGP_TRY(flags.alloc(sizeof(uint32_t) * 2 * (size_t)nblk));
  DGP_CUDA(cudaMemsetAsync(errb.p, 0, sizeof(int), st));
  DGP_CUDA(cudaMemsetAsync(flags.p, 0, sizeof(uint32_t) * 2 * (size_t)nblk, st));
  DGP_CUDA(cudaMemsetAsync(acc.p, 0, sizeof(double) * (size_t)CB * nrhs, st));
  const size_t pot_smem = POT_SMEM;
  DGP_CUDA(cudaFuncSetAttribute(k_potrf_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pot_smem));
  double *Li = linv.as<double>();
  int64_t launches = 0;
  // Lookahead on four streams forked from st: sf (high priority) factors the outer panels and
  // gives the next outer panel its update; ss and sb (high priority) take the off-chain parts of
  // each panel's work; sr (low priority) updates the rest of the matrix.
  // Outer panel p = columns [o0, oend), next panel [oend, nend):
  //   sf:  F_p   the 128-column steps of panel p on the panel's own rows: the diagonal block,
  //              the rows below it, then the next step's diagonal block (update, factorisation)
  //   ss:        beside that, the step's update of the panel's other remaining columns, which sf
  //              waits for before the next step's rows
  //   sb:        the rows under the panel, left-looking per 128-column block (the update by the
  //              panel's earlier columns, then the product with the block's inverse), off the step
  //              chain; sf waits for them at the end of the panel
  //   sf:  N_p   rows [oend, n) x columns [oend, nend) -= Q Q_next^T, Q = panel p's rows  (after
  //              R_{p-1}, which updates the same entries)
  //   sr:  R_p   the lower triangle of [nend, n)^2 -= Q Q^T  (after F_p)
  // so F_{p+1} runs while R_p does, and the trailing GEMMs keep the outer panel width as depth.
  LookaheadStreams ls;
  DGP_TRY(ls.create());
  DGP_CUDA(cudaEventRecord(ls.fork, st));
  DGP_CUDA(cudaStreamWaitEvent(ls.f, ls.fork, 0));
  DGP_CUDA(cudaStreamWaitEvent(ls.s, ls.fork, 0));
  DGP_CUDA(cudaStreamWaitEvent(ls.b, ls.fork, 0));
  DGP_CUDA(cudaStreamWaitEvent(ls.r, ls.fork, 0));
  cudaStream_t sf = ls.f, ss = ls.s, sb = ls.b, sr = ls.r;
  bool r_recorded = false;
  bool side_pending = false;   // a step's off-chain updates queued on ss that sf has not waited for
  for (int64_t o0 = 0; o0 < n; o0 += NBO) {
    const int64_t oend = std::min(n, o0 + NBO);
    const bool below = n > oend;  // rows under the outer panel: left-looking on sb, off the step chain
    bool last = false;
    for (int64_t k0 = o0; k0 < oend; k0 += CB) {
      const int64_t b = k0 / CB;
      const int nb = (int)std::min<int64_t>(CB, n - k0);
      double *Lb = Li + b * CB * CB;
      if (k0 == o0) {  // a later step's diagonal block was started by the step before it
        k_potrf_tile<<<1, PTHREADS, pot_smem, sf>>>(H, ldh, k0, nb, Lb, errb.as<int>());
        DGP_CHECK_LAUNCH();
        ++launches;
      }
      if (below) {
        // rows [oend, n) of column block k: minus the panel's earlier columns (depth k0 - o0), then
        // L = A inv(L_kk)^T in place; after this step's diagonal block and the rows of block k in
        // the earlier columns (both on sf before this point)
        DGP_CUDA(cudaEventRecord(ls.diag, sf));
        DGP_CUDA(cudaStreamWaitEvent(sb, ls.diag, 0));
        if (k0 > o0) {
          const Gemm u{H + oend * ldh + o0, ldh, H + k0 * ldh + o0, ldh, H + oend * ldh + k0, ldh, n - oend, nb,
                       k0 - o0, -1.0, 1.0, 0, 0};
          DGP_TRY(gemm_nt(u, sb));
          ++launches;
        }
        const Gemm pb{H + oend * ldh + k0, ldh, Lb, nb, H + oend * ldh + k0, ldh, n - oend, nb, nb, 1.0, 0.0, 0, 0};
        DGP_TRY(gemm_nt(pb, sb));
        ++launches;
      }
      const int64_t kend = k0 + nb, rest = n - kend;
      if (rest <= 0) {
        last = true;
        break;
      }
      const int64_t w = oend - kend;  // the outer panel's remaining columns (and rows)
      if (w == 0) continue;
      if (side_pending) {  // those rows carry the previous step's off-chain updates
        DGP_CUDA(cudaStreamWaitEvent(sf, ls.side, 0));
        side_pending = false;
      }
      // L_ik = A_ik inv(L_kk)^T for the outer panel's rows below the block (in place, one CTA per
      // 128-row strip)
      const Gemm p{H + kend * ldh + k0, ldh, Lb, nb, H + kend * ldh + k0, ldh, w, nb, nb, 1.0, 0.0, 0, 0};
      DGP_TRY(gemm_nt(p, sf));
      ++launches;
      // the next diagonal block's update, then its factorisation at once on sf; the rest of the
      // step's update of the outer panel's remaining columns on ss beside it
      const int nb2 = (int)std::min<int64_t>(CB, w);
      const int64_t k2 = kend + nb2, w2 = oend - k2;
      DGP_CUDA(cudaEventRecord(ls.step, sf));
      const Gemm a1{H + kend * ldh + k0, ldh, H + kend * ldh + k0, ldh, H + kend * ldh + kend, ldh, nb2, nb2, nb,
                    -1.0, 1.0, 1, 0};
      DGP_TRY(gemm_nt(a1, sf));
      k_potrf_tile<<<1, PTHREADS, pot_smem, sf>>>(H, ldh, kend, nb2, Li + (b + 1) * CB * CB, errb.as<int>());
      DGP_CHECK_LAUNCH();
      launches += 2;
      if (w2 > 0) {
        DGP_CUDA(cudaStreamWaitEvent(ss, ls.step, 0));
        const Gemm a2{H + k2 * ldh + k0, ldh, H + kend * ldh + k0, ldh, H + k2 * ldh + kend, ldh, w2, nb2, nb,
                      -1.0, 1.0, 0, 0};
        const Gemm a3{H + k2 * ldh + k0, ldh, H + k2 * ldh + k0, ldh, H + k2 * ldh + k2, ldh, w2, w2, nb,
                      -1.0, 1.0, 1, 0};
        DGP_TRY(gemm_nt(a2, ss));
        DGP_TRY(gemm_nt(a3, ss));
        launches += 2;
        DGP_CUDA(cudaEventRecord(ls.side, ss));
        side_pending = true;
      }
    }
    if (below) {  // the outer panel's rows below it are final before its updates of the rest
      DGP_CUDA(cudaEventRecord(ls.below, sb));
      DGP_CUDA(cudaStreamWaitEvent(sf, ls.below, 0));
    }
    if (last || n <= oend) break;
    const int64_t nend = std::min(n, oend + NBO), depth = oend - o0;
    DGP_CUDA(cudaEventRecord(ls.panel, sf));
    // N_p: the next panel's lower square, then the rows below it
    if (r_recorded) DGP_CUDA(cudaStreamWaitEvent(sf, ls.rest, 0));
    const Gemm nq{H + oend * ldh + o0, ldh, H + oend * ldh + o0, ldh, H + oend * ldh + oend, ldh, nend - oend,
                  nend - oend, depth, -1.0, 1.0, 1, 0};
    DGP_TRY(gemm_nt(nq, sf));
    ++launches;
    if (n > nend) {
      const Gemm nr{H + nend * ldh + o0, ldh, H + oend * ldh + o0, ldh, H + nend * ldh + oend, ldh, n - nend,
                    nend - oend, depth, -1.0, 1.0, 0, 0};
      DGP_TRY(gemm_nt(nr, sf));
      // R_p: the lower triangle past the next panel
      DGP_CUDA(cudaStreamWaitEvent(sr, ls.panel, 0));
      const Gemm t{H + nend * ldh + o0, ldh, H + nend * ldh + o0, ldh, H + nend * ldh + nend, ldh, n - nend,
                   n - nend, depth, -1.0, 1.0, 1, 0};
      DGP_TRY(gemm_nt(t, sr));
      DGP_CUDA(cudaEventRecord(ls.rest, sr));
      r_recorded = true;
      launches += 2;
    }
  }
  if (r_recorded) DGP_CUDA(cudaStreamWaitEvent(sf, ls.rest, 0));
  if (side_pending) DGP_CUDA(cudaStreamWaitEvent(sf, ls.side, 0));
  // L y = b, then L^T x = y: one right-hand side as two chained launches where every CTA fits on
  // the GPU at once, else (and for several right-hand sides) by 128-row blocks
  int crc = DGP_OK;
  const bool chained = nrhs == 1 && trsv_chain(H, ldh, n, Li, x, flags.as<uint32_t>(), errb.as<int>(), sf, &crc);
  if (crc) return crc;
  if (chained) launches += 2;
  const unsigned dgrid = (unsigned)ceil_div((int64_t)nrhs, (int64_t)DRHS);
  for (int64_t b = 0; b < nblk && !chained; ++b) {
    const int64_t k0 = b * CB;
    const int nb = (int)std::min<int64_t>(CB, n - k0);
    if (k0 > 0) {
      dim3 gr((unsigned)ceil_div(k0, GV), (unsigned)ceil_div(nb, 8), (unsigned)nrhs);
      k_block_gemv<false><<<gr, 256, 0, sf>>>(H, ldh, k0, nb, 0, k0, x, ldx, acc.as<double>());
      ++launches;
    }
    k_block_diag<false><<<dgrid, DTHREADS, 0, sf>>>(Li + b * CB * CB, nb, k0, x, ldx, acc.as<double>(),
                                                          nrhs);
    ++launches;
  }
  for (int64_t b = nblk - 1; b >= 0 && !chained; --b) {
    const int64_t k0 = b * CB;
    const int nb = (int)std::min<int64_t>(CB, n - k0);
    const int64_t kend = k0 + nb;
    if (kend < n) {
      dim3 gr((unsigned)ceil_div(n - kend, GVB), 1, (unsigned)nrhs);
      k_block_gemv<true><<<gr, 128, 0, sf>>>(H, ldh, k0, nb, kend, n, x, ldx, acc.as<double>());
      ++launches;
    }
    k_block_diag<true><<<dgrid, DTHREADS, 0, sf>>>(Li + b * CB * CB, nb, k0, x, ldx, acc.as<double>(),
                                                         nrhs);
    ++launches;
  }
  DGP_CUDA(cudaEventRecord(ls.join, sf));
  DGP_CUDA(cudaStreamWaitEvent(st, ls.join, 0));
  DGP_CHECK_LAUNCH();
  count_launches(launches);
  int herr = 0;
  DGP_CUDA(cudaMemcpyAsync(&herr, errb.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  if (herr & 1) return fail(DGP_ERR_ARG, "cholesky: matrix is not positive definite");
  if (herr & 2) return fail(DGP_ERR_CUDA, "cholesky: a wait of the chained solve gave up");
  return DGP_OK;
}

int cholesky_solve_run(double *H, int64_t n, int64_t ldh, double *x, cudaStream_t st) {
  return cholesky_solve_many_run(H, n, ldh, x, 1, n, st);
}

}  // namespace dgp
