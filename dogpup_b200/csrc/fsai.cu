// FSAI (factorised sparse approximate inverse) setup on the device.
//
// Pattern: the rule of FSAIP_gen (DOGPUP/dMesh.m:1361-1380) restated per row.
// The reference sorts all entries of tril(A) by (row desc, |a| desc) and keeps,
// for every row-group start s, the positions s-29..s.  Within one row of n
// entries ranked by |a| descending (ties by ascending column, MATLAB's stable
// sort of find() order) that keeps rank 0 and every rank >= n-29: all
// entries when n <= 30, otherwise the largest plus the 29 smallest.
//
// Factor: for row i with pattern P_i (m entries, diagonal last) and harmonic
// k, S = Re A[P_i,P_i] + i*k*Im A[P_i,P_i], y = S^-1 e_m by Gaussian
// elimination with partial pivoting, g_i = y / sqrt(y_m) with the principal
// square root (the arithmetic of FSAIP_CUDA.cu:92-160).  One thread per
// (row, harmonic); the row's real sub-blocks are gathered once per block into
// shared memory and reused by every harmonic of the block, instead of one
// 40.8 KB local-memory matrix and a linear search of A per thread.
#include <cub/cub.cuh>

#include "dgp_common.cuh"
#include "dgp_internal.h"

namespace dgp {

namespace {

inline unsigned grid1(int64_t n, int bs) { return (unsigned)ceil_div(n, bs); }

// number of tril entries of row i: columns <= i form a prefix of the sorted row
__device__ inline int tril_len(const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col, int64_t i) {
  int b = rowptr[i], e = rowptr[i + 1];
  int c = 0;
  for (int p = b; p < e; ++p) c += col[p] <= i;
  return c;
}

__global__ void k_pattern_count(const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col, int64_t n,
                                int cap, int32_t *cnt, int *bad) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int t = tril_len(rowptr, col, i);
  if (t == 0 || col[rowptr[i] + t - 1] != i) atomicOr(bad, 1);  // diagonal must be present
  cnt[i] = t <= cap ? t : cap;
}

__global__ void k_pattern_fill(const int32_t *__restrict__ rowptr, const int32_t *__restrict__ col,
                               const double *__restrict__ K, const double *__restrict__ M, double dfc,
                               int64_t n, int cap, const int32_t *__restrict__ rowptrG, int32_t *colG) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int b = rowptr[i];
  int t = tril_len(rowptr, col, i);
  int o = rowptrG[i];
  if (t <= cap) {
    for (int p = 0; p < t; ++p) colG[o + p] = col[b + p];
    return;
  }
  // rank by |K + i*dfc*M| descending, ties by column ascending; keep rank 0
  // and ranks >= t - (cap - 1); emit in ascending column order
  int q = 0;
  for (int p = 0; p < t; ++p) {
    double ap = hypot(K[b + p], dfc * M[b + p]);
    int rank = 0;
    for (int u = 0; u < t; ++u) {
      double au = hypot(K[b + u], dfc * M[b + u]);
      rank += (au > ap) || (au == ap && u < p);
    }
    if (rank == 0 || rank >= t - (cap - 1)) colG[o + (q++)] = col[b + p];
  }
}

// Gaussian elimination with partial pivoting on S y = e_m (S complex,
// m x m, held in a local array), then y / sqrt(y_m).
template <int MMAX>
__global__ void __launch_bounds__(128) k_fsai_factor(const int32_t *__restrict__ rowptr,
                                                     const int32_t *__restrict__ col,
                                                     const double *__restrict__ Are,
                                                     const double *__restrict__ Aim, int64_t n,
                                                     const int32_t *__restrict__ rowptrG,
                                                     const int32_t *__restrict__ colG, int nf,
                                                     double2 *__restrict__ out, int64_t s_slot, int64_t s_k,
                                                     const int32_t *__restrict__ harm) {
  constexpr int RB = 4, KT = 32;
  extern __shared__ double sh[];  // [RB][2][MMAX][MMAX]
  const int tr = threadIdx.x / KT, tk = threadIdx.x % KT;
  const int64_t row0 = (int64_t)blockIdx.x * RB;
  // cooperative gather of the RB rows' real sub-blocks (symmetric fill)
  for (int r = 0; r < RB; ++r) {
    int64_t i = row0 + r;
    if (i >= n) break;
    int gb = rowptrG[i], m = rowptrG[i + 1] - gb;
    double *s0 = sh + (size_t)r * 2 * MMAX * MMAX;
    double *s1 = s0 + MMAX * MMAX;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      int a = e / m, c = e % m;
      if (c > a) continue;
      int ra = colG[gb + a], cc = colG[gb + c];  // ra >= cc: entry of tril(A) row ra
      double vr = 0.0, vi = 0.0;
      int pb = rowptr[ra], pe = rowptr[ra + 1];
      // binary search for column cc in row ra
      int lo = pb, hi = pe;
      while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (col[mid] < cc) lo = mid + 1; else hi = mid;
      }
      if (lo < pe && col[lo] == cc) { vr = Are[lo]; vi = Aim[lo]; }
      s0[a * MMAX + c] = vr; s0[c * MMAX + a] = vr;
      s1[a * MMAX + c] = vi; s1[c * MMAX + a] = vi;
    }
  }
  __syncthreads();
  const int64_t i = row0 + tr;
  const int k = blockIdx.y * KT + tk;
  if (i >= n || k >= nf) return;
  const int gb = rowptrG[i], m = rowptrG[i + 1] - gb;
  const double *s0 = sh + (size_t)tr * 2 * MMAX * MMAX;
  const double *s1 = s0 + MMAX * MMAX;
  const double kk = (double)(harm ? harm[k] : k);
  double2 a[MMAX][MMAX];
  double2 y[MMAX];
  for (int r = 0; r < m; ++r) {
    for (int c = 0; c < m; ++c) a[r][c] = make_double2(s0[r * MMAX + c], kk * s1[r * MMAX + c]);
    y[r] = make_double2(r == m - 1 ? 1.0 : 0.0, 0.0);
  }
  // forward elimination with row pivoting on the column maximum
  for (int c = 0; c < m; ++c) {
    int piv = c;
    double best = cabs2(a[c][c]);
    for (int r = c + 1; r < m; ++r) {
      double v = cabs2(a[r][c]);
      if (v > best) { best = v; piv = r; }
    }
    if (piv != c) {
      for (int q = c; q < m; ++q) { double2 t = a[c][q]; a[c][q] = a[piv][q]; a[piv][q] = t; }
      double2 t = y[c]; y[c] = y[piv]; y[piv] = t;
    }
    for (int r = c + 1; r < m; ++r) {
      double2 f = cdiv(a[r][c], a[c][c]);
      for (int q = c; q < m; ++q) a[r][q] = csub(a[r][q], cmul(f, a[c][q]));
      y[r] = csub(y[r], cmul(f, y[c]));
    }
  }
  // back substitution
  for (int r = m - 1; r >= 0; --r) {
    double2 acc = y[r];
    for (int q = r + 1; q < m; ++q) acc = csub(acc, cmul(a[r][q], y[q]));
    y[r] = cdiv(acc, a[r][r]);
  }
  double2 sq = csqrt_ref(y[m - 1].x, y[m - 1].y);
  for (int r = 0; r < m; ++r) out[(int64_t)(gb + r) * s_slot + (int64_t)k * s_k] = cdiv(y[r], sq);
}

__global__ void k_transpose_keys(const int32_t *__restrict__ rowptrG, const int32_t *__restrict__ colG, int64_t n,
                                 uint64_t *keys, int32_t *slot) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int p = rowptrG[i]; p < rowptrG[i + 1]; ++p) {
    keys[p] = ((uint64_t)(uint32_t)colG[p] << 32) | (uint32_t)i;
    slot[p] = p;
  }
}

__global__ void k_transpose_fill(const uint64_t *__restrict__ keys, int64_t nnz, int64_t n, int32_t *rowptrT,
                                 int32_t *colT) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= nnz) return;
  int32_t r = (int32_t)(keys[p] >> 32);
  colT[p] = (int32_t)(keys[p] & 0xffffffffu);
  int32_t rprev = p == 0 ? -1 : (int32_t)(keys[p - 1] >> 32);
  for (int32_t rr = rprev + 1; rr <= r; ++rr) rowptrT[rr] = (int32_t)p;
  if (p == nnz - 1)
    for (int64_t rr = r + 1; rr <= n; ++rr) rowptrT[rr] = (int32_t)nnz;
}

__global__ void k_scale(const double *__restrict__ a, double f, int64_t n, double *out) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p < n) out[p] = f * a[p];
}

__global__ void k_max_row(const int32_t *__restrict__ rowptr, int64_t n, int *mmax) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  atomicMax(mmax, rowptr[i + 1] - rowptr[i]);
}

}  // namespace

int fsai_pattern_rows(const int32_t *d_rowptr, const int32_t *d_col, const double *d_K, const double *d_M,
                      double dfc, int64_t n, int32_t cap, int32_t *d_rowptrG, int32_t *d_colG, int32_t *h_nnzG,
                      int32_t *h_mmax, cudaStream_t st) {
  DGP_REQUIRE(n > 0 && cap >= 1 && cap <= 32, "fsai pattern: need n > 0 and 1 <= cap <= 32");
  const int bs = 256;
  DevBuf cnt, flag, tmp;
  DGP_TRY(cnt.alloc(sizeof(int32_t) * (n + 1)));
  DGP_TRY(flag.alloc(2 * sizeof(int)));
  DGP_CUDA(cudaMemsetAsync(flag.p, 0, 2 * sizeof(int), st));
  DGP_CUDA(cudaMemsetAsync(cnt.p, 0, sizeof(int32_t) * (n + 1), st));
  k_pattern_count<<<grid1(n, bs), bs, 0, st>>>(d_rowptr, d_col, n, cap, cnt.as<int32_t>(), flag.as<int>());
  DGP_CHECK_LAUNCH();
  size_t tb = 0;
  DGP_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<int32_t>(), d_rowptrG, (int)(n + 1), st));
  DGP_TRY(tmp.alloc(tb));
  DGP_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt.as<int32_t>(), d_rowptrG, (int)(n + 1), st));
  k_max_row<<<grid1(n, bs), bs, 0, st>>>(d_rowptrG, n, flag.as<int>() + 1);
  DGP_CHECK_LAUNCH();
  int hf[2] = {0, 0};
  int32_t nnzG = 0;
  DGP_CUDA(cudaMemcpyAsync(hf, flag.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaMemcpyAsync(&nnzG, d_rowptrG + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  if (hf[0]) return fail(DGP_ERR_MESH, "fsai pattern: a row of A has no diagonal entry");
  if (h_nnzG) *h_nnzG = nnzG;
  if (h_mmax) *h_mmax = hf[1];
  if (d_colG) {
    k_pattern_fill<<<grid1(n, bs), bs, 0, st>>>(d_rowptr, d_col, d_K, d_M, dfc, n, cap, d_rowptrG, d_colG);
    DGP_CHECK_LAUNCH();
  }
  return DGP_OK;
}

int fsai_factor_run(const int32_t *d_rowptr, const int32_t *d_col, const double *d_re, const double *d_im,
                    int64_t n, const int32_t *d_rowptrG, const int32_t *d_colG, int32_t mmax, int32_t nf,
                    double2 *d_out, int64_t s_slot, int64_t s_k, cudaStream_t st, const int32_t *d_harm) {
  DGP_REQUIRE(mmax >= 1 && mmax <= 32, "fsai factor: pattern rows must hold 1..32 entries");
  DGP_REQUIRE(nf >= 1 && nf <= 65535 * 32, "fsai factor: bad number of harmonics");
  dim3 grid((unsigned)ceil_div(n, 4), (unsigned)ceil_div(nf, 32));
  if (mmax <= 8) {
    size_t sm = 4 * 2 * 8 * 8 * sizeof(double);
    k_fsai_factor<8><<<grid, 128, sm, st>>>(d_rowptr, d_col, d_re, d_im, n, d_rowptrG, d_colG, nf, d_out, s_slot, s_k, d_harm);
  } else if (mmax <= 16) {
    size_t sm = 4 * 2 * 16 * 16 * sizeof(double);
    k_fsai_factor<16><<<grid, 128, sm, st>>>(d_rowptr, d_col, d_re, d_im, n, d_rowptrG, d_colG, nf, d_out, s_slot, s_k, d_harm);
  } else {
    size_t sm = 4 * 2 * 32 * 32 * sizeof(double);
    DGP_CUDA(cudaFuncSetAttribute(k_fsai_factor<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_fsai_factor<32><<<grid, 128, sm, st>>>(d_rowptr, d_col, d_re, d_im, n, d_rowptrG, d_colG, nf, d_out, s_slot, s_k, d_harm);
  }
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

int fsai_pattern_build(FsaiPattern *P, const int32_t *d_rowptr, const int32_t *d_col, const double *d_K,
                       const double *d_M, double dfc, int64_t n, int32_t cap, cudaStream_t st) {
  P->n = n;
  DGP_TRY(P->rowptr.alloc(sizeof(int32_t) * (n + 1)));
  int32_t nnzG = 0, mmax = 0;
  DGP_TRY(fsai_pattern_rows(d_rowptr, d_col, d_K, d_M, dfc, n, cap, P->rowptr.as<int32_t>(), nullptr, &nnzG,
                            &mmax, st));
  P->nnzG = nnzG;
  P->mmax = mmax;
  DGP_TRY(P->col.alloc(sizeof(int32_t) * nnzG));
  DGP_TRY(fsai_pattern_rows(d_rowptr, d_col, d_K, d_M, dfc, n, cap, P->rowptr.as<int32_t>(), P->col.as<int32_t>(),
                            nullptr, nullptr, st));
  return fsai_transpose_pattern(P, st);
}

int fsai_transpose_pattern(FsaiPattern *P, cudaStream_t st) {
  const int64_t n = P->n, nnz = P->nnzG;
  DevBuf k0, k1, s0, tmp;
  DGP_TRY(k0.alloc(sizeof(uint64_t) * nnz));
  DGP_TRY(k1.alloc(sizeof(uint64_t) * nnz));
  DGP_TRY(s0.alloc(sizeof(int32_t) * nnz));
  DGP_TRY(P->permT.alloc(sizeof(int32_t) * nnz));
  DGP_TRY(P->rowptrT.alloc(sizeof(int32_t) * (n + 1)));
  DGP_TRY(P->colT.alloc(sizeof(int32_t) * nnz));
  k_transpose_keys<<<grid1(n, 256), 256, 0, st>>>(P->rowptr.as<int32_t>(), P->col.as<int32_t>(), n,
                                                 k0.as<uint64_t>(), s0.as<int32_t>());
  DGP_CHECK_LAUNCH();
  size_t tb = 0;
  DGP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, k0.as<uint64_t>(), k1.as<uint64_t>(), s0.as<int32_t>(),
                                           P->permT.as<int32_t>(), (int)nnz, 0, 64, st));
  DGP_TRY(tmp.alloc(tb));
  DGP_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, k0.as<uint64_t>(), k1.as<uint64_t>(), s0.as<int32_t>(),
                                           P->permT.as<int32_t>(), (int)nnz, 0, 64, st));
  k_transpose_fill<<<grid1(nnz, 256), 256, 0, st>>>(k1.as<uint64_t>(), nnz, n, P->rowptrT.as<int32_t>(),
                                                   P->colT.as<int32_t>());
  DGP_CHECK_LAUNCH();
  DGP_CUDA(cudaStreamSynchronize(st));  // scratch buffers are released on return
  return DGP_OK;
}

int fsai_factor_full(const int32_t *d_rowptr, const int32_t *d_col, const double *d_K, const double *d_M, double dfc,
                     int64_t n, const int32_t *d_rowptrG, const int32_t *d_colG, int32_t nf, double2 *d_G,
                     cudaStream_t st) {
  DGP_REQUIRE(n > 0 && nf > 0, "fsai_factor: sizes must be positive");
  DGP_TRY(csr_in_range(d_rowptr, d_col, n, n, -1, 0, "fsai_factor: A", st));
  DGP_TRY(csr_in_range(d_rowptrG, d_colG, n, n, -1, 0, "fsai_factor: G pattern", st));
  DevBuf m, im;
  DGP_TRY(m.alloc(sizeof(int)));
  DGP_CUDA(cudaMemsetAsync(m.p, 0, sizeof(int), st));
  k_max_row<<<grid1(n, 256), 256, 0, st>>>(d_rowptrG, n, m.as<int>());
  DGP_CHECK_LAUNCH();
  int32_t hm = 0, nnzG = 0, nnzA = 0;
  DGP_CUDA(cudaMemcpyAsync(&hm, m.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaMemcpyAsync(&nnzG, d_rowptrG + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaMemcpyAsync(&nnzA, d_rowptr + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  // Im A = (df/c) * M, formed like the reference before the factor (dMesh.m:1241)
  DGP_TRY(im.alloc(sizeof(double) * (size_t)nnzA));
  k_scale<<<grid1(nnzA, 256), 256, 0, st>>>(d_M, dfc, nnzA, im.as<double>());
  DGP_CHECK_LAUNCH();
  DGP_TRY(fsai_factor_run(d_rowptr, d_col, d_K, im.as<double>(), n, d_rowptrG, d_colG, hm, nf, d_G, 1, nnzG, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  return DGP_OK;
}

}  // namespace dgp
