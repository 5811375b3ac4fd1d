// Batched FSAI-preconditioned BiCGSTAB (and COCG) over every source x harmonic.
//
// Replaces gpuBicstab_FSAIP + fluGPU (DOGPUP/dMesh.m:1238-1348).  The
// reference runs the iteration from MATLAB: 7 mex mat-vec calls per
// iteration, each re-copying A, x and the index arrays to fresh device
// arrays, about 20 gpuArray BLAS-1 launches and 4 device-wide waits.  Here
// one iteration is 10 sweep kernels + 5 single-block scalar kernels,
// captured once in a CUDA graph and replayed; convergence is decided on the
// device (FP64 dot products and norms) and polled by the host every
// `check_every` iterations.
//
// Arithmetic follows the reference: bilinear (unconjugated) dots r^0.v,
// r^0.r and (G t).(G s), (G t).(G t); alph = (v.r^0)/rho0 (its reciprocal
// alpha = rho0/(v.r^0) is stored and multiplied); omega in the G-weighted
// bilinear form; stop when the maximum over all columns of ||s||/||r0|| or
// ||r||/||r0|| is below tol; x = x + alpha h on the early exit.  The update
// h = x + alpha h of dMesh.m:1305 is folded into the x update
// (x = x + alpha h + omega z), which saves three vector passes.
//
// Layout of every vector: [NF][NN][NSP] complex (harmonic, node, source),
// NSP = sources padded to a power of two.  A tile of the SpMM is one
// harmonic x a block of rows; each lane carries VEC consecutive sources, so a
// row of one harmonic is one coalesced load per warp.  In the FP32 path each
// nonzero is one 16-byte record (column, K, M) for A -- combined on the fly
// into K + i w_k M -- or (column, Re G_k, Im G_k) for the FSAI factors, so a
// nonzero costs one broadcast load besides its x gather.
//
// Mixed precision: a complex-FP32 inner solve runs on the current FP64
// residual; the FP64 solution is updated and the FP64 residual b - A x is
// recomputed (FP64 K, M) with FP64 norms, until the maximum relative FP64
// residual is below tol (iterative refinement).  The inner solver is COCG
// (DGP_PREC_MIXED): A_k = K + i w_k M and the FSAI preconditioner G^T G are
// complex symmetric, so conjugate-orthogonal CG with bilinear dots applies;
// it costs one A and one G^T G application per iteration (9 launches)
// against BiCGSTAB's two of each (15 launches), for ~1.1x the iterations on
// these systems.  DGP_PREC_MIXED_BICGSTAB keeps BiCGSTAB as the inner solver.
#include <cub/cub.cuh>

#include <algorithm>
#include <initializer_list>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "dgp_common.cuh"
#include "dgp_internal.h"

namespace dgp {

namespace {

constexpr int BS = 256;
constexpr int WARPS = BS / 32;
constexpr int KERNELS_PER_ITER = 15;       // BiCGSTAB iteration
constexpr int KERNELS_PER_ITER_COCG = 9;   // COCG iteration

enum { ST_RUNNING = 0, ST_FINAL = 1, ST_DONE = 2 };
enum { ACC_D1 = 0, ACC_NS = 1, ACC_D2 = 2, ACC_D3 = 3, ACC_NR = 4, ACC_RHO = 5, NACC = 6 };

struct Ctl {
  int state;
  int iters;
  int maxit;
  int stop_rule;
  double tol;
  double max_err;
  int n_active;
  int reason;  // 0 tol reached, 1 maxit, 2 nothing to solve
  // stall guard of the device-driven loop: best max_err seen and checks since it halved
  double stall_ref;
  int stall_since;
  int loops;   // blocks of iterations the device-driven loop ran
};

struct Cols {
  int64_t C;        // columns = nf * nsp
  double *err0;     // ||r0|| per column
  double *err;      // last relative residual
  double2 *rho0, *alpha, *omega, *beta;
  double2 *acc;     // [NACC][C]
  int *active;      // 1 iterating, 2 converged at s this iteration, 0 frozen
  int *status;      // DGP_COL_*
  int *hact;        // [nf] 1 while any column of harmonic k iterates; sweeps skip the others (NULL: none skipped)
  double *tolc;     // per-column relative target of the per-column stop rule
  int nsp;
};

// a sweep block of harmonic k has nothing to do once all of k's columns are frozen
__device__ inline bool harmonic_done(const Cols &c, int k) { return c.hact && !c.hact[k]; }

// hact[k] = 1 while any column of harmonic k is active (one block; call after active[] is final)
__device__ inline void update_hact(const Cols &c) {
  if (!c.hact) return;
  const int nf = (int)(c.C / c.nsp);
  for (int k = threadIdx.x; k < nf; k += blockDim.x) {
    int any = 0;
    for (int s = 0; s < c.nsp && !any; ++s) any = c.active[(int64_t)k * c.nsp + s] != 0;
    c.hact[k] = any;
  }
}

struct Layout {
  int64_t n;
  int nf, nsp;
  int lpr;  // lanes per row (power of two <= 32)
  int rpw;  // rows per warp step
  int ipb;  // warp steps per block
  __host__ __device__ int64_t rows_per_block() const { return (int64_t)WARPS * rpw * ipb; }
};

// 16-byte record per nonzero of the FP32 path: A -> (col, K, M), G -> (col, Re, Im)
struct __align__(16) Rec32 {
  int col;
  float a, b, pad;
};

// ------------------------------------------------------------ vector I/O
template <class R> struct CT;
template <> struct CT<float> { using C = float2; };
template <> struct CT<double> { using C = double2; };

// Lane I/O.  A lane owns VEC complex values of a row as VEC/E chunks of E
// complex (16 bytes: E = 2 for complex FP32, 1 for complex FP64); chunk q
// starts cs complex after chunk q-1, with cs = E * (lanes per row), so each
// load instruction of a row group reads one contiguous run across its lanes.
template <class C> struct Chunk;
template <> struct Chunk<float2> { static constexpr int E = 2; };
template <> struct Chunk<double2> { static constexpr int E = 1; };

template <int VEC> __device__ inline void ldv(const float2 *p, int cs, float2 (&c)[VEC]) {
#pragma unroll
  for (int q = 0; q < VEC; q += 2) {
    float4 v = *reinterpret_cast<const float4 *>(p + (q / 2) * cs);
    c[q] = make_float2(v.x, v.y);
    c[q + 1] = make_float2(v.z, v.w);
  }
}
template <int VEC> __device__ inline void ldv(const double2 *p, int cs, double2 (&c)[VEC]) {
#pragma unroll
  for (int q = 0; q < VEC; ++q) c[q] = p[q * cs];
}
template <int VEC> __device__ inline void ldgv(const float2 *p, int cs, float2 (&c)[VEC]) {
#pragma unroll
  for (int q = 0; q < VEC; q += 2) {
    float4 v = __ldg(reinterpret_cast<const float4 *>(p + (q / 2) * cs));
    c[q] = make_float2(v.x, v.y);
    c[q + 1] = make_float2(v.z, v.w);
  }
}
template <int VEC> __device__ inline void ldgv(const double2 *p, int cs, double2 (&c)[VEC]) {
#pragma unroll
  for (int q = 0; q < VEC; ++q) c[q] = __ldg(p + q * cs);
}
template <int VEC> __device__ inline void stv(float2 *p, int cs, const float2 (&c)[VEC]) {
#pragma unroll
  for (int q = 0; q < VEC; q += 2)
    *reinterpret_cast<float4 *>(p + (q / 2) * cs) = make_float4(c[q].x, c[q].y, c[q + 1].x, c[q + 1].y);
}
template <int VEC> __device__ inline void stv(double2 *p, int cs, const double2 (&c)[VEC]) {
#pragma unroll
  for (int q = 0; q < VEC; ++q) p[q * cs] = c[q];
}

template <class C> __device__ inline C czero();
template <> __device__ inline float2 czero<float2>() { return make_float2(0.f, 0.f); }
template <> __device__ inline double2 czero<double2>() { return make_double2(0.0, 0.0); }

__device__ inline float2 cfmaT(float2 b, float2 c, float2 a) { return cfmaf(b, c, a); }
__device__ inline double2 cfmaT(double2 b, double2 c, double2 a) { return cfma(b, c, a); }
__device__ inline float2 cneg(float2 a) { return make_float2(-a.x, -a.y); }
__device__ inline double2 cneg(double2 a) { return make_double2(-a.x, -a.y); }

template <class R> __device__ inline typename CT<R>::C cvt(double2 a);
template <> __device__ inline float2 cvt<float>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> __device__ inline double2 cvt<double>(double2 a) { return a; }
__device__ inline double2 d2(float2 a) { return make_double2(a.x, a.y); }
__device__ inline double2 d2(double2 a) { return a; }

// bilinear product accumulated in FP64
template <class C> __device__ inline void acc_bil(double2 &s, C a, C b) {
  double2 x = d2(a), y = d2(b);
  s.x += x.x * y.x - x.y * y.y;
  s.y += x.x * y.y + x.y * y.x;
}
// FP32 partials of the FP32 solver's SpMM dots: each lane sums at most one
// block's rows (<= 32) in FP32 before the FP64 lane / warp / block reduction
__device__ inline void acc_bil(float2 &s, float2 a, float2 b) {
  s.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, s.x));
  s.y = fmaf(a.x, b.y, fmaf(a.y, b.x, s.y));
}
template <class C> __device__ inline void acc_abs2(double &s, C a) {
  double2 x = d2(a);
  s += x.x * x.x + x.y * x.y;
}

// ------------------------------------------------------------ lane mapping
struct Lane {
  int warp, sub, rsub, k;
  int64_t row0;
  __device__ Lane(const Layout &L) {
    warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    sub = lane % L.lpr;
    rsub = lane / L.lpr;
    row0 = (int64_t)blockIdx.x * L.rows_per_block();
    k = blockIdx.y;
  }
  __device__ int64_t row(const Layout &L, int it) const { return row0 + ((int64_t)it * WARPS + warp) * L.rpw + rsub; }
  // column of this lane's value v, its first column, and the stride between its chunks
  template <int E> __device__ int col(const Layout &L, int v) const { return E * ((v / E) * L.lpr + sub) + v % E; }
  template <int E> __device__ int col0() const { return E * sub; }
  template <int E> __device__ int cs(const Layout &L) const { return E * L.lpr; }
};

__device__ inline int64_t vidx(const Layout &L, int k, int64_t i, int s) {
  return ((int64_t)k * L.n + i) * L.nsp + s;
}

// Block reduction of per-lane column partials into acc[slot[q]][k*nsp + s] (FP64 atomics).
template <int VEC, int NQ, int E = 2>
__device__ inline void block_reduce(const Layout &L, const Lane &ln, double2 (&part)[VEC][NQ], double2 *acc,
                                    int64_t C, const int (&slot)[NQ], double2 *sm /*[WARPS][nsp][NQ]*/) {
#pragma unroll
  for (int v = 0; v < VEC; ++v)
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double2 x = part[v][q];
      for (int off = L.lpr; off < 32; off <<= 1) {
        x.x += __shfl_xor_sync(0xffffffffu, x.x, off);
        x.y += __shfl_xor_sync(0xffffffffu, x.y, off);
      }
      part[v][q] = x;
    }
  if (ln.rsub == 0) {
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      const int s = ln.template col<E>(L, v);
#pragma unroll
      for (int q = 0; q < NQ; ++q) sm[((int64_t)ln.warp * L.nsp + s) * NQ + q] = part[v][q];
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < L.nsp * NQ; t += blockDim.x) {
    const int s = t / NQ, q = t % NQ;
    double2 x = make_double2(0.0, 0.0);
    for (int w = 0; w < WARPS; ++w) {
      double2 y = sm[((int64_t)w * L.nsp + s) * NQ + q];
      x.x += y.x;
      x.y += y.y;
    }
    double2 *dst = acc + (int64_t)slot[q] * C + (int64_t)ln.k * L.nsp + s;
    atomicAdd(&dst->x, x.x);
    atomicAdd(&dst->y, x.y);
  }
}

// -------------------------------------------------- coefficient policies
struct CoefA32 {  // K + i w_k M from one record
  const Rec32 *rec;
  float om;
  __device__ inline void get(int p, int &j, float2 &c) const {
    int4 r = __ldg(reinterpret_cast<const int4 *>(rec + p));
    j = r.x;
    c = make_float2(__int_as_float(r.y), om * __int_as_float(r.z));
  }
};
struct CoefG32 {  // G_k (or G_k^T) from one record
  const Rec32 *rec;
  __device__ inline void get(int p, int &j, float2 &c) const {
    int4 r = __ldg(reinterpret_cast<const int4 *>(rec + p));
    j = r.x;
    c = make_float2(__int_as_float(r.y), __int_as_float(r.z));
  }
};
struct CoefA64 {
  const int32_t *col;
  const double2 *KM;
  double om;
  __device__ inline void get(int p, int &j, double2 &c) const {
    j = __ldg(col + p);
    double2 km = __ldg(KM + p);
    c = make_double2(km.x, om * km.y);
  }
};
struct CoefG64 {
  const int32_t *col;
  const double2 *G;
  __device__ inline void get(int p, int &j, double2 &c) const {
    j = __ldg(col + p);
    c = __ldg(G + p);
  }
};

// Operator descriptor handed to the SpMM kernel; make(k) gives harmonic k's coefficients.
struct OpA32 {
  const int32_t *rowptr;
  const Rec32 *rec;
  const float *omega;
  __device__ CoefA32 make(int k) const { return CoefA32{rec, omega[k]}; }
};
struct OpG32 {
  const int32_t *rowptr;
  const Rec32 *rec;
  int64_t nnz;
  __device__ CoefG32 make(int k) const { return CoefG32{rec + (int64_t)k * nnz}; }
};
struct OpA64 {
  const int32_t *rowptr, *col;
  const double2 *KM;
  const double *omega;
  __device__ CoefA64 make(int k) const { return CoefA64{col, KM, omega[k]}; }
};
struct OpG64 {
  const int32_t *rowptr, *col;
  const double2 *G;
  int64_t nnz;
  __device__ CoefG64 make(int k) const { return CoefG64{col, G + (int64_t)k * nnz}; }
};

// y[0..VEC) = sum_p coef(p) * Xk[col(p)*nsp + s0 ..]   (32-bit offsets inside one harmonic plane)
//
// Software-pipelined: the coefficient records (column, value) of batch b+1 are
// loaded before the x gathers of batch b are consumed, so the record -> column
// -> x dependency costs one memory latency per batch instead of two.
template <int VEC, class C, class Coef>
__device__ inline void row_spmv(int nsp, int cs, const int32_t *__restrict__ rowptr, int64_t i, const Coef &cf,
                                const C *__restrict__ Xk, C (&y)[VEC]) {
#pragma unroll
  for (int v = 0; v < VEC; ++v) y[v] = czero<C>();
  const int b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
  // gathers in flight per lane: UNR nonzeros x VEC complex (register budget bounds UNR*VEC)
  constexpr int UNR = VEC >= 8 ? 2 : 4;
  int p = b;
  if (p + UNR <= e) {
    int j[UNR];
    C a[UNR];
#pragma unroll
    for (int u = 0; u < UNR; ++u) cf.get(p + u, j[u], a[u]);
    for (;;) {
      C xs[UNR][VEC];
#pragma unroll
      for (int u = 0; u < UNR; ++u) ldgv<VEC>(Xk + j[u] * nsp, cs, xs[u]);
      const int pn = p + UNR;
      const bool more = pn + UNR <= e;
      int jn[UNR];
      C an[UNR];
      if (more) {
#pragma unroll
        for (int u = 0; u < UNR; ++u) cf.get(pn + u, jn[u], an[u]);
      }
#pragma unroll
      for (int u = 0; u < UNR; ++u)
#pragma unroll
        for (int v = 0; v < VEC; ++v) y[v] = cfmaT(a[u], xs[u][v], y[v]);
      p = pn;
      if (!more) break;
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        j[u] = jn[u];
        a[u] = an[u];
      }
    }
  }
  for (; p < e; ++p) {
    int j;
    C a;
    cf.get(p, j, a);
    C x[VEC];
    ldgv<VEC>(Xk + j * nsp, cs, x);
#pragma unroll
    for (int v = 0; v < VEC; ++v) y[v] = cfmaT(a, x[v], y[v]);
  }
}

// FP32 rows: the lanes of a row load the row's records in parallel (one
// coalesced 16-byte load per lane and LPR nonzeros) and hand each nonzero's
// column and coefficient to the row's lanes with shuffles, instead of every
// lane loading every record (a broadcast load costs the L1 return bandwidth
// of a full vector load); the x gathers then depend on one record load per
// LPR nonzeros.  Rows of a warp loop to the warp's longest row (masked).
template <int VEC, class Coef>
__device__ inline void row_spmv_shfl(int nsp, int cs, const int32_t *__restrict__ rowptr, int64_t i, const Coef &cf,
                                     const float2 *__restrict__ Xk, float2 (&y)[VEC], int lpr, int sub,
                                     unsigned mask /* lanes of the warp's rows that exist */) {
#pragma unroll
  for (int v = 0; v < VEC; ++v) y[v] = make_float2(0.f, 0.f);
  const int b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
  const int cmax = __reduce_max_sync(mask, e - b);
  for (int base = 0; base < cmax; base += lpr) {
    int j0 = 0;
    float2 a0 = make_float2(0.f, 0.f);
    if (b + base + sub < e) cf.get(b + base + sub, j0, a0);
    const int cnt = min(lpr, cmax - base);
    for (int u = 0; u < cnt; ++u) {
      const int j = __shfl_sync(mask, j0, u, lpr);
      const float ax = __shfl_sync(mask, a0.x, u, lpr), ay = __shfl_sync(mask, a0.y, u, lpr);
      if (b + base + u < e) {
        float2 x[VEC];
        ldgv<VEC>(Xk + j * nsp, cs, x);
        const float2 a = make_float2(ax, ay);
#pragma unroll
        for (int v = 0; v < VEC; ++v) y[v] = cfmaf(a, x[v], y[v]);
      }
    }
  }
}

// FP32 rows, U nonzeros per step (KIND 1: U = 2, KIND 2: U = 4, KIND 3: U = 4 with packed
// FP32 FMAs).  As row_spmv_shfl, but the lanes past a row's end hold a padding record
// (the row's own column, coefficient 0), so the U shuffles, U x gathers and U * VEC
// complex FMAs of a step are issued without per-nonzero predicates and the U gathers
// are in flight together.  A padding term adds 0 * x_i (exactly 0 for finite x_i).
// KIND 3 accumulates sum a.re * x and sum a.im * x as float2 pairs with one packed FMA
// each (__ffma2_rn) and combines them once per row: 2 instead of 4 FMA instructions
// per complex product.
template <int VEC, int KIND, class Coef>
__device__ inline void row_spmv_shfl_u(int nsp, int cs, const int32_t *__restrict__ rowptr, int64_t i,
                                       const Coef &cf, const float2 *__restrict__ Xk, float2 (&y)[VEC], int lpr,
                                       int sub, unsigned mask) {
  constexpr int U = KIND == 1 ? 2 : 4;
  constexpr bool PACKED = KIND == 3;
  float2 ac[VEC], as[PACKED ? VEC : 1];
#pragma unroll
  for (int v = 0; v < VEC; ++v) ac[v] = make_float2(0.f, 0.f);
#pragma unroll
  for (int v = 0; v < (PACKED ? VEC : 1); ++v) as[v] = make_float2(0.f, 0.f);
  const int b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
  const int cmax = __reduce_max_sync(mask, e - b);
  const int step = min(U, lpr);  // lpr is a power of two: every step stays inside the row's lanes
  for (int base = 0; base < cmax; base += lpr) {
    int j0 = (int)i;
    float2 a0 = make_float2(0.f, 0.f);
    if (b + base + sub < e) cf.get(b + base + sub, j0, a0);
    const int cnt = min(lpr, cmax - base);
    for (int u = 0; u < cnt; u += step) {
      int j[U];
      float2 a[U];
#pragma unroll
      for (int q = 0; q < U; ++q) {
        if (q < step) {
          j[q] = __shfl_sync(mask, j0, u + q, lpr);
          a[q].x = __shfl_sync(mask, a0.x, u + q, lpr);
          a[q].y = __shfl_sync(mask, a0.y, u + q, lpr);
        }
      }
      float2 x[U][VEC];
#pragma unroll
      for (int q = 0; q < U; ++q)
        if (q < step) ldgv<VEC>(Xk + j[q] * nsp, cs, x[q]);
#pragma unroll
      for (int q = 0; q < U; ++q) {
        if (q < step) {
          if constexpr (PACKED) {
            const float2 re = make_float2(a[q].x, a[q].x), im = make_float2(a[q].y, a[q].y);
#pragma unroll
            for (int v = 0; v < VEC; ++v) {
              ac[v] = __ffma2_rn(re, x[q][v], ac[v]);
              as[v] = __ffma2_rn(im, x[q][v], as[v]);
            }
          } else {
#pragma unroll
            for (int v = 0; v < VEC; ++v) ac[v] = cfmaf(a[q], x[q][v], ac[v]);
          }
        }
      }
    }
  }
#pragma unroll
  for (int v = 0; v < VEC; ++v) {
    if constexpr (PACKED) y[v] = make_float2(ac[v].x - as[v].y, ac[v].y + as[v].x);
    else y[v] = ac[v];
  }
}

__device__ inline bool halted(const Ctl *ctl, int need) {
  // need = ST_RUNNING: skip unless running; ST_FINAL: skip only when done
  int s = *(volatile const int *)&ctl->state;
  return need == ST_RUNNING ? (s != ST_RUNNING) : (s == ST_DONE);
}

// Y = Op_k X.  MODE 0: store.  MODE 1: store, acc[D1] += Y.W.
// MODE 2: no store, acc[D2] += Y.W, acc[D3] += Y.Y.  MODE 3: store, acc[D1] += Y.Y.
// KIND (complex FP32 only): 0 one nonzero per step (row_spmv_shfl), 1-3 row_spmv_shfl_u.
template <class R, int VEC, int MODE, class Op, int KIND = 0>
__global__ void __launch_bounds__(BS) k_spmm(Layout L, Op op, const typename CT<R>::C *__restrict__ X,
                                             typename CT<R>::C *__restrict__ Y,
                                             const typename CT<R>::C *__restrict__ W, Cols cols, const Ctl *ctl) {
  using C = typename CT<R>::C;
  if (ctl && halted(ctl, ST_RUNNING)) return;
  if (harmonic_done(cols, blockIdx.y)) return;
  extern __shared__ double2 smem[];
  Lane ln(L);
  const auto cf = op.make(ln.k);
  constexpr int E = Chunk<C>::E;
  const int c0 = ln.template col0<E>(), cs = ln.template cs<E>(L);
  const C *Xk = X + (int64_t)ln.k * L.n * L.nsp + c0;
  constexpr int NQ = MODE == 2 ? 2 : 1;
  C part[VEC][NQ];  // per-lane partial sums in the sweep's precision (FP32 lanes: <= 32 rows each)
#pragma unroll
  for (int v = 0; v < VEC; ++v)
#pragma unroll
    for (int q = 0; q < NQ; ++q) part[v][q] = czero<C>();
  for (int it = 0; it < L.ipb; ++it) {
    const int64_t i = ln.row(L, it);
    // every lane reaches this ballot each step (rows past n only `continue`), so the FP32
    // row's shuffles run on an exact mask of the warp's valid rows
    const bool valid = i < L.n;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    if (vmask == 0u) break;
    if (!valid) continue;
    C y[VEC];
    if constexpr (sizeof(R) == 4) {
      if constexpr (KIND == 0) row_spmv_shfl<VEC>(L.nsp, cs, op.rowptr, i, cf, Xk, y, L.lpr, ln.sub, vmask);
      else row_spmv_shfl_u<VEC, KIND>(L.nsp, cs, op.rowptr, i, cf, Xk, y, L.lpr, ln.sub, vmask);
    } else {
      row_spmv<VEC>(L.nsp, cs, op.rowptr, i, cf, Xk, y);
    }
    const int64_t o = vidx(L, ln.k, i, c0);
    if (MODE != 2) stv<VEC>(Y + o, cs, y);
    if constexpr (MODE == 3) {
#pragma unroll
      for (int v = 0; v < VEC; ++v) acc_bil(part[v][0], y[v], y[v]);
    } else if (MODE != 0) {
      C w[VEC];
      ldv<VEC>(W + o, cs, w);
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        acc_bil(part[v][0], y[v], w[v]);
        if (MODE == 2) acc_bil(part[v][NQ - 1], y[v], y[v]);
      }
    }
  }
  if constexpr (MODE != 0) {
    double2 pd[VEC][NQ];
#pragma unroll
    for (int v = 0; v < VEC; ++v)
#pragma unroll
      for (int q = 0; q < NQ; ++q) pd[v][q] = d2(part[v][q]);
    if constexpr (MODE == 1 || MODE == 3) {
      const int slot[1] = {ACC_D1};
      block_reduce<VEC, 1, E>(L, ln, pd, cols.acc, cols.C, slot, smem);
    } else {
      const int slot[2] = {ACC_D2, ACC_D3};
      block_reduce<VEC, 2, E>(L, ln, pd, cols.acc, cols.C, slot, smem);
    }
  }
}

// Harmonic pairs (SpMM kind 4, the A operator only: its record (column, K, M) is the same for
// every harmonic, only w_k differs).  A block computes harmonics 2 y and 2 y + 1 of its rows
// together: each nonzero's record is loaded and handed out by shuffles once for both harmonics,
// a_k = K + i w_k M is formed per harmonic, and the two harmonics' x gathers are in flight
// together.  With an odd harmonic count the last block's second harmonic is a copy of its
// first, computed and not written.
template <int VEC>
__device__ inline void row_spmv_shfl_pair(int nsp, int cs, const int32_t *__restrict__ rowptr, int64_t i,
                                          const Rec32 *__restrict__ rec, float om0, float om1,
                                          const float2 *__restrict__ X0, const float2 *__restrict__ X1,
                                          float2 (&y0)[VEC], float2 (&y1)[VEC], int lpr, int sub, unsigned mask) {
#pragma unroll
  for (int v = 0; v < VEC; ++v) {
    y0[v] = make_float2(0.f, 0.f);
    y1[v] = make_float2(0.f, 0.f);
  }
  const int b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
  const int cmax = __reduce_max_sync(mask, e - b);
  for (int base = 0; base < cmax; base += lpr) {
    int j0 = 0;
    float k0 = 0.f, m0 = 0.f;
    if (b + base + sub < e) {
      const int4 r = __ldg(reinterpret_cast<const int4 *>(rec + b + base + sub));
      j0 = r.x;
      k0 = __int_as_float(r.y);
      m0 = __int_as_float(r.z);
    }
    const int cnt = min(lpr, cmax - base);
    for (int u = 0; u < cnt; ++u) {
      const int j = __shfl_sync(mask, j0, u, lpr);
      const float kk = __shfl_sync(mask, k0, u, lpr), mm = __shfl_sync(mask, m0, u, lpr);
      if (b + base + u < e) {
        float2 x0[VEC], x1[VEC];
        ldgv<VEC>(X0 + j * nsp, cs, x0);
        ldgv<VEC>(X1 + j * nsp, cs, x1);
        const float2 a0 = make_float2(kk, om0 * mm), a1 = make_float2(kk, om1 * mm);
#pragma unroll
        for (int v = 0; v < VEC; ++v) {
          y0[v] = cfmaf(a0, x0[v], y0[v]);
          y1[v] = cfmaf(a1, x1[v], y1[v]);
        }
      }
    }
  }
}

// Y = A_k X for the harmonic pair of blockIdx.y; MODE as k_spmm.
template <int VEC, int MODE>
__global__ void __launch_bounds__(BS) k_spmm_pair(Layout L, OpA32 op, const float2 *__restrict__ X,
                                                  float2 *__restrict__ Y, const float2 *__restrict__ W, Cols cols,
                                                  const Ctl *ctl) {
  if (ctl && halted(ctl, ST_RUNNING)) return;
  const int k0 = 2 * (int)blockIdx.y, k1 = k0 + 1;
  const bool has1 = k1 < L.nf;
  const bool live0 = !harmonic_done(cols, k0), live1 = has1 && !harmonic_done(cols, k1);
  if (!live0 && !live1) return;
  extern __shared__ double2 smem[];
  Lane ln(L);
  constexpr int E = 2;
  const int c0 = ln.template col0<E>(), cs = ln.template cs<E>(L);
  const int64_t plane = L.n * (int64_t)L.nsp;
  const float2 *X0 = X + (int64_t)k0 * plane + c0;
  const float2 *X1 = has1 ? X0 + plane : X0;
  const float om0 = op.omega[k0], om1 = has1 ? op.omega[k1] : om0;
  constexpr int NQ = MODE == 2 ? 2 : 1;
  float2 p0[VEC][NQ], p1[VEC][NQ];
#pragma unroll
  for (int v = 0; v < VEC; ++v)
#pragma unroll
    for (int q = 0; q < NQ; ++q) p0[v][q] = p1[v][q] = make_float2(0.f, 0.f);
  for (int it = 0; it < L.ipb; ++it) {
    const int64_t i = ln.row(L, it);
    const bool valid = i < L.n;
    const unsigned vmask = __ballot_sync(0xffffffffu, valid);
    if (vmask == 0u) break;
    if (!valid) continue;
    float2 y0[VEC], y1[VEC];
    row_spmv_shfl_pair<VEC>(L.nsp, cs, op.rowptr, i, op.rec, om0, om1, X0, X1, y0, y1, L.lpr, ln.sub, vmask);
    const int64_t o0 = vidx(L, k0, i, c0), o1 = o0 + plane;
    if (MODE != 2) {
      if (live0) stv<VEC>(Y + o0, cs, y0);
      if (live1) stv<VEC>(Y + o1, cs, y1);
    }
    if constexpr (MODE == 3) {
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        acc_bil(p0[v][0], y0[v], y0[v]);
        acc_bil(p1[v][0], y1[v], y1[v]);
      }
    } else if (MODE != 0) {
      float2 w0[VEC], w1[VEC];
      ldv<VEC>(W + o0, cs, w0);
      ldv<VEC>(W + (has1 ? o1 : o0), cs, w1);
#pragma unroll
      for (int v = 0; v < VEC; ++v) {
        acc_bil(p0[v][0], y0[v], w0[v]);
        acc_bil(p1[v][0], y1[v], w1[v]);
        if (MODE == 2) {
          acc_bil(p0[v][NQ - 1], y0[v], y0[v]);
          acc_bil(p1[v][NQ - 1], y1[v], y1[v]);
        }
      }
    }
  }
  if constexpr (MODE != 0) {
    double2 d0[VEC][NQ], d1[VEC][NQ];
#pragma unroll
    for (int v = 0; v < VEC; ++v)
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        d0[v][q] = d2(p0[v][q]);
        d1[v][q] = d2(p1[v][q]);
      }
    constexpr int S0 = MODE == 2 ? ACC_D2 : ACC_D1;
    const int slot[NQ] = {S0};
    int slot2[2] = {ACC_D2, ACC_D3};
    Lane l0 = ln, l1 = ln;
    l0.k = k0;
    l1.k = k1;
    // (block-uniform conditions: block_reduce synchronises the block)
    if constexpr (MODE == 2) {
      if (live0) block_reduce<VEC, 2, E>(L, l0, d0, cols.acc, cols.C, slot2, smem);
      __syncthreads();
      if (live1) block_reduce<VEC, 2, E>(L, l1, d1, cols.acc, cols.C, slot2, smem);
    } else {
      if (live0) block_reduce<VEC, 1, E>(L, l0, d0, cols.acc, cols.C, slot, smem);
      __syncthreads();
      if (live1) block_reduce<VEC, 1, E>(L, l1, d1, cols.acc, cols.C, slot, smem);
    }
  }
}

// ------------------------------------------------------- tiled SpMM
// Y = Op_k X with the x rows a block needs staged in shared memory first.
// Block (b, k, z) owns rows [b*rb, b*rb + rb) of harmonic k and sources
// [z*SW, z*SW + SW): it copies its halo rows (the distinct columns of its
// rows, hcols[hptr[b] ..]) and its nonzeros' 16-byte records into shared
// memory with cp.async (all copies in flight at once, no dependent global
// loads), then each lane accumulates VEC consecutive sources of a row from
// shared memory (the record's pad word holds the column's halo position).
// MODE as k_spmm: 0 store, 1 store + Y.W, 2 Y.W and Y.Y without the store.
struct TLayout {
  int64_t n;
  int nf, nsp, rb;
  const int32_t *hptr, *hcols, *rowptr;
};

__device__ inline void cp_async16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ inline void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

template <class Op> struct TCoef;
template <> struct TCoef<OpA32> {
  float om;
  const Rec32 *rec;
  __device__ TCoef(const OpA32 &op, int k) : om(op.omega[k]), rec(op.rec) {}
  __device__ float2 of(const Rec32 &r) const { return make_float2(r.a, om * r.b); }
};
template <> struct TCoef<OpG32> {
  const Rec32 *rec;
  __device__ TCoef(const OpG32 &op, int k) : rec(op.rec + (int64_t)k * op.nnz) {}
  __device__ float2 of(const Rec32 &r) const { return make_float2(r.a, r.b); }
};

template <int MODE, int SW, class Op>
__global__ void __launch_bounds__(BS) k_tspmm(TLayout T, Op op, const float2 *__restrict__ X, float2 *__restrict__ Y,
                                              const float2 *__restrict__ W, Cols cols, const Ctl *ctl, int hcap) {
  constexpr int VEC = SW < 4 ? SW : 4;  // complex values per lane
  constexpr int LPR = SW / VEC;         // lanes per row
  constexpr int RPW = 32 / LPR;         // rows per warp
  constexpr int NQ = MODE == 2 ? 2 : 1;
  if (ctl && halted(ctl, ST_RUNNING)) return;
  if (harmonic_done(cols, blockIdx.y)) return;
  extern __shared__ float4 tsm[];
  float2 *tile = reinterpret_cast<float2 *>(tsm);                      // [hcap][SW]
  Rec32 *srec = reinterpret_cast<Rec32 *>(tile + (size_t)hcap * SW);   // [zcap]
  const int b = blockIdx.x, k = blockIdx.y, s0 = blockIdx.z * SW;
  const int64_t r0 = (int64_t)b * T.rb;
  const int64_t r1 = min(T.n, r0 + T.rb);
  const int h0 = T.hptr[b], nh = T.hptr[b + 1] - h0;
  const int p0 = T.rowptr[r0], np = T.rowptr[r1] - p0;
  const TCoef<Op> cf(op, k);
  const float2 *Xk = X + (int64_t)k * T.n * T.nsp + s0;
  constexpr int CPR = SW / 2;  // 16-byte chunks per halo row
  for (int t = threadIdx.x; t < nh * CPR; t += BS) {
    const int hr = t / CPR, c = t - hr * CPR;
    const int64_t j = T.hcols[h0 + hr];
    cp_async16(tile + hr * SW + 2 * c, Xk + j * T.nsp + 2 * c);
  }
  for (int t = threadIdx.x; t < np; t += BS) cp_async16(srec + t, cf.rec + p0 + t);
  cp_async_wait_all();
  __syncthreads();

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sub = lane % LPR, rsub = lane / LPR;
  float2 part[VEC][NQ];
#pragma unroll
  for (int v = 0; v < VEC; ++v)
#pragma unroll
    for (int q = 0; q < NQ; ++q) part[v][q] = make_float2(0.f, 0.f);
  for (int lr0 = 0; lr0 < T.rb; lr0 += WARPS * RPW) {
    const int64_t i = r0 + lr0 + warp * RPW + rsub;
    if (i >= r1) continue;
    float2 y[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) y[v] = make_float2(0.f, 0.f);
    const int pb = __ldg(T.rowptr + i) - p0, pe = __ldg(T.rowptr + i + 1) - p0;
    for (int p = pb; p < pe; ++p) {
      const Rec32 rc = srec[p];
      const float2 a = cf.of(rc);
      const float2 *xr = tile + __float_as_int(rc.pad) * SW + sub * VEC;
#pragma unroll
      for (int v = 0; v < VEC; v += 2) {
        const float4 xv = *reinterpret_cast<const float4 *>(xr + v);
        y[v] = cfmaf(a, make_float2(xv.x, xv.y), y[v]);
        if (VEC > 1) y[v + 1] = cfmaf(a, make_float2(xv.z, xv.w), y[v + 1]);
      }
    }
    const int64_t o = ((int64_t)k * T.n + i) * T.nsp + s0 + sub * VEC;
    if (MODE != 2) {
#pragma unroll
      for (int v = 0; v < VEC; v += 2)
        *reinterpret_cast<float4 *>(Y + o + v) = make_float4(y[v].x, y[v].y, y[v + 1].x, y[v + 1].y);
    }
    if (MODE != 0) {
#pragma unroll
      for (int v = 0; v < VEC; v += 2) {
        const float4 wv = *reinterpret_cast<const float4 *>(W + o + v);
        acc_bil(part[v][0], y[v], make_float2(wv.x, wv.y));
        acc_bil(part[v + 1][0], y[v + 1], make_float2(wv.z, wv.w));
        if (MODE == 2) {
          acc_bil(part[v][NQ - 1], y[v], y[v]);
          acc_bil(part[v + 1][NQ - 1], y[v + 1], y[v + 1]);
        }
      }
    }
  }
  if constexpr (MODE != 0) {
    // lanes with the same sub hold the same columns: shuffle, then warps through shared memory
    double2 pd[VEC][NQ];
#pragma unroll
    for (int v = 0; v < VEC; ++v)
#pragma unroll
      for (int q = 0; q < NQ; ++q) {
        double2 x = d2(part[v][q]);
        for (int off = LPR; off < 32; off <<= 1) {
          x.x += __shfl_xor_sync(0xffffffffu, x.x, off);
          x.y += __shfl_xor_sync(0xffffffffu, x.y, off);
        }
        pd[v][q] = x;
      }
    __syncthreads();  // the tile is no longer read: reuse its space for the warp partials
    double2 *red = reinterpret_cast<double2 *>(tsm);  // [WARPS][SW][NQ]
    if (rsub == 0) {
#pragma unroll
      for (int v = 0; v < VEC; ++v)
#pragma unroll
        for (int q = 0; q < NQ; ++q) red[(warp * SW + sub * VEC + v) * NQ + q] = pd[v][q];
    }
    __syncthreads();
    const int slot[2] = {MODE == 1 ? ACC_D1 : ACC_D2, ACC_D3};
    for (int t = threadIdx.x; t < SW * NQ; t += BS) {
      const int sc = t / NQ, q = t % NQ;
      double2 x = make_double2(0.0, 0.0);
      for (int w = 0; w < WARPS; ++w) {
        const double2 yv = red[(w * SW + sc) * NQ + q];
        x.x += yv.x;
        x.y += yv.y;
      }
      double2 *dst = cols.acc + (int64_t)slot[q] * cols.C + (int64_t)k * T.nsp + s0 + sc;
      atomicAdd(&dst->x, x.x);
      atomicAdd(&dst->y, x.y);
    }
  }
}

// per-lane column scalars
template <class R, int VEC>
__device__ inline void lane_scalars(const Cols &cols, const Lane &ln, const Layout &L, const double2 *src,
                                    typename CT<R>::C (&out)[VEC], int (&act)[VEC]) {
#pragma unroll
  for (int v = 0; v < VEC; ++v) {
    const int64_t c = (int64_t)ln.k * L.nsp + ln.template col<Chunk<typename CT<R>::C>::E>(L, v);
    act[v] = cols.active[c];
    out[v] = cvt<R>(src[c]);
  }
}

// s = r - alpha*v ; acc[NS] += |s|^2   (dMesh.m:1306-1307)
template <class R, int VEC>
__global__ void __launch_bounds__(BS) k_update_s(Layout L, const typename CT<R>::C *__restrict__ r,
                                                 const typename CT<R>::C *__restrict__ v,
                                                 typename CT<R>::C *__restrict__ s, Cols cols, const Ctl *ctl) {
  using C = typename CT<R>::C;
  if (halted(ctl, ST_RUNNING)) return;
  if (harmonic_done(cols, blockIdx.y)) return;
  extern __shared__ double2 smem[];
  Lane ln(L);
  constexpr int E = Chunk<typename CT<R>::C>::E;
  const int c0 = ln.template col0<E>(), cs = ln.template cs<E>(L);
  double2 part[VEC][1];
  C al[VEC];
  int act[VEC];
  lane_scalars<R, VEC>(cols, ln, L, cols.alpha, al, act);
#pragma unroll
  for (int q = 0; q < VEC; ++q) part[q][0] = make_double2(0, 0);
  for (int it = 0; it < L.ipb; ++it) {
    const int64_t i = ln.row(L, it);
    if (i >= L.n) break;
    const int64_t o = vidx(L, ln.k, i, c0);
    C rr[VEC], vv[VEC], ss[VEC];
    ldv<VEC>(r + o, cs, rr);
    ldv<VEC>(v + o, cs, vv);
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      ss[q] = act[q] ? cfmaT(cneg(al[q]), vv[q], rr[q]) : rr[q];
      if (act[q]) acc_abs2(part[q][0].x, ss[q]);
    }
    stv<VEC>(s + o, cs, ss);
  }
  const int slot[1] = {ACC_NS};
  block_reduce<VEC, 1, E>(L, ln, part, cols.acc, cols.C, slot, smem);
}

// x = x + alpha*h + omega*z ; r = s - omega*t ; p = p - omega*v ; acc[NR] += |r|^2 ;
// acc[RHO] += r0^.r  (dMesh.m:1305, :1327-1337).  In the FINAL state: x = x + alpha*h (:1311).
template <class R, int VEC>
__global__ void __launch_bounds__(BS) k_update_xrp(Layout L, typename CT<R>::C *__restrict__ x,
                                                   const typename CT<R>::C *__restrict__ h,
                                                   const typename CT<R>::C *__restrict__ z,
                                                   typename CT<R>::C *__restrict__ r,
                                                   const typename CT<R>::C *__restrict__ s,
                                                   const typename CT<R>::C *__restrict__ t,
                                                   typename CT<R>::C *__restrict__ p,
                                                   const typename CT<R>::C *__restrict__ v,
                                                   const typename CT<R>::C *__restrict__ rhat, Cols cols,
                                                   const Ctl *ctl) {
  using C = typename CT<R>::C;
  if (halted(ctl, ST_FINAL)) return;
  if (harmonic_done(cols, blockIdx.y)) return;
  const bool final_ = *(volatile const int *)&ctl->state == ST_FINAL;
  extern __shared__ double2 smem[];
  Lane ln(L);
  constexpr int E = Chunk<typename CT<R>::C>::E;
  const int c0 = ln.template col0<E>(), cs = ln.template cs<E>(L);
  double2 part[VEC][2];
  C al[VEC], om[VEC];
  int act[VEC];
  lane_scalars<R, VEC>(cols, ln, L, cols.omega, om, act);
  lane_scalars<R, VEC>(cols, ln, L, cols.alpha, al, act);
#pragma unroll
  for (int q = 0; q < VEC; ++q) part[q][0] = part[q][1] = make_double2(0, 0);
  for (int it = 0; it < L.ipb; ++it) {
    const int64_t i = ln.row(L, it);
    if (i >= L.n) break;
    const int64_t o = vidx(L, ln.k, i, c0);
    C xx[VEC], hh[VEC];
    ldv<VEC>(x + o, cs, xx);
    ldv<VEC>(h + o, cs, hh);
    if (final_) {
#pragma unroll
      for (int q = 0; q < VEC; ++q)
        if (act[q]) xx[q] = cfmaT(al[q], hh[q], xx[q]);
      stv<VEC>(x + o, cs, xx);
      continue;
    }
    C zz[VEC], ss[VEC], tt[VEC], pp[VEC], vv[VEC], rh[VEC], rr[VEC];
    ldv<VEC>(z + o, cs, zz);
    ldv<VEC>(s + o, cs, ss);
    ldv<VEC>(t + o, cs, tt);
    ldv<VEC>(p + o, cs, pp);
    ldv<VEC>(v + o, cs, vv);
    ldv<VEC>(rhat + o, cs, rh);
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      if (!act[q]) {
        rr[q] = ss[q];
        continue;
      }
      xx[q] = cfmaT(om[q], zz[q], cfmaT(al[q], hh[q], xx[q]));
      rr[q] = cfmaT(cneg(om[q]), tt[q], ss[q]);
      pp[q] = cfmaT(cneg(om[q]), vv[q], pp[q]);
      if (act[q] == 1) {
        acc_abs2(part[q][0].x, rr[q]);
        acc_bil(part[q][1], rh[q], rr[q]);
      }
    }
    stv<VEC>(x + o, cs, xx);
    stv<VEC>(r + o, cs, rr);
    stv<VEC>(p + o, cs, pp);
  }
  if (!final_) {
    const int slot[2] = {ACC_NR, ACC_RHO};
    block_reduce<VEC, 2, E>(L, ln, part, cols.acc, cols.C, slot, smem);
  }
}

// p = r + beta*p  (dMesh.m:1340)
template <class R, int VEC>
__global__ void __launch_bounds__(BS) k_update_p(Layout L, const typename CT<R>::C *__restrict__ r,
                                                 typename CT<R>::C *__restrict__ p, Cols cols, const Ctl *ctl) {
  using C = typename CT<R>::C;
  if (halted(ctl, ST_RUNNING)) return;
  if (harmonic_done(cols, blockIdx.y)) return;
  Lane ln(L);
  constexpr int E = Chunk<typename CT<R>::C>::E;
  const int c0 = ln.template col0<E>(), cs = ln.template cs<E>(L);
  C be[VEC];
  int act[VEC];
  lane_scalars<R, VEC>(cols, ln, L, cols.beta, be, act);
  for (int it = 0; it < L.ipb; ++it) {
    const int64_t i = ln.row(L, it);
    if (i >= L.n) break;
    const int64_t o = vidx(L, ln.k, i, c0);
    C rr[VEC], pp[VEC];
    ldv<VEC>(r + o, cs, rr);
    ldv<VEC>(p + o, cs, pp);
#pragma unroll
    for (int q = 0; q < VEC; ++q)
      if (act[q]) pp[q] = cfmaT(be[q], pp[q], rr[q]);
    stv<VEC>(p + o, cs, pp);
  }
}

// ------------------------------------------------ COCG (mixed inner solve)
// r = r - alpha q ; acc[NR] += |r|^2   (iterating columns)
template <class R, int VEC>
__global__ void __launch_bounds__(BS) k_update_r(Layout L, typename CT<R>::C *__restrict__ r,
                                                 const typename CT<R>::C *__restrict__ q, Cols cols,
                                                 const Ctl *ctl) {
  using C = typename CT<R>::C;
  if (halted(ctl, ST_RUNNING)) return;
  if (harmonic_done(cols, blockIdx.y)) return;
  extern __shared__ double2 smem[];
  Lane ln(L);
  constexpr int E = Chunk<typename CT<R>::C>::E;
  const int c0 = ln.template col0<E>(), cs = ln.template cs<E>(L);
  double2 part[VEC][1];
  C al[VEC];
  int act[VEC];
  lane_scalars<R, VEC>(cols, ln, L, cols.alpha, al, act);
#pragma unroll
  for (int v = 0; v < VEC; ++v) part[v][0] = make_double2(0, 0);
  for (int it = 0; it < L.ipb; ++it) {
    const int64_t i = ln.row(L, it);
    if (i >= L.n) break;
    const int64_t o = vidx(L, ln.k, i, c0);
    C rr[VEC], qq[VEC];
    ldv<VEC>(r + o, cs, rr);
    ldv<VEC>(q + o, cs, qq);
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      if (act[v] != 1) continue;
      rr[v] = cfmaT(cneg(al[v]), qq[v], rr[v]);
      acc_abs2(part[v][0].x, rr[v]);
    }
    stv<VEC>(r + o, cs, rr);
  }
  const int slot[1] = {ACC_NR};
  block_reduce<VEC, 1, E>(L, ln, part, cols.acc, cols.C, slot, smem);
}

// x = x + alpha p (columns iterating or pending: active 1 or 2), then p = z + beta p (columns
// still iterating, RUNNING state); in the FINAL state only the x update.  The x update of
// iteration k is taken here, before p changes, so p is read once per iteration.
template <class R, int VEC>
__global__ void __launch_bounds__(BS) k_update_px(Layout L, typename CT<R>::C *__restrict__ x,
                                                  typename CT<R>::C *__restrict__ p,
                                                  const typename CT<R>::C *__restrict__ z, Cols cols,
                                                  const Ctl *ctl) {
  using C = typename CT<R>::C;
  if (halted(ctl, ST_FINAL)) return;
  if (harmonic_done(cols, blockIdx.y)) return;
  const bool run = *(volatile const int *)&ctl->state == ST_RUNNING;
  Lane ln(L);
  constexpr int E = Chunk<typename CT<R>::C>::E;
  const int c0 = ln.template col0<E>(), cs = ln.template cs<E>(L);
  C al[VEC], be[VEC];
  int act[VEC], actb[VEC];
  lane_scalars<R, VEC>(cols, ln, L, cols.alpha, al, act);
  lane_scalars<R, VEC>(cols, ln, L, cols.beta, be, actb);
  bool any_p = false;
#pragma unroll
  for (int v = 0; v < VEC; ++v) any_p |= run && act[v] == 1;
  for (int it = 0; it < L.ipb; ++it) {
    const int64_t i = ln.row(L, it);
    if (i >= L.n) break;
    const int64_t o = vidx(L, ln.k, i, c0);
    C xx[VEC], pp[VEC], zz[VEC];
    ldv<VEC>(x + o, cs, xx);
    ldv<VEC>(p + o, cs, pp);
    if (any_p) ldv<VEC>(z + o, cs, zz);
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
      if (!act[v]) continue;
      xx[v] = cfmaT(al[v], pp[v], xx[v]);
      if (run && act[v] == 1) pp[v] = cfmaT(be[v], pp[v], zz[v]);
    }
    stv<VEC>(x + o, cs, xx);
    if (any_p) stv<VEC>(p + o, cs, pp);
  }
}

// ------------------------------------------------------------ scalar stages
__device__ inline bool finite2(double2 a) { return isfinite(a.x) && isfinite(a.y); }

// block-wide max of non-negative values; returns the result to all threads
__device__ double block_max(double v) {
  typedef cub::BlockReduce<double, 1024> BR;
  __shared__ typename BR::TempStorage tmp;
  __shared__ double res;
  double m = BR(tmp).Reduce(v, cub::Max());
  if (threadIdx.x == 0) res = m;
  __syncthreads();
  return res;
}

__device__ inline void freeze(Cols &c, int64_t j, int why) {
  c.active[j] = 0;
  c.status[j] = why;
  c.alpha[j] = make_double2(0, 0);
  c.omega[j] = make_double2(0, 0);
  c.beta[j] = make_double2(0, 0);
}

// after v = A h:  alpha = rho0 / (v.r0^)   (the reciprocal of alph, dMesh.m:1304)
__global__ void __launch_bounds__(1024) k_stage_alpha(Cols c, Ctl *ctl) {
  if (ctl->state != ST_RUNNING) return;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) {
    double2 d1 = c.acc[ACC_D1 * c.C + j];
    c.acc[ACC_D1 * c.C + j] = make_double2(0, 0);
    if (!c.active[j]) continue;
    double2 a = cdiv(c.rho0[j], d1);
    if (!(cabs2(d1) > 0.0) || !finite2(a) || !(cabs2(c.rho0[j]) > 0.0)) {
      freeze(c, j, DGP_COL_BREAKDOWN_RHO);
      continue;
    }
    c.alpha[j] = a;
  }
}

// after s: err = max ||s||/||r0||; below tol -> FINAL (x = x + alpha h), dMesh.m:1307-1313
__global__ void __launch_bounds__(1024) k_stage_check_s(Cols c, Ctl *ctl) {
  if (ctl->state != ST_RUNNING) return;
  double m = 0.0;
  const int stop_rule = ctl->stop_rule;
  const double tol = ctl->tol;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) {
    double ns = c.acc[ACC_NS * c.C + j].x;
    c.acc[ACC_NS * c.C + j] = make_double2(0, 0);
    if (!c.active[j]) continue;
    double e = sqrt(ns) / c.err0[j];
    if (!isfinite(e)) {
      freeze(c, j, DGP_COL_NONFINITE);
      continue;
    }
    c.err[j] = e;
    if (stop_rule == DGP_STOP_PER_COLUMN && e < c.tolc[j]) {
      // column done at s: x = x + alpha h in this iteration's update, then frozen
      c.omega[j] = make_double2(0, 0);
      c.status[j] = DGP_COL_CONVERGED;
      c.active[j] = 2;
    } else {
      m = fmax(m, e);
    }
  }
  m = block_max(m);
  if (threadIdx.x == 0) {
    ctl->max_err = m;
    if (stop_rule == DGP_STOP_MAX_ALL && m < tol) ctl->state = ST_FINAL;
  }
}

// after G t: omega = (Gt.Gs)/(Gt.Gt), dMesh.m:1325
__global__ void __launch_bounds__(1024) k_stage_omega(Cols c, Ctl *ctl) {
  if (ctl->state == ST_DONE) return;
  const bool fin = ctl->state == ST_FINAL;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) {
    double2 d2v = c.acc[ACC_D2 * c.C + j], d3 = c.acc[ACC_D3 * c.C + j];
    c.acc[ACC_D2 * c.C + j] = make_double2(0, 0);
    c.acc[ACC_D3 * c.C + j] = make_double2(0, 0);
    if (c.active[j] != 1 || fin) continue;
    double2 om = cdiv(d2v, d3);
    if (!(cabs2(d3) > 0.0) || !finite2(om) || !(cabs2(om) > 0.0)) {
      freeze(c, j, DGP_COL_BREAKDOWN_OMEGA);
      continue;
    }
    c.omega[j] = om;
  }
}

// after x, r: err = max ||r||/||r0|| (dMesh.m:1330-1335); beta, rho0 (:1337-1339)
__global__ void __launch_bounds__(1024) k_stage_check_r(Cols c, Ctl *ctl) {
  const int st = ctl->state;
  if (st == ST_DONE) return;
  double m = 0.0;
  const double tol = ctl->tol;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) {
    double nr = c.acc[ACC_NR * c.C + j].x;
    double2 rho = c.acc[ACC_RHO * c.C + j];
    c.acc[ACC_NR * c.C + j] = make_double2(0, 0);
    c.acc[ACC_RHO * c.C + j] = make_double2(0, 0);
    if (c.active[j] == 2) {  // finished at s this iteration
      c.active[j] = 0;
      continue;
    }
    if (!c.active[j] || st == ST_FINAL) continue;
    double e = sqrt(nr) / c.err0[j];
    if (!isfinite(e)) {
      freeze(c, j, DGP_COL_NONFINITE);
      continue;
    }
    c.err[j] = e;
    if (ctl->stop_rule == DGP_STOP_PER_COLUMN && e < c.tolc[j]) {
      c.active[j] = 0;
      c.status[j] = DGP_COL_CONVERGED;
      continue;
    }
    m = fmax(m, e);
    // beta = rho/rho0 * (1/(alph*om)) = (rho/rho0) * (alpha/omega)
    double2 b = cmul(cdiv(rho, c.rho0[j]), cdiv(c.alpha[j], c.omega[j]));
    if (!finite2(b) || !(cabs2(rho) > 0.0)) {
      freeze(c, j, DGP_COL_BREAKDOWN_RHO);
      continue;
    }
    c.beta[j] = b;
    c.rho0[j] = rho;
  }
  m = block_max(m);
  if (threadIdx.x == 0) {
    ctl->iters += 1;
    if (st == ST_FINAL) {
      ctl->state = ST_DONE;
      ctl->reason = 0;
    } else {
      ctl->max_err = m;
      // with the per-column rule the solve ends when no column is active (k_stage_count)
      if (ctl->stop_rule == DGP_STOP_MAX_ALL && m < tol) {
        ctl->state = ST_DONE;
        ctl->reason = 0;
      }
      if (ctl->state != ST_DONE && ctl->iters >= ctl->maxit) {
        ctl->state = ST_DONE;
        ctl->reason = 1;
      }
    }
  }
}

// count active columns; ends a per-column solve when none is left
__global__ void __launch_bounds__(1024) k_stage_count(Cols c, Ctl *ctl) {
  if (ctl->state == ST_DONE) return;
  typedef cub::BlockReduce<int, 1024> BR;
  __shared__ typename BR::TempStorage tmp;
  int a = 0;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) a += c.active[j] != 0;
  a = BR(tmp).Sum(a);
  update_hact(c);
  if (threadIdx.x == 0) {
    ctl->n_active = a;
    if (a == 0) {
      ctl->state = ST_DONE;
      ctl->reason = ctl->iters == 0 ? 2 : 0;
    }
  }
}

// COCG scalar stages.  rho0 holds rho = r.z (bilinear), alpha = rho / (p.Ap),
// beta = rho_new / rho.
__global__ void __launch_bounds__(1024) k_cocg_alpha(Cols c, Ctl *ctl) {
  if (ctl->state != ST_RUNNING) return;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) {
    double2 d1 = c.acc[ACC_D1 * c.C + j];
    c.acc[ACC_D1 * c.C + j] = make_double2(0, 0);
    if (!c.active[j]) continue;
    double2 a = cdiv(c.rho0[j], d1);
    if (!(cabs2(d1) > 0.0) || !finite2(a)) {
      freeze(c, j, DGP_COL_BREAKDOWN_RHO);
      continue;
    }
    c.alpha[j] = a;
  }
}

// after x, r: err = ||r||/||r0|| per column; stop rule and maxit as in k_stage_check_r
__global__ void __launch_bounds__(1024) k_cocg_check(Cols c, Ctl *ctl) {
  if (ctl->state != ST_RUNNING) return;
  double m = 0.0;
  const double tol = ctl->tol;
  const int stop_rule = ctl->stop_rule;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) {
    double nr = c.acc[ACC_NR * c.C + j].x;
    c.acc[ACC_NR * c.C + j] = make_double2(0, 0);
    if (!c.active[j]) continue;
    double e = sqrt(nr) / c.err0[j];
    if (!isfinite(e)) {
      freeze(c, j, DGP_COL_NONFINITE);
      continue;
    }
    c.err[j] = e;
    if (stop_rule == DGP_STOP_PER_COLUMN && e < c.tolc[j]) {
      c.active[j] = 2;  // converged: its last x update is still pending (k_update_px)
      c.status[j] = DGP_COL_CONVERGED;
      continue;
    }
    m = fmax(m, e);
  }
  m = block_max(m);
  if (threadIdx.x == 0) {
    ctl->iters += 1;
    ctl->max_err = m;
    // FINAL: the rest of this iteration applies the pending x updates only, k_cocg_count ends it
    if (stop_rule == DGP_STOP_MAX_ALL && m < tol) {
      ctl->state = ST_FINAL;
      ctl->reason = 0;
    } else if (ctl->iters >= ctl->maxit) {
      ctl->state = ST_FINAL;
      ctl->reason = 1;
    }
  }
}

// end of a COCG iteration: pending columns (x updated) are frozen, active columns counted,
// harmonic activity refreshed; FINAL or no active column -> DONE
__global__ void __launch_bounds__(1024) k_cocg_count(Cols c, Ctl *ctl) {
  const int st = ctl->state;
  if (st == ST_DONE) return;
  typedef cub::BlockReduce<int, 1024> BR;
  __shared__ typename BR::TempStorage tmp;
  int a = 0;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) {
    if (c.active[j] == 2) c.active[j] = 0;
    a += c.active[j] == 1;
  }
  a = BR(tmp).Sum(a);  // (its barrier also orders the active[] writes before update_hact)
  update_hact(c);
  if (threadIdx.x == 0) {
    ctl->n_active = a;
    if (st == ST_FINAL) {
      ctl->state = ST_DONE;
    } else if (a == 0) {
      ctl->state = ST_DONE;
      ctl->reason = ctl->iters == 0 ? 2 : 0;
    }
  }
}

// after z = G^T G r with acc[D1] = r.z: beta = (r.z) / rho (0 on the first call), rho = r.z
__global__ void __launch_bounds__(1024) k_cocg_rho(Cols c, Ctl *ctl, int first) {
  if (ctl->state != ST_RUNNING) return;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) {
    double2 d = c.acc[ACC_D1 * c.C + j];
    c.acc[ACC_D1 * c.C + j] = make_double2(0, 0);
    if (c.active[j] != 1) continue;
    const double2 b = first ? make_double2(0, 0) : cdiv(d, c.rho0[j]);
    if (!(cabs2(d) > 0.0) || !finite2(d) || !finite2(b)) {
      // r already holds this iteration's update: keep alpha so that x takes it too, then stop
      c.active[j] = 2;
      c.status[j] = DGP_COL_BREAKDOWN_RHO;
      c.beta[j] = make_double2(0, 0);
      continue;
    }
    c.beta[j] = b;
    c.rho0[j] = d;
  }
}

// --------------------------------------------------------- setup kernels
// initial state: x = 0, r = r^0 = p = b (dMesh.m:1283-1290); ||r0||^2 and r0.r0 per column.
template <class R, int VEC>
__global__ void __launch_bounds__(BS) k_init(Layout L, typename CT<R>::C *__restrict__ x,
                                             const typename CT<R>::C *__restrict__ r,
                                             typename CT<R>::C *__restrict__ rhat, typename CT<R>::C *__restrict__ p,
                                             Cols cols) {
  using C = typename CT<R>::C;
  extern __shared__ double2 smem[];
  Lane ln(L);
  constexpr int E = Chunk<typename CT<R>::C>::E;
  const int c0 = ln.template col0<E>(), cs = ln.template cs<E>(L);
  double2 part[VEC][2];
#pragma unroll
  for (int q = 0; q < VEC; ++q) part[q][0] = part[q][1] = make_double2(0, 0);
  for (int it = 0; it < L.ipb; ++it) {
    const int64_t i = ln.row(L, it);
    if (i >= L.n) break;
    const int64_t o = vidx(L, ln.k, i, c0);
    C bb[VEC], zz[VEC];
    ldv<VEC>(r + o, cs, bb);
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      zz[q] = czero<C>();
      acc_abs2(part[q][0].x, bb[q]);
      acc_bil(part[q][1], bb[q], bb[q]);
    }
    stv<VEC>(x + o, cs, zz);
    stv<VEC>(rhat + o, cs, bb);
    stv<VEC>(p + o, cs, bb);
  }
  const int slot[2] = {ACC_NR, ACC_RHO};
  block_reduce<VEC, 2, E>(L, ln, part, cols.acc, cols.C, slot, smem);
}

// err0 = ||r0||, rho0 = r0.r0, activity from the column index and norm.  Per-column targets:
// ctl->tol, or -- inside FP64 refinement, outer_err[j] = ||b_j - A X_j|| / ||b_j|| -- the
// larger of ctl->tol and the reduction the column still needs, 0.3 outer_tol / outer_err[j]
// (the last inner solve stops once the FP64 target is within reach instead of at ctl->tol)
__global__ void __launch_bounds__(1024) k_stage_init(Cols c, Ctl *ctl, int nsp, int ns,
                                                     const double *outer_err = nullptr, double outer_tol = 0.0) {
  typedef cub::BlockReduce<int, 1024> BR;
  __shared__ typename BR::TempStorage tmp;
  int a = 0;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) {
    double nr = c.acc[ACC_NR * c.C + j].x;
    double2 rho = c.acc[ACC_RHO * c.C + j];
    c.acc[ACC_NR * c.C + j] = make_double2(0, 0);
    c.acc[ACC_RHO * c.C + j] = make_double2(0, 0);
    const int s = (int)(j % nsp);
    c.err0[j] = sqrt(nr);
    c.err[j] = 1.0;
    c.tolc[j] = outer_err ? fmax(ctl->tol, 0.3 * outer_tol / outer_err[j]) : ctl->tol;
    c.rho0[j] = rho;
    c.alpha[j] = c.omega[j] = c.beta[j] = make_double2(0, 0);
    const bool act = s < ns && nr > 0.0 && isfinite(nr);
    c.active[j] = act ? 1 : 0;
    c.status[j] = act ? DGP_COL_MAXIT : (s < ns && !isfinite(nr) ? DGP_COL_NONFINITE : DGP_COL_ZERO_RHS);
    if (!act) c.err[j] = 0.0;
    a += act;
  }
  a = BR(tmp).Sum(a);  // (its barrier also orders the active[] writes before the loop below)
  update_hact(c);
  if (threadIdx.x == 0) {
    ctl->n_active = a;
    ctl->iters = 0;
    ctl->stall_ref = 0.0;
    ctl->stall_since = 0;
    ctl->loops = 0;
    ctl->max_err = a ? 1.0 : 0.0;
    ctl->state = a ? ST_RUNNING : ST_DONE;
    ctl->reason = a ? 1 : 2;
  }
}

// final statuses: active columns below tol are converged, the rest hit maxit
__global__ void __launch_bounds__(1024) k_stage_final(Cols c, Ctl *ctl) {
  const double tol = ctl->tol;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) {
    if (c.status[j] == DGP_COL_MAXIT || c.active[j]) {
      c.status[j] = (c.err[j] < tol || (ctl->reason == 0 && ctl->stop_rule == DGP_STOP_MAX_ALL))
                        ? DGP_COL_CONVERGED : DGP_COL_MAXIT;
    }
  }
}

// mixed precision: a column's status is decided by its FP64 residual
__global__ void k_status_outer(Cols c, const double *__restrict__ outer_err, double tol, int nsp, int ns) {
  int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j >= c.C) return;
  const int s = (int)(j % nsp);
  if (s >= ns) return;
  const int st = c.status[j];
  if (st == DGP_COL_BREAKDOWN_RHO || st == DGP_COL_BREAKDOWN_OMEGA || st == DGP_COL_NONFINITE) return;
  if (st == DGP_COL_ZERO_RHS) return;
  c.status[j] = outer_err[j] < tol ? DGP_COL_CONVERGED : DGP_COL_MAXIT;
}

// ------------------------------------------------ user layout <-> workspace
// dst[k][i][s] (nsp) = (T) src[k][i][s] (ns), zero padding
template <class R>
__global__ void k_pack(int64_t n, int nf, int nsp, int ns, const double2 *__restrict__ src,
                       typename CT<R>::C *__restrict__ dst) {
  const int64_t tot = (int64_t)nf * n * nsp;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(e % nsp);
    const int64_t ki = e / nsp;
    double2 v = s < ns ? src[ki * ns + s] : make_double2(0, 0);
    dst[e] = cvt<R>(v);
  }
}

template <class R>
__global__ void k_unpack(int64_t n, int nf, int nsp, int ns, const typename CT<R>::C *__restrict__ src,
                         double2 *__restrict__ dst) {
  const int64_t tot = (int64_t)nf * n * ns;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(e % ns);
    const int64_t ki = e / ns;
    dst[e] = d2(src[ki * nsp + s]);
  }
}

// point-source right-hand sides (dMesh.m:124-129): b[k][node][s] = w * fpsf[k]
template <class R>
__global__ void k_sources(int64_t n, int nf, int nsp, int ns, const int32_t *__restrict__ nodes,
                          const double *__restrict__ w, const double2 *__restrict__ fpsf,
                          typename CT<R>::C *__restrict__ b) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)nf * ns) return;
  const int k = (int)(t / ns), s = (int)(t % ns);
  for (int l = 0; l < 4; ++l) {
    const int32_t nd = nodes[4 * s + l];
    if (nd < 0 || nd >= n) continue;  // rejected on the host before the solve
    // the reference assigns (not accumulates) the 4 weights of a tet's distinct nodes
    double2 v = make_double2(w[4 * s + l] * fpsf[k].x, w[4 * s + l] * fpsf[k].y);
    b[((int64_t)k * n + nd) * nsp + s] = cvt<R>(v);
  }
}

__global__ void k_check_nodes(const int32_t *__restrict__ nodes, int ns, int64_t n, int *bad) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < 4 * ns && (nodes[t] < 0 || nodes[t] >= n)) atomicOr(bad, 1);
}

// ------------------------------------------------- mixed precision kernels
// X64[k][i][s] += x32[k][i][s] for s < ns (X64 is the caller's [nf][n][ns] buffer)
__global__ void k_accum_x(int64_t n, int nf, int nsp, int ns, const float2 *__restrict__ x32, double2 *__restrict__ X) {
  const int64_t tot = (int64_t)nf * n * ns;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
    const int s = (int)(e % ns);
    const int64_t ki = e / ns;
    float2 d = x32[ki * nsp + s];
    double2 v = X[e];
    v.x += (double)d.x;
    v.y += (double)d.y;
    X[e] = v;
  }
}

// FP64 residual r = b - A_k X (X in the caller's layout, stride ns; X = NULL: X = 0, no
// mat-vec), written as FP32 into r32 (the next inner right-hand side) with FP64 norms into
// acc[NR].  b is a dense caller
// buffer (stride ns) or the point sources (nodes, w, fpsf) generated on the fly.
template <int VEC>
__global__ void __launch_bounds__(BS) k_residual64(Layout L, int ns, const int32_t *__restrict__ rowptr,
                                                   const int32_t *__restrict__ col, const double2 *__restrict__ KM,
                                                   const double *__restrict__ omega, const double2 *__restrict__ X,
                                                   const double2 *__restrict__ Bd, const int32_t *__restrict__ snodes,
                                                   const double *__restrict__ sw, const double2 *__restrict__ fpsf,
                                                   float2 *__restrict__ r32, Cols cols) {
  extern __shared__ double2 smem[];
  int32_t *sn = reinterpret_cast<int32_t *>(smem + (size_t)WARPS * L.nsp);  // [nsp][4]
  double *swt = reinterpret_cast<double *>(sn + 4 * L.nsp);
  Lane ln(L);
  if (snodes) {
    for (int t = threadIdx.x; t < 4 * L.nsp; t += blockDim.x) {
      const int s = t / 4;
      sn[t] = s < ns ? snodes[t] : -1;
      swt[t] = s < ns ? sw[t] : 0.0;
    }
  }
  __syncthreads();
  const double om = omega[ln.k];
  const double2 fk = fpsf ? fpsf[ln.k] : make_double2(0, 0);
  double2 part[VEC][1];
#pragma unroll
  for (int q = 0; q < VEC; ++q) part[q][0] = make_double2(0, 0);
  const double2 *Xk = X ? X + (int64_t)ln.k * L.n * ns : nullptr;
  // columns of this lane: the strided mapping of the FP32 vectors (E = 2) it writes
  int scol[VEC];
#pragma unroll
  for (int q = 0; q < VEC; ++q) scol[q] = ln.template col<2>(L, q);
  for (int it = 0; it < L.ipb; ++it) {
    const int64_t i = ln.row(L, it);
    if (i >= L.n) break;
    double2 y[VEC];
#pragma unroll
    for (int q = 0; q < VEC; ++q) y[q] = make_double2(0, 0);
    const int b = X ? __ldg(rowptr + i) : 0, e = X ? __ldg(rowptr + i + 1) : 0;
    for (int p = b; p < e; ++p) {
      const int j = __ldg(col + p);
      const double2 km = __ldg(KM + p);
      const double2 a = make_double2(km.x, om * km.y);
#pragma unroll
      for (int q = 0; q < VEC; ++q)
        if (scol[q] < ns) y[q] = cfma(a, __ldg(Xk + (int64_t)j * ns + scol[q]), y[q]);
    }
    float2 out[VEC];
#pragma unroll
    for (int q = 0; q < VEC; ++q) {
      const int s = scol[q];
      double2 bv = make_double2(0, 0);
      if (s < ns) {
        if (Bd) {
          bv = Bd[((int64_t)ln.k * L.n + i) * ns + s];
        } else {
          for (int l = 0; l < 4; ++l)
            if (sn[4 * s + l] == i) bv = make_double2(swt[4 * s + l] * fk.x, swt[4 * s + l] * fk.y);
        }
      }
      double2 rr = make_double2(bv.x - y[q].x, bv.y - y[q].y);
      if (s >= ns) rr = make_double2(0, 0);
      acc_abs2(part[q][0].x, rr);
      out[q] = make_float2((float)rr.x, (float)rr.y);
    }
    stv<VEC>(r32 + vidx(L, ln.k, i, ln.template col0<2>()), ln.template cs<2>(L), out);
  }
  const int slot[1] = {ACC_NR};
  block_reduce<VEC, 1, 2>(L, ln, part, cols.acc, cols.C, slot, smem);
}

// mode 0: ||b|| per column from acc[NR]; mode 1: outer_err = ||r||/||b||, ctl->max_err = max
__global__ void __launch_bounds__(1024) k_outer_norms(Cols c, double *bnorm, double *outer_err, Ctl *ctl, int mode,
                                                      int nsp, int ns) {
  double m = 0.0;
  for (int64_t j = threadIdx.x; j < c.C; j += blockDim.x) {
    const double nr = c.acc[ACC_NR * c.C + j].x;
    c.acc[ACC_NR * c.C + j] = make_double2(0, 0);
    const int s = (int)(j % nsp);
    if (mode == 0) {
      bnorm[j] = sqrt(nr);
    } else {
      double e = (s < ns && bnorm[j] > 0) ? sqrt(nr) / bnorm[j] : 0.0;
      outer_err[j] = e;
      if (!isfinite(e)) e = INFINITY;
      m = fmax(m, e);
    }
  }
  m = block_max(m);
  if (threadIdx.x == 0 && mode == 1) ctl->max_err = m;
}

__global__ void k_cvt_km(const double *__restrict__ K, const double *__restrict__ M, const int32_t *__restrict__ col,
                         int64_t nnz, double2 *km64, Rec32 *rec, const int32_t *__restrict__ lcol) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= nnz) return;
  km64[p] = make_double2(K[p], M[p]);
  Rec32 r;
  r.col = col[p];
  r.a = (float)K[p];
  r.b = (float)M[p];
  r.pad = __int_as_float(lcol ? lcol[p] : 0);  // halo position for the tiled SpMM
  rec[p] = r;
}

__global__ void k_dfc_m(const double *__restrict__ M, double dfc, int64_t nnz, double *out) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p < nnz) out[p] = dfc * M[p];
}

// G^T values and the FP32 records of G and G^T
__global__ void k_gather_gt(const double2 *__restrict__ G, const int32_t *__restrict__ perm,
                            const int32_t *__restrict__ colG, const int32_t *__restrict__ colT, int64_t nnzG, int nf,
                            double2 *GT, Rec32 *recG, Rec32 *recGT, const int32_t *__restrict__ lcolG,
                            const int32_t *__restrict__ lcolT) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nnzG * nf) return;
  const int64_t k = t / nnzG, q = t % nnzG;
  const double2 gt = G[k * nnzG + perm[q]];
  GT[t] = gt;
  const double2 g = G[t];
  Rec32 a, b;
  a.col = colG[q];
  a.a = (float)g.x;
  a.b = (float)g.y;
  a.pad = __int_as_float(lcolG ? lcolG[q] : 0);
  b.col = colT[q];
  b.a = (float)gt.x;
  b.b = (float)gt.y;
  b.pad = __int_as_float(lcolT ? lcolT[q] : 0);
  recG[t] = a;
  recGT[t] = b;
}

__global__ void k_omega(int nf, double dfc, const int32_t *__restrict__ harm, double *om64, float *om32) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nf) {
    om64[k] = (double)harm[k] * dfc;
    om32[k] = (float)((double)harm[k] * dfc);
  }
}

// ------------------------------------------------------------ host side
inline unsigned g1(int64_t n, int bs) { return (unsigned)std::min<int64_t>(ceil_div(n, bs), 1 << 30); }

int pad_sources(int ns) {
  int p = 2;
  while (p < ns) p <<= 1;
  return p;
}

size_t red_smem(const Layout &L, int nq) { return sizeof(double2) * WARPS * L.nsp * nq; }

// ------------------------------------------------------- tiled SpMM plans
constexpr int TILE_RB = 32;                 // rows per block of the tiled SpMM
constexpr size_t TILE_SMEM_MAX = 200 * 1024;

inline int tile_sw(const SolverPlan *S) { return std::min(S->nsp, 32); }

// halo lists of the row blocks of one CSR pattern (host; once per plan)
int tiled_build(TiledPlan *T, const int32_t *d_rowptr, const int32_t *d_col, int64_t n, int64_t nnz, int rb,
                cudaStream_t st) {
  std::vector<int32_t> rp(n + 1), cl(nnz);
  DGP_CUDA(cudaMemcpyAsync(rp.data(), d_rowptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaMemcpyAsync(cl.data(), d_col, sizeof(int32_t) * nnz, cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  const int64_t nblk = ceil_div(n, (int64_t)rb);
  std::vector<int32_t> hptr(nblk + 1, 0), hcols, lcol(nnz), tmp;
  hcols.reserve((size_t)nnz / 2);
  int32_t hmax = 0, zmax = 0;
  for (int64_t b = 0; b < nblk; ++b) {
    const int64_t r0 = b * rb, r1 = std::min(n, r0 + rb);
    const int32_t p0 = rp[r0], p1 = rp[r1];
    tmp.assign(cl.begin() + p0, cl.begin() + p1);
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    for (int32_t p = p0; p < p1; ++p)
      lcol[p] = (int32_t)(std::lower_bound(tmp.begin(), tmp.end(), cl[p]) - tmp.begin());
    hcols.insert(hcols.end(), tmp.begin(), tmp.end());
    hptr[b + 1] = (int32_t)hcols.size();
    hmax = std::max(hmax, (int32_t)tmp.size());
    zmax = std::max(zmax, p1 - p0);
  }
  T->rb = rb;
  T->nblk = nblk;
  T->hmax = hmax;
  T->zmax = zmax;
  DGP_TRY(T->hptr.alloc(sizeof(int32_t) * hptr.size()));
  DGP_TRY(T->hcols.alloc(sizeof(int32_t) * std::max<size_t>(1, hcols.size())));
  DGP_TRY(T->lcol.alloc(sizeof(int32_t) * std::max<int64_t>(1, nnz)));
  DGP_CUDA(cudaMemcpyAsync(T->hptr.p, hptr.data(), sizeof(int32_t) * hptr.size(), cudaMemcpyHostToDevice, st));
  DGP_CUDA(cudaMemcpyAsync(T->hcols.p, hcols.data(), sizeof(int32_t) * hcols.size(), cudaMemcpyHostToDevice, st));
  DGP_CUDA(cudaMemcpyAsync(T->lcol.p, lcol.data(), sizeof(int32_t) * nnz, cudaMemcpyHostToDevice, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  return DGP_OK;
}

size_t tile_smem(const TiledPlan &T, int sw, int mode) {
  const size_t main = (size_t)T.hmax * sw * sizeof(float2) + (size_t)T.zmax * sizeof(Rec32);
  const size_t red = mode == 0 ? 0 : (size_t)WARPS * sw * (mode == 2 ? 2 : 1) * sizeof(double2);
  return std::max(main, red);
}

template <int MODE, int SW, class Op>
void tspmm_launch(const SolverPlan *S, const TiledPlan &T, const int32_t *rowptr, const Op &op, const float2 *X,
                  float2 *Y, const float2 *Wv, const Cols &cols, const Ctl *ctl, cudaStream_t st) {
  const TLayout L{S->n, S->nf, S->nsp, T.rb, T.hptr.as<int32_t>(), T.hcols.as<int32_t>(), rowptr};
  const dim3 grid((unsigned)T.nblk, (unsigned)S->nf, (unsigned)(S->nsp / SW));
  k_tspmm<MODE, SW, Op><<<grid, BS, tile_smem(T, SW, MODE), st>>>(L, op, X, Y, Wv, cols, ctl, T.hmax);
}

// dynamic shared-memory sizes of the three modes for every plan in Ts, checked against the device
template <int SW, class Op>
int tspmm_attrs(std::initializer_list<const TiledPlan *> Ts) {
  size_t b[3] = {0, 0, 0};
  for (const TiledPlan *T : Ts)
    for (int m = 0; m < 3; ++m) b[m] = std::max(b[m], tile_smem(*T, SW, m));
  DGP_TRY(allow_dyn_smem(k_tspmm<0, SW, Op>, b[0]));
  DGP_TRY(allow_dyn_smem(k_tspmm<1, SW, Op>, b[1]));
  DGP_TRY(allow_dyn_smem(k_tspmm<2, SW, Op>, b[2]));
  return DGP_OK;
}

// the tiled SpMM launch of sweep `what` (0 A, 1 G, 2 G^T) in mode MODE, dispatched on the source tile width
template <int MODE>
void tspmm(const SolverPlan *S, int what, const float2 *X, float2 *Y, const float2 *Wv, const Cols &cols,
           const Ctl *ctl, cudaStream_t st) {
  const float *om = (const float *)(S->omega.as<char>() + sizeof(double) * S->nf);
  const OpA32 A{S->rowptr.as<int32_t>(), S->RecA32.as<Rec32>(), om};
  const OpG32 G{S->P.rowptr.as<int32_t>(), S->RecG32.as<Rec32>(), S->nnzG};
  const OpG32 GT{S->P.rowptrT.as<int32_t>(), S->RecGT32.as<Rec32>(), S->nnzG};
  auto go = [&](auto sw) {
    constexpr int W_ = decltype(sw)::value;
    if (what == 0) tspmm_launch<MODE, W_>(S, S->tA, A.rowptr, A, X, Y, Wv, cols, ctl, st);
    else if (what == 1) tspmm_launch<MODE, W_>(S, S->tG, G.rowptr, G, X, Y, Wv, cols, ctl, st);
    else tspmm_launch<MODE, W_>(S, S->tGT, GT.rowptr, GT, X, Y, Wv, cols, ctl, st);
  };
  switch (tile_sw(S)) {
    case 2: go(std::integral_constant<int, 2>()); break;
    case 4: go(std::integral_constant<int, 4>()); break;
    case 8: go(std::integral_constant<int, 8>()); break;
    case 16: go(std::integral_constant<int, 16>()); break;
    default: go(std::integral_constant<int, 32>()); break;
  }
}

// builds the three halo plans and sets the kernels' shared-memory limits; tiled_ok = 1 when they fit
int tiled_setup(SolverPlan *S, cudaStream_t st) {
  DGP_TRY(tiled_build(&S->tA, S->rowptr.as<int32_t>(), S->col.as<int32_t>(), S->n, S->nnz, TILE_RB, st));
  DGP_TRY(tiled_build(&S->tG, S->P.rowptr.as<int32_t>(), S->P.col.as<int32_t>(), S->n, S->nnzG, TILE_RB, st));
  DGP_TRY(tiled_build(&S->tGT, S->P.rowptrT.as<int32_t>(), S->P.colT.as<int32_t>(), S->n, S->nnzG, TILE_RB, st));
  const int sw = tile_sw(S);
  size_t need = 0;
  for (const TiledPlan *T : {&S->tA, &S->tG, &S->tGT})
    for (int m = 0; m < 3; ++m) need = std::max(need, tile_smem(*T, sw, m));
  S->tiled_ok = need <= TILE_SMEM_MAX && S->nsp % sw == 0;
  if (!S->tiled_ok) return DGP_OK;
  auto attrs = [&](auto w) {
    constexpr int W_ = decltype(w)::value;
    int rc = tspmm_attrs<W_, OpA32>({&S->tA});
    if (rc == DGP_OK) rc = tspmm_attrs<W_, OpG32>({&S->tG, &S->tGT});
    return rc;
  };
  switch (sw) {
    case 2: return attrs(std::integral_constant<int, 2>());
    case 4: return attrs(std::integral_constant<int, 4>());
    case 8: return attrs(std::integral_constant<int, 8>());
    case 16: return attrs(std::integral_constant<int, 16>());
    default: return attrs(std::integral_constant<int, 32>());
  }
}

template <class R> struct Vecs {
  using C = typename CT<R>::C;
  C *x, *r, *rhat, *p, *v, *h, *s, *T1, *z, *t;
};

struct Work {
  Cols cols;
  Ctl *ctl;
  double *bnorm, *outer_err;
};

Work work_views(SolverPlan *S) {
  Work w;
  const int64_t C = S->ws_cols;
  char *b = S->scal.as<char>();
  w.cols.C = C;
  w.cols.err0 = (double *)b; b += sizeof(double) * C;
  w.cols.err = (double *)b; b += sizeof(double) * C;
  w.bnorm = (double *)b; b += sizeof(double) * C;
  w.outer_err = (double *)b; b += sizeof(double) * C;
  w.cols.tolc = (double *)b; b += sizeof(double) * C;
  w.cols.rho0 = (double2 *)b; b += sizeof(double2) * C;
  w.cols.alpha = (double2 *)b; b += sizeof(double2) * C;
  w.cols.omega = (double2 *)b; b += sizeof(double2) * C;
  w.cols.beta = (double2 *)b; b += sizeof(double2) * C;
  w.cols.acc = (double2 *)b; b += sizeof(double2) * C * NACC;
  w.cols.active = (int *)b;
  w.cols.hact = w.cols.active + C;
  w.cols.nsp = S->nsp;
  w.cols.status = S->status.as<int>();
  w.ctl = S->ctl.as<Ctl>();
  return w;
}

size_t scal_bytes(int64_t C) { return (sizeof(double) * 5 + sizeof(double2) * (4 + NACC) + 2 * sizeof(int)) * C + 256; }

// vector slots: COCG uses the first NVEC_COCG (x, r, r^ written by k_init, p, q, T, z),
// BiCGSTAB all NVEC_ALL; a slot that is not allocated yet views as NULL
constexpr int NVEC_COCG = 7, NVEC_ALL = 10;

template <class R> Vecs<R> vec_views(SolverPlan *S) {
  using C = typename CT<R>::C;
  Vecs<R> V;
  C **slots[NVEC_ALL] = {&V.x, &V.r, &V.rhat, &V.p, &V.v, &V.T1, &V.z, &V.h, &V.s, &V.t};
  for (int q = 0; q < NVEC_ALL; ++q) *slots[q] = S->vec[q].as<C>();
  return V;
}

// Workspace of precision `prec` with at least `nvec` vectors.  A change of precision
// reallocates everything; more vectors for the same precision are added without moving the
// existing ones (graphs captured on them stay valid).  The mixed solve with the COCG inner
// solver needs 7 of the 10 vectors (70 instead of 100 GB at 153k nodes x 64 x 128).
int ensure_workspace(SolverPlan *S, int prec, int nvec = NVEC_ALL) {
  const int64_t C = (int64_t)S->nf * S->nsp;
  const size_t esz = prec == DGP_PREC_FP64 ? sizeof(double2) : sizeof(float2);
  const size_t vb = esz * (size_t)C * S->n;
  if (S->ws_prec != prec) {
    for (auto &g : S->graph)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
    for (int &gi : S->graph_iters) gi = 0;
    for (auto &v : S->vec) v.release();
    DGP_TRY(S->scal.alloc(scal_bytes(C)));
    DGP_TRY(S->status.alloc(sizeof(int) * C));
    DGP_TRY(S->ctl.alloc(sizeof(Ctl)));
    DGP_CUDA(cudaMemset(S->scal.p, 0, scal_bytes(C)));
    S->ws_prec = prec;
    S->ws_cols = C;
  }
  for (int q = 0; q < nvec; ++q)
    if (!S->vec[q].p) DGP_TRY(S->vec[q].alloc(vb));
  return DGP_OK;
}

struct Layouts {
  Layout L, Ld;
};

// plain sweeps: ~64 rows per block; sweeps with dot products: 16x more rows per
// block, so each block issues fewer FP64 atomics per column
Layouts layouts_for(const SolverPlan *S, int vec, int rows = 64) {
  Layouts x;
  const int lpr = S->nsp / vec;
  const int rpw = 32 / lpr;
  const int ipb = std::max(1, rows / (WARPS * rpw));
  x.L = Layout{S->n, S->nf, S->nsp, lpr, rpw, ipb};
  // sweeps with dot products take 16x the rows per block: fewer block partials and FP64 atomics
  x.Ld = Layout{S->n, S->nf, S->nsp, lpr, rpw, ipb * 16};
  return x;
}

// SpMM layouts: rows per block from the autotuner when it has run; the complex-FP32 dot
// sweeps take tune_dot (default 4) times those rows per block and at most 32 rows per
// lane, the bound of their FP32 per-lane partial sums
Layouts spmm_layouts(const SolverPlan *S, int vec, bool fp32) {
  Layouts x = layouts_for(S, vec, (fp32 && S->tune_rows) ? S->tune_rows : 64);
  if (fp32) x.Ld.ipb = std::max(x.L.ipb, std::min(x.L.ipb * (S->tune_dot ? S->tune_dot : 4), 32));
  return x;
}

// complex values per lane: more per lane amortises each nonzero's coefficient load over more
// right-hand sides, fewer keep more rows in flight (FP64 up to 4 for register room)
inline int vec_for(const SolverPlan *S, bool fp32) {
  if (fp32 && S->tune_vec) return S->tune_vec;
  // untuned FP32 default: 4 per lane from 8 padded sources up, 2 below (the autotuner's choice
  // at 34,680 nodes x 32 harmonics for 3-64 sources; 8 per lane was 16-27 % slower)
  if (fp32) return S->nsp >= 8 ? 4 : 2;
  return std::min(S->nsp, 4);
}

dim3 grid_of(const Layout &L) { return dim3((unsigned)ceil_div(L.n, L.rows_per_block()), (unsigned)L.nf); }

// k_spmm launch with the plan's gather kind (complex FP32: S->tune_kind; FP64: kind 0)
template <class R, int VEC, int MODE, class Op>
void spmm_go(const SolverPlan *S, const Layout &L, size_t smem, cudaStream_t st, const Op &op,
             const typename CT<R>::C *X, typename CT<R>::C *Y, const typename CT<R>::C *W, const Cols &cols,
             const Ctl *ctl) {
  if constexpr (sizeof(R) == 4) {
    switch (S->tune_kind) {
      case 1: k_spmm<R, VEC, MODE, Op, 1><<<grid_of(L), BS, smem, st>>>(L, op, X, Y, W, cols, ctl); return;
      case 2: k_spmm<R, VEC, MODE, Op, 2><<<grid_of(L), BS, smem, st>>>(L, op, X, Y, W, cols, ctl); return;
      case 3: k_spmm<R, VEC, MODE, Op, 3><<<grid_of(L), BS, smem, st>>>(L, op, X, Y, W, cols, ctl); return;
      case 4:                                           // harmonic pairs for A; kind 0 for G, G^T
        if constexpr (std::is_same<Op, OpA32>::value) {
          const dim3 g((unsigned)ceil_div(L.n, L.rows_per_block()), (unsigned)ceil_div(L.nf, 2));
          k_spmm_pair<VEC, MODE><<<g, BS, smem, st>>>(L, op, X, Y, W, cols, ctl);
          return;
        }
        break;
      default: break;
    }
  }
  k_spmm<R, VEC, MODE, Op, 0><<<grid_of(L), BS, smem, st>>>(L, op, X, Y, W, cols, ctl);
}

// one BiCGSTAB iteration (dMesh.m:1295-1340) enqueued on st: KERNELS_PER_ITER launches
// lane widths: plain SpMM sweeps VS, SpMM sweeps with dot products VD, vector updates 2
constexpr int VU = 2;

// one BiCGSTAB iteration (dMesh.m:1295-1340) enqueued on st: KERNELS_PER_ITER launches
// one complex-FP32 iteration with the tiled SpMM (same kernel sequence as enqueue_iteration)
void enqueue_iteration_tiled(const SolverPlan *S, const Vecs<float> &V, const Work &W, cudaStream_t st) {
  const Layout Lu = layouts_for(S, VU).L, Lud = layouts_for(S, VU).Ld;
  Ctl *ctl = W.ctl;
  tspmm<0>(S, 1, V.p, V.T1, nullptr, W.cols, ctl, st);
  tspmm<0>(S, 2, V.T1, V.h, nullptr, W.cols, ctl, st);
  tspmm<1>(S, 0, V.h, V.v, V.rhat, W.cols, ctl, st);
  k_stage_alpha<<<1, 1024, 0, st>>>(W.cols, ctl);
  k_update_s<float, VU><<<grid_of(Lud), BS, red_smem(Lud, 1), st>>>(Lud, V.r, V.v, V.s, W.cols, ctl);
  k_stage_check_s<<<1, 1024, 0, st>>>(W.cols, ctl);
  tspmm<0>(S, 1, V.s, V.T1, nullptr, W.cols, ctl, st);
  tspmm<0>(S, 2, V.T1, V.z, nullptr, W.cols, ctl, st);
  tspmm<0>(S, 0, V.z, V.t, nullptr, W.cols, ctl, st);
  tspmm<2>(S, 1, V.t, nullptr, V.T1, W.cols, ctl, st);
  k_stage_omega<<<1, 1024, 0, st>>>(W.cols, ctl);
  k_update_xrp<float, VU><<<grid_of(Lud), BS, red_smem(Lud, 2), st>>>(Lud, V.x, V.h, V.z, V.r, V.s, V.t, V.p, V.v,
                                                                      V.rhat, W.cols, ctl);
  k_stage_check_r<<<1, 1024, 0, st>>>(W.cols, ctl);
  k_stage_count<<<1, 1024, 0, st>>>(W.cols, ctl);
  k_update_p<float, VU><<<grid_of(Lu), BS, 0, st>>>(Lu, V.r, V.p, W.cols, ctl);
}

template <class R, int VS, int VD, class OpA, class OpG>
void enqueue_iteration(const SolverPlan *S, const OpA &A, const OpG &G, const OpG &GT, const Vecs<R> &V,
                       const Work &W, cudaStream_t st) {
  const Layout Ls = spmm_layouts(S, VS, sizeof(R) == 4).L, Lsd = spmm_layouts(S, VD, sizeof(R) == 4).Ld;
  const Layout Lu = layouts_for(S, VU).L, Lud = layouts_for(S, VU).Ld;
  Ctl *ctl = W.ctl;
  if constexpr (sizeof(R) == 4) {
    if (S->tiled) {
      enqueue_iteration_tiled(S, V, W, st);
      return;
    }
  }
  // T1 = G p ; h = G^T T1                                       (:1295-1296)
  spmm_go<R, VS, 0>(S, Ls, 0, st, G, V.p, V.T1, nullptr, W.cols, ctl);
  spmm_go<R, VS, 0>(S, Ls, 0, st, GT, V.T1, V.h, nullptr, W.cols, ctl);
  // v = A h, d1 = v.r0^                                         (:1301, :1304)
  spmm_go<R, VD, 1>(S, Lsd, red_smem(Lsd, 1), st, A, V.h, V.v, V.rhat, W.cols, ctl);
  k_stage_alpha<<<1, 1024, 0, st>>>(W.cols, ctl);
  // s = r - alpha v ; ||s||                                     (:1306-1308)
  k_update_s<R, VU><<<grid_of(Lud), BS, red_smem(Lud, 1), st>>>(Lud, V.r, V.v, V.s, W.cols, ctl);
  k_stage_check_s<<<1, 1024, 0, st>>>(W.cols, ctl);
  // Gs = G s ; z = G^T Gs ; t = A z ; (G t).Gs, (G t).(G t)     (:1315-1325)
  spmm_go<R, VS, 0>(S, Ls, 0, st, G, V.s, V.T1, nullptr, W.cols, ctl);
  spmm_go<R, VS, 0>(S, Ls, 0, st, GT, V.T1, V.z, nullptr, W.cols, ctl);
  spmm_go<R, VS, 0>(S, Ls, 0, st, A, V.z, V.t, nullptr, W.cols, ctl);
  spmm_go<R, VD, 2>(S, Lsd, red_smem(Lsd, 2), st, G, V.t, nullptr, V.T1, W.cols, ctl);
  k_stage_omega<<<1, 1024, 0, st>>>(W.cols, ctl);
  // x += alpha h + om z ; r = s - om t ; p -= om v ; ||r|| ; r0^.r   (:1305, :1327-1337)
  k_update_xrp<R, VU><<<grid_of(Lud), BS, red_smem(Lud, 2), st>>>(Lud, V.x, V.h, V.z, V.r, V.s, V.t, V.p, V.v,
                                                                  V.rhat, W.cols, ctl);
  k_stage_check_r<<<1, 1024, 0, st>>>(W.cols, ctl);
  k_stage_count<<<1, 1024, 0, st>>>(W.cols, ctl);
  // p = r + beta p                                              (:1340)
  k_update_p<R, VU><<<grid_of(Lu), BS, 0, st>>>(Lu, V.r, V.p, W.cols, ctl);
}

// COCG preconditioner step: T1 = G r ; z = G^T T1 ; acc[D1] = r.z ; rho, beta.  The gather
// path takes r.z = r^T G^T G r as T1.T1 in the G sweep (no second read of r); the tiled path
// takes it as r.z in the G^T sweep.
template <class R, int VS, int VD, class OpG>
void enqueue_cocg_precond(const SolverPlan *S, const OpG &G, const OpG &GT, const Vecs<R> &V, const Work &W,
                          int first, cudaStream_t st) {
  Ctl *ctl = W.ctl;
  bool done = false;
  if constexpr (sizeof(R) == 4) {
    if (S->tiled) {
      tspmm<0>(S, 1, V.r, V.T1, nullptr, W.cols, ctl, st);
      tspmm<1>(S, 2, V.T1, V.z, V.r, W.cols, ctl, st);
      done = true;
    }
  }
  if (!done) {
    const Layout Ls = spmm_layouts(S, VS, sizeof(R) == 4).L, Lsd = spmm_layouts(S, VD, sizeof(R) == 4).Ld;
    spmm_go<R, VD, 3>(S, Lsd, red_smem(Lsd, 1), st, G, V.r, V.T1, nullptr, W.cols, ctl);
    spmm_go<R, VS, 0>(S, Ls, 0, st, GT, V.T1, V.z, nullptr, W.cols, ctl);
  }
  k_cocg_rho<<<1, 1024, 0, st>>>(W.cols, ctl, first);
}

// COCG start after k_stage_init: z0 = G^T G r0, rho = r0.z0, p = z0 (p holds r0 from k_init, finite)
template <class R, int VS, int VD, class OpG>
void enqueue_cocg_start(const SolverPlan *S, const OpG &G, const OpG &GT, const Vecs<R> &V, const Work &W,
                        cudaStream_t st) {
  const Layout Lu = layouts_for(S, VU).L;
  enqueue_cocg_precond<R, VS, VD>(S, G, GT, V, W, 1, st);
  k_update_p<R, VU><<<grid_of(Lu), BS, 0, st>>>(Lu, V.z, V.p, W.cols, W.ctl);
}

// one preconditioned COCG iteration (conjugate-orthogonal CG for the complex-symmetric A_k with
// the complex-symmetric FSAI preconditioner G^T G), KERNELS_PER_ITER_COCG launches:
//   q = A p, p.q ; alpha = rho/(p.q) ; r -= alpha q, ||r|| ; stop checks ;
//   z = G^T G r, rho' = r.z, beta = rho'/rho ; x += alpha p, p = z + beta p ; count
template <class R, int VS, int VD, class OpA, class OpG>
void enqueue_cocg(const SolverPlan *S, const OpA &A, const OpG &G, const OpG &GT, const Vecs<R> &V, const Work &W,
                  cudaStream_t st) {
  const Layout Lu = layouts_for(S, VU).L, Lud = layouts_for(S, VU).Ld;
  Ctl *ctl = W.ctl;
  bool done = false;
  if constexpr (sizeof(R) == 4) {
    if (S->tiled) {
      tspmm<1>(S, 0, V.p, V.v, V.p, W.cols, ctl, st);
      done = true;
    }
  }
  if (!done) {
    const Layout Lsd = spmm_layouts(S, VD, sizeof(R) == 4).Ld;
    spmm_go<R, VD, 1>(S, Lsd, red_smem(Lsd, 1), st, A, V.p, V.v, V.p, W.cols, ctl);
  }
  k_cocg_alpha<<<1, 1024, 0, st>>>(W.cols, ctl);
  k_update_r<R, VU><<<grid_of(Lud), BS, red_smem(Lud, 1), st>>>(Lud, V.r, V.v, W.cols, ctl);
  k_cocg_check<<<1, 1024, 0, st>>>(W.cols, ctl);
  enqueue_cocg_precond<R, VS, VD>(S, G, GT, V, W, 0, st);
  k_update_px<R, VU><<<grid_of(Lu), BS, 0, st>>>(Lu, V.x, V.p, V.z, W.cols, ctl);
  k_cocg_count<<<1, 1024, 0, st>>>(W.cols, ctl);
}

enum { ENQ_BICGSTAB = 0, ENQ_COCG = 1, ENQ_COCG_START = 2 };

template <class R, int VS>
int enqueue_for(SolverPlan *S, const Vecs<R> &V, const Work &W, cudaStream_t st, int what = ENQ_BICGSTAB) {
  // lane width of the SpMM sweeps with dot products: the FP32 sweeps keep their
  // partials in FP32 and afford the plain sweeps' width; FP64 ones cap at 4
  constexpr int VD = sizeof(R) == 4 ? VS : (VS < 4 ? VS : 4);
  const int32_t *rp = S->rowptr.as<int32_t>();
  if constexpr (sizeof(R) == 4) {
    OpA32 A{rp, S->RecA32.as<Rec32>(), (const float *)(S->omega.as<char>() + sizeof(double) * S->nf)};
    OpG32 G{S->P.rowptr.as<int32_t>(), S->RecG32.as<Rec32>(), S->nnzG};
    OpG32 GT{S->P.rowptrT.as<int32_t>(), S->RecGT32.as<Rec32>(), S->nnzG};
    if (what == ENQ_COCG) enqueue_cocg<R, VS, VD>(S, A, G, GT, V, W, st);
    else if (what == ENQ_COCG_START) enqueue_cocg_start<R, VS, VD>(S, G, GT, V, W, st);
    else enqueue_iteration<R, VS, VD>(S, A, G, GT, V, W, st);
  } else {
    OpA64 A{rp, S->col.as<int32_t>(), S->KM64.as<double2>(), S->omega.as<double>()};
    OpG64 G{S->P.rowptr.as<int32_t>(), S->P.col.as<int32_t>(), S->G64.as<double2>(), S->nnzG};
    OpG64 GT{S->P.rowptrT.as<int32_t>(), S->P.colT.as<int32_t>(), S->GT64.as<double2>(), S->nnzG};
    if (what == ENQ_COCG) enqueue_cocg<R, VS, VD>(S, A, G, GT, V, W, st);
    else if (what == ENQ_COCG_START) enqueue_cocg_start<R, VS, VD>(S, G, GT, V, W, st);
    else enqueue_iteration<R, VS, VD>(S, A, G, GT, V, W, st);
  }
  DGP_CUDA(cudaGetLastError());
  return DGP_OK;
}

// run BiCGSTAB iterations (graph-captured blocks) until the control block says done
// dispatch of enqueue_for on the plan's lane width
template <class R>
int enqueue_vec(SolverPlan *S, const Vecs<R> &V, const Work &W, cudaStream_t st, int what) {
  switch (vec_for(S, sizeof(R) == 4)) {
    case 2: return enqueue_for<R, 2>(S, V, W, st, what);
    case 4: return enqueue_for<R, 4>(S, V, W, st, what);
    default:
      if constexpr (sizeof(R) == 4) return enqueue_for<R, 8>(S, V, W, st, what);
      return DGP_OK;
  }
}

// End of one block of iterations in the device-driven loop: keep looping while the control block
// is not DONE, the iteration count is below maxit + one block (the iteration kernels stop at
// maxit themselves; this bound ends the loop even if they did not), and -- with the stall guard
// of the mixed path's inner solves -- the largest residual of the active columns halved within
// the last `patience` blocks.
__global__ void k_loop_cond(cudaGraphConditionalHandle h, Ctl *ctl, int stall_guard, int patience, int block) {
  if (threadIdx.x != 0) return;
  int cont = ctl->state != ST_DONE;
  ctl->loops += 1;
  if (cont && ctl->iters >= ctl->maxit + block) cont = 0;
  if (cont && ctl->loops > ctl->maxit + 2) cont = 0;  // blocks run without counting iterations
  if (cont && stall_guard) {
    const double e = ctl->max_err;
    if (ctl->stall_ref == 0.0 || e < 0.5 * ctl->stall_ref) {
      ctl->stall_ref = e;
      ctl->stall_since = 0;
    } else if (++ctl->stall_since >= patience) {
      cont = 0;
    }
  }
  cudaGraphSetConditional(h, cont ? 1u : 0u);
}

// Device-driven form of run_iterations: ONE graph launch whose WHILE node replays blocks of
// check_every iterations until k_loop_cond clears the condition; the host waits once for the
// control block.
template <class R>
int run_iterations_device(SolverPlan *S, const Vecs<R> &V, const Work &W, int check_every, cudaStream_t st,
                          int *iters_out, bool stall_guard, bool cocg) {
  const int gi = 3 + (sizeof(R) == 4 ? (cocg ? 2 : 1) : 0);
  const int per_iter = cocg ? KERNELS_PER_ITER_COCG : KERNELS_PER_ITER;
  const int patience = std::max(3, 40 / check_every);
  if (!S->graph[gi] || S->graph_iters[gi] != check_every) {
    if (S->graph[gi]) {
      cudaGraphExecDestroy(S->graph[gi]);
      S->graph[gi] = nullptr;
    }
    cudaGraph_t g;
    DGP_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &p);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g);
      return cuda_fail(e, "solver: conditional graph node", __FILE__, __LINE__);
    }
    cudaGraph_t body = p.conditional.phGraph_out[0];
    cudaStream_t cs;
    DGP_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    int rc = DGP_OK;
    if (e == cudaSuccess) {
      for (int q = 0; q < check_every && rc == DGP_OK; ++q)
        rc = enqueue_vec<R>(S, V, W, cs, cocg ? ENQ_COCG : ENQ_BICGSTAB);
      k_loop_cond<<<1, 32, 0, cs>>>(h, W.ctl, stall_guard ? 1 : 0, patience, check_every);
      cudaGraph_t out = nullptr;
      e = cudaStreamEndCapture(cs, &out);
    }
    cudaStreamDestroy(cs);
    if (rc == DGP_OK && e == cudaSuccess) e = cudaGraphInstantiate(&S->graph[gi], g, 0);
    cudaGraphDestroy(g);
    if (rc != DGP_OK) return rc;
    DGP_CUDA(e);
    S->graph_iters[gi] = check_every;
  }
  Ctl *hb = (Ctl *)S->h_ctl;
  DGP_CUDA(cudaGraphLaunch(S->graph[gi], st));
  DGP_CUDA(cudaMemcpyAsync(hb, W.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  count_launches((int64_t)hb->loops * (per_iter * check_every + 1));
  *iters_out = hb->iters;
  return DGP_OK;
}

template <class R>
int run_iterations(SolverPlan *S, const Vecs<R> &V, const Work &W, int check_every, int maxit, cudaStream_t st,
                   int *iters_out, bool stall_guard = false, bool cocg = false) {
  const int gi = sizeof(R) == 4 ? (cocg ? 2 : 1) : 0;
  const int per_iter = cocg ? KERNELS_PER_ITER_COCG : KERNELS_PER_ITER;
  if (check_every < 1) check_every = 1;
  if (S->device_loop) return run_iterations_device<R>(S, V, W, check_every, st, iters_out, stall_guard, cocg);
  if (!S->graph[gi] || S->graph_iters[gi] != check_every) {
    if (S->graph[gi]) {
      cudaGraphExecDestroy(S->graph[gi]);
      S->graph[gi] = nullptr;
    }
    cudaStream_t cs;
    DGP_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g;
    DGP_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    int rc = DGP_OK;
    for (int q = 0; q < check_every && rc == DGP_OK; ++q)
      rc = enqueue_vec<R>(S, V, W, cs, cocg ? ENQ_COCG : ENQ_BICGSTAB);
    cudaError_t e = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (rc != DGP_OK) return rc;
    DGP_CUDA(e);
    cudaError_t e2 = cudaGraphInstantiate(&S->graph[gi], g, 0);
    cudaGraphDestroy(g);
    DGP_CUDA(e2);
    S->graph_iters[gi] = check_every;
  }
  // two pinned mirrors of the control block: while the host waits for one block of iterations'
  // state, the next block is already queued, so the GPU never idles on the host's poll (after the
  // stop the queued block's kernels return at once)
  Ctl *hb = (Ctl *)S->h_ctl;
  for (auto &pe : S->poll_ev)
    if (!pe) DGP_CUDA(cudaEventCreateWithFlags(&pe, cudaEventDisableTiming));
  cudaEvent_t *ev = S->poll_ev;
  auto launch_block = [&](int slot) -> cudaError_t {
    cudaError_t e = cudaGraphLaunch(S->graph[gi], st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hb[slot], W.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev[slot], st);
    count_launches((int64_t)per_iter * check_every);
    return e;
  };
  auto done = [](int rc) { return rc; };
  // the device stops at maxit; the host bound only guards against a logic error
  const int64_t max_launches = maxit / check_every + 4;
  // stall guard (inner solves of the mixed path): stop when the largest residual among the
  // still-active columns has not halved for ~40 iterations -- complex-FP32 BiCGSTAB can
  // stall at its rounding floor, and the FP64 refinement that follows restarts from the
  // true residual, so stopping there loses nothing
  const int patience = std::max(3, 40 / check_every);
  double ref_err = 0.0;
  int since = 0;
  cudaError_t e = launch_block(0);
  if (e != cudaSuccess) return done(cuda_fail(e, "solver: graph launch", __FILE__, __LINE__));
  int cur = 0;
  for (int64_t launches = 1;; ++launches) {
    if (launches > max_launches) return done(fail(DGP_ERR_CUDA, "solver: control block never reached DONE"));
    e = launch_block(cur ^ 1);  // the next block of iterations, queued before this poll
    if (e == cudaSuccess) e = cudaEventSynchronize(ev[cur]);
    if (e != cudaSuccess) return done(cuda_fail(e, "solver: iteration block", __FILE__, __LINE__));
    const Ctl &h = hb[cur];
    if (h.state == ST_DONE) break;
    if (stall_guard) {
      if (ref_err == 0.0 || h.max_err < 0.5 * ref_err) {
        ref_err = h.max_err;
        since = 0;
      } else if (++since >= patience) {
        break;
      }
    }
    cur ^= 1;
  }
  // wait for the queued block (it returns at once after a stop on the device, or runs one more
  // block of iterations after a stall-guard stop) and report the final count
  e = cudaMemcpyAsync(&hb[0], W.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return done(cuda_fail(e, "solver: iteration block", __FILE__, __LINE__));
  *iters_out = hb[0].iters;
  done(DGP_OK);
  return DGP_OK;
}

int set_ctl(Ctl *d, double tol, int maxit, int stop_rule, cudaStream_t st, void *h_ctl) {
  Ctl *h = (Ctl *)h_ctl;
  std::memset(h, 0, sizeof(Ctl));
  h->tol = tol;
  h->maxit = maxit;
  h->stop_rule = stop_rule;
  // only the static fields: state/iters are set by k_stage_init
  DGP_CUDA(cudaMemcpyAsync(&d->maxit, &h->maxit, sizeof(int) * 2, cudaMemcpyHostToDevice, st));
  DGP_CUDA(cudaMemcpyAsync(&d->tol, &h->tol, sizeof(double), cudaMemcpyHostToDevice, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  return DGP_OK;
}

template <class R, int VEC>
void launch_init(const Layout &Ld, const Vecs<R> &V, const Work &W, cudaStream_t st) {
  k_init<R, VEC><<<grid_of(Ld), BS, red_smem(Ld, 2), st>>>(Ld, V.x, V.r, V.rhat, V.p, W.cols);
}

// FP64 residual sweep b - A x with the solver's lane layout for its source count
void launch_residual(SolverPlan *S, int ns, const double *d_X, const double *d_B, const int32_t *d_nodes,
                     const double *d_w, const double *d_fpsf, float2 *r32, const Work &W, cudaStream_t st) {
  const int vec = vec_for(S, false);
  const Layout Ld = layouts_for(S, vec).Ld;
  const size_t sm = red_smem(Ld, 1) + (sizeof(int32_t) + sizeof(double)) * 4 * Ld.nsp;
  if (vec == 2)
    k_residual64<2><<<grid_of(Ld), BS, sm, st>>>(Ld, ns, S->rowptr.as<int32_t>(), S->col.as<int32_t>(),
                                                 S->KM64.as<double2>(), S->omega.as<double>(), (const double2 *)d_X,
                                                 (const double2 *)d_B, d_nodes, d_w, (const double2 *)d_fpsf, r32,
                                                 W.cols);
  else
    k_residual64<4><<<grid_of(Ld), BS, sm, st>>>(Ld, ns, S->rowptr.as<int32_t>(), S->col.as<int32_t>(),
                                                 S->KM64.as<double2>(), S->omega.as<double>(), (const double2 *)d_X,
                                                 (const double2 *)d_B, d_nodes, d_w, (const double2 *)d_fpsf, r32,
                                                 W.cols);
  count_launches(1);
}

}  // namespace

SolverPlan::~SolverPlan() {
  for (auto &g : graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto &e : poll_ev)
    if (e) cudaEventDestroy(e);
  if (h_ctl) cudaFreeHost(h_ctl);
}

int solver_update(SolverPlan *S, const double *d_K, const double *d_M, cudaStream_t st) {
  const int64_t nnz = S->nnz;
  k_cvt_km<<<g1(nnz, 256), 256, 0, st>>>(d_K, d_M, S->col.as<int32_t>(), nnz, S->KM64.as<double2>(),
                                          S->RecA32.as<Rec32>(), S->tA.lcol.as<int32_t>());
  DGP_CHECK_LAUNCH();
  // FSAI of tril(K + i*k*dfc*M) for every harmonic (scratch kept in the plan: no allocation per update)
  if (!S->dfcM.p) DGP_TRY(S->dfcM.alloc(sizeof(double) * nnz));
  k_dfc_m<<<g1(nnz, 256), 256, 0, st>>>(d_M, S->dfc, nnz, S->dfcM.as<double>());
  DGP_CHECK_LAUNCH();
  DGP_TRY(fsai_factor_run(S->rowptr.as<int32_t>(), S->col.as<int32_t>(), d_K, S->dfcM.as<double>(), S->n,
                          S->P.rowptr.as<int32_t>(), S->P.col.as<int32_t>(), S->P.mmax, S->nf,
                          S->G64.as<double2>(), 1, S->nnzG, st, S->harm.as<int32_t>()));
  k_gather_gt<<<g1(S->nnzG * S->nf, 256), 256, 0, st>>>(S->G64.as<double2>(), S->P.permT.as<int32_t>(),
                                                       S->P.col.as<int32_t>(), S->P.colT.as<int32_t>(), S->nnzG,
                                                       S->nf, S->GT64.as<double2>(), S->RecG32.as<Rec32>(),
                                                       S->RecGT32.as<Rec32>(), S->tG.lcol.as<int32_t>(),
                                                       S->tGT.lcol.as<int32_t>());
  DGP_CHECK_LAUNCH();
  DGP_CUDA(cudaStreamSynchronize(st));
  return DGP_OK;
}

int solver_build(SolverPlan *S, const int32_t *d_rowptr, const int32_t *d_col, int64_t n, int64_t nnz,
                 const double *d_K, const double *d_M, double dfc, int32_t nf, int32_t ns_max,
                 const dgp_solve_opts *opts, cudaStream_t st, const int32_t *h_harm) {
  DGP_REQUIRE(n > 0 && nnz > 0 && nf > 0 && nf <= 65535, "solver: bad sizes");
  std::vector<int32_t> hl(nf);
  for (int j = 0; j < nf; ++j) {
    hl[j] = h_harm ? h_harm[j] : j;
    DGP_REQUIRE(hl[j] >= 0, "solver: harmonic indices must be >= 0");
  }
  DGP_REQUIRE(ns_max >= 1 && ns_max <= 128, "solver: 1 <= ns_max <= 128 sources per harmonic");
  DGP_REQUIRE(nnz < INT32_MAX && n < (1 << 24), "solver: nnz must fit int32 and n < 2^24");
  DGP_TRY(csr_in_range(d_rowptr, d_col, n, n, nnz, 0, "solver: pattern", st));
  S->n = n;
  S->nnz = nnz;
  S->nf = nf;
  S->ns_max = ns_max;
  S->nsp = pad_sources(ns_max);
  S->dfc = dfc;
  if (opts) S->opts = *opts; else dgp_solve_opts_default(&S->opts);
  DGP_TRY(S->rowptr.alloc(sizeof(int32_t) * (n + 1)));
  DGP_TRY(S->col.alloc(sizeof(int32_t) * nnz));
  DGP_CUDA(cudaMemcpyAsync(S->rowptr.p, d_rowptr, sizeof(int32_t) * (n + 1), cudaMemcpyDeviceToDevice, st));
  DGP_CUDA(cudaMemcpyAsync(S->col.p, d_col, sizeof(int32_t) * nnz, cudaMemcpyDeviceToDevice, st));
  DGP_TRY(S->KM64.alloc(sizeof(double2) * nnz));
  DGP_TRY(S->RecA32.alloc(sizeof(Rec32) * nnz));
  DGP_TRY(S->omega.alloc((sizeof(double) + sizeof(float)) * nf));
  DGP_TRY(S->harm.alloc(sizeof(int32_t) * nf));
  DGP_CUDA(cudaMemcpyAsync(S->harm.p, hl.data(), sizeof(int32_t) * nf, cudaMemcpyHostToDevice, st));
  k_omega<<<g1(nf, 128), 128, 0, st>>>(nf, dfc, S->harm.as<int32_t>(), S->omega.as<double>(),
                                        (float *)(S->omega.as<char>() + sizeof(double) * nf));
  DGP_CHECK_LAUNCH();
  DGP_TRY(fsai_pattern_build(&S->P, S->rowptr.as<int32_t>(), S->col.as<int32_t>(), d_K, d_M, dfc, n,
                             S->opts.fsai_cap, st));
  S->nnzG = S->P.nnzG;
  const size_t gcount = (size_t)S->nnzG * nf;
  DGP_TRY(S->G64.alloc(sizeof(double2) * gcount));
  DGP_TRY(S->GT64.alloc(sizeof(double2) * gcount));
  DGP_TRY(S->RecG32.alloc(sizeof(Rec32) * gcount));
  DGP_TRY(S->RecGT32.alloc(sizeof(Rec32) * gcount));
  DGP_CUDA(cudaMallocHost(&S->h_ctl, 2 * sizeof(Ctl)));  // two mirrors (run_iterations' pipelined polls)
  DGP_TRY(tiled_setup(S, st));
  return solver_update(S, d_K, d_M, st);
}

// FP64 reference-semantics solve (DGP_PREC_FP64)
static int solve_fp64(SolverPlan *S, const double *d_B, const int32_t *d_nodes, const double *d_w,
                      const double *d_fpsf, double *d_X, int ns, const dgp_solve_opts &o, dgp_solve_report *rep,
                      cudaStream_t st) {
  DGP_TRY(ensure_workspace(S, DGP_PREC_FP64));
  Work W = work_views(S);
  Vecs<double> V = vec_views<double>(S);
  const int vec = vec_for(S, false);
  const Layouts LL = layouts_for(S, vec);
  const size_t vbytes = sizeof(double2) * (size_t)S->ws_cols * S->n;
  // b -> r (workspace layout)
  if (d_B) {
    k_pack<double><<<g1((int64_t)S->ws_cols * S->n, 256), 256, 0, st>>>(S->n, S->nf, S->nsp, ns,
                                                                         (const double2 *)d_B, V.r);
  } else {
    DGP_CUDA(cudaMemsetAsync(V.r, 0, vbytes, st));
    k_sources<double><<<g1((int64_t)S->nf * ns, 128), 128, 0, st>>>(S->n, S->nf, S->nsp, ns, d_nodes, d_w,
                                                                      (const double2 *)d_fpsf, V.r);
  }
  DGP_CHECK_LAUNCH();
  DGP_TRY(set_ctl(W.ctl, o.tol, o.maxit, o.stop_rule, st, S->h_ctl));
  launch_init<double, VU>(layouts_for(S, VU).Ld, V, W, st);
  DGP_CHECK_LAUNCH();
  k_stage_init<<<1, 1024, 0, st>>>(W.cols, W.ctl, S->nsp, ns);
  DGP_CHECK_LAUNCH();
  int iters = 0;
  DGP_TRY(run_iterations<double>(S, V, W, o.check_every, o.maxit, st, &iters));
  k_stage_final<<<1, 1024, 0, st>>>(W.cols, W.ctl);
  DGP_CHECK_LAUNCH();
  k_unpack<double><<<g1((int64_t)S->nf * S->n * ns, 256), 256, 0, st>>>(S->n, S->nf, S->nsp, ns, V.x,
                                                                          (double2 *)d_X);
  DGP_CHECK_LAUNCH();
  // true FP64 residual of the returned solution, for the report (||b|| = ||r0|| since x0 = 0)
  DGP_CUDA(cudaMemcpyAsync(W.bnorm, W.cols.err0, sizeof(double) * W.cols.C, cudaMemcpyDeviceToDevice, st));
  DGP_CUDA(cudaMemsetAsync(W.cols.acc + ACC_NR * W.cols.C, 0, sizeof(double2) * W.cols.C, st));
  launch_residual(S, ns, d_X, d_B, d_nodes, d_w, d_fpsf, (float2 *)V.T1, W, st);
  k_outer_norms<<<1, 1024, 0, st>>>(W.cols, W.bnorm, W.outer_err, W.ctl, 1, S->nsp, ns);
  DGP_CHECK_LAUNCH();
  Ctl hc;
  DGP_CUDA(cudaMemcpyAsync(&hc, W.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  rep->iterations = iters;
  rep->refinements = 0;
  rep->max_rel_residual = hc.max_err;
  return hc.reason == 1 ? DGP_ERR_NOT_CONVERGED : DGP_OK;
}

// mixed precision: complex-FP32 inner solves (COCG, or BiCGSTAB for DGP_PREC_MIXED_BICGSTAB)
// inside FP64 iterative refinement
static int solve_mixed(SolverPlan *S, const double *d_B, const int32_t *d_nodes, const double *d_w,
                       const double *d_fpsf, double *d_X, int ns, const dgp_solve_opts &o, dgp_solve_report *rep,
                       cudaStream_t st) {
  const bool cocg = o.precision == DGP_PREC_MIXED;
  DGP_TRY(ensure_workspace(S, DGP_PREC_MIXED, cocg ? NVEC_COCG : NVEC_ALL));
  Work W = work_views(S);
  Vecs<float> V = vec_views<float>(S);
  const int vec = vec_for(S, true);
  const Layouts LL = layouts_for(S, vec);
  DGP_CUDA(cudaMemsetAsync(d_X, 0, sizeof(double2) * (size_t)S->nf * S->n * ns, st));
  DGP_CUDA(cudaMemsetAsync(W.cols.acc, 0, sizeof(double2) * W.cols.C * NACC, st));
  // r = b (x = 0, no mat-vec): ||b|| per column
  launch_residual(S, ns, nullptr, d_B, d_nodes, d_w, d_fpsf, V.r, W, st);
  k_outer_norms<<<1, 1024, 0, st>>>(W.cols, W.bnorm, W.outer_err, W.ctl, 0, S->nsp, ns);
  DGP_CHECK_LAUNCH();
  int total_iters = 0, refinements = 0;
  double max_err = 1.0;
  Ctl *h = (Ctl *)S->h_ctl;
  int status = DGP_OK;
  const int max_ref = std::max(1, o.max_refine);
  for (int ref = 0; ref < max_ref; ++ref) {
    // inner FP32 solve on the current residual (already in V.r)
    const int inner_maxit = std::max(1, o.maxit - total_iters);
    // inner columns stop individually: each column freezes at inner_tol and a harmonic whose
    // columns are all frozen drops out of every sweep (low harmonics need ~4x the iterations of
    // high ones, so this halves the inner work); the FP64 residual of every column is checked
    // against tol after each inner solve.  The stall guard of run_iterations ends inner solves
    // that stop making progress in FP32.
    DGP_TRY(set_ctl(W.ctl, o.inner_tol, inner_maxit, DGP_STOP_PER_COLUMN, st, S->h_ctl));
    launch_init<float, VU>(layouts_for(S, VU).Ld, V, W, st);
    DGP_CHECK_LAUNCH();
    k_stage_init<<<1, 1024, 0, st>>>(W.cols, W.ctl, S->nsp, ns, ref > 0 ? W.outer_err : nullptr, o.tol);
    DGP_CHECK_LAUNCH();
    if (cocg) {
      DGP_TRY(enqueue_vec<float>(S, V, W, st, ENQ_COCG_START));
      count_launches(3);
    }
    int it = 0;
    DGP_TRY(run_iterations<float>(S, V, W, o.check_every, inner_maxit, st, &it, true, cocg));
    total_iters += it;
    refinements += 1;
    // X += x32 ; r = b - A X in FP64
    k_accum_x<<<g1((int64_t)S->nf * S->n * ns, 256), 256, 0, st>>>(S->n, S->nf, S->nsp, ns, V.x, (double2 *)d_X);
    DGP_CHECK_LAUNCH();
    launch_residual(S, ns, d_X, d_B, d_nodes, d_w, d_fpsf, V.r, W, st);
    k_outer_norms<<<1, 1024, 0, st>>>(W.cols, W.bnorm, W.outer_err, W.ctl, 1, S->nsp, ns);
    DGP_CHECK_LAUNCH();
    DGP_CUDA(cudaMemcpyAsync(h, W.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaStreamSynchronize(st));
    max_err = h->max_err;
    if (max_err < o.tol) break;
    if (total_iters >= o.maxit || ref == max_ref - 1) {
      status = DGP_ERR_NOT_CONVERGED;
      break;
    }
  }
  k_status_outer<<<g1(W.cols.C, 256), 256, 0, st>>>(W.cols, W.outer_err, o.tol, S->nsp, ns);
  DGP_CHECK_LAUNCH();
  rep->iterations = total_iters;
  rep->refinements = refinements;
  rep->max_rel_residual = max_err;
  return status;
}

int solver_solve(SolverPlan *S, const double *d_B, const int32_t *d_nodes, const double *d_w, const double *d_fpsf,
                 double *d_X, int32_t ns, const dgp_solve_opts *opts, dgp_solve_report *rep, cudaStream_t st) {
  DGP_REQUIRE(ns >= 1 && ns <= S->ns_max, "solve: ns must be in 1..ns_max");
  DGP_REQUIRE(d_X, "solve: null output");
  DGP_REQUIRE(d_B || (d_nodes && d_w && d_fpsf), "solve: need a dense right-hand side or point sources");
  dgp_solve_opts o = opts ? *opts : S->opts;
  DGP_REQUIRE(o.tol > 0 && o.maxit >= 1, "solve: tol > 0 and maxit >= 1 required");
  DGP_REQUIRE(o.precision == DGP_PREC_FP64 || o.precision == DGP_PREC_MIXED || o.precision == DGP_PREC_MIXED_BICGSTAB,
              "solve: unknown precision");
  if (o.check_every < 1) o.check_every = 1;
  if (d_nodes) {
    if (!S->node_flag.p) DGP_TRY(S->node_flag.alloc(sizeof(int)));
    DGP_CUDA(cudaMemsetAsync(S->node_flag.p, 0, sizeof(int), st));
    k_check_nodes<<<g1(4 * ns, 128), 128, 0, st>>>(d_nodes, ns, S->n, S->node_flag.as<int>());
    DGP_CHECK_LAUNCH();
    int hb = 0;
    DGP_CUDA(cudaMemcpyAsync(&hb, S->node_flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaStreamSynchronize(st));
    if (hb) return fail(DGP_ERR_ARG, "solve: source node index out of range");
  }
  dgp_solve_report local{};
  dgp_solve_report *r = rep ? rep : &local;
  const int rc = o.precision == DGP_PREC_FP64 ? solve_fp64(S, d_B, d_nodes, d_w, d_fpsf, d_X, ns, o, r, st)
                                              : solve_mixed(S, d_B, d_nodes, d_w, d_fpsf, d_X, ns, o, r, st);
  if (rc != DGP_OK && rc != DGP_ERR_NOT_CONVERGED) return rc;
  // per-column statuses for the caller (harmonic-major, ns columns per harmonic)
  std::vector<int> hs((size_t)S->ws_cols);
  DGP_CUDA(cudaMemcpyAsync(hs.data(), S->status.p, sizeof(int) * S->ws_cols, cudaMemcpyDeviceToHost, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  int bad = 0;
  std::vector<int> out((size_t)S->nf * ns);
  for (int k = 0; k < S->nf; ++k)
    for (int s = 0; s < ns; ++s) {
      int v = hs[(size_t)k * S->nsp + s];
      if (v == DGP_COL_ZERO_RHS) v = DGP_COL_CONVERGED;  // x = 0 solves b = 0 exactly
      out[(size_t)k * ns + s] = v;
      bad += v != DGP_COL_CONVERGED;
    }
  r->n_not_converged = bad;
  if (r->d_status)
    DGP_CUDA(cudaMemcpyAsync(r->d_status, out.data(), sizeof(int) * out.size(), cudaMemcpyHostToDevice, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  // any column that missed tol -- maxit, a breakdown or a non-finite value -- makes the call NOT_CONVERGED
  if (rc == DGP_ERR_NOT_CONVERGED || bad > 0)
    return fail(DGP_ERR_NOT_CONVERGED, "solve: " + std::to_string(bad) + " of " + std::to_string(out.size()) +
                                           " columns did not reach tol (per-column status in the report)");
  return DGP_OK;
}

// ------------------------------------------------------ kernel timing hook
namespace {
// every column iterating (the update kernels skip frozen columns' work)
__global__ void k_all_active(Cols c) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < c.C; j += (int64_t)gridDim.x * blockDim.x)
    c.active[j] = 1;
}

template <int VEC>
void profile_launch(int which, const SolverPlan *S, const OpA32 &A, const OpG32 &G, const Vecs<float> &V,
                    const Work &W, const Ctl *ctl, cudaStream_t st) {
  const Layout L = spmm_layouts(S, VEC, true).L, Ld = spmm_layouts(S, VEC, true).Ld;
  const Layout Lu = layouts_for(S, VU).L, Lud = layouts_for(S, VU).Ld;
  switch (which) {
    case 0: spmm_go<float, VEC, 0>(S, L, 0, st, A, V.z, V.x, nullptr, W.cols, ctl); break;
    case 1: spmm_go<float, VEC, 0>(S, L, 0, st, G, V.p, V.T1, nullptr, W.cols, ctl); break;
    case 4: spmm_go<float, VEC, 1>(S, Ld, red_smem(Ld, 1), st, A, V.p, V.v, V.p, W.cols, ctl); break;
    case 5: spmm_go<float, VEC, 3>(S, Ld, red_smem(Ld, 1), st, G, V.r, V.T1, nullptr, W.cols, ctl); break;
    case 6: k_update_r<float, VU><<<grid_of(Lud), BS, red_smem(Lud, 1), st>>>(Lud, V.r, V.v, W.cols, ctl); break;
    case 7: k_update_px<float, VU><<<grid_of(Lu), BS, 0, st>>>(Lu, V.x, V.p, V.z, W.cols, ctl); break;
    case 2:
      k_update_xrp<float, VU><<<grid_of(Lud), BS, red_smem(Lud, 2), st>>>(Lud, V.x, V.h, V.z, V.r, V.s, V.t, V.p,
                                                                          V.v, V.rhat, W.cols, ctl);
      break;
    default:
      k_update_s<float, VU><<<grid_of(Lud), BS, red_smem(Lud, 1), st>>>(Lud, V.r, V.v, V.s, W.cols, ctl);
      break;
  }
}
}  // namespace

// Times one sweep kernel of the complex-FP32 iteration on the solver's own
// workspace (same shapes and launch configuration as inside the solve) with
// CUDA events on `st`, and returns its algorithmic bytes per launch.
int solver_profile(SolverPlan *S, int which, int reps, float *ms, double *bytes, cudaStream_t st) {
  DGP_REQUIRE(S->ws_prec == DGP_PREC_MIXED, "profile: run a mixed-precision solve first");
  DGP_REQUIRE(reps >= 1 && which >= 0 && which <= 7, "profile: bad arguments");
  if (which == 2 || which == 3) DGP_TRY(ensure_workspace(S, DGP_PREC_MIXED, NVEC_ALL));  // BiCGSTAB updates
  Vecs<float> V = vec_views<float>(S);
  Work W = work_views(S);
  W.cols.hact = nullptr;  // timing / checking runs sweep every harmonic
  DevBuf dctl;
  DGP_TRY(dctl.alloc(sizeof(Ctl)));
  Ctl hc{};
  hc.state = ST_RUNNING;
  hc.maxit = 1 << 30;
  DGP_CUDA(cudaMemcpyAsync(dctl.p, &hc, sizeof(Ctl), cudaMemcpyHostToDevice, st));
  Ctl *ctl = dctl.as<Ctl>();
  const int vec = vec_for(S, true);
  const float *om = (const float *)(S->omega.as<char>() + sizeof(double) * S->nf);
  OpA32 A{S->rowptr.as<int32_t>(), S->RecA32.as<Rec32>(), om};
  OpG32 G{S->P.rowptr.as<int32_t>(), S->RecG32.as<Rec32>(), S->nnzG};
  const double pass = 8.0 * (double)S->nf * S->n * S->nsp;
  auto launch = [&]() {
    switch (vec) {
      case 2: profile_launch<2>(which, S, A, G, V, W, ctl, st); break;
      case 4: profile_launch<4>(which, S, A, G, V, W, ctl, st); break;
      default: profile_launch<8>(which, S, A, G, V, W, ctl, st); break;
    }
  };
  if (which == 2 || which == 3 || which == 6 || which == 7) {  // update kernels: time full work
    k_all_active<<<g1(W.cols.C, 256), 256, 0, st>>>(W.cols);
    count_launches(1);
  }
  switch (which) {
    case 0: *bytes = 2 * pass + (double)S->nf * (16.0 * S->nnz + 4.0 * (S->n + 1)); break;
    case 1: *bytes = 2 * pass + (double)S->nf * (16.0 * S->nnzG + 4.0 * (S->n + 1)); break;
    case 2: *bytes = 11 * pass; break;
    case 4: *bytes = 3 * pass + (double)S->nf * (16.0 * S->nnz + 4.0 * (S->n + 1)); break;
    case 5: *bytes = 2 * pass + (double)S->nf * (16.0 * S->nnzG + 4.0 * (S->n + 1)); break;
    case 7: *bytes = 5 * pass; break;
    default: *bytes = 3 * pass; break;
  }
  launch();  // warm
  DGP_CHECK_LAUNCH();
  cudaEvent_t e0, e1;
  DGP_CUDA(cudaEventCreate(&e0));
  DGP_CUDA(cudaEventCreate(&e1));
  DGP_CUDA(cudaEventRecord(e0, st));
  for (int r = 0; r < reps; ++r) launch();
  DGP_CUDA(cudaEventRecord(e1, st));
  DGP_CUDA(cudaEventSynchronize(e1));
  float t = 0;
  DGP_CUDA(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  DGP_CHECK_LAUNCH();
  count_launches(reps + 1);
  DGP_CUDA(cudaMemsetAsync(W.cols.acc, 0, sizeof(double2) * W.cols.C * NACC, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  *ms = t / reps;
  return DGP_OK;
}

// ------------------------------------------------------------ autotuner
namespace {
// the complex-FP32 SpMM sweeps of one iteration (enqueue_iteration's 7 SpMM launches)
template <int VEC>
void spmm_set(const SolverPlan *S, const OpA32 &A, const OpG32 &G, const OpG32 &GT, const Vecs<float> &V,
              const Work &W, const Ctl *ctl, cudaStream_t st) {
  const Layouts LL = spmm_layouts(S, VEC, true);
  const Layout Ls = LL.L, Lsd = LL.Ld;
  // scratch vectors from the first NVEC_COCG slots only (x, r and r^ stand in for h, s and t)
  spmm_go<float, VEC, 0>(S, Ls, 0, st, G, V.p, V.T1, nullptr, W.cols, ctl);
  spmm_go<float, VEC, 0>(S, Ls, 0, st, GT, V.T1, V.x, nullptr, W.cols, ctl);
  spmm_go<float, VEC, 1>(S, Lsd, red_smem(Lsd, 1), st, A, V.x, V.v, V.rhat, W.cols, ctl);
  spmm_go<float, VEC, 0>(S, Ls, 0, st, G, V.r, V.T1, nullptr, W.cols, ctl);
  spmm_go<float, VEC, 0>(S, Ls, 0, st, GT, V.T1, V.z, nullptr, W.cols, ctl);
  spmm_go<float, VEC, 0>(S, Ls, 0, st, A, V.z, V.rhat, nullptr, W.cols, ctl);
  spmm_go<float, VEC, 2>(S, Lsd, red_smem(Lsd, 2), st, G, V.rhat, nullptr, V.T1, W.cols, ctl);
}
}  // namespace

void tspmm_set(const SolverPlan *S, const Vecs<float> &V, const Work &W, const Ctl *ctl, cudaStream_t st) {
  tspmm<0>(S, 1, V.p, V.T1, nullptr, W.cols, ctl, st);
  tspmm<0>(S, 2, V.T1, V.x, nullptr, W.cols, ctl, st);
  tspmm<1>(S, 0, V.x, V.v, V.rhat, W.cols, ctl, st);
  tspmm<0>(S, 1, V.r, V.T1, nullptr, W.cols, ctl, st);
  tspmm<0>(S, 2, V.T1, V.z, nullptr, W.cols, ctl, st);
  tspmm<0>(S, 0, V.z, V.rhat, nullptr, W.cols, ctl, st);
  tspmm<2>(S, 1, V.rhat, nullptr, V.T1, W.cols, ctl, st);
}

// deterministic test pattern in [-1, 1) for the operator self-check
__global__ void k_fill_pattern(float2 *x, int64_t n, uint32_t seed) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t h = (uint32_t)i * 2654435761u ^ seed;
  h ^= h >> 15;
  h *= 2246822519u;
  h ^= h >> 13;
  const float a = (float)(h & 0xffff) / 32768.f - 1.f, b = (float)(h >> 16) / 32768.f - 1.f;
  x[i] = make_float2(a, b);
}

// out[0] = max |a - b|, out[1] = max |b| as float bits (non-negative floats order like their bits)
__global__ void k_maxdiff(const float2 *__restrict__ a, const float2 *__restrict__ b, int64_t n, unsigned *out) {
  float d = 0.f, m = 0.f;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 u = a[i], v = b[i];
    d = fmaxf(d, fmaxf(fabsf(u.x - v.x), fabsf(u.y - v.y)));
    m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
  for (int off = 16; off > 0; off >>= 1) {
    d = fmaxf(d, __shfl_xor_sync(0xffffffffu, d, off));
    m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, __float_as_uint(d));
    atomicMax(out + 1, __float_as_uint(m));
  }
}

// Chooses the lane width (complex values per lane) and the rows per block of
// the complex-FP32 SpMM sweeps for this plan's shape by timing the seven
// SpMM launches of one iteration, with CUDA events on `st`, for every
// candidate on the plan's own workspace; keeps the fastest and drops captured
// graphs so the next solve records the new launch shapes.  The vector
// contents are scratch here (every solve re-initialises them).
int solver_autotune(SolverPlan *S, int32_t *tiled_out, int32_t *vec_out, int32_t *rows_out, float *ms_out,
                    cudaStream_t st) {
  DGP_TRY(ensure_workspace(S, DGP_PREC_MIXED, NVEC_COCG));
  Vecs<float> V = vec_views<float>(S);
  Work W = work_views(S);
  W.cols.hact = nullptr;  // timing / checking runs sweep every harmonic
  DevBuf dctl;
  DGP_TRY(dctl.alloc(sizeof(Ctl)));
  Ctl hc{};
  hc.state = ST_RUNNING;
  hc.maxit = 1 << 30;
  DGP_CUDA(cudaMemcpyAsync(dctl.p, &hc, sizeof(Ctl), cudaMemcpyHostToDevice, st));
  const Ctl *ctl = dctl.as<Ctl>();
  const float *om = (const float *)(S->omega.as<char>() + sizeof(double) * S->nf);
  OpA32 A{S->rowptr.as<int32_t>(), S->RecA32.as<Rec32>(), om};
  OpG32 G{S->P.rowptr.as<int32_t>(), S->RecG32.as<Rec32>(), S->nnzG};
  OpG32 GT{S->P.rowptrT.as<int32_t>(), S->RecGT32.as<Rec32>(), S->nnzG};
  cudaEvent_t e0, e1;
  DGP_CUDA(cudaEventCreate(&e0));
  DGP_CUDA(cudaEventCreate(&e1));
  const int32_t old_vec = S->tune_vec, old_rows = S->tune_rows, old_tiled = S->tiled, old_kind = S->tune_kind;
  S->tiled = 0;
  float best = 3.4e38f;
  int32_t bv = 0, br = 0, bk = 0;
  int launches = 0;
  int rc = DGP_OK;
  for (int kind = 0; kind < 5 && rc == DGP_OK; ++kind)
  for (int vec : {8, 4, 2}) {
    if (vec > S->nsp || S->nsp / vec > 32) continue;
    int last_ipb = -1;
    for (int rows : {32, 64, 128, 256}) {
      S->tune_vec = vec;
      S->tune_rows = rows;
      S->tune_kind = kind;
      const int ipb = spmm_layouts(S, vec, true).L.ipb;
      if (ipb == last_ipb) continue;  // same launch shape as the previous candidate
      last_ipb = ipb;
      auto run = [&]() {
        switch (vec) {
          case 2: spmm_set<2>(S, A, G, GT, V, W, ctl, st); break;
          case 4: spmm_set<4>(S, A, G, GT, V, W, ctl, st); break;
          default: spmm_set<8>(S, A, G, GT, V, W, ctl, st); break;
        }
      };
      run();  // warm
      cudaEventRecord(e0, st);
      run();
      run();
      cudaEventRecord(e1, st);
      launches += 21;
      cudaError_t e = cudaEventSynchronize(e1);
      if (e != cudaSuccess) {
        rc = cuda_fail(e, "autotune", __FILE__, __LINE__);
        break;
      }
      float t = 0;
      cudaEventElapsedTime(&t, e0, e1);
      t *= 0.5f;
      if (t < best) {
        best = t;
        bv = vec;
        br = rows;
        bk = kind;
      }
    }
    if (rc != DGP_OK) break;
  }
  int32_t bt = 0;
  if (rc == DGP_OK && S->tiled_ok) {  // the tiled SpMM as one more candidate
    S->tiled = 1;
    tspmm_set(S, V, W, ctl, st);
    cudaEventRecord(e0, st);
    tspmm_set(S, V, W, ctl, st);
    tspmm_set(S, V, W, ctl, st);
    cudaEventRecord(e1, st);
    launches += 21;
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) {
      rc = cuda_fail(e, "autotune", __FILE__, __LINE__);
    } else {
      float t = 0;
      cudaEventElapsedTime(&t, e0, e1);
      t *= 0.5f;
      if (t < best) {
        best = t;
        bt = 1;
      }
    }
    S->tiled = 0;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  count_launches(launches);
  if (rc != DGP_OK || bv == 0) {
    S->tune_vec = old_vec;
    S->tune_rows = old_rows;
    S->tiled = old_tiled;
    S->tune_kind = old_kind;
    return rc != DGP_OK ? rc : fail(DGP_ERR_UNSUPPORTED, "autotune: no launch shape fits this plan");
  }
  DGP_CHECK_LAUNCH();
  S->tune_vec = bv;
  S->tune_rows = br;
  S->tune_kind = bk;
  S->tiled = bt;
  for (auto &g : S->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  for (int &gi : S->graph_iters) gi = 0;
  DGP_CUDA(cudaMemsetAsync(W.cols.acc, 0, sizeof(double2) * W.cols.C * NACC, st));
  DGP_CUDA(cudaStreamSynchronize(st));
  if (tiled_out) *tiled_out = bt;
  if (vec_out) *vec_out = bv;
  if (rows_out) *rows_out = br;
  if (ms_out) *ms_out = best;
  return DGP_OK;
}

int solver_set_spmm(SolverPlan *S, int32_t tiled, int32_t vec, int32_t rows) {
  DGP_REQUIRE(tiled == 0 || tiled == 1, "set_spmm: tiled must be 0 or 1");
  DGP_REQUIRE(!tiled || S->tiled_ok, "set_spmm: the tiled SpMM does not fit this plan's shared memory");
  if (!tiled && vec != 0) {
    DGP_REQUIRE((vec == 2 || vec == 4 || vec == 8) && vec <= S->nsp && S->nsp / vec <= 32,
                "set_spmm: vec must be 2, 4 or 8, at most the padded source count and at least nsp/32");
    DGP_REQUIRE(rows == 0 || rows == 32 || rows == 64 || rows == 128 || rows == 256,
                "set_spmm: rows must be 0 (default), 32, 64, 128 or 256");
  }
  S->tiled = tiled;
  if (!tiled) {
    S->tune_vec = vec;
    S->tune_rows = vec ? rows : 0;
  }
  for (auto &g : S->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  for (int &gi : S->graph_iters) gi = 0;
  return DGP_OK;
}

int solver_set_spmm_kind(SolverPlan *S, int32_t kind) {
  DGP_REQUIRE(kind >= 0 && kind <= 4, "set_spmm_kind: kind must be 0, 1, 2, 3 or 4");
  S->tune_kind = kind;
  for (auto &g : S->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  for (int &gi : S->graph_iters) gi = 0;
  return DGP_OK;
}

int solver_set_device_loop(SolverPlan *S, int32_t on) {
  DGP_REQUIRE(on == 0 || on == 1, "set_device_loop: 0 (host polling) or 1 (device-driven loop)");
  S->device_loop = on;
  return DGP_OK;
}

int solver_set_dot_rows(SolverPlan *S, int32_t mult) {
  DGP_REQUIRE(mult == 0 || mult == 1 || mult == 2 || mult == 4 || mult == 8 || mult == 16,
              "set_dot_rows: multiple must be 0 (default 4), 1, 2, 4, 8 or 16");
  S->tune_dot = mult;
  for (auto &g : S->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  for (int &gi : S->graph_iters) gi = 0;
  return DGP_OK;
}

// Runs the gather and the tiled SpMM of A, G and G^T on one test pattern and
// returns the largest |difference| over the largest |value| (FP32 roundoff:
// only the summation order differs).
int solver_check_spmm(SolverPlan *S, double *max_rel, cudaStream_t st) {
  DGP_REQUIRE(max_rel, "check_spmm: null output");
  DGP_REQUIRE(S->tiled_ok, "check_spmm: the tiled SpMM does not fit this plan");
  DGP_TRY(ensure_workspace(S, DGP_PREC_MIXED, NVEC_COCG));
  Vecs<float> V = vec_views<float>(S);
  Work W = work_views(S);
  W.cols.hact = nullptr;  // timing / checking runs sweep every harmonic
  DevBuf dctl, dm;
  DGP_TRY(dctl.alloc(sizeof(Ctl)));
  DGP_TRY(dm.alloc(2 * sizeof(unsigned)));
  Ctl hc{};
  hc.state = ST_RUNNING;
  hc.maxit = 1 << 30;
  DGP_CUDA(cudaMemcpyAsync(dctl.p, &hc, sizeof(Ctl), cudaMemcpyHostToDevice, st));
  const Ctl *ctl = dctl.as<Ctl>();
  const int64_t cnt = (int64_t)S->nf * S->n * S->nsp;
  k_fill_pattern<<<g1(cnt, 256), 256, 0, st>>>(V.p, cnt, 12345u);
  const float *om = (const float *)(S->omega.as<char>() + sizeof(double) * S->nf);
  const OpA32 A{S->rowptr.as<int32_t>(), S->RecA32.as<Rec32>(), om};
  const OpG32 G{S->P.rowptr.as<int32_t>(), S->RecG32.as<Rec32>(), S->nnzG};
  const OpG32 GT{S->P.rowptrT.as<int32_t>(), S->RecGT32.as<Rec32>(), S->nnzG};
  const int gv = std::min(S->nsp, 8);  // gather kernel at its built-in shape
  auto gather = [&](auto vv, int what) {
    constexpr int VV = decltype(vv)::value;
    const Layout L = layouts_for(S, VV).L;
    if (what == 0) k_spmm<float, VV, 0><<<grid_of(L), BS, 0, st>>>(L, A, V.p, V.T1, nullptr, W.cols, ctl);
    else k_spmm<float, VV, 0><<<grid_of(L), BS, 0, st>>>(L, what == 1 ? G : GT, V.p, V.T1, nullptr, W.cols, ctl);
  };
  double worst = 0.0;
  for (int what = 0; what < 3; ++what) {
    if (gv == 2) gather(std::integral_constant<int, 2>(), what);
    else if (gv == 4) gather(std::integral_constant<int, 4>(), what);
    else gather(std::integral_constant<int, 8>(), what);
    tspmm<0>(S, what, V.p, V.x, nullptr, W.cols, ctl, st);
    DGP_CUDA(cudaMemsetAsync(dm.p, 0, 2 * sizeof(unsigned), st));
    k_maxdiff<<<1184, 256, 0, st>>>(V.x, V.T1, cnt, dm.as<unsigned>());
    unsigned h[2] = {0, 0};
    DGP_CUDA(cudaMemcpyAsync(h, dm.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaStreamSynchronize(st));
    float d, m;
    memcpy(&d, &h[0], 4);
    memcpy(&m, &h[1], 4);
    worst = std::max(worst, m > 0 ? (double)d / m : (double)d);
  }
  count_launches(3 * 3 + 1);
  DGP_CHECK_LAUNCH();
  *max_rel = worst;
  return DGP_OK;
}

// --------------------------------------------------- standalone operators
int spmm_A_f64(const int32_t *rowptr, const int32_t *col, const double2 *KM, const double *omega, int64_t n,
               int32_t nf, int32_t ns, const double2 *X, double2 *Y, cudaStream_t st) {
  DGP_REQUIRE(ns >= 2 && (ns & (ns - 1)) == 0 && ns <= 64,
              "spmm_A: ns must be a power of two in 2..64 (pad the source axis)");
  const int lpr = ns / 2, rpw = 32 / lpr;
  Layout L{n, nf, ns, lpr, rpw, std::max(1, 64 / (WARPS * rpw))};
  Cols c{};
  OpA64 A{rowptr, col, KM, omega};
  k_spmm<double, 2, 0><<<grid_of(L), BS, 0, st>>>(L, A, X, Y, nullptr, c, nullptr);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

int fsai_apply_f64(const int32_t *rowptr, const int32_t *col, const double2 *G, int64_t n, int64_t nnzG, int32_t nf,
                   int32_t ns, const double2 *X, double2 *Y, cudaStream_t st) {
  DGP_REQUIRE(ns >= 2 && (ns & (ns - 1)) == 0 && ns <= 64,
              "fsai_apply: ns must be a power of two in 2..64 (pad the source axis)");
  const int lpr = ns / 2, rpw = 32 / lpr;
  Layout L{n, nf, ns, lpr, rpw, std::max(1, 64 / (WARPS * rpw))};
  Cols c{};
  OpG64 Gop{rowptr, col, G, nnzG};
  k_spmm<double, 2, 0><<<grid_of(L), BS, 0, st>>>(L, Gop, X, Y, nullptr, c, nullptr);
  DGP_CHECK_LAUNCH();
  return DGP_OK;
}

}  // namespace dgp
