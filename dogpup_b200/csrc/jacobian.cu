// Adjoint absorption Jacobian, its time-gated form and vector-Jacobian product.
//
//   J_complex  DOGPUP/dMesh.m:206-247
//     J[m,k,v] = -(P phi_s)[v,k] (P phiA_d)[v,k] w_v / s_fpsf[k],  m <-> (s,d) by link
//   fc2tg on J (tutorials/tut_2_fluence_and_sensitivity.m:147, wghtd_LM_recon.m:61)
//     J_tg[m,g,v] = Nt 2 Re sum_k conj(gate_fc[g,k]) c~_k,  c~_0 = J_0 / 2
//   optional Rytov normalisation J_tg[m,g,v] / data_tg[m,g] (wghtd_LM_recon.m:61)
//
// Everything per voxel is folded into one complex table
//   C[g,k] = -2 Nt h_k conj(gate_fc[g,k]) / s_fpsf[k]     (h_0 = 1/2, else 1)
// so that J_tg[m,g,v] = w_v * sum_k Re(C[g,k] a_k),  a_k = (P phi_s)_k (P phiA_d)_k.
//
// P is the mesh-to-voxel interpolation (mesh.m2g, <= 8 entries per row) or the
// identity (nodal basis, P = NULL).  Output layouts follow the reference's
// memory order (MATLAB column-major [NM x NF x NV] / [NM x NG x NV]): voxel
// slowest, measurement fastest, i.e. [nv][nf][nm] and [nv][ng][nm].  The TG
// layout is J^T row-major with the measurement index g*NM + m, the K-major
// operand of the J^T W J contraction.
//
// One block per voxel (grid-stride): the block gathers P phi and P phiA for
// all harmonics and optodes into shared memory once (FP64 sums, stored as
// complex FP32), then each thread owns measurements m and accumulates all NG
// gates in registers; consecutive threads write consecutive m (coalesced).
// The time-gated form (k_jacobian_tg) blocks MT measurements per thread so that
// each gate coefficient read from shared memory feeds MT complex products.
#include <algorithm>
#include <type_traits>
#include <vector>

#include "dgp_common.cuh"
#include "dgp_internal.h"
#include "tc_common.cuh"

namespace dgp {

namespace {

constexpr int JBS = 256;
constexpr int NGMAX = 32;
constexpr int PMAX = 8;

struct JArgs {
  const int32_t *prow, *pcol;
  const double *pval;
  int64_t nv, nn;
  const double *w;           // [nv] voxel weights
  const double2 *phi, *phiA; // [nf][nn][ns], [nf][nn][nd]
  int ns, nd, nf, nm, ng;
  const int32_t *link;       // [nm][2]
};

// stage (P phi)[v] -> sh[k*cnt + o] for o < cnt optodes of field f [nf][nn][cnt]
__device__ void stage_field(const JArgs &a, int64_t v, const double2 *__restrict__ f, int cnt, float2 *sh) {
  int32_t nodes[PMAX];
  double wts[PMAX];
  int np;
  if (a.prow) {
    int b = a.prow[v], e = a.prow[v + 1];
    np = min(e - b, PMAX);
    for (int q = 0; q < np; ++q) {
      nodes[q] = a.pcol[b + q];
      wts[q] = a.pval[b + q];
    }
  } else {
    np = 1;
    nodes[0] = (int32_t)v;
    wts[0] = 1.0;
  }
  for (int t = threadIdx.x; t < a.nf * cnt; t += blockDim.x) {
    int k = t / cnt, o = t % cnt;
    double2 acc = make_double2(0, 0);
    for (int q = 0; q < np; ++q) {
      double2 x = f[((int64_t)k * a.nn + nodes[q]) * cnt + o];
      acc.x += wts[q] * x.x;
      acc.y += wts[q] * x.y;
    }
    sh[t] = make_float2((float)acc.x, (float)acc.y);
  }
}

// Complex Jacobian J[v][k][m] (double2 [nv][nf][nm]): one block per voxel, threads over m.
__global__ void __launch_bounds__(JBS) k_jacobian_complex(JArgs a, const double2 *__restrict__ fpsf_inv,
                                                          double2 *__restrict__ Jfd) {
  extern __shared__ float2 sh[];
  float2 *Ps = sh;                         // [nf][ns]
  float2 *Pd = Ps + a.nf * a.ns;           // [nf][nd]
  for (int64_t v = blockIdx.x; v < a.nv; v += gridDim.x) {
    __syncthreads();
    stage_field(a, v, a.phi, a.ns, Ps);
    stage_field(a, v, a.phiA, a.nd, Pd);
    __syncthreads();
    const double wv = a.w ? a.w[v] : 1.0;
    for (int m = threadIdx.x; m < a.nm; m += blockDim.x) {
      const int s = a.link[2 * m], d = a.link[2 * m + 1];
      for (int k = 0; k < a.nf; ++k) {
        float2 x = Ps[k * a.ns + s], y = Pd[k * a.nd + d];
        double2 p = make_double2((double)x.x * y.x - (double)x.y * y.y, (double)x.x * y.y + (double)x.y * y.x);
        double2 r = cmul(p, fpsf_inv[k]);  // -1 / s_fpsf[k]
        Jfd[((int64_t)v * a.nf + k) * a.nm + m] = make_double2(wv * r.x, wv * r.y);
      }
    }
  }
}

// Time-gated Jacobian with register blocking: a thread owns MT measurements (m = m0 + j*JBS)
// and all NGC (>= ng, zero-padded) gates of each; per harmonic it forms the MT products
// a_k(m) once and reads the gate coefficients C[k][0..NGC) as 128-bit shared loads, each
// used for MT complex products (the DFT over harmonics is 2*MT*NGC FMAs per harmonic).
template <int MT, int NGC>
__global__ void __launch_bounds__(JBS) k_jacobian_tg(JArgs a, const float2 *__restrict__ Ckg /*[nf][NGC]*/,
                                                     const double *__restrict__ rytov, float *__restrict__ Jtg) {
  extern __shared__ float2 sh[];
  float2 *Ps = sh;                         // [nf][ns]
  float2 *Pd = Ps + a.nf * a.ns;           // [nf][nd]
  // [nf][NGC], read as float4: start at an even float2 offset (16-byte aligned)
  float2 *Cs = Pd + a.nf * a.nd + ((a.nf * (a.ns + a.nd)) & 1);
  for (int t = threadIdx.x; t < a.nf * NGC; t += blockDim.x) Cs[t] = Ckg[t];
  for (int64_t v = blockIdx.x; v < a.nv; v += gridDim.x) {
    __syncthreads();
    stage_field(a, v, a.phi, a.ns, Ps);
    stage_field(a, v, a.phiA, a.nd, Pd);
    __syncthreads();
    const double wv = a.w ? a.w[v] : 1.0;
    for (int m0 = 0; m0 < a.nm; m0 += JBS * MT) {
      int sj[MT], dj[MT];
#pragma unroll
      for (int j = 0; j < MT; ++j) {
        const int m = m0 + j * JBS + threadIdx.x;
        const bool ok = m < a.nm;
        sj[j] = ok ? a.link[2 * m] : 0;
        dj[j] = ok ? a.link[2 * m + 1] : 0;
      }
      float acc[MT][NGC];
#pragma unroll
      for (int j = 0; j < MT; ++j)
#pragma unroll
        for (int g = 0; g < NGC; ++g) acc[j][g] = 0.f;
#pragma unroll 1
      for (int k = 0; k < a.nf; ++k) {
        float ar[MT], ai[MT];
#pragma unroll
        for (int j = 0; j < MT; ++j) {
          const float2 x = Ps[k * a.ns + sj[j]], y = Pd[k * a.nd + dj[j]];
          ar[j] = x.x * y.x - x.y * y.y;
          ai[j] = x.x * y.y + x.y * y.x;
        }
        const float4 *c4 = reinterpret_cast<const float4 *>(Cs + k * NGC);
#pragma unroll
        for (int g2 = 0; g2 < NGC / 2; ++g2) {
          const float4 c = c4[g2];  // (C[k][2 g2], C[k][2 g2 + 1])
#pragma unroll
          for (int j = 0; j < MT; ++j) {
            acc[j][2 * g2] = fmaf(c.x, ar[j], fmaf(-c.y, ai[j], acc[j][2 * g2]));
            acc[j][2 * g2 + 1] = fmaf(c.z, ar[j], fmaf(-c.w, ai[j], acc[j][2 * g2 + 1]));
          }
        }
      }
      // epilogue in FP32 (the output precision): w_v scaling and the Rytov division
      const float wf = (float)wv;
#pragma unroll
      for (int j = 0; j < MT; ++j) {
        const int m = m0 + j * JBS + threadIdx.x;
        if (m >= a.nm) continue;
#pragma unroll
        for (int g = 0; g < NGC; ++g) {
          if (g < a.ng) {
            float val = wf * acc[j][g];
            if (rytov) val = val / (float)rytov[(int64_t)m * a.ng + g];
            Jtg[((int64_t)v * a.ng + g) * a.nm + m] = val;
          }
        }
      }
    }
  }
}

// ------------------------------------------------------------------------------------------
// Time-gated Jacobian on the tensor cores (tcgen05, kind::tf32, split operands), nodal basis.
//
// Per voxel v the DFT over harmonics is a real GEMM over the (gate, source) x detector block:
//   J_tg[v][g][m(s,d)] = w_v Re sum_k Q[g,s,k] Pd[k][d],   Q[g,s,k] = C[g,k] Ps[k][s]
//                      = w_v sum_K' A'[(g,s)][K'] B'[d][K']
// with A' = [Re Q | -Im Q] and B' = [Re Pd | Im Pd] over K' = 2 NF, Ps / Pd the source and
// detector fields at node v.  An MMA tile is M = 128 rows (4 gates x 32 sources), K' in chunks
// of 16 harmonics ([16 real | 16 imaginary]).  Of the two ways to form the per-voxel operand
// this one builds NG x NS x NF products (the gate coefficient times the source field) instead
// of NS x ND x NF (the field products per link), and no MMA column is spent on padded gates.
//
// Split operands: FP32 values x enter as hi and lo = x - hi, hi = tf32(x) rounded (B'') or x
// with its 13 low mantissa bits cleared (A', one logic operation).  The B operand of
// each MMA is the 64 rows [B'_hi ; B'_lo] (N = 64), so two MMAs per K step, A'_hi [B'_hi ; B'_lo]
// and A'_lo [B'_hi ; B'_lo], leave (A'_hi + A'_lo) B'_hi in accumulator columns 0-31 and
// (A'_hi + A'_lo) B'_lo in columns 32-63, which the epilogue adds.  A tf32 MMA of M = 128, K = 8
// takes about the same time at N = 64 as at N = 32 on B200 (48 vs 46 cycles measured), so this
// forms the three products of a 3xTF32 scheme (and lo x lo) in 2/3 of the MMAs.
//
// Data paths.  Shared-memory bandwidth bounded earlier forms of this kernel (the A' operand
// written to shared memory and read back by every MMA: ~100 KB per stage), so here:
//   - the A' stages go from the builders' registers straight into tensor memory (tcgen05.st;
//     warp 4+q writes lanes 32q.. = the rows of gate 4t+q) and the MMAs read A' from there;
//   - the fields of the next voxel are copied into shared memory by cp.async while the current
//     one is built (completion counted on an mbarrier), and each builder keeps its source
//     fields in registers for the whole voxel.
//
// Persistent CTA (one per SM), warp-specialised, all hand-offs through mbarriers:
//   warps 0-3   epilogue: per tile, tensor memory -> hi + lo halves, w_v (and Rytov) -> J
//               (warp q reads accumulator lanes 32q.. = gate 4t+q of tile t, lane = source)
//   warps 4-11  builders: field copies, A' stages tile by tile (lane = source, warp = gate
//               within the tile x harmonic half)
//   warp 12     one thread issues the MMAs (tile by tile: every chunk of a tile, after which
//               its accumulator is complete); tensor-memory allocation
//   warps 13-14 B'' of each voxel as soon as its fields are staged (lane = detector), ahead of
//               the MMAs that need it
// Tensor memory: 2 accumulator slots of 64 columns (a tile's slot is released as soon as the
// epilogue has read it), then 3 A' stages of two chunks each (128 columns: hi 0-63, lo 64-127),
// so the MMA thread waits once per 16 MMAs (an mbarrier wait right after a burst of MMAs costs
// a few hundred cycles on B200).  Every mbarrier
// wait is bounded: a timeout sets err, raises the abort flag that every role polls, and the
// MMA thread waits (bounded) for all of its MMAs before the tensor memory is freed.
constexpr int T2_EPI = 4, T2_BLD = 8, T2_BB = 2;    // epilogue, A' builder, B'' builder warps
constexpr int T2_THREADS = 32 * (T2_EPI + T2_BLD + 1 + T2_BB);
constexpr int T2_BT = 32 * T2_BLD;                 // builder threads
constexpr int T2_NSLOT = 2;                        // accumulator slots (64 columns each)
constexpr int T2_NST = 3;                          // A' stages in tensor memory (2 chunks, 128 columns each)
constexpr uint32_t T2_ACOL = 64u * T2_NSLOT;       // first A' column
constexpr int T2_BCH = 2 * 32 * 128;               // one chunk of B'': 32 hi rows, then 32 lo rows
constexpr uint32_t T2_IDESC = tc::idesc(2, 2, 128, 64);

struct T2Layout {
  uint32_t b_off, f_off, c_off, l_off, bytes;      // shared memory, from the 1 KB-aligned base
  uint32_t fbuf;                                   // bytes of one voxel's staged fields
  int nch, ntile, nkp;
};

__host__ __device__ inline T2Layout t2_layout(int nf, int ng) {
  T2Layout L;
  L.nch = (nf + 15) / 16;
  L.ntile = (ng + 3) / 4;
  L.nkp = 16 * L.nch;
  L.fbuf = (uint32_t)(2 * 32 * 16 * L.nkp);                      // [2 fields][NKP][32] complex FP64
  L.b_off = 0;
  L.f_off = L.b_off + 2 * L.nch * T2_BCH;                        // two voxels' staged fields
  L.c_off = L.f_off + 2 * L.fbuf;                                // gate table [4 NTILE][NKP] float2
  L.l_off = L.c_off + (uint32_t)(8 * 4 * L.ntile * L.nkp);        // link lookup [32][32] int
  L.bytes = L.l_off + 4 * 32 * 32;
  return L;
}

// cp.async copies of voxel v's fields into a staging buffer [2][NKP][32] (source, then detector;
// zero past NF and past the optode counts): builder thread bt copies elements bt + 256 q
__device__ inline void t2_stage_fields(const JArgs &a, int64_t v, int nkp, unsigned char *dst, int bt) {
  const int per = nkp * 32;
  for (int e = bt; e < 2 * per; e += T2_BT) {
    const bool det = e >= per;
    const int r = det ? e - per : e, k = r >> 5, o = r & 31, cnt = det ? a.nd : a.ns;
    const double2 *f = det ? a.phiA : a.phi;
    const bool ok = o < cnt && k < a.nf;
    tc::cp_async16(dst + 16 * (size_t)e, ok ? f + ((int64_t)k * a.nn + v) * cnt + o : f, ok);
  }
}

// x -> (tf32(x), tf32(x - tf32(x))) for 4 values, stored as 16-byte chunks of the hi and lo images
__device__ inline void st_split4(unsigned char *hi, unsigned char *lo, uint32_t off, const float (&x)[4]) {
  float h[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    h[i] = tc::to_tf32(x[i]);
    l[i] = tc::to_tf32(x[i] - h[i]);
  }
  *reinterpret_cast<float4 *>(hi + off) = make_float4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<float4 *>(lo + off) = make_float4(l[0], l[1], l[2], l[3]);
}

__global__ void __launch_bounds__(T2_THREADS, 1) k_jacobian_tg_tc(JArgs a, const float2 *__restrict__ C /*[ng][nf]*/,
                                                                 const double *__restrict__ rytov, int dense,
                                                                 float *__restrict__ Jtg, int *err) {
  extern __shared__ __align__(1024) unsigned char t2_raw[];
  __shared__ __align__(8) uint64_t full[T2_NST], empty[T2_NST], bfull[2], bempty[2], fready[2], fdone[2];
  __shared__ __align__(8) uint64_t tfull[T2_NSLOT], tempty[T2_NSLOT], done;
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(t2_raw) + 1023) & ~uintptr_t(1023));
  const T2Layout L = t2_layout(a.nf, a.ng);
  float2 *Ct = reinterpret_cast<float2 *>(sm + L.c_off);
  int *lk = reinterpret_cast<int *>(sm + L.l_off);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  constexpr unsigned FULL = 0xffffffffu;
  volatile int *abort_v = &abort_flag;

  if (tid == 0) {
    for (int i = 0; i < T2_NST; ++i) {
      tc::mbar_init(&full[i], T2_BLD);                 // one arrival per builder warp
      tc::mbar_init(&empty[i], 1);
    }
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&bfull[b], T2_BB);
      tc::mbar_init(&bempty[b], 1);
      tc::mbar_init(&fready[b], T2_BT);                // one cp.async arrival per builder thread
      tc::mbar_init(&fdone[b], T2_BLD + T2_BB);        // readers of a staged voxel's fields
    }
    for (int q = 0; q < T2_NSLOT; ++q) {
      tc::mbar_init(&tfull[q], 1);
      tc::mbar_init(&tempty[q], T2_EPI);
    }
    tc::mbar_init(&done, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == T2_EPI + T2_BLD) tc::tmem_alloc(&tmem_slot, 512);
  for (int t = tid; t < 4 * L.ntile * L.nkp; t += T2_THREADS) {
    const int g = t / L.nkp, k = t % L.nkp;
    Ct[t] = (g < a.ng && k < a.nf) ? C[g * a.nf + k] : make_float2(0.f, 0.f);
  }
  for (int t = tid; t < 32 * 32; t += T2_THREADS) lk[t] = -1;
  __syncthreads();
  if (!dense)
    for (int m = tid; m < a.nm; m += T2_THREADS) lk[a.link[2 * m] * 32 + a.link[2 * m + 1]] = m;  // unique links
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;

  if (warp == T2_EPI + T2_BLD) {
    // ---------------------------------------------------------------- MMA issue (one thread)
    if (lane == 0) {
      uint32_t st_idx = 0, tl_idx = 0;
      int i = 0;
      bool ok = true;
      for (int64_t v = blockIdx.x; v < a.nv && ok; v += gridDim.x, ++i) {
        if (*abort_v) break;
        const int buf = i & 1;
        ok = tc::mbar_wait(&bfull[buf], (i >> 1) & 1);
        tc::fence_after_sync();
        // B'' descriptors: one per chunk, K steps of 32 bytes = +2 in the descriptor's address field
        const uint64_t bdesc0 = tc::sdesc_k_sw128(tc::smem_u32(sm + L.b_off + buf * L.nch * T2_BCH));
        for (int t = 0; t < L.ntile && ok; ++t, ++tl_idx) {
          const uint32_t slot = tl_idx % T2_NSLOT, use = tl_idx / T2_NSLOT;
          if (use >= 1) ok = tc::mbar_wait(&tempty[slot], (use - 1) & 1);   // the epilogue has read it
          tc::fence_after_sync();
          const uint32_t d_tm = tmem + 64u * slot;
          // one wait per tile: on its last stage.  Every builder warp fills a tile's stages in
          // order and its arrival on a stage's barrier releases all of its earlier writes, so the
          // last stage's completion covers the tile's earlier stages too (an mbarrier wait right
          // after a burst of MMAs costs a few hundred cycles).
          {
            const int nst_tile = (L.nch + 1) / 2;
            const uint32_t sl = st_idx + (uint32_t)nst_tile - 1u;
            ok = tc::mbar_wait(&full[sl % T2_NST], (sl / T2_NST) & 1);
            tc::fence_after_sync();
          }
          for (int c0 = 0; c0 < L.nch && ok; c0 += 2) {   // a stage = chunks c0, c0 + 1
            const uint32_t s = st_idx % T2_NST;
            for (int cc = 0; cc < 2 && c0 + cc < L.nch; ++cc) {
              const int c = c0 + cc;
              const uint32_t ah = tmem + T2_ACOL + 128u * s + 32u * cc, al = ah + 64u;   // A' in tensor memory
              const uint64_t bd = bdesc0 + (uint64_t)((c * T2_BCH) >> 4);             // B'' = [hi ; lo] rows
              tc::umma_tf32_ts<T2_IDESC>(d_tm, ah, bd, c ? 1u : 0u);
              tc::umma_tf32_ts<T2_IDESC>(d_tm, al, bd, 1u);
#pragma unroll
              for (int kk = 1; kk < 4; ++kk) {         // K = 8 tf32: 8 columns of A', 32 bytes of B''
                tc::umma_tf32_ts<T2_IDESC>(d_tm, ah + 8u * kk, bd + 2u * kk, 1u);
                tc::umma_tf32_ts<T2_IDESC>(d_tm, al + 8u * kk, bd + 2u * kk, 1u);
              }
            }
            tc::umma_commit(&empty[s]);
            ++st_idx;
          }
          if (ok) tc::umma_commit(&tfull[slot]);
        }
        if (ok) tc::umma_commit(&bempty[buf]);
      }
      if (!ok) {
        atomicOr(err, 4);
        *abort_v = 1;
      }
      tc::umma_commit(&done);                            // arrives once every MMA issued has completed
      if (!tc::mbar_wait(&done, 0)) atomicOr(err, 4);
    }
    __syncwarp();
  } else if (warp > T2_EPI + T2_BLD) {
    // ---------------------------------------------------------------- B'' builders
    // Voxel i's detector operand into buffer i % 2 as soon as its fields are staged (fready) and
    // the MMAs of voxel i - 2 are done with the buffer (bempty): warp w takes the 8-harmonic
    // blocks p = w, w + 2, .. (chunk p / 2, half p % 2), lane = detector.
    const int w = warp - (T2_EPI + T2_BLD + 1);
    unsigned char *fst = sm + L.f_off;
    int i = 0;
    bool fail = false;
    for (int64_t v = blockIdx.x; v < a.nv; v += gridDim.x, ++i) {
      if (__any_sync(FULL, *abort_v != 0)) break;
      const int bj = i & 1;
      if (!__all_sync(FULL, tc::mbar_wait(&fready[bj], (i >> 1) & 1)) ||
          (i >= 2 && !__all_sync(FULL, tc::mbar_wait(&bempty[bj], ((i >> 1) - 1) & 1)))) {
        fail = true;
        break;
      }
      const double2 *fd = reinterpret_cast<const double2 *>(fst + bj * L.fbuf) + L.nkp * 32;
      unsigned char *bb = sm + L.b_off + bj * L.nch * T2_BCH;
      for (int p = w; p < 2 * L.nch; p += T2_BB) {
        float re[8], im[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const double2 y = fd[(8 * p + q) * 32 + lane];
          re[q] = (float)y.x;
          im[q] = (float)y.y;
        }
        unsigned char *bh = bb + (p >> 1) * T2_BCH;
        const float r0[4] = {re[0], re[1], re[2], re[3]}, r1[4] = {re[4], re[5], re[6], re[7]};
        const float i0[4] = {im[0], im[1], im[2], im[3]}, i1[4] = {im[4], im[5], im[6], im[7]};
        const int h = p & 1;                             // hi rows 0-31, lo rows 32-63
        st_split4(bh, bh + 4096, tc::sw128_chunk(lane, 2 * h + 0), r0);
        st_split4(bh, bh + 4096, tc::sw128_chunk(lane, 2 * h + 1), r1);
        st_split4(bh, bh + 4096, tc::sw128_chunk(lane, 4 + 2 * h + 0), i0);
        st_split4(bh, bh + 4096, tc::sw128_chunk(lane, 4 + 2 * h + 1), i1);
      }
      tc::fence_async_smem();                            // B'' -> async proxy
      __syncwarp();
      if (lane == 0) {
        tc::mbar_arrive(&bfull[bj]);
        tc::mbar_arrive(&fdone[bj]);
      }
    }
    if (fail && lane == 0) {
      atomicOr(err, 32);
      *abort_v = 1;
    }
  } else if (warp >= T2_EPI) {
    // ---------------------------------------------------------------- builders
    // Per voxel i (staging buffer i % 2): copy voxel i+1's fields into the other buffer once
    // every reader of voxel i-1's is done with them (fdone), wait for voxel i's copies (fready),
    // read this thread's source fields into registers (harmonics 16 c + 8 half + j), then build
    // the A' stages tile by tile into tensor memory.  Waits are warp-uniform.
    const int bt = tid - 32 * T2_EPI, bw = bt >> 5, gl = bw & 3, half = bw >> 2, s = lane;
    unsigned char *fst = sm + L.f_off;
    int64_t v = blockIdx.x;
    if (v < a.nv) t2_stage_fields(a, v, L.nkp, fst, bt);
    tc::cp_async_arrive(&fready[0]);
    uint32_t st_idx = 0;
    int i = 0;
    bool fail = false;
    for (; v < a.nv && !fail; v += gridDim.x, ++i) {
      if (__any_sync(FULL, *abort_v != 0)) break;
      const int buf = i & 1;
      const int64_t vn = v + gridDim.x;
      if (vn < a.nv) {
        if (i >= 1 && !__all_sync(FULL, tc::mbar_wait(&fdone[buf ^ 1], ((i - 1) >> 1) & 1))) {
          fail = true;
          break;
        }
        t2_stage_fields(a, vn, L.nkp, fst + (buf ^ 1) * L.fbuf, bt);
        tc::cp_async_arrive(&fready[buf ^ 1]);
      }
      if (!__all_sync(FULL, tc::mbar_wait(&fready[buf], (i >> 1) & 1))) {
        fail = true;
        break;
      }
      const double2 *fs = reinterpret_cast<const double2 *>(fst + buf * L.fbuf);
      float pr[4][8], pi[4][8];
#pragma unroll
      for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const double2 y = c < L.nch ? fs[(16 * c + 8 * half + j) * 32 + s] : make_double2(0.0, 0.0);
          pr[c][j] = (float)y.x;
          pi[c][j] = (float)y.y;
        }
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(&fdone[buf]);
      for (int t = 0; t < L.ntile && !fail; ++t) {
#pragma unroll
        for (int c0 = 0; c0 < 4; c0 += 2) {             // a stage = chunks c0, c0 + 1
          if (c0 >= L.nch || fail) break;
          const uint32_t si = st_idx % T2_NST;
          if (st_idx >= T2_NST && !__all_sync(FULL, tc::mbar_wait(&empty[si], ((st_idx / T2_NST) - 1) & 1))) {
            fail = true;
            break;
          }
          tc::fence_after_sync();                        // after the MMAs that read this stage
#pragma unroll
          for (int cc = 0; cc < 2; ++cc) {
            const int c = c0 + cc;
            if (c >= L.nch) break;
            const float2 *cg = Ct + (4 * t + gl) * L.nkp + 16 * c + 8 * half;
            float hr[8], lr[8], hm[8], lm[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
              const float2 q = cg[j];
              const float qr = q.x * pr[c][j] - q.y * pi[c][j], qi = -(q.x * pi[c][j] + q.y * pr[c][j]);
              // hi = x with the 13 low mantissa bits cleared (a TF32 value), lo = x - hi (exact);
              // the MMA reads lo as TF32 too, which drops ~2^-22 of x
              hr[j] = __uint_as_float(__float_as_uint(qr) & 0xffffe000u);
              lr[j] = qr - hr[j];
              hm[j] = __uint_as_float(__float_as_uint(qi) & 0xffffe000u);
              lm[j] = qi - hm[j];
            }
            // row gl * 32 + s = lane s of this warp's quadrant; chunk cc of the stage: K' = 8 half + j
            // (real), 16 + 8 half + j (imaginary); lo 64 columns after hi
            const uint32_t tq = tmem + ((uint32_t)(32 * gl) << 16) + T2_ACOL + 128u * si + 32u * cc + 8u * half;
            tc::tmem_st8(tq, hr);
            tc::tmem_st8(tq + 16u, hm);
            tc::tmem_st8(tq + 64u, lr);
            tc::tmem_st8(tq + 80u, lm);
          }
          tc::tmem_wait_st();                            // the stores have landed, then
          tc::fence_before_sync();                       // ordered before the arrival
          __syncwarp();
          if (lane == 0) tc::mbar_arrive(&full[si]);
          ++st_idx;
        }
      }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");    // no copy outlives the kernel
    if (fail && lane == 0) {
      atomicOr(err, 8);
      *abort_v = 1;
    }
  } else {
    // ---------------------------------------------------------------- epilogue
    const int gl = warp, s = lane;
    uint32_t tl_idx = 0;
    bool ok = true;
    for (int64_t v = blockIdx.x; v < a.nv && ok; v += gridDim.x) {
      if (__any_sync(FULL, *abort_v != 0)) break;
      const float wv = (float)(a.w ? a.w[v] : 1.0);
      for (int t = 0; t < L.ntile; ++t, ++tl_idx) {
        const uint32_t slot = tl_idx % T2_NSLOT, use = tl_idx / T2_NSLOT;
        ok = __all_sync(FULL, tc::mbar_wait(&tfull[slot], use & 1));
        if (!ok) {
          if (lane == 0) {
            atomicOr(err, 16);
            *abort_v = 1;
          }
          break;
        }
        tc::fence_after_sync();
        uint32_t r[32], q[32];
        const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16) + 64u * slot;
        tc::tmem_ld32(ta, r);                            // (A_hi + A_lo) B_hi
        tc::tmem_ld32(ta + 32u, q);                      // (A_hi + A_lo) B_lo
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&tempty[slot]);
        const int g = 4 * t + gl;
        if (g >= a.ng || s >= a.ns) continue;
        float *row = Jtg + ((int64_t)v * a.ng + g) * a.nm;
        if (dense == 2) {                                // m = s nd + d, nd and nm multiples of 4
          float4 *dst = reinterpret_cast<float4 *>(row + s * a.nd);
#pragma unroll
          for (int d4 = 0; d4 < 8; ++d4)
            if (4 * d4 < a.nd) {
              const int d = 4 * d4;
              dst[d4] = make_float4(wv * (__uint_as_float(r[d]) + __uint_as_float(q[d])),
                                    wv * (__uint_as_float(r[d + 1]) + __uint_as_float(q[d + 1])),
                                    wv * (__uint_as_float(r[d + 2]) + __uint_as_float(q[d + 2])),
                                    wv * (__uint_as_float(r[d + 3]) + __uint_as_float(q[d + 3])));
            }
        } else {
#pragma unroll
          for (int d = 0; d < 32; ++d) {
            if (d >= a.nd) break;
            const int m = dense ? s * a.nd + d : lk[s * 32 + d];
            if (m < 0) continue;
            float val = wv * (__uint_as_float(r[d]) + __uint_as_float(q[d]));
            if (rytov) val = val / (float)rytov[(int64_t)m * a.ng + g];
            row[m] = val;
          }
        }
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == T2_EPI + T2_BLD) tc::tmem_free(tmem, 512);
}

// ------------------------------------------------------------------------------------------
// Vector-Jacobian product on the tensor cores.
//
//   vjp[v] = w_v Re sum_k sum_s (P phi)_k[v][s] Y_k[v][s],   Y_k = (P phiA)_k Chat_k^T,
//
// with Chat_k[s][d] = sum over links m = (s, d) of Chat[m][k] (the upstream gradient folded into
// the DFT, zero for source-detector pairs without a link).  Per harmonic this is a complex GEMM
// over all voxels, [NV x ND] x [ND x NS], written as a real one with K' = 2 ND (re, im of each
// detector, interleaved) and N' = 2 NS (re, im of each source, interleaved), on the tensor cores
// (kind::tf32, 3xTF32 split, M = 128 voxels, N' = 64, K' = 64: NS, ND <= 32, padded with zeros).
// The per-harmonic operand B'_k = the real embedding of Chat_k^T is built once per call in
// global memory, already split and swizzled (k_vjp_btab), and copied into shared memory.
//
// CTA = 256 threads over a tile of 128 voxels, looping over the harmonics: the threads convert
// this tile's (P phiA)_k rows to the split A' operand (coalesced FP64 loads), thread 0 issues the
// 24 MMAs, and in the epilogue each warp reads its 32 voxel rows x 32 columns of Y_k from tensor
// memory, dots them with (P phi)_k read from global memory and accumulates in FP64.  96 KB of
// shared memory: two CTAs per SM overlap one's loads with the other's MMAs and epilogue.
constexpr int VT_THREADS = 256;
constexpr int VT_ROWS = 128;                       // voxels per tile (MMA M)
constexpr int VT_NP = 64;                          // N' = 2 x 32 sources
constexpr int VT_KP = 64;                          // K' = 2 x 32 detectors
constexpr int VT_A = VT_ROWS * VT_KP * 4;          // 32 KB: 128 rows x 64 fp32 (two 128-byte atoms)
constexpr int VT_B = VT_NP * VT_KP * 4;            // 16 KB
constexpr int VT_SMEM = 2 * VT_A + 2 * VT_B + 1024;
constexpr uint32_t VT_IDESC = tc::idesc(2, 2, VT_ROWS, VT_NP);

// K-major split operand image: element (row, j) of a [rows][64] fp32 tile stored as two 128-byte
// swizzled sub-tiles (j < 32, j >= 32) of rows x 128 B
__host__ __device__ inline uint32_t kmaj64(uint32_t row, uint32_t j, uint32_t rows) {
  return (j >> 5) * rows * 128u + tc::sw128_chunk(row, (j & 31u) >> 2) + (j & 3u) * 4u;
}

// Btab[k] = (hi, lo) images of B'_k [64 rows n'][64 K'] (16 KB each), from Chat [nm][nf]:
//   B'[2s][2d] = Re C, B'[2s][2d+1] = -Im C, B'[2s+1][2d] = Im C, B'[2s+1][2d+1] = Re C,
// C = Chat_k[s][d]; one thread per (k, s, d).
__global__ void k_vjp_btab(const float2 *__restrict__ Chat, const int32_t *__restrict__ link, int nm, int nf,
                           unsigned char *__restrict__ Btab) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)nf * 32 * 32) return;
  const int k = (int)(t / 1024), s = (int)(t / 32 % 32), d = (int)(t % 32);
  float2 c = make_float2(0.f, 0.f);
  for (int m = 0; m < nm; ++m)  // link tables are small (nm <= 1024 here): a scan per entry
    if (link[2 * m] == s && link[2 * m + 1] == d) {
      const float2 x = Chat[(int64_t)m * nf + k];
      c.x += x.x;
      c.y += x.y;
    }
  unsigned char *hi = Btab + (size_t)k * 2 * VT_B, *lo = hi + VT_B;
  const float v[2][2] = {{c.x, -c.y}, {c.y, c.x}};
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const float x = v[a][b], h = tc::to_tf32(x), l = tc::to_tf32(x - h);
      const uint32_t off = kmaj64(2 * s + a, 2 * d + b, VT_NP);
      *reinterpret_cast<float *>(hi + off) = h;
      *reinterpret_cast<float *>(lo + off) = l;
    }
}

// (P f)_k[v][o] for o < cnt optodes of field f [nf][nn][cnt], FP64
__device__ inline double2 basis_field(const JArgs &a, int64_t v, int k, int o, const double2 *__restrict__ f, int cnt) {
  if (!a.prow) return f[((int64_t)k * a.nn + v) * cnt + o];
  double2 acc = make_double2(0.0, 0.0);
  const int b = a.prow[v], e = min(a.prow[v + 1], b + PMAX);
  for (int q = b; q < e; ++q) {
    const double2 x = f[((int64_t)k * a.nn + a.pcol[q]) * cnt + o];
    acc.x += a.pval[q] * x.x;
    acc.y += a.pval[q] * x.y;
  }
  return acc;
}

__global__ void __launch_bounds__(VT_THREADS, 2) k_jacobian_vjp_tc(JArgs a, const unsigned char *__restrict__ Btab,
                                                                  double *__restrict__ vjp, int *err) {
  extern __shared__ __align__(1024) unsigned char vt_raw[];
  __shared__ __align__(8) uint64_t bar_mma;
  __shared__ uint32_t tmem_slot;
  __shared__ double part[VT_THREADS];
  unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(vt_raw) + 1023) & ~uintptr_t(1023));
  unsigned char *Ahi = sm, *Alo = sm + VT_A, *Bhi = sm + 2 * VT_A, *Blo = Bhi + VT_B;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    tc::mbar_init(&bar_mma, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tc::tmem_alloc(&tmem_slot, VT_NP);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const int quad = warp & 3, chalf = warp >> 2;    // TMEM lanes 32 quad.., columns 32 chalf.. (sources 16 chalf..)
  uint32_t phase = 0;
  bool ok = true;
  for (int64_t v0 = (int64_t)blockIdx.x * VT_ROWS; v0 < a.nv && ok; v0 += (int64_t)gridDim.x * VT_ROWS) {
    const int64_t vr = v0 + 32 * quad + lane;      // this thread's voxel row in the epilogue
    double acc = 0.0;
    for (int k = 0; k < a.nf && ok; ++k) {
      // A' = split real embedding of (P phiA)_k for the tile's voxels: element (row, d) -> K' 2d, 2d+1
      for (int e = tid; e < VT_ROWS * 32; e += VT_THREADS) {
        const int row = e >> 5, d = e & 31;
        const int64_t v = v0 + row;
        double2 x = make_double2(0.0, 0.0);
        if (v < a.nv && d < a.nd) x = basis_field(a, v, k, d, a.phiA, a.nd);
        const float xr = (float)x.x, xi = (float)x.y;
        const float hr = tc::to_tf32(xr), hi_ = tc::to_tf32(xi);
        const uint32_t off = kmaj64(row, 2 * d, VT_ROWS);
        *reinterpret_cast<float2 *>(Ahi + off) = make_float2(hr, hi_);
        *reinterpret_cast<float2 *>(Alo + off) = make_float2(tc::to_tf32(xr - hr), tc::to_tf32(xi - hi_));
      }
      // B'_k: a straight copy of its (hi, lo) images
      {
        const uint4 *src = reinterpret_cast<const uint4 *>(Btab + (size_t)k * 2 * VT_B);
        uint4 *dst = reinterpret_cast<uint4 *>(Bhi);
        for (int e = tid; e < 2 * VT_B / 16; e += VT_THREADS) dst[e] = __ldg(src + e);
      }
      tc::fence_async_smem();
      tc::fence_before_sync();
      __syncthreads();
      if (tid == 0) {
        tc::fence_after_sync();
        const uint32_t ah = tc::smem_u32(Ahi), al = tc::smem_u32(Alo), bh = tc::smem_u32(Bhi), bl = tc::smem_u32(Blo);
#pragma unroll
        for (int kk = 0; kk < VT_KP / 8; ++kk) {       // K = 8 tf32 per MMA; 4 per 128-byte atom
          const uint32_t oa = (kk >> 2) * VT_ROWS * 128u + 32u * (kk & 3);
          const uint32_t ob = (kk >> 2) * VT_NP * 128u + 32u * (kk & 3);
          tc::umma_tf32<VT_IDESC>(tmem, tc::sdesc_k_sw128(ah + oa), tc::sdesc_k_sw128(bh + ob), kk ? 1u : 0u);
          tc::umma_tf32<VT_IDESC>(tmem, tc::sdesc_k_sw128(ah + oa), tc::sdesc_k_sw128(bl + ob), 1u);
          tc::umma_tf32<VT_IDESC>(tmem, tc::sdesc_k_sw128(al + oa), tc::sdesc_k_sw128(bh + ob), 1u);
        }
        tc::umma_commit(&bar_mma);
      }
      bool w = tc::mbar_wait(&bar_mma, phase);
      phase ^= 1u;
      if (!w) atomicOr(err, 1);
      w = __all_sync(0xffffffffu, w);
      tc::fence_after_sync();
      if (w) {
        uint32_t y[32];                                // Y_k[vr][s], s = 16 chalf + i: (re, im) pairs
        tc::tmem_ld32(tmem + ((uint32_t)(32 * quad) << 16) + 32u * chalf, y);
        if (vr < a.nv) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const int sidx = 16 * chalf + i;
            if (sidx < a.ns) {
              const double2 p = basis_field(a, vr, k, sidx, a.phi, a.ns);
              acc += p.x * (double)__uint_as_float(y[2 * i]) - p.y * (double)__uint_as_float(y[2 * i + 1]);
            }
          }
        }
      }
      tc::fence_before_sync();
      ok = __syncthreads_and(w);                       // operands and accumulator are free again
    }
    part[tid] = acc;
    __syncthreads();
    if (chalf == 0 && vr < a.nv && ok) vjp[vr] = (a.w ? a.w[vr] : 1.0) * (part[tid] + part[tid + 128]);
    __syncthreads();
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tmem, VT_NP);
}

// Vector-Jacobian product out[v] = w_v sum_m sum_k Re(Chat[m,k] a_k(m)) for VB voxels per block
// pass: the fields of VB voxels are staged together, so each Chat[m,k] read from global memory
// (L2) serves VB voxels.
template <int VB>
__global__ void __launch_bounds__(JBS) k_jacobian_vjp(JArgs a, const float2 *__restrict__ Chat,
                                                      double *__restrict__ vjp) {
  extern __shared__ float2 sh[];
  const int per = a.nf * (a.ns + a.nd);
  __shared__ double red[JBS / 32][VB];
  for (int64_t v0 = (int64_t)blockIdx.x * VB; v0 < a.nv; v0 += (int64_t)gridDim.x * VB) {
    __syncthreads();
#pragma unroll
    for (int b = 0; b < VB; ++b) {
      if (v0 + b >= a.nv) break;
      stage_field(a, v0 + b, a.phi, a.ns, sh + b * per);
      stage_field(a, v0 + b, a.phiA, a.nd, sh + b * per + a.nf * a.ns);
    }
    __syncthreads();
    double part[VB];
#pragma unroll
    for (int b = 0; b < VB; ++b) part[b] = 0.0;
    for (int m = threadIdx.x; m < a.nm; m += blockDim.x) {
      const int s = a.link[2 * m], d = a.link[2 * m + 1];
      double acc[VB];
#pragma unroll
      for (int b = 0; b < VB; ++b) acc[b] = 0.0;
      for (int k = 0; k < a.nf; ++k) {
        const float2 c = Chat[(int64_t)m * a.nf + k];
#pragma unroll
        for (int b = 0; b < VB; ++b) {
          const float2 x = sh[b * per + k * a.ns + s], y = sh[b * per + a.nf * a.ns + k * a.nd + d];
          const float ar = x.x * y.x - x.y * y.y, ai = x.x * y.y + x.y * y.x;
          acc[b] += (double)(c.x * ar - c.y * ai);
        }
      }
#pragma unroll
      for (int b = 0; b < VB; ++b) part[b] += acc[b];
    }
#pragma unroll
    for (int b = 0; b < VB; ++b) {
      double q = part[b];
      for (int off = 16; off > 0; off >>= 1) q += __shfl_xor_sync(0xffffffffu, q, off);
      if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5][b] = q;
    }
    __syncthreads();
    if (threadIdx.x < VB && v0 + threadIdx.x < a.nv) {
      double tot = 0.0;
      for (int q = 0; q < JBS / 32; ++q) tot += red[q][threadIdx.x];
      vjp[v0 + threadIdx.x] = (a.w ? a.w[v0 + threadIdx.x] : 1.0) * tot;
    }
  }
}

// Ckg[k][g] = C[g][k] for g < ng, 0 for ng <= g < ngc (the register-blocked kernel's layout)
__global__ void k_ctab_kg(const float2 *__restrict__ C, int ng, int nf, int ngc, float2 *Ckg) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nf * ngc) return;
  const int k = t / ngc, g = t % ngc;
  Ckg[t] = g < ng ? C[g * nf + k] : make_float2(0.f, 0.f);
}

// C[g,k] = -2 Nt h_k conj(gate[g,k]) / fpsf[k]; also -1/fpsf[k] for the FD form
__global__ void k_ctab(const double2 *__restrict__ gate, const double2 *__restrict__ fpsf, int ng, int nf, int nt,
                       float2 *C, double2 *finv) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < nf) finv[t] = cdiv(make_double2(-1.0, 0.0), fpsf[t]);
  if (t >= ng * nf || !gate) return;
  const int k = t % nf;  // t = g * nf + k
  double h = k == 0 ? 0.5 : 1.0;
  double2 gc = make_double2(gate[t].x, -gate[t].y);
  double2 r = cdiv(gc, fpsf[k]);
  double s = -2.0 * (double)nt * h;
  C[t] = make_float2((float)(s * r.x), (float)(s * r.y));
}

// Chat[m,k] = sum_g gin[m,g] C[g,k]   (the upstream gradient folded into the DFT)
__global__ void k_chat(const double *__restrict__ gin, const float2 *__restrict__ C, const double *__restrict__ rytov,
                       int nm, int ng, int nf, float2 *Chat) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)nm * nf) return;
  int m = (int)(t / nf), k = (int)(t % nf);
  double re = 0, im = 0;
  for (int g = 0; g < ng; ++g) {
    double q = gin[(int64_t)m * ng + g];
    if (rytov) q /= rytov[(int64_t)m * ng + g];
    float2 c = C[g * nf + k];
    re += q * c.x;
    im += q * c.y;
  }
  Chat[t] = make_float2((float)re, (float)im);
}

int launch_common(JArgs &a, size_t &smem, int &grid) {
  DGP_REQUIRE(a.nv > 0 && a.nn > 0 && a.ns > 0 && a.nd > 0 && a.nf > 0 && a.nm > 0, "jacobian: sizes must be positive");
  smem = sizeof(float2) * ((size_t)a.nf * (a.ns + a.nd) + (size_t)a.ng * a.nf);
  DGP_REQUIRE(smem <= 200 * 1024, "jacobian: NF*(NS+ND+NG) too large for one block's shared memory");
  grid = (int)std::min<int64_t>(a.nv, (int64_t)sm_count() * 8);
  return DGP_OK;
}

}  // namespace

// 0 (default) and 2: the tensor cores where the shapes fit (TG Jacobian: nodal basis, unique
//   links, up to 32 sources and detectors, shared memory for the operand rings; vjp: up to 32
//   sources and detectors), else the CUDA cores.  Measured at the sensitivity configuration
//   (100k voxels, 32 x 32 optodes, 64 harmonics, 20 gates, one B200): TG Jacobian 11.9 ms
//   against 20.0 ms, vjp 5.2 ms against 16.4 ms.
// 1: both on the CUDA cores (cross-checks, timing)
static int g_jacobian_engine = 0;

int set_jacobian_engine(int engine) {
  DGP_REQUIRE(engine >= 0 && engine <= 2,
              "jacobian engine must be 0 (default), 1 (CUDA cores) or 2 (tensor cores where the shapes fit)");
  g_jacobian_engine = engine;
  return DGP_OK;
}

int jacobian_run(int mode, const int32_t *prow, const int32_t *pcol, const double *pval, int64_t nv, const double *w,
                 const double *phi, int ns, const double *phiA, int nd, int64_t nn, int nf, const double *fpsf,
                 const int32_t *link, int nm, const double *gate, int ng, int nt, const double *rytov, void *out,
                 const double *gin, cudaStream_t st) {
  DGP_REQUIRE(phi && phiA && fpsf && link && out, "jacobian: null pointer");
  DGP_REQUIRE(mode == 1 || (gate && ng >= 1 && ng <= NGMAX), "jacobian: need gate coefficients, 1 <= NG <= 32");
  DGP_REQUIRE(prow || nv == nn, "jacobian: the nodal basis (P = NULL) needs nv == nn");
  JArgs a{prow, pcol, pval, nv, nn, w, (const double2 *)phi, (const double2 *)phiA, ns, nd, nf, nm, mode == 1 ? 0 : ng,
          link};
  size_t smem;
  int grid;
  DGP_TRY(launch_common(a, smem, grid));
  // the link table addresses the staged fields in shared memory and P's columns address the
  // fields in HBM: both are checked before the first kernel uses them
  // links_unique: every (s, d) pair at most once (the tensor-core epilogue writes each pair's
  // entries from one accumulator row); links_dense: link m is (m / nd, m % nd) for all NS x ND
  bool links_unique = ns <= 32 && nd <= 32, links_dense = nm == ns * nd;
  {
    std::vector<int32_t> hl(2 * (size_t)nm);
    DGP_CUDA(cudaMemcpyAsync(hl.data(), link, sizeof(int32_t) * 2 * nm, cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaStreamSynchronize(st));
    std::vector<char> seen(links_unique ? 32 * 32 : 0, 0);
    for (int m = 0; m < nm; ++m) {
      const int32_t s_ = hl[2 * m], d_ = hl[2 * m + 1];
      if (s_ < 0 || s_ >= ns || d_ < 0 || d_ >= nd) return fail(DGP_ERR_ARG, "jacobian: link index out of range");
      if (links_unique) {
        if (seen[s_ * 32 + d_]) links_unique = false;
        else seen[s_ * 32 + d_] = 1;
      }
      if (s_ != m / nd || d_ != m % nd) links_dense = false;
    }
  }
  if (prow) {
    DGP_REQUIRE(pcol && pval, "jacobian: null basis column or value array");
    DGP_TRY(csr_in_range(prow, pcol, nv, nn, -1, PMAX, "jacobian basis", st));
  }
  DevBuf ctab, finv, chat;
  DGP_TRY(ctab.alloc(sizeof(float2) * (size_t)std::max(1, ng) * nf));
  DGP_TRY(finv.alloc(sizeof(double2) * nf));
  int nt_ = std::max(ng * nf, nf);
  k_ctab<<<(unsigned)ceil_div(nt_, 256), 256, 0, st>>>((const double2 *)gate, (const double2 *)fpsf, mode == 1 ? 0 : ng,
                                                        nf, nt, ctab.as<float2>(), finv.as<double2>());
  DGP_CHECK_LAUNCH();
  if (mode == 1) DGP_TRY(allow_dyn_smem(k_jacobian_complex, smem));
  const T2Layout tl = t2_layout(nf, std::max(1, ng));
  const size_t smem_tc = tl.bytes + 1024;
  // (+ 1 KB of the kernel's own static shared memory)
  const bool tc_fits = mode == 0 && !prow && links_unique && nf <= 64 && smem_tc + 1024 <= 227 * 1024;
  if (tc_fits && g_jacobian_engine != 1) {
    // tensor cores: one persistent warp-specialised CTA per SM
    const int dense = !links_dense ? 0 : (!rytov && nd % 4 == 0 && nm % 4 == 0) ? 2 : 1;
    DevBuf flag;
    DGP_TRY(flag.alloc(sizeof(int)));
    DGP_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    DGP_TRY(allow_dyn_smem(k_jacobian_tg_tc, smem_tc));
    const int gtc = (int)std::min<int64_t>(nv, (int64_t)sm_count());
    k_jacobian_tg_tc<<<gtc, T2_THREADS, smem_tc, st>>>(a, ctab.as<float2>(), rytov, dense, (float *)out,
                                                       flag.as<int>());
    DGP_CHECK_LAUNCH();
    int h = 0;
    DGP_CUDA(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaStreamSynchronize(st));
    if (h) return fail(DGP_ERR_CUDA, "jacobian_tg: a tensor-core pipeline wait timed out");
    return DGP_OK;
  }
  if (mode == 0) {
    // register-blocked TG kernel: gates padded to 8/16/24/32, MT measurements per thread
    const int ngc = ng <= 8 ? 8 : ng <= 16 ? 16 : ng <= 24 ? 24 : 32;
    // measurements per thread: 4 while the accumulators fit two blocks per SM (<= 16 gates), else 2
    const int mt = (nm > 2 * JBS && ngc <= 16) ? 4 : nm > JBS ? 2 : 1;
    DevBuf ckg;
    DGP_TRY(ckg.alloc(sizeof(float2) * (size_t)nf * ngc));
    k_ctab_kg<<<(unsigned)ceil_div((int64_t)nf * ngc, 256), 256, 0, st>>>(ctab.as<float2>(), ng, nf, ngc,
                                                                          ckg.as<float2>());
    DGP_CHECK_LAUNCH();
    const size_t smem_tg = sizeof(float2) * ((size_t)nf * (ns + nd) + 1 + (size_t)nf * ngc);
    DGP_REQUIRE(smem_tg <= 200 * 1024, "jacobian: NF*(NS+ND+NG) too large for one block's shared memory");
    int arc = DGP_OK;
    auto go = [&](auto mtc, auto ngcc) {
      constexpr int MT_ = decltype(mtc)::value, NGC_ = decltype(ngcc)::value;
      arc = allow_dyn_smem(k_jacobian_tg<MT_, NGC_>, smem_tg);
      if (arc == DGP_OK) k_jacobian_tg<MT_, NGC_><<<grid, JBS, smem_tg, st>>>(a, ckg.as<float2>(), rytov, (float *)out);
    };
    auto by_ngc = [&](auto mtc) {
      switch (ngc) {
        case 8: go(mtc, std::integral_constant<int, 8>()); break;
        case 16: go(mtc, std::integral_constant<int, 16>()); break;
        case 24: go(mtc, std::integral_constant<int, 24>()); break;
        default: go(mtc, std::integral_constant<int, 32>()); break;
      }
    };
    if (mt == 4) by_ngc(std::integral_constant<int, 4>());
    else if (mt == 2) by_ngc(std::integral_constant<int, 2>());
    else by_ngc(std::integral_constant<int, 1>());
    DGP_TRY(arc);
    DGP_CHECK_LAUNCH();
    DGP_CUDA(cudaStreamSynchronize(st));  // ckg is released on return
  } else if (mode == 1) {
    k_jacobian_complex<<<grid, JBS, smem, st>>>(a, finv.as<double2>(), (double2 *)out);
  } else {
    DGP_REQUIRE(gin, "jacobian vjp: null upstream gradient");
    DGP_TRY(chat.alloc(sizeof(float2) * (size_t)nm * nf));
    k_chat<<<(unsigned)ceil_div((int64_t)nm * nf, 256), 256, 0, st>>>(gin, ctab.as<float2>(), rytov, nm, ng, nf,
                                                                      chat.as<float2>());
    DGP_CHECK_LAUNCH();
    if (g_jacobian_engine != 1 && ns <= 32 && nd <= 32 && nm <= 4096) {
      // tensor cores: per-harmonic complex GEMM over voxel tiles
      DevBuf btab, flag;
      DGP_TRY(btab.alloc((size_t)nf * 2 * VT_B));
      DGP_TRY(flag.alloc(sizeof(int)));
      DGP_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
      k_vjp_btab<<<(unsigned)ceil_div((int64_t)nf * 1024, 256), 256, 0, st>>>(chat.as<float2>(), link, nm, nf,
                                                                              btab.as<unsigned char>());
      DGP_CHECK_LAUNCH();
      DGP_CUDA(cudaFuncSetAttribute(k_jacobian_vjp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, VT_SMEM));
      const int gv = (int)std::min<int64_t>(ceil_div(nv, VT_ROWS), (int64_t)sm_count() * 2);
      k_jacobian_vjp_tc<<<gv, VT_THREADS, VT_SMEM, st>>>(a, btab.as<unsigned char>(), (double *)out, flag.as<int>());
      DGP_CHECK_LAUNCH();
      int h = 0;
      DGP_CUDA(cudaMemcpyAsync(&h, flag.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      DGP_CUDA(cudaStreamSynchronize(st));
      if (h) return fail(DGP_ERR_CUDA, "jacobian_tg_vjp: a tensor-core pipeline wait timed out");
      return DGP_OK;
    }
    // voxels per block pass: as many as 200 KB of staged fields allow, up to 4
    const size_t per = sizeof(float2) * (size_t)nf * (ns + nd);
    const int vb = (int)std::min<size_t>(4, std::max<size_t>(1, (200 * 1024) / per));
    const size_t smem_v = per * vb;
    int arc = DGP_OK;
    auto go = [&](auto vbc) {
      constexpr int VB_ = decltype(vbc)::value;
      arc = allow_dyn_smem(k_jacobian_vjp<VB_>, smem_v);
      const int gv = (int)std::min<int64_t>(ceil_div(nv, VB_), (int64_t)sm_count() * 8);
      if (arc == DGP_OK) k_jacobian_vjp<VB_><<<gv, JBS, smem_v, st>>>(a, chat.as<float2>(), (double *)out);
    };
    if (vb >= 4) go(std::integral_constant<int, 4>());
    else if (vb == 3) go(std::integral_constant<int, 3>());
    else if (vb == 2) go(std::integral_constant<int, 2>());
    else go(std::integral_constant<int, 1>());
    DGP_TRY(arc);
  }
  DGP_CHECK_LAUNCH();
  DGP_CUDA(cudaStreamSynchronize(st));  // scratch tables are released on return
  return DGP_OK;
}

}  // namespace dgp
