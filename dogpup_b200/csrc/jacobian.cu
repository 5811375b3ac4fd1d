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
// Time-gated Jacobian on the tensor cores (tcgen05, kind::tf32, 3xTF32 split).
//
// Per voxel v and tile of 128 links m, J_tg[v][g][m] = w_v * sum_K' A'[m][K'] B'[K'][g] with
//   A'[m][K'] = Re / Im of a_k(m) = (P phi_s)_k (P phiA_d)_k  and  B'[K'][g] = Re / -Im of C[g,k],
// K' = 2 NF (the real and imaginary parts of the DFT's complex products).  K' runs in chunks of
// 16 harmonics = 32 values ([16 real | 16 imaginary], one 128-byte row of a 128B-swizzled
// K-major tile).  FP32 values x are split x = hi + lo with hi = tf32(x), lo = tf32(x - hi), and
// each chunk issues hi*hi + hi*lo + lo*hi into an FP32 accumulator in tensor memory (the lo*lo
// term, ~2^-22 relative, is dropped).
//
// CTA = 256 threads, persistent over voxels (one CTA per SM).  All threads build the A' chunks
// (two threads per link row, 8 harmonics each) from the voxel's fields staged in shared memory;
// thread 0 issues the chunk's 12 MMAs (M = 128, N = 32 gate columns, K = 8) and commits them to
// the chunk buffer's mbarrier.  Two chunk buffers: the next chunk is built while the tensor core
// works on the previous one.  Two accumulators in tensor memory (2 x 32 columns): a tile's
// epilogue (tcgen05.ld, w_v and Rytov scaling, coalesced FP32 stores) runs while the next tile's
// MMAs are in flight.  Every mbarrier wait is bounded; a timeout raises err and ends the kernel
// after waiting (bounded) for the MMAs it issued, and the tensor memory is always freed.
constexpr int TC_THREADS = 256;
constexpr int TC_CH = 16;                    // harmonics per K' chunk
constexpr int TC_ROWS = 128;                 // links per tile (MMA M)
constexpr int TC_N = 32;                     // gate columns (MMA N), NG <= 32
constexpr int TC_ATILE = TC_ROWS * 128;      // one 128 x 32 fp32 operand tile: 16 KB
constexpr int TC_BTILE = TC_N * 128;         // one 32 x 32 fp32 operand tile: 4 KB
constexpr uint32_t TC_IDESC = tc::idesc(2, 2, TC_ROWS, TC_N);

struct TcLayout {
  uint32_t a_off, b_off, f_off, bytes;       // A' buffers, B' table, staged fields, total (from the 1 KB-aligned base)
  int nch;
};

__host__ __device__ inline TcLayout tc_layout(int nf, int ns, int nd) {
  TcLayout L;
  L.nch = (nf + TC_CH - 1) / TC_CH;
  L.a_off = 0;                                               // 2 buffers x (hi, lo)
  L.b_off = 4 * TC_ATILE;                                    // nch x (hi) then nch x (lo)
  L.f_off = L.b_off + 2 * L.nch * TC_BTILE;
  L.bytes = L.f_off + (uint32_t)(sizeof(float2) * (size_t)nf * (ns + nd));
  return L;
}

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

__global__ void __launch_bounds__(TC_THREADS, 1) k_jacobian_tg_tc(JArgs a, const float2 *__restrict__ C /*[ng][nf]*/,
                                                                 const double *__restrict__ rytov,
                                                                 float *__restrict__ Jtg, int *err) {
  extern __shared__ __align__(1024) unsigned char tc_raw[];
  __shared__ __align__(8) uint64_t bar_buf[2], bar_d[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  unsigned char *sm = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~uintptr_t(1023));
  const TcLayout L = tc_layout(a.nf, a.ns, a.nd);
  unsigned char *Ab = sm + L.a_off;                   // buffer b: hi at b*2*ATILE, lo at +ATILE
  unsigned char *Bhi = sm + L.b_off, *Blo = Bhi + L.nch * TC_BTILE;
  float2 *Ps = reinterpret_cast<float2 *>(sm + L.f_off), *Pd = Ps + a.nf * a.ns;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (tid == 0) {
    for (int b = 0; b < 2; ++b) {
      tc::mbar_init(&bar_buf[b], 1);
      tc::mbar_init(&bar_d[b], 1);
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) tc::tmem_alloc(&tmem_slot, 2 * TC_N);
  // B' = the gate table, split: row g (MMA N), K' = chunk c's [Re C[g][16c..16c+15] | -Im C[g][..]]
  for (int t = tid; t < L.nch * TC_N * 8; t += TC_THREADS) {
    const int c = t / (TC_N * 8), g = (t / 8) % TC_N, q = t % 8;   // 16-byte chunk q of row g in chunk c
    float x[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int j = 4 * q + i, k = c * TC_CH + (j & 15);
      const float2 v = (g < a.ng && k < a.nf) ? C[g * a.nf + k] : make_float2(0.f, 0.f);
      x[i] = j < 16 ? v.x : -v.y;
    }
    st_split4(Bhi + c * TC_BTILE, Blo + c * TC_BTILE, tc::sw128_chunk(g, q), x);
  }
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_slot;

  const int r = tid & (TC_ROWS - 1), half = tid >> 7;   // link row of the tile, harmonic half of a chunk
  uint32_t q = 0, t = 0;                               // chunks and tiles issued by this CTA
  bool have_prev = false, stop = false;
  int64_t pv = 0;
  int pm0 = 0;
  uint32_t pt = 0;
  float pw = 0.f;

  // epilogue of tile tp (voxel vp, links m0p..): TMEM accumulator tp & 1 -> J
  auto epilogue = [&](uint32_t tp, int64_t vp, int m0p, float wp) {
    bool ok = tc::mbar_wait(&bar_d[tp & 1], (tp >> 1) & 1);
    if (!ok) atomicOr(err, 1);
    ok = __all_sync(0xffffffffu, ok);
    tc::fence_after_sync();
    if (ok) {
      const int quad = warp & 3, cbase = (warp >> 2) * 16;
      uint32_t v[16];
      tc::tmem_ld16(tmem + ((uint32_t)(32 * quad) << 16) + (tp & 1) * TC_N + cbase, v);
      const int m = m0p + 32 * quad + lane;
      if (m < a.nm) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int g = cbase + i;
          if (g < a.ng) {
            float val = wp * __uint_as_float(v[i]);
            if (rytov) val = val / (float)rytov[(int64_t)m * a.ng + g];
            Jtg[((int64_t)vp * a.ng + g) * a.nm + m] = val;
          }
        }
      }
    }
    tc::fence_before_sync();
    return ok;
  };

  for (int64_t v = blockIdx.x; v < a.nv && !stop; v += gridDim.x) {
    __syncthreads();                                   // the previous voxel's chunks are built
    stage_field(a, v, a.phi, a.ns, Ps);
    stage_field(a, v, a.phiA, a.nd, Pd);
    __syncthreads();
    const float wv = (float)(a.w ? a.w[v] : 1.0);
    for (int m0 = 0; m0 < a.nm && !stop; m0 += TC_ROWS) {
      const int m = m0 + r;
      const bool valid = m < a.nm;
      const int s = valid ? a.link[2 * m] : 0, d = valid ? a.link[2 * m + 1] : 0;
      for (int c = 0; c < L.nch; ++c) {
        const uint32_t b = q & 1;
        bool ok = true;
        if (q >= 2) ok = tc::mbar_wait(&bar_buf[b], ((q >> 1) - 1) & 1);   // chunk q-2 has been consumed
        if (!ok) {
          atomicOr(err, 2);
          abort_flag = 1;
        }
        unsigned char *hi = Ab + b * 2 * TC_ATILE, *lo = hi + TC_ATILE;
        if (ok) {
          // this thread's 8 harmonics of chunk c: K' = 8 half + i (real) and 16 + 8 half + i (imaginary)
          float re[8], im[8];
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            const int k = c * TC_CH + 8 * half + i;
            re[i] = im[i] = 0.f;
            if (valid && k < a.nf) {
              const float2 x = Ps[k * a.ns + s], y = Pd[k * a.nd + d];
              re[i] = x.x * y.x - x.y * y.y;
              im[i] = x.x * y.y + x.y * y.x;
            }
          }
          const float r0[4] = {re[0], re[1], re[2], re[3]}, r1[4] = {re[4], re[5], re[6], re[7]};
          const float i0[4] = {im[0], im[1], im[2], im[3]}, i1[4] = {im[4], im[5], im[6], im[7]};
          st_split4(hi, lo, tc::sw128_chunk(r, 2 * half + 0), r0);
          st_split4(hi, lo, tc::sw128_chunk(r, 2 * half + 1), r1);
          st_split4(hi, lo, tc::sw128_chunk(r, 4 + 2 * half + 0), i0);
          st_split4(hi, lo, tc::sw128_chunk(r, 4 + 2 * half + 1), i1);
        }
        tc::fence_async_smem();
        tc::fence_before_sync();
        if (__syncthreads_or(abort_flag)) {
          stop = true;
          break;
        }
        if (tid == 0) {
          tc::fence_after_sync();
          const uint32_t d_tm = tmem + (t & 1) * TC_N;
          const uint32_t ah = tc::smem_u32(hi), al = tc::smem_u32(lo);
          const uint32_t bh = tc::smem_u32(Bhi + c * TC_BTILE), bl = tc::smem_u32(Blo + c * TC_BTILE);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {             // K = 8 tf32 = 32 bytes per MMA
            const uint32_t o = 32u * kk;
            tc::umma_tf32<TC_IDESC>(d_tm, tc::sdesc_k_sw128(ah + o), tc::sdesc_k_sw128(bh + o), (c | kk) ? 1u : 0u);
            tc::umma_tf32<TC_IDESC>(d_tm, tc::sdesc_k_sw128(ah + o), tc::sdesc_k_sw128(bl + o), 1u);
            tc::umma_tf32<TC_IDESC>(d_tm, tc::sdesc_k_sw128(al + o), tc::sdesc_k_sw128(bh + o), 1u);
          }
          tc::umma_commit(&bar_buf[b]);
          if (c == L.nch - 1) tc::umma_commit(&bar_d[t & 1]);
        }
        ++q;
        if (have_prev && c == (L.nch > 1 ? 1 : 0)) {   // the previous tile's MMAs are done by now
          if (!epilogue(pt, pv, pm0, pw)) abort_flag = 1;
          have_prev = false;
        }
      }
      if (stop) break;
      have_prev = true;
      pt = t;
      pv = v;
      pm0 = m0;
      pw = wv;
      ++t;
    }
  }
  if (!stop && have_prev) epilogue(pt, pv, pm0, pw);
  // teardown: every MMA this CTA issued has completed (bounded) before the tensor memory is freed
  if (q > 0 && tid == 0) {
    const uint32_t last = q - 1;
    tc::mbar_wait(&bar_buf[last & 1], (last >> 1) & 1);
    if (q > 1) tc::mbar_wait(&bar_buf[(last - 1) & 1], ((last - 1) >> 1) & 1);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_free(tmem, 2 * TC_N);
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

// 0 (auto): for each kernel the engine measured faster at the sensitivity configuration's
//   shapes (100k voxels, 32 x 32 optodes, 64 harmonics, 20 gates, one B200): the TG Jacobian on
//   the CUDA cores (20.0 ms; its tensor-core form, latency-bound in every phase with one CTA per
//   SM, 42.5 ms), the vjp on the tensor cores (5.2 ms against 16.4 ms);
// 1: both on the CUDA cores;  2: both on the tensor cores where their shapes fit
static int g_jacobian_engine = 0;

int set_jacobian_engine(int engine) {
  DGP_REQUIRE(engine >= 0 && engine <= 2,
              "jacobian engine must be 0 (auto), 1 (CUDA cores) or 2 (tensor cores where the shapes fit)");
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
  {
    std::vector<int32_t> hl(2 * (size_t)nm);
    DGP_CUDA(cudaMemcpyAsync(hl.data(), link, sizeof(int32_t) * 2 * nm, cudaMemcpyDeviceToHost, st));
    DGP_CUDA(cudaStreamSynchronize(st));
    for (int m = 0; m < nm; ++m)
      if (hl[2 * m] < 0 || hl[2 * m] >= ns || hl[2 * m + 1] < 0 || hl[2 * m + 1] >= nd)
        return fail(DGP_ERR_ARG, "jacobian: link index out of range");
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
  if (smem > 48 * 1024)
    DGP_CUDA(cudaFuncSetAttribute(k_jacobian_complex, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const TcLayout tl = tc_layout(nf, ns, nd);
  const size_t smem_tc = tl.bytes + 1024;
  if (mode == 0 && g_jacobian_engine == 2 && smem_tc <= 227 * 1024) {
    // tensor cores: one persistent CTA per SM
    DevBuf flag;
    DGP_TRY(flag.alloc(sizeof(int)));
    DGP_CUDA(cudaMemsetAsync(flag.p, 0, sizeof(int), st));
    DGP_CUDA(cudaFuncSetAttribute(k_jacobian_tg_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_tc));
    const int gtc = (int)std::min<int64_t>(nv, (int64_t)sm_count());
    k_jacobian_tg_tc<<<gtc, TC_THREADS, smem_tc, st>>>(a, ctab.as<float2>(), rytov, (float *)out, flag.as<int>());
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
    auto go = [&](auto mtc, auto ngcc) {
      constexpr int MT_ = decltype(mtc)::value, NGC_ = decltype(ngcc)::value;
      cudaFuncSetAttribute(k_jacobian_tg<MT_, NGC_>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_tg);
      k_jacobian_tg<MT_, NGC_><<<grid, JBS, smem_tg, st>>>(a, ckg.as<float2>(), rytov, (float *)out);
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
    auto go = [&](auto vbc) {
      constexpr int VB_ = decltype(vbc)::value;
      cudaFuncSetAttribute(k_jacobian_vjp<VB_>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_v);
      const int gv = (int)std::min<int64_t>(ceil_div(nv, VB_), (int64_t)sm_count() * 8);
      k_jacobian_vjp<VB_><<<gv, JBS, smem_v, st>>>(a, chat.as<float2>(), (double *)out);
    };
    if (vb >= 4) go(std::integral_constant<int, 4>());
    else if (vb == 3) go(std::integral_constant<int, 3>());
    else if (vb == 2) go(std::integral_constant<int, 2>());
    else go(std::integral_constant<int, 1>());
  }
  DGP_CHECK_LAUNCH();
  DGP_CUDA(cudaStreamSynchronize(st));  // scratch tables are released on return
  return DGP_OK;
}

}  // namespace dgp
