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
