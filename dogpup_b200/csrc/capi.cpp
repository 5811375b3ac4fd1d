// C ABI of libdogpup_b200: argument checks, error reporting, plan handles.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "dgp_common.cuh"
#include "dgp_internal.h"
#include "dogpup_b200.h"
#include "dogpup_b200_mex.hpp"

namespace dgp {

static thread_local std::string g_err;
static std::atomic<int64_t> g_launches{0};
static std::atomic<int64_t> g_device_allocs{0};

void count_launches(int64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
int64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

void set_error(const std::string &msg) { g_err = msg; }

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
  char buf[512];
  std::snprintf(buf, sizeof buf, "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file,
                line);
  g_err = buf;
  return e == cudaErrorMemoryAllocation ? DGP_ERR_NOMEM : DGP_ERR_CUDA;
}

int DevBuf::alloc(size_t n) {
  release();
  if (n == 0) n = 16;
  cudaError_t e = cudaMalloc(&p, n);
  g_device_allocs.fetch_add(1, std::memory_order_relaxed);
  if (e != cudaSuccess) {
    p = nullptr;
    cudaGetLastError();
    char buf[160];
    std::snprintf(buf, sizeof buf, "device allocation of %zu bytes failed: %s", n, cudaGetErrorString(e));
    return fail(DGP_ERR_NOMEM, buf);
  }
  bytes = n;
  return DGP_OK;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

int sm_count() {
  static int cache[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && cache[dev]) return cache[dev];
  int n = 148;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  if (dev >= 0 && dev < 64) cache[dev] = n;
  return n;
}

int allow_dyn_smem_impl(const void *kernel, size_t bytes) {
  int dev = 0, optin = 0;
  DGP_CUDA(cudaGetDevice(&dev));
  DGP_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  DGP_CUDA(cudaFuncGetAttributes(&fa, kernel));
  const int64_t cap = (int64_t)optin - (int64_t)fa.sharedSizeBytes;
  if ((int64_t)bytes > cap)
    return fail(DGP_ERR_ARG, "shared memory per block (" + std::to_string(bytes) + " bytes) above the device's " +
                                 std::to_string(cap) + " for this kernel");
  DGP_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap));
  return DGP_OK;
}

int mex_spmv(int mode, double *out_re, double *out_im, const double *x_re, const double *x_im, const double *fAxis,
             const double *v_re, const double *v_im, const int *rPtr, const int *cPtr, int64_t nnz, int nrows,
             int ncols, int nfreqs, cudaStream_t st, int es = 1);
int td2fc_run(const double *x, int64_t nr, int nt, const double *t, const double *f, int nf, double *c,
              cudaStream_t st);
int fc2td_run(const double *c, int64_t nr, int nf, const double *f, const double *t, int nt, double *x,
              cudaStream_t st);
int fc2tg_run(const double *c, int64_t nr, int nf, const double *gate, int ng, int nt, double *y, cudaStream_t st);
int meas_run(const int32_t *dn, const double *dw, int nd, const int32_t *link, int nm, const double *phi, int64_t n,
             int nf, int ns, double *data, cudaStream_t st);
int csr_spmv_run(const int32_t *rowptr, const int32_t *col, const double *val, int64_t nrows, int64_t ncols,
                 const double *x, double *y, cudaStream_t st);
int mex_fsaip(double *out_re, double *out_im, const double *A_re, const double *A_im, const int *rPtrA,
              const int *cPtrA, const int *rPtrG, const int *cPtrG, int nfreqs, int nrows, cudaStream_t st,
              int es = 1);
int set_jacobian_engine(int engine);
int jacobian_run(int mode, const int32_t *prow, const int32_t *pcol, const double *pval, int64_t nv, const double *w,
                 const double *phi, int ns, const double *phiA, int nd, int64_t nn, int nf, const double *fpsf,
                 const int32_t *link, int nm, const double *gate, int ng, int nt, const double *rytov, void *out,
                 const double *gin, cudaStream_t st);
int normal_eq_run(const float *Jt, int64_t nv, int64_t nm, const double *W, const double *y, double lam, int mode,
                  double *H, int64_t ldh, double *rhs, cudaStream_t st);
int cholesky_solve_run(double *H, int64_t n, int64_t ldh, double *x, cudaStream_t st);
int times_jt_run(const double *A, int64_t na, int64_t nv, const float *Jt, int64_t nm, double *out, cudaStream_t st);
int row_dots_run(const float *Jt, int64_t nv, int64_t nm, const double *W, const double *y, double *diag, double *rhs,
                 cudaStream_t st);
int lm_update_run(const float *Jt, int64_t nv, int64_t nm, const double *W, const double *y, double lam, double *x,
                  int32_t form, int32_t *form_used, cudaStream_t st);
int cholesky_solve_many_run(double *H, int64_t n, int64_t ldh, double *x, int32_t nrhs, int64_t ldx,
                            cudaStream_t st);

}  // namespace dgp

using namespace dgp;

struct dgp_fem_s {
  FemPlan plan;
};
struct dgp_solver_s {
  SolverPlan plan;
};

#define DGP_GUARD(expr)                                                        \
  try {                                                                        \
    return (expr);                                                             \
  } catch (const std::bad_alloc &) {                                           \
    return fail(DGP_ERR_NOMEM, "host allocation failed");                      \
  } catch (...) {                                                              \
    return fail(DGP_ERR_ARG, "unexpected exception");                          \
  }

extern "C" {

const char *dgp_last_error(void) { return g_err.c_str(); }

const char *dgp_status_string(int s) {
  switch (s) {
    case DGP_OK: return "ok";
    case DGP_ERR_ARG: return "invalid argument";
    case DGP_ERR_CUDA: return "CUDA error";
    case DGP_ERR_NOMEM: return "out of memory";
    case DGP_ERR_MESH: return "invalid mesh";
    case DGP_ERR_NOT_CONVERGED: return "not converged";
    case DGP_ERR_BREAKDOWN: return "BiCGSTAB breakdown";
    case DGP_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

int dgp_version(void) { return 10000; }

int64_t dgp_kernel_launches(void) { return launch_count(); }

int64_t dgp_device_allocations(void) { return g_device_allocs.load(std::memory_order_relaxed); }

// ------------------------------------------------------------ mex layouts
int dgp_smv_mex(double *d_out_real, double *d_out_imag, const double *d_x_real, const double *d_x_imag,
                const double *d_fAxis, const double *d_valA_real, const double *d_valA_imag, const int *d_rPtr,
                const int *d_cPtr, int nrows, int ncols, int nfreqs, dgp_stream_t stream) {
  DGP_GUARD(mex_spmv(0, d_out_real, d_out_imag, d_x_real, d_x_imag, d_fAxis, d_valA_real, d_valA_imag, d_rPtr,
                     d_cPtr, 0, nrows, ncols, nfreqs, (cudaStream_t)stream));
}

int dgp_fsaimv_mex(double *d_out_real, double *d_out_imag, const double *d_x_real, const double *d_x_imag,
                   const double *d_valG_real, const double *d_valG_imag, const int *d_rPtr, const int *d_cPtr,
                   int nnz, int nrows, int ncols, int nfreqs, dgp_stream_t stream) {
  DGP_GUARD(mex_spmv(1, d_out_real, d_out_imag, d_x_real, d_x_imag, nullptr, d_valG_real, d_valG_imag, d_rPtr,
                     d_cPtr, nnz, nrows, ncols, nfreqs, (cudaStream_t)stream));
}

int dgp_fsaip_mex(double *d_out_real, double *d_out_imag, const double *d_valA_real, const double *d_valA_imag,
                  const int *d_rPtrA, const int *d_cPtrA, const int *d_rPtrG, const int *d_cPtrG, int nfreqs,
                  int nrows, dgp_stream_t stream) {
  DGP_GUARD(mex_fsaip(d_out_real, d_out_imag, d_valA_real, d_valA_imag, d_rPtrA, d_cPtrA, d_rPtrG, d_cPtrG, nfreqs,
                      nrows, (cudaStream_t)stream));
}

int dgp_smv_mex_ic(double *d_out, const double *d_x, const double *d_fAxis, const double *d_valA, const int *d_rPtr,
                   const int *d_cPtr, int nrows, int ncols, int nfreqs, dgp_stream_t stream) {
  if (!d_out || !d_x || !d_valA) return fail(DGP_ERR_ARG, "smv_mex_ic: null pointer");
  DGP_GUARD(mex_spmv(0, d_out, d_out + 1, d_x, d_x + 1, d_fAxis, d_valA, d_valA + 1, d_rPtr, d_cPtr, 0, nrows, ncols,
                     nfreqs, (cudaStream_t)stream, 2));
}

int dgp_fsaimv_mex_ic(double *d_out, const double *d_x, const double *d_valG, const int *d_rPtr, const int *d_cPtr,
                      int nnz, int nrows, int ncols, int nfreqs, dgp_stream_t stream) {
  if (!d_out || !d_x || !d_valG) return fail(DGP_ERR_ARG, "FSAImv_mex_ic: null pointer");
  DGP_GUARD(mex_spmv(1, d_out, d_out + 1, d_x, d_x + 1, nullptr, d_valG, d_valG + 1, d_rPtr, d_cPtr, nnz, nrows,
                     ncols, nfreqs, (cudaStream_t)stream, 2));
}

int dgp_fsaip_mex_ic(double *d_out, const double *d_valA, const int *d_rPtrA, const int *d_cPtrA, const int *d_rPtrG,
                     const int *d_cPtrG, int nfreqs, int nrows, dgp_stream_t stream) {
  if (!d_out || !d_valA) return fail(DGP_ERR_ARG, "FSAIP_mex_ic: null pointer");
  DGP_GUARD(mex_fsaip(d_out, d_out + 1, d_valA, d_valA + 1, d_rPtrA, d_cPtrA, d_rPtrG, d_cPtrG, nfreqs, nrows,
                      (cudaStream_t)stream, 2));
}

// -------------------------------------------------------------------- FEM
int dgp_fem_create(dgp_fem_t *fem, const double *d_node, const int32_t *d_elem, int64_t nn, int64_t ne, double nr,
                   dgp_stream_t stream) {
  if (!fem || !d_node || !d_elem) return fail(DGP_ERR_ARG, "fem_create: null pointer");
  *fem = nullptr;
  dgp_fem_s *h = new (std::nothrow) dgp_fem_s();
  if (!h) return fail(DGP_ERR_NOMEM, "fem_create: host allocation failed");
  int rc;
  try {
    rc = fem_create(&h->plan, d_node, d_elem, nn, ne, nr, (cudaStream_t)stream);
  } catch (...) {
    rc = fail(DGP_ERR_NOMEM, "fem_create: exception");
  }
  if (rc != DGP_OK) {
    delete h;
    return rc;
  }
  *fem = h;
  return DGP_OK;
}

int dgp_fem_destroy(dgp_fem_t fem) {
  delete fem;
  return DGP_OK;
}

int dgp_fem_info(dgp_fem_t fem, int64_t *nnz, int64_t *n_robin_faces, int64_t *n_boundary, double *c_medium) {
  if (!fem) return fail(DGP_ERR_ARG, "fem_info: null handle");
  if (nnz) *nnz = fem->plan.nnz;
  if (n_robin_faces) *n_robin_faces = fem->plan.nfaces;
  if (n_boundary) *n_boundary = fem->plan.nbnd;
  if (c_medium) *c_medium = fem->plan.c;
  return DGP_OK;
}

int dgp_fem_pattern(dgp_fem_t fem, const int32_t **d_rowptr, const int32_t **d_col) {
  if (!fem || !d_rowptr || !d_col) return fail(DGP_ERR_ARG, "fem_pattern: null pointer");
  *d_rowptr = fem->plan.rowptr.as<int32_t>();
  *d_col = fem->plan.col.as<int32_t>();
  return DGP_OK;
}

int dgp_fem_boundary(dgp_fem_t fem, int32_t *d_bnd, dgp_stream_t stream) {
  if (!fem || !d_bnd) return fail(DGP_ERR_ARG, "fem_boundary: null pointer");
  DGP_CUDA(cudaMemcpyAsync(d_bnd, fem->plan.bnd.p, sizeof(int32_t) * fem->plan.nn, cudaMemcpyDeviceToDevice,
                           (cudaStream_t)stream));
  return DGP_OK;
}

int dgp_fem_assemble(dgp_fem_t fem, const double *d_mua, const double *d_musp, double *d_K, double *d_M,
                     dgp_stream_t stream) {
  if (!fem) return fail(DGP_ERR_ARG, "fem_assemble: null handle");
  DGP_GUARD(fem_assemble(&fem->plan, d_mua, d_musp, d_K, d_M, (cudaStream_t)stream));
}

int dgp_fem_adjoint_grad(dgp_fem_t fem, const double *d_mua, const double *d_musp, const double *d_phi,
                         const double *d_lam, int32_t nf, int32_t ns, double *d_gmua, double *d_gmusp,
                         dgp_stream_t stream) {
  if (!fem) return fail(DGP_ERR_ARG, "fem_adjoint_grad: null handle");
  DGP_GUARD(fem_adjoint_grad(&fem->plan, d_mua, d_musp, d_phi, d_lam, nf, ns, d_gmua, d_gmusp,
                             (cudaStream_t)stream));
}

// ----------------------------------------------------------------- solver
void dgp_solve_opts_default(dgp_solve_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->tol = 1e-12;       // dMesh.m:1243
  o->maxit = 1000;      // dMesh.m:1243
  o->precision = DGP_PREC_FP64;
  o->inner_tol = 3e-5;  // per-column inner stop: final FP64 residual ~10x below tol
  o->max_refine = 8;
  o->fsai_cap = 30;     // dMesh.m:1363
  o->stop_rule = DGP_STOP_MAX_ALL;
  o->check_every = 8;
}

int dgp_solver_create(dgp_solver_t *solver, const int32_t *d_rowptr, const int32_t *d_col, int64_t n, int64_t nnz,
                      const double *d_K, const double *d_M, double dfc, int32_t nf, int32_t ns_max,
                      const dgp_solve_opts *opts, dgp_stream_t stream) {
  return dgp_solver_create_harmonics(solver, d_rowptr, d_col, n, nnz, d_K, d_M, dfc, nullptr, nf, ns_max, opts,
                                     stream);
}

int dgp_solver_create_harmonics(dgp_solver_t *solver, const int32_t *d_rowptr, const int32_t *d_col, int64_t n,
                                int64_t nnz, const double *d_K, const double *d_M, double dfc,
                                const int32_t *h_harmonics, int32_t nf, int32_t ns_max, const dgp_solve_opts *opts,
                                dgp_stream_t stream) {
  if (!solver || !d_rowptr || !d_col || !d_K || !d_M) return fail(DGP_ERR_ARG, "solver_create: null pointer");
  *solver = nullptr;
  dgp_solver_s *h = new (std::nothrow) dgp_solver_s();
  if (!h) return fail(DGP_ERR_NOMEM, "solver_create: host allocation failed");
  int rc;
  try {
    rc = solver_build(&h->plan, d_rowptr, d_col, n, nnz, d_K, d_M, dfc, nf, ns_max, opts, (cudaStream_t)stream,
                      h_harmonics);
  } catch (...) {
    rc = fail(DGP_ERR_NOMEM, "solver_create: exception");
  }
  if (rc != DGP_OK) {
    delete h;
    return rc;
  }
  *solver = h;
  return DGP_OK;
}

int dgp_solver_update(dgp_solver_t s, const double *d_K, const double *d_M, dgp_stream_t stream) {
  if (!s || !d_K || !d_M) return fail(DGP_ERR_ARG, "solver_update: null pointer");
  DGP_GUARD(solver_update(&s->plan, d_K, d_M, (cudaStream_t)stream));
}

int dgp_solver_destroy(dgp_solver_t s) {
  delete s;
  return DGP_OK;
}

int dgp_solver_memory(dgp_solver_t s, int64_t *bytes) {
  if (!s || !bytes) return fail(DGP_ERR_ARG, "solver_memory: null pointer");
  const SolverPlan &p = s->plan;
  int64_t b = 0;
  const DevBuf *bufs[] = {&p.rowptr, &p.col, &p.KM64, &p.RecA32, &p.dfcM, &p.omega, &p.G64, &p.GT64, &p.RecG32, &p.RecGT32,
                          &p.P.rowptr, &p.P.col, &p.P.rowptrT, &p.P.colT, &p.P.permT, &p.scal, &p.ctl, &p.status};
  for (auto *d : bufs) b += (int64_t)d->bytes;
  for (auto &v : p.vec) b += (int64_t)v.bytes;
  *bytes = b;
  return DGP_OK;
}

int dgp_solve(dgp_solver_t s, const double *d_B, double *d_X, int32_t ns, const dgp_solve_opts *opts,
              dgp_solve_report *report, dgp_stream_t stream) {
  if (!s || !d_B || !d_X) return fail(DGP_ERR_ARG, "solve: null pointer");
  DGP_GUARD(solver_solve(&s->plan, d_B, nullptr, nullptr, nullptr, d_X, ns, opts, report, (cudaStream_t)stream));
}

int dgp_solver_autotune(dgp_solver_t s, int32_t *tiled, int32_t *vec, int32_t *rows, float *ms,
                        dgp_stream_t stream) {
  if (!s) return fail(DGP_ERR_ARG, "solver_autotune: null handle");
  DGP_GUARD(solver_autotune(&s->plan, tiled, vec, rows, ms, (cudaStream_t)stream));
}

int dgp_solver_set_spmm(dgp_solver_t s, int32_t tiled, int32_t vec, int32_t rows) {
  if (!s) return fail(DGP_ERR_ARG, "solver_set_spmm: null handle");
  DGP_GUARD(solver_set_spmm(&s->plan, tiled, vec, rows));
}

int dgp_solver_set_spmm_kind(dgp_solver_t s, int32_t kind) {
  if (!s) return fail(DGP_ERR_ARG, "solver_set_spmm_kind: null handle");
  DGP_GUARD(solver_set_spmm_kind(&s->plan, kind));
}

int dgp_solver_set_device_loop(dgp_solver_t s, int32_t on) {
  if (!s) return fail(DGP_ERR_ARG, "solver_set_device_loop: null handle");
  DGP_GUARD(solver_set_device_loop(&s->plan, on));
}

int dgp_solver_spmm_shape(dgp_solver_t s, int32_t *tiled, int32_t *vec, int32_t *rows, int32_t *kind) {
  if (!s) return fail(DGP_ERR_ARG, "solver_spmm_shape: null handle");
  if (tiled) *tiled = s->plan.tiled;
  if (vec) *vec = s->plan.tune_vec;
  if (rows) *rows = s->plan.tune_rows;
  if (kind) *kind = s->plan.tune_kind;
  return DGP_OK;
}

int dgp_solver_set_dot_rows(dgp_solver_t s, int32_t mult) {
  if (!s) return fail(DGP_ERR_ARG, "solver_set_dot_rows: null handle");
  DGP_GUARD(solver_set_dot_rows(&s->plan, mult));
}

int dgp_solver_check_spmm(dgp_solver_t s, double *max_rel, dgp_stream_t stream) {
  if (!s) return fail(DGP_ERR_ARG, "solver_check_spmm: null handle");
  DGP_GUARD(solver_check_spmm(&s->plan, max_rel, (cudaStream_t)stream));
}

int dgp_solve_mex(dgp_solver_t s, const double *d_Q, double *d_X, int32_t ns, int32_t layout,
                  const dgp_solve_opts *opts, dgp_solve_report *report, dgp_stream_t stream) {
  if (!s) return fail(DGP_ERR_ARG, "solve_mex: null handle");
  DGP_GUARD(solve_mexlayout(&s->plan, d_Q, d_X, ns, layout, opts, report, (cudaStream_t)stream));
}

int dgp_solve_sources(dgp_solver_t s, const int32_t *d_nodes, const double *d_w, const double *d_fpsf, int32_t ns,
                      double *d_X, const dgp_solve_opts *opts, dgp_solve_report *report, dgp_stream_t stream) {
  if (!s || !d_nodes || !d_w || !d_fpsf || !d_X) return fail(DGP_ERR_ARG, "solve_sources: null pointer");
  DGP_GUARD(solver_solve(&s->plan, nullptr, d_nodes, d_w, d_fpsf, d_X, ns, opts, report, (cudaStream_t)stream));
}

int dgp_solver_profile_kernel(dgp_solver_t s, int32_t which, int32_t reps, float *ms, double *bytes,
                              dgp_stream_t stream) {
  if (!s || !ms || !bytes) return fail(DGP_ERR_ARG, "solver_profile_kernel: null pointer");
  DGP_GUARD(solver_profile(&s->plan, which, reps, ms, bytes, (cudaStream_t)stream));
}

// ------------------------------------------------------ batched operators
int dgp_spmm_A(const int32_t *d_rowptr, const int32_t *d_col, const double *d_KM, const double *d_omega, int64_t n,
               int32_t nf, int32_t ns, const double *d_X, double *d_Y, dgp_stream_t stream) {
  if (!d_rowptr || !d_col || !d_KM || !d_omega || !d_X || !d_Y) return fail(DGP_ERR_ARG, "spmm_A: null pointer");
  DGP_GUARD(spmm_A_f64(d_rowptr, d_col, (const double2 *)d_KM, d_omega, n, nf, ns, (const double2 *)d_X,
                       (double2 *)d_Y, (cudaStream_t)stream));
}

int dgp_fsai_pattern(const int32_t *d_rowptr, const int32_t *d_col, const double *d_K, const double *d_M, double dfc,
                     int64_t n, int32_t cap, int32_t *d_rowptrG, int32_t *d_colG, dgp_stream_t stream) {
  if (!d_rowptr || !d_col || !d_K || !d_M || !d_rowptrG) return fail(DGP_ERR_ARG, "fsai_pattern: null pointer");
  if (n <= 0) return fail(DGP_ERR_ARG, "fsai pattern: need n > 0 and 1 <= cap <= 32");
  DGP_GUARD([&] {
    DGP_TRY(csr_in_range(d_rowptr, d_col, n, n, -1, 0, "fsai_pattern: A", (cudaStream_t)stream));
    return fsai_pattern_rows(d_rowptr, d_col, d_K, d_M, dfc, n, cap, d_rowptrG, d_colG, nullptr, nullptr,
                             (cudaStream_t)stream);
  }());
}

int dgp_fsai_factor(const int32_t *d_rowptr, const int32_t *d_col, const double *d_K, const double *d_M, double dfc,
                    int64_t n, const int32_t *d_rowptrG, const int32_t *d_colG, int32_t nf, double *d_G,
                    dgp_stream_t stream) {
  if (!d_rowptr || !d_col || !d_K || !d_M || !d_rowptrG || !d_colG || !d_G)
    return fail(DGP_ERR_ARG, "fsai_factor: null pointer");
  DGP_GUARD(fsai_factor_full(d_rowptr, d_col, d_K, d_M, dfc, n, d_rowptrG, d_colG, nf, (double2 *)d_G,
                             (cudaStream_t)stream));
}

int dgp_fsai_apply(const int32_t *d_rowptrG, const int32_t *d_colG, const double *d_G, int64_t n, int64_t nnzG,
                   int32_t nf, int32_t ns, int32_t transpose, const double *d_X, double *d_Y, dgp_stream_t stream) {
  if (!d_rowptrG || !d_colG || !d_G || !d_X || !d_Y) return fail(DGP_ERR_ARG, "fsai_apply: null pointer");
  if (transpose) return fail(DGP_ERR_UNSUPPORTED, "fsai_apply: pass the transposed pattern and values instead");
  DGP_GUARD(fsai_apply_f64(d_rowptrG, d_colG, (const double2 *)d_G, n, nnzG, nf, ns, (const double2 *)d_X,
                           (double2 *)d_Y, (cudaStream_t)stream));
}

// ------------------------------------------------ measurement, transforms
int dgp_meas(const int32_t *d_det_nodes, const double *d_det_w, int32_t nd, const int32_t *d_link, int32_t nm,
             const double *d_phi, int64_t n, int32_t nf, int32_t ns, double *d_data, dgp_stream_t stream) {
  DGP_GUARD(meas_run(d_det_nodes, d_det_w, nd, d_link, nm, d_phi, n, nf, ns, d_data, (cudaStream_t)stream));
}

int dgp_csr_spmv(const int32_t *d_rowptr, const int32_t *d_col, const double *d_val, int64_t nrows, int64_t ncols,
                 const double *d_x, double *d_y, dgp_stream_t stream) {
  DGP_GUARD(csr_spmv_run(d_rowptr, d_col, d_val, nrows, ncols, d_x, d_y, (cudaStream_t)stream));
}

int dgp_td2fc(const double *d_x, int64_t nr, int32_t nt, const double *d_t, const double *d_f, int32_t nf,
              double *d_c, dgp_stream_t stream) {
  DGP_GUARD(td2fc_run(d_x, nr, nt, d_t, d_f, nf, d_c, (cudaStream_t)stream));
}

int dgp_fc2td(const double *d_c, int64_t nr, int32_t nf, const double *d_f, const double *d_t, int32_t nt,
              double *d_x, dgp_stream_t stream) {
  DGP_GUARD(fc2td_run(d_c, nr, nf, d_f, d_t, nt, d_x, (cudaStream_t)stream));
}

int dgp_fc2tg(const double *d_c, int64_t nr, int32_t nf, const double *d_gate_fc, int32_t ng, int32_t nt,
              double *d_y, dgp_stream_t stream) {
  DGP_GUARD(fc2tg_run(d_c, nr, nf, d_gate_fc, ng, nt, d_y, (cudaStream_t)stream));
}

// --------------------------------------------------------------- Jacobian
int dgp_set_jacobian_engine(int32_t engine) { DGP_GUARD(set_jacobian_engine(engine)); }

int dgp_jacobian_complex(const int32_t *d_P_rowptr, const int32_t *d_P_col, const double *d_P_val, int64_t nv,
                         const double *d_w, const double *d_phi, int32_t ns, const double *d_phiA, int32_t nd,
                         int64_t nn, int32_t nf, const double *d_fpsf, const int32_t *d_link, int32_t nm, double *d_J,
                         dgp_stream_t stream) {
  DGP_GUARD(jacobian_run(1, d_P_rowptr, d_P_col, d_P_val, nv, d_w, d_phi, ns, d_phiA, nd, nn, nf, d_fpsf, d_link, nm,
                         nullptr, 0, 0, nullptr, d_J, nullptr, (cudaStream_t)stream));
}

int dgp_jacobian_tg(const int32_t *d_P_rowptr, const int32_t *d_P_col, const double *d_P_val, int64_t nv,
                    const double *d_w, const double *d_phi, int32_t ns, const double *d_phiA, int32_t nd, int64_t nn,
                    int32_t nf, const double *d_fpsf, const int32_t *d_link, int32_t nm, const double *d_gate_fc,
                    int32_t ng, int32_t nt, const double *d_data_tg, float *d_J, dgp_stream_t stream) {
  DGP_GUARD(jacobian_run(0, d_P_rowptr, d_P_col, d_P_val, nv, d_w, d_phi, ns, d_phiA, nd, nn, nf, d_fpsf, d_link, nm,
                         d_gate_fc, ng, nt, d_data_tg, d_J, nullptr, (cudaStream_t)stream));
}

int dgp_jacobian_tg_vjp(const int32_t *d_P_rowptr, const int32_t *d_P_col, const double *d_P_val, int64_t nv,
                        const double *d_w, const double *d_phi, int32_t ns, const double *d_phiA, int32_t nd,
                        int64_t nn, int32_t nf, const double *d_fpsf, const int32_t *d_link, int32_t nm,
                        const double *d_gate_fc, int32_t ng, int32_t nt, const double *d_data_tg, const double *d_g,
                        double *d_out, dgp_stream_t stream) {
  DGP_GUARD(jacobian_run(2, d_P_rowptr, d_P_col, d_P_val, nv, d_w, d_phi, ns, d_phiA, nd, nn, nf, d_fpsf, d_link, nm,
                         d_gate_fc, ng, nt, d_data_tg, d_out, d_g, (cudaStream_t)stream));
}

int dgp_tg_adjoint_rhs(const int32_t *d_det_nodes, const double *d_det_w, int32_t nd, const int32_t *d_link,
                       int32_t nm, const double *d_gate_fc, int32_t ng, int32_t nt, const double *d_g, int64_t n,
                       int32_t nf, int32_t ns, double *d_B, dgp_stream_t stream) {
  DGP_GUARD(tg_adjoint_rhs(d_det_nodes, d_det_w, nd, d_link, nm, d_gate_fc, ng, nt, d_g, n, nf, ns, d_B,
                           (cudaStream_t)stream));
}

// ----------------------------------------------------------- point location
int dgp_locate_points(const double *d_node, const int32_t *d_elem, int64_t nn, int64_t ne, const double *d_pts,
                      int64_t np, double eps, int32_t *d_eid, double *d_w, dgp_stream_t stream) {
  DGP_GUARD(locate_points(d_node, d_elem, nn, ne, d_pts, np, eps, d_eid, d_w, (cudaStream_t)stream));
}

int dgp_grid_to_mesh(const double *d_node, int64_t nn, const double *origin, const double *spacing, const int32_t *n,
                     const uint8_t *d_inmesh, int32_t *d_col, double *d_val, dgp_stream_t stream) {
  if (!origin || !spacing || !n) return fail(DGP_ERR_ARG, "grid_to_mesh: null lattice description");
  DGP_GUARD(grid_to_mesh(d_node, nn, origin, spacing, n, d_inmesh, d_col, d_val, (cudaStream_t)stream));
}

int dgp_snap_to_surface(const double *d_node, int64_t nn, const int32_t *d_bnd, const int32_t *d_face,
                        int64_t nface, const double *d_pos, int64_t n, double *d_out_pos, double *d_out_dir,
                        int32_t *d_out_face, dgp_stream_t stream) {
  DGP_GUARD(snap_to_surface(d_node, nn, d_bnd, d_face, nface, d_pos, n, d_out_pos, d_out_dir, d_out_face,
                            (cudaStream_t)stream));
}

// -------------------------------------------------------- normal equations
int dgp_normal_eq(const float *d_Jt, int64_t nv, int64_t nmeas, const double *d_w, const double *d_y, double lambda,
                  int32_t damping, double *d_H, int64_t ldh, double *d_rhs, dgp_stream_t stream) {
  DGP_GUARD(normal_eq_run(d_Jt, nv, nmeas, d_w, d_y, lambda, damping, d_H, ldh, d_rhs, (cudaStream_t)stream));
}

int dgp_times_jt(const double *d_A, int64_t na, int64_t nv, const float *d_Jt, int64_t nmeas, double *d_out,
                 dgp_stream_t stream) {
  DGP_GUARD(times_jt_run(d_A, na, nv, d_Jt, nmeas, d_out, (cudaStream_t)stream));
}

int dgp_cholesky_solve(double *d_H, int64_t n, int64_t ldh, double *d_x, dgp_stream_t stream) {
  DGP_GUARD(cholesky_solve_run(d_H, n, ldh, d_x, (cudaStream_t)stream));
}

int dgp_row_dots(const float *d_Jt, int64_t nv, int64_t nmeas, const double *d_w, const double *d_y, double *d_diag,
                 double *d_rhs, dgp_stream_t stream) {
  DGP_GUARD(row_dots_run(d_Jt, nv, nmeas, d_w, d_y, d_diag, d_rhs, (cudaStream_t)stream));
}

int dgp_lm_update(const float *d_Jt, int64_t nv, int64_t nmeas, const double *d_w, const double *d_y, double lambda,
                  double *d_x, int32_t form, int32_t *form_used, dgp_stream_t stream) {
  DGP_GUARD(lm_update_run(d_Jt, nv, nmeas, d_w, d_y, lambda, d_x, form, form_used, (cudaStream_t)stream));
}

int dgp_cholesky_solve_many(double *d_H, int64_t n, int64_t ldh, double *d_X, int32_t nrhs, int64_t ldx,
                            dgp_stream_t stream) {
  DGP_GUARD(cholesky_solve_many_run(d_H, n, ldh, d_X, nrhs, ldx, (cudaStream_t)stream));
}

}  // extern "C"

// ----------------------------------------------- C++-linkage drop-ins
void smv_call(double *const d_out_real, double *const d_out_imag, const double *const d_x_real,
              const double *const d_x_imag, const double *const d_fAxis, const double *const d_valA_real,
              const double *const d_valA_imag, const int *const d_rPtr, const int *const d_cPtr, const int nrows,
              const int ncols, const int nfreqs) {
  dgp_smv_mex(d_out_real, d_out_imag, d_x_real, d_x_imag, d_fAxis, d_valA_real, d_valA_imag, d_rPtr, d_cPtr, nrows,
              ncols, nfreqs, nullptr);
}

void FSAImv_call(double *const d_out_real, double *const d_out_imag, const double *const d_x_real,
                 const double *const d_x_imag, const double *const d_valG_real, const double *const d_valG_imag,
                 const int *const d_rPtr, const int *const d_cPtr, const int nnz, const int nrows, const int ncols,
                 const int nfreqs) {
  dgp_fsaimv_mex(d_out_real, d_out_imag, d_x_real, d_x_imag, d_valG_real, d_valG_imag, d_rPtr, d_cPtr, nnz, nrows,
                 ncols, nfreqs, nullptr);
}

void FSAIP_call(double *const d_out_real, double *const d_out_imag, const double *const d_valA_real,
                const double *const d_valA_imag, const int *const d_rPtrA, const int *const d_cPtrA,
                const int *const d_rPtrG, const int *const d_cPtrG, const int nfreqs, const int nrows) {
  dgp_fsaip_mex(d_out_real, d_out_imag, d_valA_real, d_valA_imag, d_rPtrA, d_cPtrA, d_rPtrG, d_cPtrG, nfreqs, nrows,
                nullptr);
}
