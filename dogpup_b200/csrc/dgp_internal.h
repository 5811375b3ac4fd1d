// Internal plan structures shared by the dogpup_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dgp_common.cuh"

namespace dgp {

// ------------------------------------------------------------------ FEM
struct FemPlan {
  int64_t nn = 0, ne = 0, nfaces = 0, nnz = 0, nk = 0, nbnd = 0;
  double nr = 0, c = 0, rfac = 0;
  DevBuf node, elem;      // copies of the mesh
  DevBuf bnd;             // int32 [nn]
  DevBuf faces;           // int32 [nfaces][3] Robin face set
  DevBuf rowptr, col;     // int32 CSR pattern (full symmetric)
  DevBuf cstart, payload; // per-slot contribution lists
  DevBuf Ke, Me, Be;      // element / face blocks (scratch of every assembly)
  DevBuf flag;            // int: degenerate-element flag of the element kernel (kept: no per-call allocation)
};

int fem_create(FemPlan *F, const double *d_node, const int32_t *d_elem, int64_t nn, int64_t ne, double nr,
               cudaStream_t st);
int fem_assemble(FemPlan *F, const double *d_mua, const double *d_musp, double *d_K, double *d_M,
                 cudaStream_t st);
// dL/dmua (and dL/dmusp when d_gmusp is not NULL) = -Re sum lam^T (dA/dp) phi
int fem_adjoint_grad(FemPlan *F, const double *d_mua, const double *d_musp, const double *d_phi,
                     const double *d_lam, int32_t nf, int32_t ns, double *d_gmua, double *d_gmusp,
                     cudaStream_t st);
// adjoint sources of L = sum g . fc2tg(meas(phi))
int tg_adjoint_rhs(const int32_t *d_det_nodes, const double *d_det_w, int32_t nd, const int32_t *d_link, int32_t nm,
                   const double *d_gate_fc, int32_t ng, int32_t nt, const double *d_g, int64_t n, int32_t nf,
                   int32_t ns, double *d_B, cudaStream_t st);

// ----------------------------------------------------------------- FSAI
struct FsaiPattern {
  int64_t n = 0, nnzG = 0;
  int32_t mmax = 0;          // longest pattern row
  DevBuf rowptr, col;        // lower-triangular pattern of G
  DevBuf rowptrT, colT;      // pattern of G^T
  DevBuf permT;              // G^T slot t holds G slot permT[t]
};

int fsai_pattern_build(FsaiPattern *P, const int32_t *d_rowptr, const int32_t *d_col, const double *d_K,
                       const double *d_M, double dfc, int64_t n, int32_t cap, cudaStream_t st);
// pattern counts / fill as exposed by the C ABI
int fsai_pattern_rows(const int32_t *d_rowptr, const int32_t *d_col, const double *d_K, const double *d_M,
                      double dfc, int64_t n, int32_t cap, int32_t *d_rowptrG, int32_t *d_colG,
                      int32_t *h_nnzG, int32_t *h_mmax, cudaStream_t st);
// G values of A_h = Re + i*h*Im for the harmonics h = d_harm[j] (j = 0 .. nf-1;
// h = j when d_harm is NULL), written to out[slot * s_slot + j * s_k]
// (complex128 interleaved).
int fsai_factor_run(const int32_t *d_rowptr, const int32_t *d_col, const double *d_re, const double *d_im,
                    int64_t n, const int32_t *d_rowptrG, const int32_t *d_colG, int32_t mmax, int32_t nf,
                    double2 *d_out, int64_t s_slot, int64_t s_k, cudaStream_t st, const int32_t *d_harm = nullptr);
int fsai_transpose_pattern(FsaiPattern *P, cudaStream_t st);
int fsai_factor_full(const int32_t *d_rowptr, const int32_t *d_col, const double *d_K, const double *d_M, double dfc,
                     int64_t n, const int32_t *d_rowptrG, const int32_t *d_colG, int32_t nf, double2 *d_G,
                     cudaStream_t st);

// ---------------------------------------------------------------- solver
// Row-block halo plan of the tiled SpMM (complex-FP32 sweeps): rows are cut
// into blocks of rb consecutive rows; block b stages the distinct columns
// hcols[hptr[b] .. hptr[b+1]) of its rows in shared memory, and each nonzero
// p carries its column's position in that list, lcol[p].
struct TiledPlan {
  int32_t rb = 0, hmax = 0, zmax = 0;  // rows per block, largest halo, most nonzeros in a block
  int64_t nblk = 0;
  DevBuf hptr, hcols, lcol;
};

struct SolverPlan {
  int64_t n = 0, nnz = 0, nnzG = 0;
  int32_t nf = 0, ns_max = 0, nsp = 0;  // nsp: padded sources per harmonic
  double dfc = 0;
  dgp_solve_opts opts{};
  DevBuf rowptr, col;            // A pattern
  DevBuf KM64;                   // interleaved (K, M) per slot, FP64
  DevBuf RecA32;                 // FP32 path: one 16-byte (col, K, M) record per slot
  DevBuf dfcM;                   // [nnz] dfc * M, the imaginary part of the FSAI input (update scratch)
  DevBuf node_flag;              // int: out-of-range source node flag (solve scratch)
  DevBuf omega;                  // [nf] h_j * dfc (FP64), then [nf] FP32
  DevBuf harm;                   // [nf] harmonic index h_j of batch slot j
  FsaiPattern P;
  DevBuf G64, GT64;              // [nf][nnzG] complex128
  DevBuf RecG32, RecGT32;        // FP32 path: [nf][nnzG] 16-byte (col, Re, Im) records
  // workspace (allocated lazily per precision)
  int ws_prec = -1;
  int64_t ws_cols = 0;
  DevBuf vec[12];                // solver vectors
  DevBuf scal;                   // per-column scalars
  DevBuf ctl;                    // control block
  DevBuf status;                 // per-column status
  void *h_ctl = nullptr;         // pinned mirrors of the control block (two)
  cudaEvent_t poll_ev[2] = {nullptr, nullptr};  // the two mirrors' copy-done events
  // blocks of iterations captured as graphs -- [0..2]: FP64 BiCGSTAB, FP32 BiCGSTAB, FP32 COCG
  // (replayed and polled by the host); [3..5]: the same inside a device-driven WHILE loop
  cudaGraphExec_t graph[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  int graph_iters[6] = {0, 0, 0, 0, 0, 0};
  int32_t device_loop = 1;       // 1: an inner solve is one graph launch (WHILE node), 0: host polling
  // SpMM launch shape of the complex-FP32 sweeps chosen by solver_autotune (0 = built-in default)
  int32_t tune_vec = 0, tune_rows = 0;
  int32_t tune_kind = 0;  // gather SpMM inner loop: 0 one nonzero per step, 1 two, 2 four, 3 four + packed FMAs
  int32_t tune_dot = 0;  // rows per block of the FP32 dot-product sweeps, as a multiple of tune_rows (0: 4)
  // tiled SpMM (halo rows staged in shared memory) for A, G and G^T; tiled = 1 selects it
  TiledPlan tA, tG, tGT;
  int32_t tiled_ok = 0, tiled = 0;
  int64_t bytes = 0;
  ~SolverPlan();
};

// h_harm: host list of the nf harmonic indices the plan solves (NULL = 0 .. nf-1)
int solver_build(SolverPlan *S, const int32_t *d_rowptr, const int32_t *d_col, int64_t n, int64_t nnz,
                 const double *d_K, const double *d_M, double dfc, int32_t nf, int32_t ns_max,
                 const dgp_solve_opts *opts, cudaStream_t st, const int32_t *h_harm = nullptr);
int solver_update(SolverPlan *S, const double *d_K, const double *d_M, cudaStream_t st);
int solver_solve(SolverPlan *S, const double *d_B, const int32_t *d_nodes, const double *d_w,
                 const double *d_fpsf, double *d_X, int32_t ns, const dgp_solve_opts *opts,
                 dgp_solve_report *rep, cudaStream_t st);

// gpuBicstab_FSAIP on MATLAB's [N x NS x NF] interleaved layout (transposes around solver_solve)
int solve_mexlayout(SolverPlan *S, const double *d_Q, double *d_X, int32_t ns, int32_t layout,
                    const dgp_solve_opts *opts, dgp_solve_report *rep, cudaStream_t st);

int solver_profile(SolverPlan *S, int which, int reps, float *ms, double *bytes, cudaStream_t st);
// times the complex-FP32 SpMM sweeps of one iteration for each candidate lane width x rows per
// block on the plan's own workspace and keeps the fastest (tune_vec, tune_rows)
int solver_autotune(SolverPlan *S, int32_t *tiled, int32_t *vec, int32_t *rows, float *ms, cudaStream_t st);
// sets the SpMM kind / shape explicitly (tiled 0: gather kernel with vec, rows; 1: tiled)
int solver_set_spmm(SolverPlan *S, int32_t tiled, int32_t vec, int32_t rows);
int solver_set_spmm_kind(SolverPlan *S, int32_t kind);
int solver_set_device_loop(SolverPlan *S, int32_t on);
int solver_set_dot_rows(SolverPlan *S, int32_t mult);
// largest relative difference between the tiled and the gather SpMM on the plan's operators
int solver_check_spmm(SolverPlan *S, double *max_rel, cudaStream_t st);

// DGP_ERR_MESH unless every id in d_ids[0..count) lies in [0, limit) (synchronises the stream)
int ids_in_range(const int32_t *d_ids, int64_t count, int64_t limit, const char *who, cudaStream_t st);
// DGP_ERR_MESH unless d_rowptr[0..nrows] starts at 0, never decreases and (nnz >= 0) ends at nnz, no
// row holds more than max_row entries (max_row > 0), and every column id lies in [0, ncols)
// (synchronises the stream)
int csr_in_range(const int32_t *d_rowptr, const int32_t *d_col, int64_t nrows, int64_t ncols, int64_t nnz,
                 int64_t max_row, const char *who, cudaStream_t st);

// containing tetrahedron (-1: none) and barycentric weights [np][4] of points [np][3]
int locate_points(const double *d_node, const int32_t *d_elem, int64_t nn, int64_t ne, const double *d_pts,
                  int64_t np, double eps, int32_t *d_eid, double *d_w, cudaStream_t st);

// grid-to-mesh interpolation rows [nn][4] (voxel index or -1, weight) on a rectilinear lattice
int grid_to_mesh(const double *d_node, int64_t nn, const double origin[3], const double spacing[3], const int32_t n[3],
                 const uint8_t *d_inmesh, int32_t *d_col, double *d_val, cudaStream_t st);

// optode snapping: closest surface point, inward normal and face of each position
int snap_to_surface(const double *d_node, int64_t nn, const int32_t *d_bnd, const int32_t *d_face, int64_t nface,
                    const double *d_pos, int64_t n, double *d_out_pos, double *d_out_dir, int32_t *d_out_face,
                    cudaStream_t st);

// batched operators (layout [nf][n][ns] complex)
int spmm_A_f64(const int32_t *rowptr, const int32_t *col, const double2 *KM, const double *omega, int64_t n,
               int32_t nf, int32_t ns, const double2 *X, double2 *Y, cudaStream_t st);
int fsai_apply_f64(const int32_t *rowptr, const int32_t *col, const double2 *G, int64_t n, int64_t nnzG,
                   int32_t nf, int32_t ns, const double2 *X, double2 *Y, cudaStream_t st);

// FP64 Cholesky H = L L^T (lower triangle of the row-major H, overwritten by L) and the solve of
// L L^T x = b for one (cholesky_solve_run) or nrhs right-hand sides stored as the rows of x
int cholesky_solve_run(double *H, int64_t n, int64_t ldh, double *x, cudaStream_t st);
int cholesky_solve_many_run(double *H, int64_t n, int64_t ldh, double *x, int32_t nrhs, int64_t ldx,
                            cudaStream_t st);

}  // namespace dgp
