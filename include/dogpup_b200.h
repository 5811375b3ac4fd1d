/*
 * dogpup_b200.h -- C ABI of the B200 (sm_100a) forward/sensitivity path of
 * DOGPUP (diffuse optical tomography: frequency-domain diffusion FEM,
 * FSAI-preconditioned BiCGSTAB over all source x harmonic right-hand sides,
 * adjoint absorption Jacobian, Fourier-series time-domain / time-gate
 * transforms, weighted Levenberg-Marquardt normal-equation step).
 *
 * Conventions
 *   - Every pointer named d_* is device memory owned by the caller unless a
 *     function says otherwise; h_* is host memory.
 *   - Complex numbers are interleaved (re, im) pairs of double or float.
 *   - Batched fields use the layout [NF][NN][NS]: harmonic k slowest, node i,
 *     source s fastest (element (k,i,s) at ((k*NN)+i)*NS+s).  The
 *     MATLAB-facing drop-ins below keep the reference's own layouts.
 *   - Indices are 0-based int32; element counts and offsets are int64.
 *   - Functions return 0 (DGP_OK) or a dgp_status code; dgp_last_error()
 *     returns a message for the calling thread's last failure.
 *   - Work is enqueued on the given stream and is asynchronous unless a
 *     function says it synchronises.
 */
#ifndef DOGPUP_B200_H
#define DOGPUP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *dgp_stream_t; /* same type as cudaStream_t */

typedef enum dgp_status {
  DGP_OK = 0,
  DGP_ERR_ARG = 1,        /* invalid argument or size                       */
  DGP_ERR_CUDA = 2,       /* a CUDA runtime call failed                     */
  DGP_ERR_NOMEM = 3,      /* device allocation failed                       */
  DGP_ERR_MESH = 4,       /* degenerate mesh / pattern (e.g. zero volume)   */
  DGP_ERR_NOT_CONVERGED = 5, /* solver hit maxit before tol (x still valid) */
  DGP_ERR_BREAKDOWN = 6,  /* reserved: solves report a breakdown per column
                           (DGP_COL_BREAKDOWN_*) under DGP_ERR_NOT_CONVERGED */
  DGP_ERR_UNSUPPORTED = 7
} dgp_status;

/* Per-column solver status words written to dgp_solve_report.d_status. */
enum {
  DGP_COL_CONVERGED = 0,
  DGP_COL_MAXIT = 1,
  DGP_COL_BREAKDOWN_RHO = 2,
  DGP_COL_BREAKDOWN_OMEGA = 3,
  DGP_COL_NONFINITE = 4,
  DGP_COL_ZERO_RHS = 5
};

const char *dgp_last_error(void);
const char *dgp_status_string(int status);
int dgp_version(void);
/* Number of kernels this library has launched in the process so far
 * (kernels inside its CUDA graphs included). */
int64_t dgp_kernel_launches(void);
/* Number of device allocations (cudaMalloc calls, failed ones included) this
 * library's own code has made in the process so far; allocations made inside
 * cuBLAS are not counted. */
int64_t dgp_device_allocations(void);

/* ====================================================================== *
 *  Drop-in host functions of the reference mex sources.  Same names,
 *  argument order and layouts (split real/imag planes, column-major
 *  [N x NS x NF]); C++ linkage like the reference headers, declared in
 *  dogpup_b200_mex.hpp.  The extern "C" forms below add a stream and a
 *  status return.
 * ====================================================================== */

/* Replaces smv_call, cuda_lib/mex_sources/smvMex.hpp:4-15 (smv_CUDA.cu:59-82):
 * y[:,s,f] = (Re A + i*fAxis[f]*Im A) x[:,s,f], A full symmetric CSR. */
int dgp_smv_mex(double *d_out_real, double *d_out_imag, const double *d_x_real,
                const double *d_x_imag, const double *d_fAxis,
                const double *d_valA_real, const double *d_valA_imag,
                const int *d_rPtr, const int *d_cPtr, int nrows, int ncols,
                int nfreqs, dgp_stream_t stream);

/* Replaces FSAImv_call, cuda_lib/mex_sources/FSAImvMex.hpp:4-15
 * (FSAImv_CUDA.cu:58-81): y[:,s,f] = G_f x[:,s,f], G values [nnz x NF]. */
int dgp_fsaimv_mex(double *d_out_real, double *d_out_imag,
                   const double *d_x_real, const double *d_x_imag,
                   const double *d_valG_real, const double *d_valG_imag,
                   const int *d_rPtr, const int *d_cPtr, int nnz, int nrows,
                   int ncols, int nfreqs, dgp_stream_t stream);

/* Replaces FSAIP_call, cuda_lib/mex_sources/FSAIP.hpp:4-13
 * (FSAIP_CUDA.cu:162-180): FSAI factor of tril(A) for harmonics
 * 0..nfreqs-1, output [NF x nnzG] (harmonic fastest) like the reference. */
int dgp_fsaip_mex(double *d_out_real, double *d_out_imag,
                  const double *d_valA_real, const double *d_valA_imag,
                  const int *d_rPtrA, const int *d_cPtrA, const int *d_rPtrG,
                  const int *d_cPtrG, int nfreqs, int nrows,
                  dgp_stream_t stream);

/* The same three operations on interleaved complex data (MATLAB's
 * interleaved-complex API, R2018a+): each complex array is one pointer to
 * (re, im) pairs in the layout above, which saves the gateways the
 * real/imaginary split copies the reference makes (mxGPUCopyReal/Imag). */
int dgp_smv_mex_ic(double *d_out, const double *d_x, const double *d_fAxis,
                   const double *d_valA, const int *d_rPtr, const int *d_cPtr,
                   int nrows, int ncols, int nfreqs, dgp_stream_t stream);
int dgp_fsaimv_mex_ic(double *d_out, const double *d_x, const double *d_valG,
                      const int *d_rPtr, const int *d_cPtr, int nnz, int nrows,
                      int ncols, int nfreqs, dgp_stream_t stream);
int dgp_fsaip_mex_ic(double *d_out, const double *d_valA, const int *d_rPtrA,
                     const int *d_cPtrA, const int *d_rPtrG, const int *d_cPtrG,
                     int nfreqs, int nrows, dgp_stream_t stream);

/* No counterpart in the reference.  dgp_fsaip_mex for callers that must not
 * allocate device memory -- a MATLAB mex gateway whose device memory has to
 * come from MATLAB's gpuArray pool, or an application whose own pooling
 * allocator owns the GPU.  Same arguments and output; it allocates nothing
 * and stages its work in one fixed 16 MiB device array that every GPU loading
 * the library keeps until exit.  Limit: nfreqs * (longest pattern row)
 * <= 1048576, else DGP_ERR_ARG; a G row pointer that does not start at 0 or
 * decreases is DGP_ERR_MESH.  All calls share that array: calls that overlap
 * on the GPU race, so serialise them.  The first call in each CUDA context
 * (a new one after a device reset included) looks the array up; make it
 * before any stream capture.  Synchronises the stream. */
int dgp_fsaip_mex_noalloc(double *d_out_real, double *d_out_imag,
                          const double *d_valA_real, const double *d_valA_imag,
                          const int *d_rPtrA, const int *d_cPtrA,
                          const int *d_rPtrG, const int *d_cPtrG, int nfreqs,
                          int nrows, dgp_stream_t stream);

/* ====================================================================== *
 *  FEM topology and assembly on the device.
 *  Replaces prepare_mesh + gen_fwdmat + update_properties,
 *  DOGPUP/dMesh.m:80-88, :945-1030, :1033-1235.
 * ====================================================================== */
typedef struct dgp_fem_s *dgp_fem_t;

/* Builds, on the device: element volumes and inverse-Jacobians, the
 * boundary-node flags (faces owned by one tet), the Robin face set of
 * dMesh.m:1129-1140, the full symmetric CSR pattern of the FEM matrix and
 * the element-to-slot gather map.  d_node [nn][3] f64, d_elem [ne][4].
 * Synchronises the stream (it reads sizes back). */
int dgp_fem_create(dgp_fem_t *fem, const double *d_node, const int32_t *d_elem,
                   int64_t nn, int64_t ne, double nr, dgp_stream_t stream);
int dgp_fem_destroy(dgp_fem_t fem);
/* nnz of the pattern, number of Robin faces, number of boundary nodes,
 * and the speed of light in the medium c = cVac/nr (mm/s). */
int dgp_fem_info(dgp_fem_t fem, int64_t *nnz, int64_t *n_robin_faces,
                 int64_t *n_boundary, double *c_medium);
/* Borrowed device pointers to the CSR pattern (valid until destroy). */
int dgp_fem_pattern(dgp_fem_t fem, const int32_t **d_rowptr,
                    const int32_t **d_col);
/* Boundary flags (int32 0/1) of every node. */
int dgp_fem_boundary(dgp_fem_t fem, int32_t *d_bnd, dgp_stream_t stream);
/* K (stiffness with kappa = 1/(3(mua+musp)) + absorption + Robin) and M
 * (mass) values on the pattern, float64, from nodal mua and musp. */
int dgp_fem_assemble(dgp_fem_t fem, const double *d_mua, const double *d_musp,
                     double *d_K, double *d_M, dgp_stream_t stream);
/* Reverse-mode gradient of a real functional L(phi) through the assembly:
 *   d_gmua[v]  = dL/dmua_v  = -Re sum_{k,s} lam_{k,s}^T (dA_k/dmua_v)  phi_{k,s}
 *   d_gmusp[v] = dL/dmusp_v = -Re sum_{k,s} lam_{k,s}^T (dA_k/dmusp_v) phi_{k,s}
 * (d_gmusp may be NULL) where phi [nf][nn][ns] complex128 are the forward
 * fields and lam the adjoint fields A_k^-1 (dL/dphi_{k,s}) of the same
 * layout.  dA/dp follows the element quadrature of dgp_fem_assemble exactly,
 * kappa's dependence on mua and musp included; the reference's absorption
 * Jacobian (J_complex, dMesh.m:206-247) holds kappa fixed, which is
 * d_gmua - d_gmusp here.  No reference counterpart as one call: the
 * reference forms J explicitly and multiplies. */
int dgp_fem_adjoint_grad(dgp_fem_t fem, const double *d_mua,
                         const double *d_musp, const double *d_phi,
                         const double *d_lam, int32_t nf, int32_t ns,
                         double *d_gmua, double *d_gmusp, dgp_stream_t stream);

/* ====================================================================== *
 *  Batched solver: FSAI setup + BiCGSTAB over every source x harmonic.
 *  Replaces fluGPU + gpuBicstab_FSAIP + FSAIP_gen, dMesh.m:1238-1385,
 *  as one call instead of a MATLAB loop over mex mat-vecs.
 * ====================================================================== */
/* FP64: the reference's BiCGSTAB in FP64.  MIXED: complex-FP32 COCG
 * (conjugate-orthogonal CG: A_k and the FSAI preconditioner G^T G are
 * complex symmetric; one A and one G^T G application per iteration) inside
 * FP64 iterative refinement.  MIXED_BICGSTAB: as MIXED with complex-FP32
 * BiCGSTAB (the reference's recurrences) as the inner solver. */
enum { DGP_PREC_FP64 = 0, DGP_PREC_MIXED = 1, DGP_PREC_MIXED_BICGSTAB = 2 };
enum { DGP_STOP_MAX_ALL = 0, DGP_STOP_PER_COLUMN = 1 };

typedef struct dgp_solve_opts {
  double tol;          /* relative residual target (reference: 1e-12)      */
  int32_t maxit;       /* iterations (reference: 1000; mixed: summed over
                        * the inner solves)                                */
  int32_t precision;   /* DGP_PREC_FP64 | _MIXED | _MIXED_BICGSTAB         */
  double inner_tol;    /* mixed: complex-FP32 inner target per refinement  */
  int32_t max_refine;  /* mixed: maximum FP64 refinement steps             */
  int32_t fsai_cap;    /* FSAI pattern cap per row (reference: 30)         */
  int32_t stop_rule;   /* FP64: DGP_STOP_MAX_ALL (reference: every column
                        * iterates until the largest residual is below tol)
                        * | PER_COLUMN (each column freezes at tol; sweeps
                        * skip harmonics whose columns are all frozen).
                        * Mixed: the inner complex-FP32 solves always stop
                        * per column; every column's FP64 residual must
                        * reach tol. */
  int32_t check_every; /* iterations per host convergence poll (>= 1)      */
} dgp_solve_opts;

void dgp_solve_opts_default(dgp_solve_opts *opts);

typedef struct dgp_solve_report {
  int32_t iterations;       /* inner iterations (summed over refinement)    */
  int32_t refinements;      /* FP64 refinement steps (mixed)                */
  double max_rel_residual;  /* max over columns of ||b-Ax||/||b|| (FP64)    */
  int32_t n_not_converged;  /* columns whose status is not CONVERGED        */
  int32_t *d_status;        /* optional [NF*NS] per-column status (in/out)  */
} dgp_solve_report;

typedef struct dgp_solver_s *dgp_solver_t;

/* Creates a solver for A_k = K + i*k*dfc*M, k = 0..nf-1, on the CSR pattern
 * (d_rowptr, d_col) with values d_K, d_M (float64, copied), for up to
 * ns_max sources per harmonic.  dfc = df/c (rad/s over mm/s).  Builds the
 * FSAI pattern and factors for all harmonics and allocates the workspace.
 * DGP_ERR_MESH unless d_rowptr starts at 0, never decreases and ends at nnz
 * and every column lies in [0, n). */
int dgp_solver_create(dgp_solver_t *solver, const int32_t *d_rowptr,
                      const int32_t *d_col, int64_t n, int64_t nnz,
                      const double *d_K, const double *d_M, double dfc,
                      int32_t nf, int32_t ns_max, const dgp_solve_opts *opts,
                      dgp_stream_t stream);
/* As dgp_solver_create for an arbitrary set of harmonics: batch slot j
 * solves A_h = K + i*h*dfc*M with h = h_harmonics[j] (a host array of nf
 * indices >= 0; NULL = 0 .. nf-1, which is dgp_solver_create).  Right-hand
 * sides, d_fpsf and solutions are then indexed by slot j.  Used to shard the
 * harmonics of one mesh over several GPUs and to solve one harmonic alone;
 * the reference always solves harmonics 0 .. NF-1 together (dMesh.m:1243). */
int dgp_solver_create_harmonics(dgp_solver_t *solver, const int32_t *d_rowptr,
                                const int32_t *d_col, int64_t n, int64_t nnz,
                                const double *d_K, const double *d_M,
                                double dfc, const int32_t *h_harmonics,
                                int32_t nf, int32_t ns_max,
                                const dgp_solve_opts *opts,
                                dgp_stream_t stream);
/* New K, M values on the same pattern (e.g. after a property update):
 * re-copies them and refactors FSAI. */
int dgp_solver_update(dgp_solver_t solver, const double *d_K, const double *d_M,
                      dgp_stream_t stream);
int dgp_solver_destroy(dgp_solver_t solver);
/* Bytes of device memory the solver holds. */
int dgp_solver_memory(dgp_solver_t solver, int64_t *bytes);
/* Autotuner of the complex-FP32 (DGP_PREC_MIXED) sweeps: times the seven
 * SpMM launches of one BiCGSTAB iteration for each candidate -- the gather
 * SpMM of each inner-loop kind (dgp_solver_set_spmm_kind) at each lane width
 * (8, 4, 2 complex values per lane) x rows per block (32 .. 256) that fits
 * the plan, and the tiled SpMM (32-row blocks whose
 * halo rows are staged in shared memory) when it fits -- on the plan's own
 * workspace (allocating it if needed), and keeps the fastest for later
 * solves.  Outputs (each may be NULL): 1 if the tiled SpMM won, the best
 * gather lane width and rows per block, and the winner's time for the seven
 * launches in ms.  Synchronises the stream.  No reference counterpart (the
 * reference's launch shapes are fixed, smv_CUDA.cu:57-82). */
int dgp_solver_autotune(dgp_solver_t solver, int32_t *tiled, int32_t *vec,
                        int32_t *rows, float *ms, dgp_stream_t stream);
/* Sets the complex-FP32 SpMM explicitly: tiled = 1 selects the tiled SpMM
 * (DGP_ERR_ARG if it does not fit the plan); tiled = 0 the gather SpMM with
 * vec complex values per lane (2, 4, 8; 0 = built-in default) and rows per
 * block (32, 64, 128, 256; 0 = 64). */
int dgp_solver_set_spmm(dgp_solver_t solver, int32_t tiled, int32_t vec,
                        int32_t rows);
/* Inner loop of the complex-FP32 gather SpMM: kind 0 handles one nonzero
 * per step; 1 and 2 issue the gathers of 2 or 4 nonzeros together (lanes
 * past a row's end carry a zero coefficient on the row's own column); 3 is
 * kind 2 with packed FP32 FMAs (two instead of four FMA instructions per
 * complex product); 4 computes two harmonics of A per block, so that each
 * nonzero's record (column, K, M) is loaded and handed out once for both (the
 * G sweeps run kind 0).  dgp_solver_autotune searches the kinds with the lane widths and
 * block heights; dgp_solver_spmm_shape reports the plan's current choice. */
int dgp_solver_set_spmm_kind(dgp_solver_t solver, int32_t kind);
/* How a solve runs its iterations.  1 (default): each inner solve is ONE
 * graph launch -- a CUDA-graph WHILE node replays blocks of check_every
 * iterations and a device kernel ends the loop on convergence, at maxit, or
 * (mixed precision's inner solves) when the largest residual has stopped
 * halving; the host waits once per inner solve.  0: the host replays the
 * block graph and polls the control block between blocks. */
int dgp_solver_set_device_loop(dgp_solver_t solver, int32_t on);
int dgp_solver_spmm_shape(dgp_solver_t solver, int32_t *tiled, int32_t *vec,
                          int32_t *rows, int32_t *kind);
/* Rows per block of the complex-FP32 SpMM sweeps that also reduce a dot
 * product (v = A h with v.r^, the COCG sweeps q = A p with p.q and T = G r
 * with T.T), as a multiple of the plain sweeps' rows per block: 1, 2, 4, 8
 * or 16 (0 = default 4; at most 32 warp steps per block).  Taller blocks
 * issue fewer FP64 atomics, shorter ones more blocks (at 153k nodes x 128
 * harmonics: 4 and 2 give the shortest solve, 16 is 1 % slower, 1 is 6 %
 * slower). */
int dgp_solver_set_dot_rows(dgp_solver_t solver, int32_t mult);
/* Self-check of the two SpMM kinds: applies A_k, G_k and G_k^T to one
 * deterministic test pattern with the gather and with the tiled kernel and
 * returns max |difference| / max |value| over all three (FP32 roundoff
 * from the different summation order, ~1e-7).  Synchronises the stream. */
int dgp_solver_check_spmm(dgp_solver_t solver, double *max_rel,
                          dgp_stream_t stream);

/* Solves A_k X[k] = B[k] for every harmonic, B and X complex128
 * [NF][NN][NS] with ns <= ns_max.  Synchronises the stream; returns
 * DGP_ERR_NOT_CONVERGED if any column missed tol -- maxit, a breakdown or a
 * non-finite value, told apart by the per-column status words (X is still
 * written). */
int dgp_solve(dgp_solver_t solver, const double *d_B, double *d_X, int32_t ns,
              const dgp_solve_opts *opts, dgp_solve_report *report,
              dgp_stream_t stream);

/* dgp_solve on MATLAB's layouts: d_Q and d_X are column-major complex128
 * with interleaved real/imaginary parts (the data of a complex array under
 * MATLAB's interleaved-complex API):
 *   DGP_LAYOUT_N_NS_NF: [N x NS x NF] (x of smv_mex, gpuBicstab_FSAIP's
 *                       working layout, dMesh.m:1264)
 *   DGP_LAYOUT_N_NF_NS: [N x NF x NS] (fluGPU's Q and phi, dMesh.m:1238-1243)
 * This is the entry the bicgstab_fsai_mex gateway calls; the reference has
 * no single-call counterpart (it drives smv_mex / FSAImv_mex from a MATLAB
 * loop, dMesh.m:1247-1348). */
enum { DGP_LAYOUT_N_NS_NF = 0, DGP_LAYOUT_N_NF_NS = 1 };
int dgp_solve_mex(dgp_solver_t solver, const double *d_Q, double *d_X,
                  int32_t ns, int32_t layout, const dgp_solve_opts *opts,
                  dgp_solve_report *report, dgp_stream_t stream);

/* Same solve with the point-source right-hand sides of flu_solve /
 * adj_flu_solve (dMesh.m:124-129, :191-196) generated on the device:
 * B[k][node_s[l]][s] = w_s[l] * fpsf[k] for the 4 nodes of each optode's
 * tet.  d_nodes [ns][4] int32, d_w [ns][4] f64, d_fpsf [nf] complex128. */
int dgp_solve_sources(dgp_solver_t solver, const int32_t *d_nodes,
                      const double *d_w, const double *d_fpsf, int32_t ns,
                      double *d_X, const dgp_solve_opts *opts,
                      dgp_solve_report *report, dgp_stream_t stream);

/* Times one sweep kernel of the complex-FP32 iteration on the solver's
 * workspace with CUDA events on `stream` (which: 0 = t = A z SpMM,
 * 1 = G p SpMM, 2 = BiCGSTAB x/r/p update, 3 = h/s update, 4 = q = A p SpMM
 * with p.q, 5 = T = G r SpMM with T.T, 6 = COCG r update, 7 = COCG x/p
 * update) and returns the average
 * milliseconds per launch and the kernel's algorithmic bytes per launch.
 * Needs a prior DGP_PREC_MIXED solve; overwrites workspace vectors. */
int dgp_solver_profile_kernel(dgp_solver_t solver, int32_t which, int32_t reps,
                              float *ms, double *bytes, dgp_stream_t stream);

/* ====================================================================== *
 *  Batched sparse operators (the solver's building blocks), layout
 *  [NF][NN][NS] complex128.
 * ====================================================================== */
/* Y[k] = (K + i*omega[k]*M) X[k]; d_KM interleaved (K_ij, M_ij) per slot. */
int dgp_spmm_A(const int32_t *d_rowptr, const int32_t *d_col,
               const double *d_KM, const double *d_omega, int64_t n,
               int32_t nf, int32_t ns, const double *d_X, double *d_Y,
               dgp_stream_t stream);
/* FSAI pattern (rule of dMesh.m:1361-1380) of tril(K + i*dfc*M): counts
 * rows first (d_rowptrG [n+1]), then fills columns with a second call that
 * passes d_colG (size from d_rowptrG[n]).  DGP_ERR_MESH for a malformed CSR
 * (row pointer not starting at 0 or decreasing, column outside [0, n)). */
int dgp_fsai_pattern(const int32_t *d_rowptr, const int32_t *d_col,
                     const double *d_K, const double *d_M, double dfc,
                     int64_t n, int32_t cap, int32_t *d_rowptrG,
                     int32_t *d_colG, dgp_stream_t stream);
/* FSAI factor values G[k][slot] (complex128) for k = 0..nf-1 of
 * A_k = K + i*k*dfc*M on the pattern (arithmetic of FSAIP_CUDA.cu:92-160).
 * DGP_ERR_MESH when the CSR of A or of the G pattern is malformed. */
int dgp_fsai_factor(const int32_t *d_rowptr, const int32_t *d_col,
                    const double *d_K, const double *d_M, double dfc,
                    int64_t n, const int32_t *d_rowptrG, const int32_t *d_colG,
                    int32_t nf, double *d_G, dgp_stream_t stream);
/* Y[k] = G_k X[k] (transpose = 0) or G_k^T X[k] (transpose = 1). */
int dgp_fsai_apply(const int32_t *d_rowptrG, const int32_t *d_colG,
                   const double *d_G, int64_t n, int64_t nnzG, int32_t nf,
                   int32_t ns, int32_t transpose, const double *d_X,
                   double *d_Y, dgp_stream_t stream);

/* ====================================================================== *
 *  Detector data, Jacobian, transforms (dMesh.m:144-171, :206-247;
 *  td2fc.m, fc2td.m, fc2tg.m).
 * ====================================================================== */
/* data[m][k] = sum_l w_d[l] * phi[k][node_d[l]][s] for link m = (s, d).
 * d_nodes/d_w are the detectors' tet nodes and barycentric weights [nd][4]. */
int dgp_meas(const int32_t *d_det_nodes, const double *d_det_w, int32_t nd,
             const int32_t *d_link, int32_t nm, const double *d_phi,
             int64_t n, int32_t nf, int32_t ns, double *d_data,
             dgp_stream_t stream);

/* y = A x for a real FP64 CSR matrix A [nrows x ncols] (int32 0-based
 * row pointer and columns).  The voxel-basis maps of the LM update use it:
 * G = m2g * mua and d_mu = g2m * x (wghtd_LM_recon.m:105, :133).  Entries
 * whose column lies outside [0, ncols) are skipped. */
int dgp_csr_spmv(const int32_t *d_rowptr, const int32_t *d_col,
                 const double *d_val, int64_t nrows, int64_t ncols,
                 const double *d_x, double *d_y, dgp_stream_t stream);

/* Fourier coefficients of sampled signals: c[r][k] = dt/t_end *
 * sum_t exp(-i f_k t) x[r][t]  (td2fc.m:26-32).  x [nr][nt] f64. */
int dgp_td2fc(const double *d_x, int64_t nr, int32_t nt, const double *d_t,
              const double *d_f, int32_t nf, double *d_c, dgp_stream_t stream);
/* x[r][t] = 2 Re sum_k exp(i f_k t) c~[r][k], c~_0 = c_0/2 (fc2td.m:24-31). */
int dgp_fc2td(const double *d_c, int64_t nr, int32_t nf, const double *d_f,
              const double *d_t, int32_t nt, double *d_x, dgp_stream_t stream);
/* y[r][g] = nt * 2 Re sum_k conj(gate[g][k]) c~[r][k] (fc2tg.m:25-32). */
int dgp_fc2tg(const double *d_c, int64_t nr, int32_t nf, const double *d_gate_fc,
              int32_t ng, int32_t nt, double *d_y, dgp_stream_t stream);
/* Adjoint sources of L = sum_{m,g} d_g[m][g] * fc2tg(meas(phi))[m][g]:
 * d_B[k][node][s] = dL/dphi_{k,s}[node] (complex128 [nf][n][ns], overwritten),
 * c[m][k] = 2 nt h_k sum_g g[m][g] conj(gate[g][k]) (h_0 = 1/2, else 1)
 * scattered through detector d's weights for every link m = (s, d).  Solving
 * A_k lam = B (dgp_solve) gives the adjoint fields of dgp_fem_adjoint_grad.
 * The chain rule of fc2tg.m:25-32 and meas_flu (dMesh.m:144-171). */
int dgp_tg_adjoint_rhs(const int32_t *d_det_nodes, const double *d_det_w,
                       int32_t nd, const int32_t *d_link, int32_t nm,
                       const double *d_gate_fc, int32_t ng, int32_t nt,
                       const double *d_g, int64_t n, int32_t nf, int32_t ns,
                       double *d_B, dgp_stream_t stream);

/* ====================================================================== *
 *  Absorption Jacobian (J_complex, dMesh.m:206-247) and its time-gated
 *  form (fc2tg along the harmonic axis, tut_2...m:147, wghtd_LM_recon.m:61).
 *
 *  Basis: d_P_* is the CSR of the mesh-to-voxel interpolation m2g
 *  ([nv x nn], <= 8 entries per row, dMesh.m:286-327) or NULL for the nodal
 *  basis (nv == nn).  d_w [nv]: voxel weight (dxyz^3 for the voxel grid, the
 *  lumped nodal mass for the nodal basis), NULL = 1.
 *  Fields: d_phi [nf][nn][ns], d_phiA [nf][nn][nd] complex128 (forward and
 *  adjoint fluence as dgp_solve writes them); d_fpsf [nf] complex128;
 *  d_link [nm][2] (source, detector).  Outputs use the reference's memory
 *  order: voxel slowest, measurement fastest.
 *  Checked before any kernel runs: a link entry outside [0, ns) x [0, nd) is
 *  DGP_ERR_ARG; a malformed P (row pointer not starting at 0 or decreasing,
 *  a row of more than 8 entries, a column outside [0, nn)) is DGP_ERR_MESH.
 * ====================================================================== */
/* J[v][k][m] complex128 = -(P phi_s)(P phiA_d) w_v / s_fpsf[k]. */
int dgp_jacobian_complex(const int32_t *d_P_rowptr, const int32_t *d_P_col,
                         const double *d_P_val, int64_t nv, const double *d_w,
                         const double *d_phi, int32_t ns, const double *d_phiA,
                         int32_t nd, int64_t nn, int32_t nf,
                         const double *d_fpsf, const int32_t *d_link,
                         int32_t nm, double *d_J, dgp_stream_t stream);
/* J_tg[v][g][m] float32 = Nt 2 Re sum_k conj(gate_fc[g][k]) J~[m][k][v]
 * (J~_0 = J_0/2), divided by d_data_tg[m][g] when that is not NULL (Rytov
 * normalisation).  1 <= ng <= 32.  Row v of the output is row v of J^T
 * with measurement index g*nm + m.  The DFT over harmonics runs on the tensor
 * cores (tcgen05: per voxel a GEMM over (gate, source) x detector with TF32
 * operands split in two, so that three products keep FP32 accuracy) where the
 * shapes fit (dgp_set_jacobian_engine), else on the CUDA cores. */
/* Engines of dgp_jacobian_tg and dgp_jacobian_tg_vjp, process-wide: 0 (default)
 * and 2 the tensor cores where the shapes fit, else the CUDA cores; 1 both on
 * the CUDA cores (cross-checks, timing).  The tensor-core TG Jacobian takes the
 * nodal basis (P = NULL), at most 32 sources and 32 detectors, each (source,
 * detector) pair at most once in the link table, and at most 64 harmonics; the
 * tensor-core vjp the nodal basis or a basis P, at most 32 sources and 32
 * detectors and 4096 links. */
int dgp_set_jacobian_engine(int32_t engine);
int dgp_jacobian_tg(const int32_t *d_P_rowptr, const int32_t *d_P_col,
                    const double *d_P_val, int64_t nv, const double *d_w,
                    const double *d_phi, int32_t ns, const double *d_phiA,
                    int32_t nd, int64_t nn, int32_t nf, const double *d_fpsf,
                    const int32_t *d_link, int32_t nm, const double *d_gate_fc,
                    int32_t ng, int32_t nt, const double *d_data_tg,
                    float *d_J, dgp_stream_t stream);
/* out[v] = sum_{m,g} J_tg[v][g][m] * d_g[m][g]: the TG Jacobian's transpose
 * applied to an upstream gradient without forming J (same arguments). */
int dgp_jacobian_tg_vjp(const int32_t *d_P_rowptr, const int32_t *d_P_col,
                        const double *d_P_val, int64_t nv, const double *d_w,
                        const double *d_phi, int32_t ns, const double *d_phiA,
                        int32_t nd, int64_t nn, int32_t nf,
                        const double *d_fpsf, const int32_t *d_link,
                        int32_t nm, const double *d_gate_fc, int32_t ng,
                        int32_t nt, const double *d_data_tg, const double *d_g,
                        double *d_out, dgp_stream_t stream);

/* ====================================================================== *
 *  Point location for the voxel basis (mesh2grid, dMesh.m:286-327; the
 *  reference uses MATLAB's pointLocation on the host).
 * ====================================================================== */
/* For each point d_pts[i][0..2]: d_eid[i] = the element whose smallest
 * barycentric weight is largest (ties: lower element id) when that weight is
 * >= -eps, else -1; d_w[i][0..3] its barycentric weights for the vertices
 * d_elem[e][0..3] (zeros when d_eid[i] == -1).  d_node [nn][3] float64,
 * d_elem [ne][4] int32 (0-based; DGP_ERR_MESH when an id is outside
 * [0, nn)).  Bins the elements on the device; the call synchronises the
 * stream. */
int dgp_locate_points(const double *d_node, const int32_t *d_elem, int64_t nn,
                      int64_t ne, const double *d_pts, int64_t np, double eps,
                      int32_t *d_eid, double *d_w, dgp_stream_t stream);

/* Optode snapping (snap_pos, dOptode.m:155-190): for each position
 * d_pos[i][0..2], the nearest boundary node (d_bnd[v] != 0; ties: lower
 * index), then the closest point on the surface triangles d_face[f][0..2]
 * (int32, 0-based) that contain that node (ties: lower face index):
 * d_out_pos[i] = that point, d_out_dir[i] = the face's normal
 * -cross(b - a, c - a) normalised (inward for outward-ordered faces),
 * d_out_face[i] = the face.  DGP_ERR_MESH when a face node id is outside
 * [0, nn); DGP_ERR_ARG when a position finds no boundary node or face.
 * Synchronises the stream. */
int dgp_snap_to_surface(const double *d_node, int64_t nn, const int32_t *d_bnd,
                        const int32_t *d_face, int64_t nface, const double *d_pos,
                        int64_t n, double *d_out_pos, double *d_out_dir,
                        int32_t *d_out_face, dgp_stream_t stream);

/* Grid-to-mesh interpolation g2m (dMesh.m:330-373) on the lattice of voxel
 * centres origin[d] + i*spacing[d], i < n[d], spacing != 0 (host arrays of 3;
 * voxel index
 * i + n0*(j + n1*k), MATLAB's ndgrid order).  Row r of g2m is written to
 * d_col[r][0..3] (voxel index, -1 = empty) and d_val[r][0..3]: the
 * barycentric weights of node r in the lattice's Kuhn triangulation (one of
 * the Delaunay triangulations of a rectilinear lattice), restricted to voxels
 * with d_inmesh[v] != 0 and normalised to sum 1; a node none of whose four
 * voxels is in the mesh (or that lies outside the lattice) gets its nearest
 * in-mesh voxel with weight 1 (ties: lower index).  Zero weights are
 * dropped. */
int dgp_grid_to_mesh(const double *d_node, int64_t nn, const double *origin,
                     const double *spacing, const int32_t *n,
                     const uint8_t *d_inmesh, int32_t *d_col, double *d_val,
                     dgp_stream_t stream);

/* ====================================================================== *
 *  Levenberg-Marquardt normal equations (tik_inv, reconstruction/
 *  tik_inv.m:1-20, with a diagonal data weight W = 1/sigma^2).
 * ====================================================================== */
enum { DGP_DAMP_MAX_DIAG = 0, DGP_DAMP_DIAG = 1, DGP_DAMP_ADD = 2 };
/* H = J^T W J (lower triangle of d_H [nv][ldh] in FP64, from split-BF16
 * tensor-core products with FP32 accumulation), H_ii = (J^T W J)_ii (exact
 * FP64) + lambda * (max_j (J^T W J)_jj for DGP_DAMP_MAX_DIAG, the tik_inv
 * rule; (J^T W J)_ii for DGP_DAMP_DIAG; 1 for DGP_DAMP_ADD), and d_rhs = J^T W y (FP64) when
 * d_y and d_rhs are not NULL.  d_Jt is J transposed, [nv][nmeas] float32
 * (the dgp_jacobian_tg output); d_w [nmeas] or NULL (W = I).  The strict
 * upper triangle of d_H is not written. */
int dgp_normal_eq(const float *d_Jt, int64_t nv, int64_t nmeas, const double *d_w,
                  const double *d_y, double lambda, int32_t damping, double *d_H,
                  int64_t ldh, double *d_rhs, dgp_stream_t stream);
/* out[a][m] = sum_v A[a][v] Jt[v][m] (FP64 accumulation): A [na][nv] f64,
 * Jt [nv][nmeas] f32 (J transposed, the TG Jacobian's layout), out [na][nmeas]
 * f64.  The spots-times-J^T product of reshape_J (reconstruction/reshape_J.m:
 * 15, Js*J'). */
int dgp_times_jt(const double *d_A, int64_t na, int64_t nv, const float *d_Jt,
                 int64_t nmeas, double *d_out, dgp_stream_t stream);

/* Solves H x = b in place (d_x: b in, x out) by an FP64 Cholesky
 * factorisation of the lower triangle of d_H (overwritten by L).
 * Returns DGP_ERR_ARG if H is not positive definite.  A 16-byte aligned d_H
 * with an even ldh keeps every row 16-byte aligned, and the factorisation's
 * GEMMs then move their operands with 16-byte copies (an odd ldh works, about
 * 8 % slower at n = 22,971).  One right-hand side is solved by two
 * cooperative launches when the GPU holds every 128-row block's CTA at once. */
int dgp_cholesky_solve(double *d_H, int64_t n, int64_t ldh, double *d_x,
                       dgp_stream_t stream);
/* d_diag[v] = sum_m w_m Jt[v][m]^2 and, when d_y and d_rhs are not NULL,
 * d_rhs[v] = sum_m Jt[v][m] w_m y_m (FP64 sums; d_w NULL = 1): the diagonal of
 * J^T W J and J^T W y without forming J^T W J. */
int dgp_row_dots(const float *d_Jt, int64_t nv, int64_t nmeas, const double *d_w,
                 const double *d_y, double *d_diag, double *d_rhs, dgp_stream_t stream);
/* The tik_inv update (reconstruction/tik_inv.m:13-20, with a diagonal data
 * weight W): d_x = (J^T W J + lambda max_i (J^T W J)_ii I)^-1 J^T W y.
 * form 1 factors the nv x nv system (dgp_normal_eq + dgp_cholesky_solve);
 * form 2 the nmeas x nmeas one, J_w^T (J_w J_w^T + mu I)^-1 W^1/2 y with
 * J_w = W^1/2 J and mu = lambda max_i (J^T W J)_ii (the same update, far less
 * work when nmeas < nv); form 0 picks the smaller.  *form_used (may be NULL)
 * reports 1 or 2.  Both forms return DGP_ERR_ARG unless every weight is finite
 * and non-negative.  Allocates its work arrays; synchronises the stream. */
int dgp_lm_update(const float *d_Jt, int64_t nv, int64_t nmeas, const double *d_w,
                  const double *d_y, double lambda, double *d_x, int32_t form,
                  int32_t *form_used, dgp_stream_t stream);
/* dgp_cholesky_solve for nrhs right-hand sides: row r of d_X [nrhs][ldx]
 * (ldx >= n) is b_r in and x_r out; one factorisation, one pair of triangular solves.
 * Used for reshape_J's w = (Js J^T)(J J^T + lam max diag I)^-1
 * (reconstruction/reshape_J.m:13-15) with the rows of Js J^T as b_r.
 * nrhs > 1 solves by 128-row blocks, a partial-sum and a diagonal launch each. */
int dgp_cholesky_solve_many(double *d_H, int64_t n, int64_t ldh, double *d_X,
                            int32_t nrhs, int64_t ldx, dgp_stream_t stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* DOGPUP_B200_H */
