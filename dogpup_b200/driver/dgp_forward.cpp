// dgp_forward: standalone C++ driver of the forward hot path through the C ABI
// (include/dogpup_b200.h), no Python or MATLAB involved.
//
//   dgp_forward CASE OUT [--precision fp64|mixed|mixed_bicgstab] [--tol T] [--maxit N] [--repeat R]
//
// Reads a case file (mesh, nodal mua / musp, optode barycentrics, links,
// source spectrum; format below), then on the GPU: builds the FEM plan,
// assembles K and M (gen_fwdmat, DOGPUP/dMesh.m:1033-1194), builds the FSAI
// solver plan, solves every source x harmonic with point-source right-hand
// sides (flu_solve, dMesh.m:106-141) and measures the detectors (meas_flu,
// :144-171).  Writes the detector data and prints one JSON line of timings.
// With --repeat R the property update + solve + measurement step runs R more
// times (CUDA-event timed), as an LM loop would (wghtd_LM_recon.m:155).
//
// Case file (little endian; written by dogpup_b200.caseio.write_case):
//   char[8] "DGPCASE1"; int64 nn, ne, ns, nd, nm, nf; double nr, dfc;
//   f64 node[nn][3]; i32 elem[ne][4]; f64 mua[nn], musp[nn];
//   i32 src_nodes[ns][4]; f64 src_w[ns][4]; i32 det_nodes[nd][4]; f64 det_w[nd][4];
//   i32 link[nm][2] (source, detector; 0-based); f64 fpsf[nf][2] (re, im)
// Output file: char[8] "DGPDATA1"; int64 nm, nf; f64 data[nm][nf][2].
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "dogpup_b200.h"

namespace {

[[noreturn]] void die(const char *what, const char *msg) {
  fprintf(stderr, "dgp_forward: %s: %s\n", what, msg);
  exit(1);
}

void ok(int rc, const char *what) {
  if (rc != DGP_OK && rc != DGP_ERR_NOT_CONVERGED) die(what, dgp_last_error());
}

void cu(cudaError_t e, const char *what) {
  if (e != cudaSuccess) die(what, cudaGetErrorString(e));
}

template <class T>
struct Dev {
  T *p = nullptr;
  size_t n = 0;
  explicit Dev(size_t count) : n(count) { cu(cudaMalloc(&p, sizeof(T) * (count ? count : 1)), "cudaMalloc"); }
  Dev(const std::vector<T> &h) : Dev(h.size()) {
    cu(cudaMemcpy(p, h.data(), sizeof(T) * n, cudaMemcpyHostToDevice), "upload");
  }
  ~Dev() { cudaFree(p); }
  Dev(const Dev &) = delete;
  Dev &operator=(const Dev &) = delete;
};

struct Case {
  int64_t nn = 0, ne = 0, ns = 0, nd = 0, nm = 0, nf = 0;
  double nr = 0, dfc = 0;
  std::vector<double> node, mua, musp, src_w, det_w, fpsf;
  std::vector<int32_t> elem, src_nodes, det_nodes, link;
};

template <class T>
void rd(FILE *f, std::vector<T> &v, int64_t count) {
  if (count < 0 || count > (int64_t)1 << 34) die("case", "bad array size");
  v.resize((size_t)count);
  if (count && fread(v.data(), sizeof(T), (size_t)count, f) != (size_t)count) die("case", "truncated file");
}

Case read_case(const char *path) {
  FILE *f = fopen(path, "rb");
  if (!f) die("case", "cannot open");
  char magic[8];
  Case c;
  int64_t h[6];
  double d[2];
  if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "DGPCASE1", 8) != 0) die("case", "not a DGPCASE1 file");
  if (fread(h, sizeof(int64_t), 6, f) != 6 || fread(d, sizeof(double), 2, f) != 2) die("case", "truncated header");
  c.nn = h[0]; c.ne = h[1]; c.ns = h[2]; c.nd = h[3]; c.nm = h[4]; c.nf = h[5];
  c.nr = d[0]; c.dfc = d[1];
  rd(f, c.node, 3 * c.nn);
  rd(f, c.elem, 4 * c.ne);
  rd(f, c.mua, c.nn);
  rd(f, c.musp, c.nn);
  rd(f, c.src_nodes, 4 * c.ns);
  rd(f, c.src_w, 4 * c.ns);
  rd(f, c.det_nodes, 4 * c.nd);
  rd(f, c.det_w, 4 * c.nd);
  rd(f, c.link, 2 * c.nm);
  rd(f, c.fpsf, 2 * c.nf);
  fclose(f);
  return c;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  cu(cudaEventElapsedTime(&ms, a, b), "event");
  return ms;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s CASE OUT [--precision fp64|mixed|mixed_bicgstab] [--tol T] [--maxit N] [--repeat R]\n", argv[0]);
    return 2;
  }
  dgp_solve_opts o;
  dgp_solve_opts_default(&o);
  int repeat = 0;
  for (int i = 3; i + 1 < argc; i += 2) {
    const std::string k = argv[i], v = argv[i + 1];
    if (k == "--precision")
      o.precision = v == "mixed" ? DGP_PREC_MIXED : v == "mixed_bicgstab" ? DGP_PREC_MIXED_BICGSTAB : DGP_PREC_FP64;
    else if (k == "--tol") o.tol = atof(v.c_str());
    else if (k == "--maxit") o.maxit = atoi(v.c_str());
    else if (k == "--repeat") repeat = atoi(v.c_str());
    else die("arguments", ("unknown option " + k).c_str());
  }
  const Case c = read_case(argv[1]);
  cudaStream_t st;
  cu(cudaStreamCreate(&st), "stream");
  cudaEvent_t e0, e1, e2, e3;
  for (cudaEvent_t *e : {&e0, &e1, &e2, &e3}) cu(cudaEventCreate(e), "event");

  Dev<double> node(c.node), mua(c.mua), musp(c.musp), src_w(c.src_w), det_w(c.det_w), fpsf(c.fpsf);
  Dev<int32_t> elem(c.elem), src_nodes(c.src_nodes), det_nodes(c.det_nodes), link(c.link);

  cu(cudaEventRecord(e0, st), "event");
  dgp_fem_t fem = nullptr;
  ok(dgp_fem_create(&fem, node.p, elem.p, c.nn, c.ne, c.nr, st), "fem_create");
  int64_t nnz = 0, nrob = 0, nbnd = 0;
  double cmed = 0;
  ok(dgp_fem_info(fem, &nnz, &nrob, &nbnd, &cmed), "fem_info");
  const int32_t *rowptr = nullptr, *col = nullptr;
  ok(dgp_fem_pattern(fem, &rowptr, &col), "fem_pattern");
  Dev<double> K(nnz), M(nnz);
  ok(dgp_fem_assemble(fem, mua.p, musp.p, K.p, M.p, st), "fem_assemble");
  dgp_solver_t S = nullptr;
  ok(dgp_solver_create(&S, rowptr, col, c.nn, nnz, K.p, M.p, c.dfc, (int32_t)c.nf, (int32_t)c.ns, &o, st),
     "solver_create");
  cu(cudaEventRecord(e1, st), "event");

  Dev<double> phi((size_t)2 * c.nf * c.nn * c.ns), data((size_t)2 * c.nm * c.nf);
  dgp_solve_report rep;
  memset(&rep, 0, sizeof(rep));
  ok(dgp_solve_sources(S, src_nodes.p, src_w.p, fpsf.p, (int32_t)c.ns, phi.p, &o, &rep, st), "solve_sources");
  ok(dgp_meas(det_nodes.p, det_w.p, (int32_t)c.nd, link.p, (int32_t)c.nm, phi.p, c.nn, (int32_t)c.nf,
              (int32_t)c.ns, data.p, st),
     "meas");
  cu(cudaEventRecord(e2, st), "event");
  cu(cudaStreamSynchronize(st), "sync");
  const float setup_ms = elapsed(e0, e1), solve_ms = elapsed(e1, e2);

  // repeated steps: property update (re-assembly + FSAI refactor) + solve + measurement
  float step_ms = 0;
  if (repeat > 0) {
    cu(cudaEventRecord(e2, st), "event");
    for (int r = 0; r < repeat; ++r) {
      ok(dgp_fem_assemble(fem, mua.p, musp.p, K.p, M.p, st), "fem_assemble");
      ok(dgp_solver_update(S, K.p, M.p, st), "solver_update");
      ok(dgp_solve_sources(S, src_nodes.p, src_w.p, fpsf.p, (int32_t)c.ns, phi.p, &o, &rep, st), "solve_sources");
      ok(dgp_meas(det_nodes.p, det_w.p, (int32_t)c.nd, link.p, (int32_t)c.nm, phi.p, c.nn, (int32_t)c.nf,
                  (int32_t)c.ns, data.p, st),
         "meas");
    }
    cu(cudaEventRecord(e3, st), "event");
    cu(cudaStreamSynchronize(st), "sync");
    step_ms = elapsed(e2, e3) / repeat;
  }

  std::vector<double> h((size_t)2 * c.nm * c.nf);
  cu(cudaMemcpy(h.data(), data.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost), "download");
  FILE *f = fopen(argv[2], "wb");
  if (!f) die("output", "cannot open");
  const int64_t hdr[2] = {c.nm, c.nf};
  fwrite("DGPDATA1", 1, 8, f);
  fwrite(hdr, sizeof(int64_t), 2, f);
  fwrite(h.data(), sizeof(double), h.size(), f);
  fclose(f);

  printf("{\"nodes\": %lld, \"nnz\": %lld, \"sources\": %lld, \"harmonics\": %lld, \"precision\": \"%s\", "
         "\"iterations\": %d, \"refinements\": %d, \"max_rel_residual\": %.3e, \"not_converged\": %d, "
         "\"setup_ms\": %.3f, \"solve_ms\": %.3f, \"step_ms\": %.3f, \"solves_per_s\": %.1f}\n",
         (long long)c.nn, (long long)nnz, (long long)c.ns, (long long)c.nf,
         o.precision == DGP_PREC_MIXED ? "mixed" : o.precision == DGP_PREC_MIXED_BICGSTAB ? "mixed_bicgstab" : "fp64",
         rep.iterations, rep.refinements, rep.max_rel_residual,
         rep.n_not_converged, setup_ms, solve_ms, step_ms, c.ns * c.nf / (solve_ms * 1e-3));
  dgp_solver_destroy(S);
  dgp_fem_destroy(fem);
  for (cudaEvent_t e : {e0, e1, e2, e3}) cudaEventDestroy(e);
  cudaStreamDestroy(st);
  return rep.n_not_converged > 0 ? 3 : 0;
}
