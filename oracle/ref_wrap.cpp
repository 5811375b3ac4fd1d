// extern "C" entry points around the reference's own host functions
// (smvMex.hpp:4-15, FSAImvMex.hpp:4-15, FSAIP.hpp:4-13), so the test-suite can
// call the unmodified reference kernels through ctypes.  Checker only.
#include <cuda_runtime.h>

#include "FSAIP.hpp"
#include "FSAImvMex.hpp"
#include "smvMex.hpp"

extern "C" {

int ref_smv(double *o_re, double *o_im, const double *x_re, const double *x_im, const double *f, const double *a_re,
            const double *a_im, const int *rp, const int *cp, int nrows, int ncols, int nfreqs) {
  smv_call(o_re, o_im, x_re, x_im, f, a_re, a_im, rp, cp, nrows, ncols, nfreqs);
  return (int)cudaDeviceSynchronize();
}

int ref_fsaimv(double *o_re, double *o_im, const double *x_re, const double *x_im, const double *g_re,
               const double *g_im, const int *rp, const int *cp, int nnz, int nrows, int ncols, int nfreqs) {
  FSAImv_call(o_re, o_im, x_re, x_im, g_re, g_im, rp, cp, nnz, nrows, ncols, nfreqs);
  return (int)cudaDeviceSynchronize();
}

int ref_fsaip(double *o_re, double *o_im, const double *a_re, const double *a_im, const int *rpa, const int *cpa,
              const int *rpg, const int *cpg, int nfreqs, int nrows) {
  FSAIP_call(o_re, o_im, a_re, a_im, rpa, cpa, rpg, cpg, nfreqs, nrows);
  return (int)cudaDeviceSynchronize();
}
}
