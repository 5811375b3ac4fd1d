// C++-linkage drop-ins with the exact signatures of the reference mex host
// functions, so the reference's own mex gateways link against this library
// unchanged.  Each runs on the default stream like the reference and records
// a failure for dgp_last_error() (the reference functions return void and
// check nothing).
#ifndef DOGPUP_B200_MEX_HPP
#define DOGPUP_B200_MEX_HPP

// cuda_lib/mex_sources/smvMex.hpp:4-15
void smv_call(double *const d_out_real, double *const d_out_imag, const double *const d_x_real,
              const double *const d_x_imag, const double *const d_fAxis, const double *const d_valA_real,
              const double *const d_valA_imag, const int *const d_rPtr, const int *const d_cPtr, const int nrows,
              const int ncols, const int nfreqs);

// cuda_lib/mex_sources/FSAImvMex.hpp:4-15
void FSAImv_call(double *const d_out_real, double *const d_out_imag, const double *const d_x_real,
                 const double *const d_x_imag, const double *const d_valG_real, const double *const d_valG_imag,
                 const int *const d_rPtr, const int *const d_cPtr, const int nnz, const int nrows, const int ncols,
                 const int nfreqs);

// cuda_lib/mex_sources/FSAIP.hpp:4-13
void FSAIP_call(double *const d_out_real, double *const d_out_imag, const double *const d_valA_real,
                const double *const d_valA_imag, const int *const d_rPtrA, const int *const d_cPtrA,
                const int *const d_rPtrG, const int *const d_cPtrG, const int nfreqs, const int nrows);

#endif
