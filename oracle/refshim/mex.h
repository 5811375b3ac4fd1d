/* Empty stand-in for MATLAB's mex.h: the reference CUDA kernels include it
 * but use none of its API.  Used only to compile those kernels as a checker. */
#ifndef DGP_REFSHIM_MEX_H
#define DGP_REFSHIM_MEX_H
#endif
