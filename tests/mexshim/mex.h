/* Test double of MATLAB's mex.h (interleaved-complex model, R2018a+): the
 * subset of the documented C API that dogpup_b200's gateways use, so they can
 * be compiled and driven from the test suite without MATLAB.  TEST
 * INFRASTRUCTURE ONLY; a real build uses MATLAB's own headers (mexcuda). */
#ifndef DGP_TEST_MEX_H
#define DGP_TEST_MEX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef size_t mwSize;
typedef size_t mwIndex;
typedef struct mxArray_tag mxArray;
typedef enum { mxUNKNOWN_CLASS = 0, mxCHAR_CLASS = 4, mxDOUBLE_CLASS = 6, mxSINGLE_CLASS = 7, mxINT32_CLASS = 12 } mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;
typedef struct { double real, imag; } mxComplexDouble;

/* the gateway entry point, C linkage as in MATLAB's mex.h */
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
void mexWarnMsgIdAndTxt(const char *id, const char *fmt, ...);
void mxFree(void *p);

int mxIsComplex(const mxArray *a);
int mxIsSparse(const mxArray *a);
int mxIsChar(const mxArray *a);
size_t mxGetM(const mxArray *a);
size_t mxGetN(const mxArray *a);
size_t mxGetNumberOfElements(const mxArray *a);
double mxGetScalar(const mxArray *a);
double *mxGetDoubles(const mxArray *a);
mxComplexDouble *mxGetComplexDoubles(const mxArray *a);
mwIndex *mxGetJc(const mxArray *a);
mwIndex *mxGetIr(const mxArray *a);
int mxGetString(const mxArray *a, char *buf, mwSize len);
mxArray *mxCreateDoubleScalar(double v);

#ifdef __cplusplus
}
#endif

#endif
