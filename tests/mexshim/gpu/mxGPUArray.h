/* Test double of MATLAB's gpu/mxGPUArray.h: the documented gpuArray C API
 * subset that dogpup_b200's gateways use.  TEST INFRASTRUCTURE ONLY. */
#ifndef DGP_TEST_MXGPUARRAY_H
#define DGP_TEST_MXGPUARRAY_H

#include "../mex.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mxGPUArray_tag mxGPUArray;
typedef enum { MX_GPU_DO_NOT_INITIALIZE = 0, MX_GPU_INITIALIZE_VALUES = 1 } mxGPUInitialize;
enum { MX_GPU_SUCCESS = 0, MX_GPU_FAILURE = 1 };

int mxInitGPU(void);
int mxIsGPUArray(const mxArray *a);
const mxGPUArray *mxGPUCreateFromMxArray(const mxArray *a);
mxGPUArray *mxGPUCreateGPUArray(mwSize ndims, const mwSize *dims, mxClassID cid, mxComplexity cx,
                                mxGPUInitialize init);
const void *mxGPUGetDataReadOnly(const mxGPUArray *g);
void *mxGPUGetData(mxGPUArray *g);
mwSize mxGPUGetNumberOfDimensions(const mxGPUArray *g);
const mwSize *mxGPUGetDimensions(const mxGPUArray *g);
mwSize mxGPUGetNumberOfElements(const mxGPUArray *g);
mxClassID mxGPUGetClassID(const mxGPUArray *g);
mxComplexity mxGPUGetComplexity(const mxGPUArray *g);
mxArray *mxGPUCreateMxArrayOnGPU(const mxGPUArray *g);
mxArray *mxGPUCreateMxArrayOnCPU(const mxGPUArray *g);
void mxGPUDestroyGPUArray(const mxGPUArray *g);

#ifdef __cplusplus
}
#endif

#endif
