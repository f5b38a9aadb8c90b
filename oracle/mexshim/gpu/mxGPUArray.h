/* gpu/mxGPUArray.h -- TEST-ONLY stand-in for MATLAB's mxGPUArray API (see ../mex.h). */
#ifndef TOPGPU_TEST_MXGPU_SHIM_H
#define TOPGPU_TEST_MXGPU_SHIM_H
#include "../mex.h"
#ifdef __cplusplus
extern "C" {
#endif
typedef struct shim_array mxGPUArray;
int mxInitGPU(void);
int mxIsGPUArray(const mxArray *a);
const mxGPUArray *mxGPUCreateFromMxArray(const mxArray *a);
mxClassID mxGPUGetClassID(const mxGPUArray *a);
mxComplexity mxGPUGetComplexity(const mxGPUArray *a);
const mwSize *mxGPUGetDimensions(const mxGPUArray *a);
mwSize mxGPUGetNumberOfDimensions(const mxGPUArray *a);
mwSize mxGPUGetNumberOfElements(const mxGPUArray *a);
void *mxGPUGetData(mxGPUArray *a);
const void *mxGPUGetDataReadOnly(const mxGPUArray *a);
void mxGPUDestroyGPUArray(const mxGPUArray *a);
mxArray *mxGPUCreateMxArrayOnGPU(const mxGPUArray *a);
#ifdef __cplusplus
}
#endif
#endif
