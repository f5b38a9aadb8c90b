/* mex.h -- TEST-ONLY stand-in for MATLAB's MEX API, enough to compile the
 * reference's CUDA MEX files unmodified (oracle/ref_build.sh) and call their
 * mexFunction on raw device buffers from the parity tests.  Not part of the
 * product.  mexErrMsgIdAndTxt throws; shim_call() turns that into a status. */
#ifndef TOPGPU_TEST_MEX_SHIM_H
#define TOPGPU_TEST_MEX_SHIM_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef size_t mwSize;
typedef enum {
    mxUNKNOWN_CLASS = 0, mxCELL_CLASS, mxSTRUCT_CLASS, mxLOGICAL_CLASS, mxCHAR_CLASS, mxVOID_CLASS,
    mxDOUBLE_CLASS, mxSINGLE_CLASS, mxINT8_CLASS, mxUINT8_CLASS, mxINT16_CLASS, mxUINT16_CLASS,
    mxINT32_CLASS, mxUINT32_CLASS, mxINT64_CLASS, mxUINT64_CLASS
} mxClassID;
typedef enum { mxREAL = 0, mxCOMPLEX } mxComplexity;
typedef struct shim_array {
    mxClassID cls;
    mwSize ndim;
    mwSize dims[8];
    void *data;
    int on_gpu;
} mxArray;
void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...);
void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);
#ifdef __cplusplus
}
#endif
#endif
