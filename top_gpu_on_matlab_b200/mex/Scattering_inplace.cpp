// Scattering_inplace(Y, eNodMat, uMat) over top_scatter; replaces the
// reference's Scattering_inplace.cu:81-146.  The reference reads uMat with Y's
// class whatever uMat's is; a different class is refused here instead.
#include "topgpu_mex.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)nlhs; (void)plhs;
    if (nrhs != 3) mexErrMsgIdAndTxt("Scattering_inplace:arity", "Expected 3 inputs: (Y, eNodMat, uMat). No outputs.");
    mxInitGPU();
    GpuArgs g;
    const mxGPUArray *Y = g.wrap(prhs[0]);
    const mxClassID clsY = mxGPUGetClassID(Y);
    const mwSize *dY = mxGPUGetDimensions(Y);
    if (mxGPUGetNumberOfDimensions(Y) != 2 || dY[1] != 3) TOPGPU_MEX_FAIL(g, "Scattering_inplace:shape", "Y must be [numNodes x 3].");
    const mxGPUArray *EN = g.wrap(prhs[1]);
    if (mxGPUGetClassID(EN) != mxINT32_CLASS || mxGPUGetComplexity(EN) != mxREAL)
        TOPGPU_MEX_FAIL(g, "Scattering_inplace:type", "eNodMat must be gpuArray(int32).");
    const mwSize *dE = mxGPUGetDimensions(EN);
    if (mxGPUGetNumberOfDimensions(EN) != 2 || dE[1] != 8)
        TOPGPU_MEX_FAIL(g, "Scattering_inplace:shape", "eNodMat must be [Ne x %d] int32 (1-based).", 8);
    const mxGPUArray *U = g.wrap(prhs[2]);
    const mwSize *dU = mxGPUGetDimensions(U);
    if (mxGPUGetNumberOfDimensions(U) != 2 || dU[0] != dE[0] || dU[1] != 24)
        TOPGPU_MEX_FAIL(g, "Scattering_inplace:shape", "uMat must be [Ne x 24] double.");
    if (clsY != mxSINGLE_CLASS && clsY != mxDOUBLE_CLASS) TOPGPU_MEX_FAIL(g, "Scattering_inplace:type", "Y must be single or double.");
    if (mxGPUGetClassID(U) != clsY) TOPGPU_MEX_FAIL(g, "Scattering_inplace:type", "uMat class must match Y.");
    const int st = top_scatter(mxGPUGetData(const_cast<mxGPUArray *>(Y)), (const int32_t *)mxGPUGetDataReadOnly(EN),
                               mxGPUGetDataReadOnly(U), (int64_t)dE[0], (int64_t)dY[0], topgpu_dtype(clsY), nullptr);
    if (st != TOP_OK) TOPGPU_MEX_FAIL(g, "Scattering_inplace:cuda", "%s", top_last_error());
}
