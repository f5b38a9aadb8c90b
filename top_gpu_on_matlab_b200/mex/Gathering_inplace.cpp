// Gathering_inplace(gUMat, gU, gE) over top_gather; replaces the reference's
// Gathering_inplace.cu:75-171 (checks and identifiers in the same order).
#include "topgpu_mex.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)plhs;
    if (nrhs != 3) mexErrMsgIdAndTxt("Gathering_inplace:Args", "Usage: Gathering_inplace(gUMat, gU, gE)");
    if (nlhs != 0) mexErrMsgIdAndTxt("Gathering_inplace:Args", "This function returns no outputs. gUMat is modified in-place.");
    mxInitGPU();
    GpuArgs g;
    const mxGPUArray *gUMat = g.wrap(prhs[0]), *gU = g.wrap(prhs[1]), *gE = g.wrap(prhs[2]);
    const mxClassID clsU = mxGPUGetClassID(gU), clsE = mxGPUGetClassID(gE);
    if (clsU != mxSINGLE_CLASS && clsU != mxDOUBLE_CLASS) TOPGPU_MEX_FAIL(g, "Gathering_inplace:Type", "gU must be single or double gpuArray.");
    if (mxGPUGetClassID(gUMat) != clsU) TOPGPU_MEX_FAIL(g, "Gathering_inplace:Type", "gUMat precision must match gU.");
    if (clsE != mxINT32_CLASS && clsE != mxUINT32_CLASS) TOPGPU_MEX_FAIL(g, "Gathering_inplace:Type", "gE must be int32 or uint32 gpuArray.");
    const mwSize *dU = mxGPUGetDimensions(gU), *dE = mxGPUGetDimensions(gE), *dO = mxGPUGetDimensions(gUMat);
    if (mxGPUGetNumberOfDimensions(gU) != 2 || dU[1] != 3) TOPGPU_MEX_FAIL(g, "Gathering_inplace:Shape", "gU must be (numNodes x 3).");
    if (mxGPUGetNumberOfDimensions(gE) != 2 || dE[1] != 8) TOPGPU_MEX_FAIL(g, "Gathering_inplace:Shape", "gE must be (nElem x 8).");
    if (mxGPUGetNumberOfDimensions(gUMat) != 2 || dO[0] != dE[0] || dO[1] != 24)
        TOPGPU_MEX_FAIL(g, "Gathering_inplace:Shape", "gUMat must be (nElem x 24).");
    const int st = top_gather(mxGPUGetData(const_cast<mxGPUArray *>(gUMat)), mxGPUGetDataReadOnly(gU),
                              mxGPUGetDataReadOnly(gE), clsE == mxUINT32_CLASS, (int64_t)dE[0], (int64_t)dU[0],
                              topgpu_dtype(clsU), nullptr);
    if (st != TOP_OK) TOPGPU_MEX_FAIL(g, "Gathering_inplace:CUDA", "%s", top_last_error());
}
