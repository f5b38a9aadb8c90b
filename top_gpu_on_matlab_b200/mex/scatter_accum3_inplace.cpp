// scatter_accum3_inplace(keys, Tmp, xF) over top_scatter_accum3; replaces the
// reference's scatter_accum3_inplace.cu:115-145 (identifiers "scatter_accum3:*").
#include "topgpu_mex.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    (void)plhs;
    if (nrhs != 3)
        mexErrMsgIdAndTxt("scatter_accum3:args", "Usage: scatter_accum3_inplace(transferMatGPU[int32], TmpGPU[Nx3], xFinerGPU[Mx3]).");
    if (nlhs != 0) mexErrMsgIdAndTxt("scatter_accum3:nlhs", "No output. xFiner is updated in-place.");
    mxInitGPU();
    for (int i = 0; i < 3; ++i)
        if (!mxIsGPUArray(prhs[i])) mexErrMsgIdAndTxt("scatter_accum3:gpu", "All inputs must be gpuArray.");
    GpuArgs g;
    const mxGPUArray *keys = g.wrap(prhs[0]), *tmp = g.wrap(prhs[1]), *xf = g.wrap(prhs[2]);
    const mwSize *dT = mxGPUGetDimensions(tmp), *dX = mxGPUGetDimensions(xf);
    if (mxGPUGetNumberOfDimensions(tmp) != 2 || dT[1] != 3) TOPGPU_MEX_FAIL(g, "scatter_accum3:shape", "`Tmp` must be [N x 3] gpuArray.");
    if (mxGPUGetNumberOfDimensions(xf) != 2 || dX[1] != 3) TOPGPU_MEX_FAIL(g, "scatter_accum3:shape", "`xFiner` must be [M x 3] gpuArray.");
    if (mxGPUGetClassID(keys) != mxINT32_CLASS) TOPGPU_MEX_FAIL(g, "scatter_accum3:type", "`transferMat` must be int32 gpuArray.");
    const mxClassID cls = mxGPUGetClassID(tmp);
    if (cls != mxGPUGetClassID(xf))
        TOPGPU_MEX_FAIL(g, "scatter_accum3:type", "`Tmp` and `xFiner` must have the same class (single/double).");
    if (cls != mxSINGLE_CLASS && cls != mxDOUBLE_CLASS)
        TOPGPU_MEX_FAIL(g, "scatter_accum3:type", "Only single or double supported for `Tmp`/`xFiner`.");
    const int st = top_scatter_accum3((const int32_t *)mxGPUGetDataReadOnly(keys), mxGPUGetDataReadOnly(tmp), (int64_t)dT[0],
                                      mxGPUGetData(const_cast<mxGPUArray *>(xf)), (int64_t)dX[0], topgpu_dtype(cls), nullptr);
    if (st != TOP_OK) TOPGPU_MEX_FAIL(g, "scatter_accum3:cuda", "%s", top_last_error());
}
