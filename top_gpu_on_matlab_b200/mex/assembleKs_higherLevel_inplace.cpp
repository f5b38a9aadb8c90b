// assembleKs_higherLevel_inplace(d_Ks, d_upMap, d_KsPrev, d_Psub) over
// top_assemble_ks_higher; replaces the reference's
// assembleKs_higherLevel_inplace.cu:134-217.
#include "topgpu_mex.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    if (nrhs != 4)
        mexErrMsgIdAndTxt("assembleKs_higherLevel_inplace:Input", "Expected 4 inputs: (d_Ks, d_upMap, d_KsPrev, d_Psub).");
    mxInitGPU();
    GpuArgs g;
    const mxGPUArray *Ks = g.wrap(prhs[0]), *up = g.wrap(prhs[1]), *prev = g.wrap(prhs[2]), *P = g.wrap(prhs[3]);
    const mxClassID cls = mxGPUGetClassID(Ks);
    if (cls != mxSINGLE_CLASS && cls != mxDOUBLE_CLASS)
        TOPGPU_MEX_FAIL(g, "assembleKs_higherLevel_inplace:Type", "d_Ks must be single/double gpuArray.");
    if (mxGPUGetClassID(up) != mxINT32_CLASS) TOPGPU_MEX_FAIL(g, "assembleKs_higherLevel_inplace:Type", "d_upMap must be int32 gpuArray.");
    if (mxGPUGetClassID(prev) != cls || mxGPUGetClassID(P) != cls)
        TOPGPU_MEX_FAIL(g, "assembleKs_higherLevel_inplace:Type", "d_KsPrev and d_Psub must match d_Ks class.");
    const mwSize *dK = mxGPUGetDimensions(Ks);
    if (mxGPUGetNumberOfDimensions(Ks) != 3 || dK[0] != 24 || dK[1] != 24)
        TOPGPU_MEX_FAIL(g, "assembleKs_higherLevel_inplace:Shape", "d_Ks must be [24 x 24 x nElem].");
    const int64_t nElem = (int64_t)dK[2];
    const mwSize *dU = mxGPUGetDimensions(up);
    if (mxGPUGetNumberOfDimensions(up) != 2 || (int64_t)dU[0] != nElem)
        TOPGPU_MEX_FAIL(g, "assembleKs_higherLevel_inplace:Shape", "d_upMap must be [nElem x nSub].");
    const int nSub = (int)dU[1];
    const mwSize *dV = mxGPUGetDimensions(prev);
    if (mxGPUGetNumberOfDimensions(prev) != 3 || dV[0] != 24 || dV[1] != 24)
        TOPGPU_MEX_FAIL(g, "assembleKs_higherLevel_inplace:Shape", "d_KsPrev must be [24 x 24 x nFinElem].");
    const mwSize *dP = mxGPUGetDimensions(P);
    if (mxGPUGetNumberOfDimensions(P) != 3 || dP[0] != 24 || dP[1] != 24 || (int)dP[2] != nSub)
        TOPGPU_MEX_FAIL(g, "assembleKs_higherLevel_inplace:Shape", "d_Psub must be [24 x 24 x nSub].");
    const int st = top_assemble_ks_higher(mxGPUGetData(const_cast<mxGPUArray *>(Ks)), (const int32_t *)mxGPUGetDataReadOnly(up),
                                          mxGPUGetDataReadOnly(prev), mxGPUGetDataReadOnly(P), nElem, nSub, (int64_t)dV[2],
                                          topgpu_dtype(cls), nullptr);
    if (st != TOP_OK) TOPGPU_MEX_FAIL(g, "assembleKs_higherLevel_inplace:CUDA", "%s", top_last_error());
    if (nlhs > 0) plhs[0] = mxGPUCreateMxArrayOnGPU(Ks);
}
