// assembleKs_level2_inplace(d_Ks, d_upMap, d_eleModulus, d_K_0, d_Pch,
//   d_mapUnique, d_uniqueFree, d_uniqueFixed) over top_assemble_ks_level2;
// replaces the reference's assembleKs_level2_inplace.cu:165-284.
#include "topgpu_mex.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    if (nrhs != 8) mexErrMsgIdAndTxt("assembleKs_level2_inplace:Input", "Expected 8 inputs.");
    mxInitGPU();
    GpuArgs g;
    const mxGPUArray *Ks = g.wrap(prhs[0]), *up = g.wrap(prhs[1]), *E = g.wrap(prhs[2]), *K0 = g.wrap(prhs[3]),
                     *P = g.wrap(prhs[4]), *mu = g.wrap(prhs[5]), *uf = g.wrap(prhs[6]), *ux = g.wrap(prhs[7]);
    const mxClassID cls = mxGPUGetClassID(Ks);
    if (cls != mxSINGLE_CLASS && cls != mxDOUBLE_CLASS) TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:Type", "d_Ks must be single/double gpuArray.");
    if (mxGPUGetClassID(up) != mxINT32_CLASS || mxGPUGetClassID(mu) != mxINT32_CLASS)
        TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:Type", "d_upMap and d_mapUnique must be int32 gpuArray.");
    const mwSize *dK = mxGPUGetDimensions(Ks);
    if (mxGPUGetNumberOfDimensions(Ks) != 3 || dK[0] != 24 || dK[1] != 24)
        TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:Shape", "d_Ks must be [24 x 24 x nElem].");
    const int64_t nElem = (int64_t)dK[2];
    const mwSize *dU = mxGPUGetDimensions(up);
    if (mxGPUGetNumberOfDimensions(up) != 2 || (int64_t)dU[0] != nElem)
        TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:Shape", "d_upMap must be [nElem x nCh].");
    const int nCh = (int)dU[1];
    const mwSize *dP = mxGPUGetDimensions(P);
    if (mxGPUGetNumberOfDimensions(P) != 3 || dP[0] != 24 || dP[1] != 24 || (int)dP[2] != nCh)
        TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:Shape", "d_Pch must be [24 x 24 x nCh].");
    const mwSize *d0 = mxGPUGetDimensions(K0);
    if (mxGPUGetNumberOfDimensions(K0) != 2 || d0[0] * d0[1] != 576)
        TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:Shape", "d_K_0 must contain 576 elements.");
    int64_t nUnique = 0;
    if (mxGPUGetNumberOfElements(uf) > 0) {
        const mwSize *df = mxGPUGetDimensions(uf);
        if (mxGPUGetNumberOfDimensions(uf) != 2 || df[0] != 576)
            TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:Shape", "d_uniqueFree must be [576 x nUnique] or empty.");
        nUnique = (int64_t)df[1];
    }
    if (mxGPUGetNumberOfElements(ux) > 0) {
        const mwSize *dx = mxGPUGetDimensions(ux);
        if (mxGPUGetNumberOfDimensions(ux) != 2 || dx[0] != 576 || (int64_t)dx[1] != nUnique)
            TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:Shape", "d_uniqueFixed must be [576 x nUnique] matching d_uniqueFree.");
    }
    if (mxGPUGetClassID(E) != cls || mxGPUGetClassID(K0) != cls || mxGPUGetClassID(P) != cls)
        TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:Type", "d_eleModulus/d_K_0/d_Pch must match d_Ks class.");
    if (mxGPUGetNumberOfElements(uf) > 0 && mxGPUGetClassID(uf) != cls)
        TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:Type", "d_uniqueFree class must match d_Ks.");
    if (mxGPUGetNumberOfElements(ux) > 0 && mxGPUGetClassID(ux) != cls)
        TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:Type", "d_uniqueFixed class must match d_Ks.");
    const int st = top_assemble_ks_level2(mxGPUGetData(const_cast<mxGPUArray *>(Ks)), (const int32_t *)mxGPUGetDataReadOnly(up),
                                          mxGPUGetDataReadOnly(E), mxGPUGetDataReadOnly(K0), mxGPUGetDataReadOnly(P),
                                          (const int32_t *)mxGPUGetDataReadOnly(mu), topgpu_opt_ptr(uf), topgpu_opt_ptr(ux),
                                          nElem, nCh, (int64_t)mxGPUGetNumberOfElements(E), nUnique, topgpu_dtype(cls), nullptr);
    if (st != TOP_OK) TOPGPU_MEX_FAIL(g, "assembleKs_level2_inplace:CUDA", "%s", top_last_error());
    if (nlhs > 0) plhs[0] = mxGPUCreateMxArrayOnGPU(Ks);      // optional output, as the reference returns d_Ks
}
