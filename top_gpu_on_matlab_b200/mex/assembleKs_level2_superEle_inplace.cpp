// assembleKs_level2_superEle_inplace(d_Ks, d_upMap, d_Ks0, d_Psub,
//   d_mapUnique, d_eleModulus, d_uniqueFree, d_uniqueFixed) over
// top_assemble_ks_level2_super; replaces the reference's
// assembleKs_level2_superEle_inplace.cu:178-325.
#include "topgpu_mex.h"

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[])
{
    if (nrhs != 8)
        mexErrMsgIdAndTxt("assembleKs_level2_superEle_inplace:Input",
                          "Expected 8 inputs: d_Ks, d_upMap, d_Ks0, d_Psub, d_mapUnique, d_eleModulus, d_uniqueFree, d_uniqueFixed.");
    mxInitGPU();
    GpuArgs g;
    const mxGPUArray *Ks = g.wrap(prhs[0]), *up = g.wrap(prhs[1]), *K0 = g.wrap(prhs[2]), *P = g.wrap(prhs[3]),
                     *mu = g.wrap(prhs[4]), *E = g.wrap(prhs[5]), *uf = g.wrap(prhs[6]), *ux = g.wrap(prhs[7]);
    const char *T = "assembleKs_level2_superEle_inplace:Type", *S = "assembleKs_level2_superEle_inplace:Shape";
    const mxClassID cls = mxGPUGetClassID(Ks);
    if (cls != mxSINGLE_CLASS && cls != mxDOUBLE_CLASS) TOPGPU_MEX_FAIL(g, T, "d_Ks must be single/double gpuArray.");
    if (mxGPUGetClassID(up) != mxINT32_CLASS || mxGPUGetClassID(mu) != mxINT32_CLASS)
        TOPGPU_MEX_FAIL(g, T, "d_upMap and d_mapUnique must be int32 gpuArray.");
    if (mxGPUGetClassID(K0) != cls || mxGPUGetClassID(P) != cls || mxGPUGetClassID(E) != cls)
        TOPGPU_MEX_FAIL(g, T, "d_Ks0, d_Psub, d_eleModulus must match d_Ks class.");
    if (mxGPUGetNumberOfElements(uf) > 0 && mxGPUGetClassID(uf) != cls) TOPGPU_MEX_FAIL(g, T, "d_uniqueFree class must match d_Ks.");
    if (mxGPUGetNumberOfElements(ux) > 0 && mxGPUGetClassID(ux) != cls) TOPGPU_MEX_FAIL(g, T, "d_uniqueFixed class must match d_Ks.");
    const mwSize *dK = mxGPUGetDimensions(Ks);
    if (mxGPUGetNumberOfDimensions(Ks) != 3 || dK[0] != 24 || dK[1] != 24) TOPGPU_MEX_FAIL(g, S, "d_Ks must be [24 x 24 x nElem].");
    const int64_t nElem = (int64_t)dK[2];
    const mwSize *dU = mxGPUGetDimensions(up);
    if (mxGPUGetNumberOfDimensions(up) != 2 || (int64_t)dU[0] != nElem) TOPGPU_MEX_FAIL(g, S, "d_upMap must be [nElem x nSub].");
    const int nSub = (int)dU[1];
    if (mxGPUGetNumberOfElements(K0) % 576 != 0) TOPGPU_MEX_FAIL(g, S, "d_Ks0 total elements must be a multiple of 576.");
    const mwSize *dP = mxGPUGetDimensions(P);
    if (mxGPUGetNumberOfDimensions(P) != 3 || dP[0] != 24 || dP[1] != 24 || (int)dP[2] != nSub)
        TOPGPU_MEX_FAIL(g, S, "d_Psub must be [24 x 24 x nSub].");
    if (mxGPUGetNumberOfElements(E) % 64 != 0) TOPGPU_MEX_FAIL(g, S, "d_eleModulus total elements must be a multiple of 64.");
    int64_t nUnique = 0;
    if (mxGPUGetNumberOfElements(uf) > 0) {
        const mwSize *df = mxGPUGetDimensions(uf);
        const mwSize nd = mxGPUGetNumberOfDimensions(uf);
        if (nd == 3) {
            if (df[0] != 576 || df[1] != 64) TOPGPU_MEX_FAIL(g, S, "d_uniqueFree must be [576 x 64 x nUnique].");
            nUnique = (int64_t)df[2];
        } else if (nd == 2) {
            if (df[0] != 576 * 64) TOPGPU_MEX_FAIL(g, S, "d_uniqueFree must be [576*64 x nUnique] or [576 x 64 x nUnique].");
            nUnique = (int64_t)df[1];
        } else {
            TOPGPU_MEX_FAIL(g, S, "d_uniqueFree must be 2-D or 3-D.");
        }
    }
    if (mxGPUGetNumberOfElements(ux) > 0) {
        const mwSize *dx = mxGPUGetDimensions(ux);
        if (mxGPUGetNumberOfDimensions(ux) != 2 || dx[0] != 576 || (int64_t)dx[1] != nUnique)
            TOPGPU_MEX_FAIL(g, S, "d_uniqueFixed must be [576 x nUnique] matching d_uniqueFree.");
    }
    const int st = top_assemble_ks_level2_super(mxGPUGetData(const_cast<mxGPUArray *>(Ks)), (const int32_t *)mxGPUGetDataReadOnly(up),
                                                mxGPUGetDataReadOnly(K0), mxGPUGetDataReadOnly(P),
                                                (const int32_t *)mxGPUGetDataReadOnly(mu), mxGPUGetDataReadOnly(E),
                                                topgpu_opt_ptr(uf), topgpu_opt_ptr(ux), nElem, nSub,
                                                (int64_t)(mxGPUGetNumberOfElements(K0) / 576), nUnique, topgpu_dtype(cls), nullptr);
    if (st != TOP_OK) TOPGPU_MEX_FAIL(g, "assembleKs_level2_superEle_inplace:CUDA", "%s", top_last_error());
    if (nlhs > 0) plhs[0] = mxGPUCreateMxArrayOnGPU(Ks);
}
