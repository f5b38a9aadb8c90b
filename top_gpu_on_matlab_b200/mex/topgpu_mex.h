/* topgpu_mex.h -- shared helpers of the six MEX gateways over libtopgpu.so.
 *
 * Each gateway keeps the reference gateway's name, argument order, in-place
 * semantics, argument checks (in the same order) and error identifiers, and
 * forwards to the C ABI in include/topgpu.h on the legacy default stream, the
 * stream MATLAB's MEX calls use.  Build one MEX file per gateway, e.g.
 *   mexcuda Gathering_inplace.cpp -I<repo>/include -L<repo>/top_gpu_on_matlab_b200 -ltopgpu
 */
#ifndef TOPGPU_MEX_H
#define TOPGPU_MEX_H
#include "mex.h"
#include "gpu/mxGPUArray.h"
#include "topgpu.h"

/* the mxGPUArray wrappers of a call, released on every exit path */
struct GpuArgs {
    const mxGPUArray *a[8];
    int n;
    GpuArgs() : n(0) {}
    const mxGPUArray *wrap(const mxArray *m) { return a[n++] = mxGPUCreateFromMxArray(m); }
    void release() { for (int i = 0; i < n; ++i) mxGPUDestroyGPUArray(a[i]); n = 0; }
    ~GpuArgs() { release(); }
};

/* raise `id` with `msg` after releasing the wrappers (mexErrMsgIdAndTxt does
 * not return) */
#define TOPGPU_MEX_FAIL(args, id, ...) do { (args).release(); mexErrMsgIdAndTxt(id, __VA_ARGS__); } while (0)

static inline int topgpu_dtype(mxClassID c) { return c == mxDOUBLE_CLASS ? TOP_F64 : TOP_F32; }

static inline const void *topgpu_opt_ptr(const mxGPUArray *a)
{
    return mxGPUGetNumberOfElements(a) > 0 ? mxGPUGetDataReadOnly(a) : (const void *)0;
}

#endif
