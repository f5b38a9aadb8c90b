// mexshim.cpp -- TEST-ONLY implementation of the MEX stand-in (see mex.h).
// Linked into each reference kernel library built by oracle/ref_build.sh.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include "mex.h"
#include "gpu/mxGPUArray.h"

namespace {
struct MexError { std::string id, msg; };
}

extern "C" void mexErrMsgIdAndTxt(const char *id, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    throw MexError{id ? id : "", buf};
}
extern "C" int mxInitGPU(void) { return 0; }
extern "C" int mxIsGPUArray(const mxArray *a) { return a && a->on_gpu; }
extern "C" const mxGPUArray *mxGPUCreateFromMxArray(const mxArray *a) { return a; }
extern "C" mxClassID mxGPUGetClassID(const mxGPUArray *a) { return a->cls; }
extern "C" mxComplexity mxGPUGetComplexity(const mxGPUArray *) { return mxREAL; }
extern "C" const mwSize *mxGPUGetDimensions(const mxGPUArray *a) { return a->dims; }
extern "C" mwSize mxGPUGetNumberOfDimensions(const mxGPUArray *a) { return a->ndim; }
extern "C" mwSize mxGPUGetNumberOfElements(const mxGPUArray *a)
{
    mwSize n = 1;
    for (mwSize i = 0; i < a->ndim; ++i) n *= a->dims[i];
    return n;
}
extern "C" void *mxGPUGetData(mxGPUArray *a) { return a->data; }
extern "C" const void *mxGPUGetDataReadOnly(const mxGPUArray *a) { return a->data; }
extern "C" void mxGPUDestroyGPUArray(const mxGPUArray *) {}
extern "C" mxArray *mxGPUCreateMxArrayOnGPU(const mxGPUArray *a) { return const_cast<mxArray *>(a); }

// Call the library's mexFunction; returns 0, or 1 with the MATLAB error id.
extern "C" int shim_call(int nlhs, mxArray **plhs, int nrhs, const mxArray **prhs, char *errid, int errlen)
{
    try {
        mexFunction(nlhs, plhs, nrhs, prhs);
    } catch (const MexError &e) {
        if (errid && errlen > 0) {
            std::snprintf(errid, errlen, "%s|%s", e.id.c_str(), e.msg.c_str());
        }
        return 1;
    }
    return 0;
}
