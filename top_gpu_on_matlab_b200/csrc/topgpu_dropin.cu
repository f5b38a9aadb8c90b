// topgpu_dropin.cu -- the six MEX kernels of TOP_GPU as C-ABI entry points
// for sm_100a.  Same arguments, layouts and in-place semantics as the MEX
// gateways (see include/topgpu.h for the file:line each one replaces).
#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>
#include "topgpu_kernels.cuh"

using namespace topgpu;

namespace {

inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// ---------------------------------------------------------------------------
// gather: one thread per element; node ids held in registers; 24 coalesced
// column stores (uMat is column-major [nElem x 24]).  An out-of-range node
// id yields 0 instead of an out-of-bounds read.
template <typename T, typename IDX>
__global__ void gather_kernel(T *__restrict__ uMat, const T *__restrict__ u,
                              const IDX *__restrict__ eNod, int64_t nElem, int64_t nNodes)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nElem) return;
    int64_t node[8];
#pragma unroll
    for (int n = 0; n < 8; ++n) node[n] = (int64_t)__ldg(&eNod[e + n * nElem]) - 1;
#pragma unroll
    for (int n = 0; n < 8; ++n) {
        const bool ok = node[n] >= 0 && node[n] < nNodes;
#pragma unroll
        for (int c = 0; c < 3; ++c)
            uMat[e + (int64_t)(3 * n + c) * nElem] = ok ? __ldg(&u[node[n] + c * nNodes]) : T(0);
    }
}

// scatter: one thread per element; each of the 24 contributions is a single
// fire-and-forget reduction into the L2-resident node array.
template <typename T>
__global__ void scatter_kernel(T *__restrict__ Y, const int32_t *__restrict__ eNod,
                               const T *__restrict__ uMat, int64_t Ne, int64_t nNodes)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Ne) return;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int64_t nid = (int64_t)__ldg(&eNod[e + j * Ne]) - 1;
        if (nid < 0 || nid >= nNodes) continue;
#pragma unroll
        for (int c = 0; c < 3; ++c) atomicAdd(&Y[nid + c * nNodes], __ldg(&uMat[e + (int64_t)(c + 3 * j) * Ne]));
    }
}

template <typename T>
__global__ void scatter_accum3_kernel(const int32_t *__restrict__ keys, const T *__restrict__ Tmp,
                                      int64_t N, T *__restrict__ xF, int64_t M)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int64_t key = (int64_t)__ldg(&keys[i]) - 1;
    if (key < 0 || key >= M) return;
#pragma unroll
    for (int c = 0; c < 3; ++c) atomicAdd(&xF[key + c * M], __ldg(&Tmp[i + c * N]));
}

// Q_s = P_s^T K0 P_s for every child slot (one CTA each): the child-
// independent part of the level-2 Galerkin product.
template <typename T>
struct K0Child {
    const T *K0;
    __device__ T operator()(int32_t, int i) const { return K0[i]; }
};
struct NoSkip { __device__ bool operator()(int32_t) const { return false; } };

// [n x n] identity child map: CTA e of ptkp_kernel then processes slot e only
__global__ void eye_upmap_kernel(int32_t *up, int n)
{ int i = blockIdx.x * blockDim.x + threadIdx.x; if (i < n * n) up[i] = (i % (n + 1) == 0) ? 1 : 0; }

// A row of the level-2 GEMM: the moduli of a coarse cell's regular children
// (0 for void children and for children with fixed DOFs).
struct Level2Row {
    const int32_t *upMap; const double *E; const int32_t *mapUnique; int64_t nElem; int nCh; int hasFixed;
    __device__ double operator()(int64_t m, int k) const {
        if (k >= nCh) return 0.0;
        const int32_t f1 = upMap[m + (int64_t)k * nElem];
        if (f1 <= 0) return 0.0;
        if (hasFixed && mapUnique[f1 - 1] > 0) return 0.0;
        return E[f1 - 1];
    }
};

template <typename T>
struct Level2Child {   // K_child of assembleKs_level2_inplace.cu:104-115
    const T *E; const T *K0; const int32_t *mapUnique; const T *uFree; const T *uFixed; int hasFixed;
    __device__ T operator()(int32_t f0, int i) const {
        const T mod = E[f0];
        const int32_t uid0 = hasFixed ? mapUnique[f0] - 1 : -1;
        if (uid0 >= 0) return uFree[(size_t)uid0 * 576 + i] * mod + uFixed[(size_t)uid0 * 576 + i];
        return K0[i] * mod;
    }
};
struct RegularChild {  // skip children with fixed DOFs (handled by the GEMM otherwise)
    const int32_t *mapUnique; int hasFixed; int invert;
    __device__ bool operator()(int32_t f0) const {
        const bool bnd = hasFixed && mapUnique[f0] > 0;
        return invert ? !bnd : bnd;
    }
};
template <typename T>
struct PrevChild {
    const T *KsPrev;
    __device__ T operator()(int32_t f0, int i) const { return KsPrev[(size_t)f0 * 576 + i]; }
};
template <typename T>
struct SuperChild {   // assembleKs_level2_superEle_inplace.cu:113-140
    const T *Ks0; const int32_t *mapUnique; const T *E; const T *uFree; const T *uFixed; int hasFixed;
    __device__ T operator()(int32_t f0, int i) const {
        const int32_t uid1 = hasFixed ? mapUnique[f0] : 0;
        if (uid1 > 0) {
            const size_t fb = (size_t)(uid1 - 1) * 576 * 64, mb = (size_t)f0 * 64;
            T acc = T(0);
            for (int q = 0; q < 64; ++q) acc += uFree[fb + (size_t)q * 576 + i] * E[mb + q];
            return acc + uFixed[(size_t)(uid1 - 1) * 576 + i];
        }
        return Ks0[(size_t)f0 * 576 + i];
    }
};

inline int blocks_for(int64_t n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

extern "C" int top_gather(void *uMat, const void *u, const void *eNod, int eNodIsU32,
                          int64_t nElem, int64_t nNodes, int dtype, void *stream)
{
    if (nElem < 0 || nNodes < 0) { set_error("Gathering_inplace:Shape negative size"); return TOP_ERR_SHAPE; }
    if (dtype != TOP_F32 && dtype != TOP_F64) { set_error("Gathering_inplace:Type gU must be single or double."); return TOP_ERR_TYPE; }
    if (nElem == 0) return TOP_OK;
    if (!uMat || !u || !eNod) { set_error("Gathering_inplace:Args null pointer"); return TOP_ERR_ARGS; }
    const int T = 256, G = blocks_for(nElem, T);
    if (dtype == TOP_F64) {
        if (eNodIsU32) gather_kernel<double, uint32_t><<<G, T, 0, S(stream)>>>((double *)uMat, (const double *)u, (const uint32_t *)eNod, nElem, nNodes);
        else gather_kernel<double, int32_t><<<G, T, 0, S(stream)>>>((double *)uMat, (const double *)u, (const int32_t *)eNod, nElem, nNodes);
    } else {
        if (eNodIsU32) gather_kernel<float, uint32_t><<<G, T, 0, S(stream)>>>((float *)uMat, (const float *)u, (const uint32_t *)eNod, nElem, nNodes);
        else gather_kernel<float, int32_t><<<G, T, 0, S(stream)>>>((float *)uMat, (const float *)u, (const int32_t *)eNod, nElem, nNodes);
    }
    TOP_CUDA_CHECK(cudaGetLastError(), "Gathering_inplace");
    return TOP_OK;
}

extern "C" int top_scatter(void *Y, const int32_t *eNod, const void *uMat,
                           int64_t nElem, int64_t nNodes, int dtype, void *stream)
{
    if (nElem < 0 || nNodes < 0) { set_error("Scattering_inplace:shape negative size"); return TOP_ERR_SHAPE; }
    if (dtype != TOP_F32 && dtype != TOP_F64) { set_error("Scattering_inplace:type unsupported class"); return TOP_ERR_TYPE; }
    if (nElem > 0) {
        if (!Y || !eNod || !uMat) { set_error("Scattering_inplace:arity null pointer"); return TOP_ERR_ARGS; }
        const int T = 256, G = blocks_for(nElem, T);
        if (dtype == TOP_F64) scatter_kernel<double><<<G, T, 0, S(stream)>>>((double *)Y, eNod, (const double *)uMat, nElem, nNodes);
        else scatter_kernel<float><<<G, T, 0, S(stream)>>>((float *)Y, eNod, (const float *)uMat, nElem, nNodes);
        TOP_CUDA_CHECK(cudaGetLastError(), "Scattering_inplace");
    }
    TOP_CUDA_CHECK(cudaStreamSynchronize(S(stream)), "Scattering_inplace");
    return TOP_OK;
}

extern "C" int top_scatter_accum3(const int32_t *keys, const void *Tmp, int64_t N,
                                  void *xF, int64_t M, int dtype, void *stream)
{
    if (N < 0 || M < 0) { set_error("scatter_accum3:shape negative size"); return TOP_ERR_SHAPE; }
    if (dtype != TOP_F32 && dtype != TOP_F64) { set_error("scatter_accum3:type Only single or double supported for `Tmp`/`xFiner`."); return TOP_ERR_TYPE; }
    if (N == 0) return TOP_OK;
    if (!keys || !Tmp || !xF) { set_error("scatter_accum3:gpu All inputs must be gpuArray."); return TOP_ERR_ARGS; }
    const int T = 256, G = blocks_for(N, T);
    if (dtype == TOP_F64) scatter_accum3_kernel<double><<<G, T, 0, S(stream)>>>(keys, (const double *)Tmp, N, (double *)xF, M);
    else scatter_accum3_kernel<float><<<G, T, 0, S(stream)>>>(keys, (const float *)Tmp, N, (float *)xF, M);
    TOP_CUDA_CHECK(cudaGetLastError(), "scatter_accum3");
    return TOP_OK;
}

namespace topgpu {
// Level-2 Galerkin assembly in the form Ks = (moduli of regular children) x Q
// on the FP64 tensor cores, plus the full triple product for children with
// fixed DOFs.  Shared with the fused solver.  Qscratch: [64 x 576] doubles,
// zero-filled by the caller; eyeScratch: [nCh x nCh] int32.
int assemble_level2_f64(double *Ks, const int32_t *upMap, const double *E, const double *K0,
                        const double *Pch, const int32_t *mapUnique, const double *uFree,
                        const double *uFixed, int64_t nElem, int nCh, int64_t nUnique,
                        double *Qscratch, int32_t *eyeScratch, cudaStream_t st,
                        const int32_t *bndList, int64_t nBnd)
{
    const int hasFixed = (nUnique > 0 && mapUnique && uFree && uFixed) ? 1 : 0;
    // Q_s = P_s^T K0 P_s, one CTA per child slot
    if (nCh > 0) {
        eye_upmap_kernel<<<(nCh * nCh + 255) / 256, 256, 0, st>>>(eyeScratch, nCh);
        ptkp_f64(st, Qscratch, eyeScratch, nCh, nCh, Pch, K0Child<double>{K0}, NoSkip{}, 0, nullptr, nCh);
    }
    if (nElem == 0) return TOP_OK;
    if (nCh <= kGemmK) {
        cudaFuncSetAttribute(dgemm_k64_kernel<Level2Row>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem);
        // one CTA per row block, looping over the column tiles (the gathered A
        // tile loaded once instead of once per column tile)
        dim3 grid((unsigned)((nElem + kGemmBM - 1) / kGemmBM), 1);
        // B = Qscratch has 64 rows whatever nCh is: the GEMM's K tiles load rows
        // nCh..63 too and multiply them by the zero A entries that ARow returns
        // there, so those rows must exist and hold finite values (0 * NaN = NaN)
        dgemm_k64_kernel<<<grid, 128, kGemmSmem, st>>>(Ks, nElem, 576, 576, Qscratch, 576,
                                                       Level2Row{upMap, E, mapUnique, nElem, nCh, hasFixed});
        // children with fixed DOFs: full triple products, accumulated; only the
        // coarse cells in bndList when the caller knows them (-1: all cells)
        if (hasFixed && nBnd != 0)
            ptkp_f64(st, Ks, upMap, nElem, nCh, Pch, Level2Child<double>{E, K0, mapUnique, uFree, uFixed, hasFixed},
                     RegularChild{mapUnique, hasFixed, 1}, 1, nBnd > 0 ? bndList : nullptr, nBnd > 0 ? nBnd : nElem);
    } else {
        ptkp_f64(st, Ks, upMap, nElem, nCh, Pch, Level2Child<double>{E, K0, mapUnique, uFree, uFixed, hasFixed}, NoSkip{}, 0,
                 nullptr, nElem);
    }
    return cudaGetLastError() == cudaSuccess ? TOP_OK : TOP_ERR_CUDA;
}

int assemble_higher_f64(double *Ks, const int32_t *upMap, const double *KsPrev, const double *Psub,
                        int64_t nElem, int nSub, cudaStream_t st)
{
    if (nElem == 0) return TOP_OK;
    ptkp_f64(st, Ks, upMap, nElem, nSub, Psub, PrevChild<double>{KsPrev}, NoSkip{}, 0, nullptr, nElem);
    return cudaGetLastError() == cudaSuccess ? TOP_OK : TOP_ERR_CUDA;
}
}  // namespace topgpu

extern "C" int top_assemble_ks_level2(void *Ks, const int32_t *upMap, const void *eleModulus,
                                      const void *K0, const void *Pch, const int32_t *mapUnique,
                                      const void *uniqueFree, const void *uniqueFixed,
                                      int64_t nElem, int nCh, int64_t nFine, int64_t nUnique,
                                      int dtype, void *stream)
{
    const char *N = "assembleKs_level2_inplace";
    if (dtype != TOP_F32 && dtype != TOP_F64) { set_error("%s:Type d_Ks must be single/double gpuArray.", N); return TOP_ERR_TYPE; }
    if (nElem < 0 || nCh < 0 || nFine < 0 || nUnique < 0) { set_error("%s:Shape negative size", N); return TOP_ERR_SHAPE; }
    if (nElem == 0) return TOP_OK;
    if (!Ks || !upMap || !eleModulus || !K0 || !Pch) { set_error("%s:Input null pointer", N); return TOP_ERR_ARGS; }
    const int hasFixed = (nUnique > 0 && mapUnique && uniqueFree && uniqueFixed) ? 1 : 0;
    cudaStream_t st = S(stream);
    if (dtype == TOP_F64) {
        struct Scratch {             // stream-ordered frees on every exit of this block
            void *p = nullptr; cudaStream_t st;
            explicit Scratch(cudaStream_t q) : st(q) {}
            ~Scratch() { if (p) cudaFreeAsync(p, st); }
        } q(st), o(st);
        const size_t qn = (size_t)576 * (nCh > 64 ? nCh : 64);
        TOP_CUDA_CHECK(cudaMallocAsync(&q.p, sizeof(double) * qn, st), N);
        TOP_CUDA_CHECK(cudaMemsetAsync(q.p, 0, sizeof(double) * qn, st), N);
        TOP_CUDA_CHECK(cudaMallocAsync(&o.p, sizeof(int32_t) * (size_t)nCh * nCh + 4, st), N);
        double *Q = static_cast<double *>(q.p);
        int32_t *one = static_cast<int32_t *>(o.p);
        int rc = assemble_level2_f64((double *)Ks, upMap, (const double *)eleModulus, (const double *)K0,
                                     (const double *)Pch, mapUnique, (const double *)uniqueFree,
                                     (const double *)uniqueFixed, nElem, nCh, hasFixed ? nUnique : 0, Q, one, st, nullptr, -1);
        if (rc) { set_error("%s:CUDA launch failed: %s", N, cudaGetErrorString(cudaGetLastError())); return rc; }
    } else {
        ptkp_kernel<float><<<(unsigned)nElem, kPtkpThreads, 0, st>>>(
            (float *)Ks, upMap, nElem, nCh, (const float *)Pch,
            Level2Child<float>{(const float *)eleModulus, (const float *)K0, mapUnique,
                               (const float *)uniqueFree, (const float *)uniqueFixed, hasFixed},
            NoSkip{}, 0, nullptr);
    }
    TOP_CUDA_CHECK(cudaGetLastError(), N);
    TOP_CUDA_CHECK(cudaStreamSynchronize(st), N);   // assembleKs_level2_inplace.cu:272
    return TOP_OK;
}

extern "C" int top_assemble_ks_higher(void *Ks, const int32_t *upMap, const void *KsPrev,
                                      const void *Psub, int64_t nElem, int nSub, int64_t nFine,
                                      int dtype, void *stream)
{
    const char *N = "assembleKs_higherLevel_inplace";
    if (dtype != TOP_F32 && dtype != TOP_F64) { set_error("%s:Type d_Ks must be single/double gpuArray.", N); return TOP_ERR_TYPE; }
    if (nElem < 0 || nSub < 0 || nFine < 0) { set_error("%s:Shape negative size", N); return TOP_ERR_SHAPE; }
    if (nElem == 0) return TOP_OK;
    if (!Ks || !upMap || !KsPrev || !Psub) { set_error("%s:Input null pointer", N); return TOP_ERR_ARGS; }
    cudaStream_t st = S(stream);
    if (dtype == TOP_F64)
        ptkp_f64(st, (double *)Ks, upMap, nElem, nSub, (const double *)Psub, PrevChild<double>{(const double *)KsPrev},
                 NoSkip{}, 0, nullptr, nElem);
    else
        ptkp_kernel<float><<<(unsigned)nElem, kPtkpThreads, 0, st>>>((float *)Ks, upMap, nElem, nSub, (const float *)Psub,
                                                                     PrevChild<float>{(const float *)KsPrev}, NoSkip{}, 0, nullptr);
    TOP_CUDA_CHECK(cudaGetLastError(), N);
    TOP_CUDA_CHECK(cudaStreamSynchronize(st), N);   // assembleKs_higherLevel_inplace.cu:209
    return TOP_OK;
}

extern "C" int top_assemble_ks_level2_super(void *Ks, const int32_t *upMap, const void *Ks0,
                                            const void *Psub, const int32_t *mapUnique,
                                            const void *eleModulus, const void *uniqueFree,
                                            const void *uniqueFixed, int64_t nElem, int nSub,
                                            int64_t nFine, int64_t nUnique, int dtype, void *stream)
{
    const char *N = "assembleKs_level2_superEle_inplace";
    if (dtype != TOP_F32 && dtype != TOP_F64) { set_error("%s:Type d_Ks must be single/double gpuArray.", N); return TOP_ERR_TYPE; }
    if (nElem < 0 || nSub < 0 || nFine < 0 || nUnique < 0) { set_error("%s:Shape negative size", N); return TOP_ERR_SHAPE; }
    if (nElem == 0) return TOP_OK;
    if (!Ks || !upMap || !Ks0 || !Psub || !eleModulus) { set_error("%s:Input null pointer", N); return TOP_ERR_ARGS; }
    const int hasFixed = (nUnique > 0 && mapUnique && uniqueFree && uniqueFixed) ? 1 : 0;
    cudaStream_t st = S(stream);
    if (dtype == TOP_F64)
        ptkp_f64(st, (double *)Ks, upMap, nElem, nSub, (const double *)Psub,
                 SuperChild<double>{(const double *)Ks0, mapUnique, (const double *)eleModulus,
                                    (const double *)uniqueFree, (const double *)uniqueFixed, hasFixed}, NoSkip{}, 0, nullptr, nElem);
    else
        ptkp_kernel<float><<<(unsigned)nElem, kPtkpThreads, 0, st>>>(
            (float *)Ks, upMap, nElem, nSub, (const float *)Psub,
            SuperChild<float>{(const float *)Ks0, mapUnique, (const float *)eleModulus,
                              (const float *)uniqueFree, (const float *)uniqueFixed, hasFixed}, NoSkip{}, 0, nullptr);
    TOP_CUDA_CHECK(cudaGetLastError(), N);
    TOP_CUDA_CHECK(cudaStreamSynchronize(st), N);   // ..._superEle_inplace.cu:313
    return TOP_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of top_assemble_ks_level2.
//
// Some callers cannot let this library allocate device memory during a
// call: a MEX gateway running inside MATLAB, whose gpuArray pool keeps most
// of the device memory and expects to be the only allocator, and
// applications that reserve their memory once up front and must not pay the
// implicit device synchronisation of cudaMalloc/cudaFree inside an
// optimisation loop.  This entry point takes its scratch (the child matrices
// Q_s = P_s' K0 P_s and the slot map of the level-2 Galerkin GEMM) from the
// fixed device arrays below, which every GPU that loads the library holds
// until the process exits (about 311 KB per device).
//
// Limits and behaviour:
//  * at most kNoAllocMaxChildren (64) children per coarse element -- the
//    level-2 case of the reference (span 4); larger nCh is rejected with
//    TOP_ERR_SHAPE before anything runs;
//  * the first call on a device (and the first call after that device's
//    context was replaced, e.g. by cudaDeviceReset) resolves the arrays'
//    device addresses with cudaGetSymbolAddress, with that device current;
//    make that call before any stream capture on that device;
//  * all calls share the arrays and each call clears the part it reads, so
//    calls that run concurrently on the GPU (different streams or threads)
//    race -- serialise them.
namespace {
constexpr int kNoAllocMaxChildren = 64;
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) double g_noalloc_Q[576 * kNoAllocMaxChildren];
static __device__ __align__(256) int32_t g_noalloc_eye[kNoAllocMaxChildren * kNoAllocMaxChildren];

// The resolved addresses are valid for one context of one device: a device
// reset unloads the module and the next context may place the arrays
// elsewhere, so the cache is keyed on (device, current context).  The context
// handle comes from the driver's cuCtxGetCurrent, looked up through the
// runtime (no link against libcuda).
struct NoAllocScratch { double *Q = nullptr; int32_t *eye = nullptr; void *ctx = nullptr; };
std::mutex g_noalloc_mu;
NoAllocScratch g_noalloc_dev[kNoAllocMaxDevices];
bool g_noalloc_ready[kNoAllocMaxDevices] = {};
typedef int (*CtxGetCurrentFn)(void **);

int current_context(void **ctx, const char *N)
{
    static CtxGetCurrentFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        TOP_CUDA_CHECK(cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q), N);
        if (q != cudaDriverEntryPointSuccess || !p) { set_error("%s:CUDA cuCtxGetCurrent not available", N); return TOP_ERR_CUDA; }
        fn = reinterpret_cast<CtxGetCurrentFn>(p);
    }
    *ctx = nullptr;
    if (fn(ctx) != 0 || !*ctx) { set_error("%s:CUDA no current context", N); return TOP_ERR_CUDA; }
    return TOP_OK;
}

int noalloc_scratch(NoAllocScratch *out, const char *N)
{
    int dev = 0;
    TOP_CUDA_CHECK(cudaGetDevice(&dev), N);
    if (dev < 0 || dev >= kNoAllocMaxDevices) { set_error("%s:CUDA device %d out of range", N, dev); return TOP_ERR_CUDA; }
    TOP_CUDA_CHECK(cudaSetDevice(dev), N);         // binds the device's primary context to this thread
    void *ctx = nullptr;
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    int rc = current_context(&ctx, N);
    if (rc) return rc;
    if (!g_noalloc_ready[dev] || g_noalloc_dev[dev].ctx != ctx) {
        NoAllocScratch s;
        TOP_CUDA_CHECK(cudaGetSymbolAddress((void **)&s.Q, g_noalloc_Q), N);
        TOP_CUDA_CHECK(cudaGetSymbolAddress((void **)&s.eye, g_noalloc_eye), N);
        s.ctx = ctx;
        g_noalloc_dev[dev] = s;
        g_noalloc_ready[dev] = true;
    }
    *out = g_noalloc_dev[dev];
    return TOP_OK;
}
}  // namespace

extern "C" int top_assemble_ks_level2_noalloc(void *Ks, const int32_t *upMap, const void *eleModulus,
                                              const void *K0, const void *Pch, const int32_t *mapUnique,
                                              const void *uniqueFree, const void *uniqueFixed,
                                              int64_t nElem, int nCh, int64_t nFine, int64_t nUnique,
                                              int dtype, void *stream)
{
    const char *N = "assembleKs_level2_inplace";
    if (dtype != TOP_F32 && dtype != TOP_F64) { set_error("%s:Type d_Ks must be single/double gpuArray.", N); return TOP_ERR_TYPE; }
    if (nElem < 0 || nCh < 0 || nFine < 0 || nUnique < 0) { set_error("%s:Shape negative size", N); return TOP_ERR_SHAPE; }
    if (nCh > kNoAllocMaxChildren) {
        set_error("%s:Shape %d children per coarse element exceed the allocation-free limit of %d", N, nCh, kNoAllocMaxChildren);
        return TOP_ERR_SHAPE;
    }
    if (nElem == 0) return TOP_OK;
    if (!Ks || !upMap || !eleModulus || !K0 || !Pch) { set_error("%s:Input null pointer", N); return TOP_ERR_ARGS; }
    const int hasFixed = (nUnique > 0 && mapUnique && uniqueFree && uniqueFixed) ? 1 : 0;
    cudaStream_t st = S(stream);
    if (dtype == TOP_F64) {
        NoAllocScratch sc;
        int rc = noalloc_scratch(&sc, N);
        if (rc) return rc;
        // the GEMM loads all 64 rows of Q and multiplies rows nCh..63 by zero:
        // clear them all, so that no value left by an earlier call (NaN or Inf
        // included) reaches this call's result
        TOP_CUDA_CHECK(cudaMemsetAsync(sc.Q, 0, sizeof(double) * 576 * kNoAllocMaxChildren, st), N);
        rc = assemble_level2_f64((double *)Ks, upMap, (const double *)eleModulus, (const double *)K0,
                                 (const double *)Pch, mapUnique, (const double *)uniqueFree,
                                 (const double *)uniqueFixed, nElem, nCh, hasFixed ? nUnique : 0, sc.Q, sc.eye, st, nullptr, -1);
        if (rc) { set_error("%s:CUDA launch failed: %s", N, cudaGetErrorString(cudaGetLastError())); return rc; }
    } else {
        ptkp_kernel<float><<<(unsigned)nElem, kPtkpThreads, 0, st>>>(
            (float *)Ks, upMap, nElem, nCh, (const float *)Pch,
            Level2Child<float>{(const float *)eleModulus, (const float *)K0, mapUnique,
                               (const float *)uniqueFree, (const float *)uniqueFixed, hasFixed},
            NoSkip{}, 0, nullptr);
    }
    TOP_CUDA_CHECK(cudaGetLastError(), N);
    TOP_CUDA_CHECK(cudaStreamSynchronize(st), N);
    return TOP_OK;
}
