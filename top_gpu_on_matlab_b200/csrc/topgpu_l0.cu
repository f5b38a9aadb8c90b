// topgpu_l0.cu -- level-0 stiffness product dispatch of the fused solver:
// the node-centric kernel with the dense 24x24 Ke (topgpu_grid.cuh) or the
// Walsh-basis tile kernel (topgpu_walsh.cuh), per precision, with the
// operand/epilogue combinations the solver uses instantiated here.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include "topgpu_solver_impl.cuh"
#include "topgpu_stage.cuh"

namespace topgpu {
namespace {

template <typename T> const KeParam<T> &keparam(const top_solver *s);
template <> const KeParam<double> &keparam<double>(const top_solver *s) { return s->Ke64; }
template <> const KeParam<float> &keparam<float>(const top_solver *s) { return s->Ke32; }
template <typename T> const T *egrid(const top_solver *s);
template <> const double *egrid<double>(const top_solver *s) { return s->Eg64; }
template <> const float *egrid<float>(const top_solver *s) { return s->Eg32; }
template <typename T> const WalshParam<T> &walshparam(const top_solver *s);
template <> const WalshParam<double> &walshparam<double>(const top_solver *s) { return s->W64; }
template <> const WalshParam<float> &walshparam<float>(const top_solver *s) { return s->W32; }
template <typename T> const WalshPairParam<T> &walshpair(const top_solver *s);
template <> const WalshPairParam<double> &walshpair<double>(const top_solver *s) { return s->WP64; }
template <> const WalshPairParam<float> &walshpair<float>(const top_solver *s) { return s->WP32; }
template <typename T> constexpr int prec_slot() { return sizeof(T) == 8 ? 0 : 1; }

// thread-tile shapes the Walsh-basis kernels are built for
#define TOPGPU_WALSH_SHAPES(X) X(16, 16) X(16, 8)

bool walsh_shape_ok(int ty, int tx)
{
#define TOPGPU_SHAPE_OK(A, B) if (ty == A && tx == B) return true;
    TOPGPU_WALSH_SHAPES(TOPGPU_SHAPE_OK)
#undef TOPGPU_SHAPE_OK
    return false;
}
int tiles_of(const Geom &g, int kind, int ty, int tx)
{
    if (kind == 6) return stg::tiles(g, ty, tx);
    return (kind == 2 || kind == 4) ? walsh_pair_tiles(g, ty, tx) : walsh_tiles(g, ty, tx);
}

// ---- kind 6: tensor maps of the staged level-0 product -------------------
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda)
PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}
// node vector: (y, x', z', component, right-hand side) over a level-0 grid
// vector (base = slot 0 of component 0 = node (0, -1, -1)); box = one staged
// node layer of a tile
bool encode_nodes(CUtensorMap *m, const float *base, const Geom &g, int64_t vs, int nv, int boxY, int boxX)
{
    auto fn = encode_fn();
    if (!fn) return false;
    const int64_t PX = g.NX + 2, PZ = g.NZ + 2;
    const cuuint64_t dims[5] = {(cuuint64_t)g.PY, (cuuint64_t)PX, (cuuint64_t)PZ, 3, (cuuint64_t)(nv > 0 ? nv : 1)};
    const cuuint64_t strides[4] = {(cuuint64_t)g.PY * 4, (cuuint64_t)g.plane * 4, (cuuint64_t)g.cs * 4,
                                   (cuuint64_t)(vs > 0 ? vs : 3 * g.cs) * 4};
    const cuuint32_t box[5] = {(cuuint32_t)boxY, (cuuint32_t)boxX, 1, 3, 1};
    const cuuint32_t es[5] = {1, 1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, const_cast<float *>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
// element moduli on the node grid (element at its base node's slot)
bool encode_moduli(CUtensorMap *m, const float *base, const Geom &g, int boxY, int boxX)
{
    auto fn = encode_fn();
    if (!fn) return false;
    const int64_t PX = g.NX + 2, PZ = g.NZ + 2;
    const cuuint64_t dims[3] = {(cuuint64_t)g.PY, (cuuint64_t)PX, (cuuint64_t)PZ};
    const cuuint64_t strides[2] = {(cuuint64_t)g.PY * 4, (cuuint64_t)g.plane * 4};
    const cuuint32_t box[3] = {(cuuint32_t)boxY, (cuuint32_t)boxX, 1};
    const cuuint32_t es[3] = {1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
// the staged kernel needs 16-byte aligned vectors and multiple-of-four
// pitches (TMA strides and the paired epilogue accesses)
bool stage_geom_ok(const Geom &g) { return ((g.PY | g.plane | g.origin | g.cs) & 3) == 0; }

template <int A, int B, class Out>
void launch_stage(top_solver *s, const top_solver::L0Kernel &k, const VecIn<float, float> &in, const Out &out,
                  Reduce red, const int *done, int nv)
{
    using Tl = stg::Tile<A, B>;
    DevLevel &lv = s->L[0];
    static const int occ = [] {
        int n = 0;
        if (cudaFuncSetAttribute(l0s_kernel<A, B, Out>, cudaFuncAttributeMaxDynamicSharedMemorySize, Tl::SMEM) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, l0s_kernel<A, B, Out>, Tl::NTHREADS, Tl::SMEM) != cudaSuccess)
            n = 1;
        return n > 0 ? n : 1;
    }();
    const int64_t work = (int64_t)stg::tiles(lv.g, A, B) * lv.g.NZ;
    int64_t n = k.ctas > 0 ? k.ctas : (int64_t)s->numSMs * occ;
    n = std::max<int64_t>(std::min<int64_t>(std::min<int64_t>(n, work), s->nPartials), 1);
    CUtensorMap mu, me;
    const float *ub = in.u.p0;
    const int64_t vs = in.vs;
    const bool ok = encode_nodes(&mu, ub, lv.g, vs, vs > 0 ? nv : 1, Tl::BY, Tl::BXU) &&
                    encode_moduli(&me, s->Eg32, lv.g, Tl::BY, B);
    if (!ok) { s->stageErr = true; return; }
    launch_k(s, l0s_kernel<A, B, Out>, dim3((unsigned)n, (unsigned)nv), Tl::NTHREADS, (size_t)Tl::SMEM, s->st,
             mu, me, s->WP32, in, out, lv.flags, k.mask, lv.g, float(s->p.E0), red, done, s->tcErr);
}

// grid of the Walsh kernel: the configured CTA count (0: the CTAs that fit
// on the GPU at once), at most one per (tile, layer) work item
template <typename T, int A, int B, class In, class Out, int KIND>
unsigned l0w_ctas(const top_solver *s, const top_solver::L0Kernel &k)
{
    static const int occ = [] {
        int n = 0;
        cudaError_t e;
        if constexpr (KIND == 2) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, l0p_kernel<T, A, B, In, Out>, A * B, 0);
        else if constexpr (KIND == 3) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, l0d_kernel<T, A, B, In, Out>, A * B, 0);
        else if constexpr (KIND == 4) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, l0q_kernel<T, A, B, In, Out>, A * B, 0);
        else if constexpr (KIND == 5) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, l0t_kernel<A, B, In, Out>, A * B, tc::kSmemBytes);
        else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, l0w_kernel<T, A, B, In, Out>, A * B, 0);
        if (e != cudaSuccess) n = 1;
        return n > 0 ? n : 1;
    }();
    const DevLevel &lv = s->L[0];
    const int64_t work = (int64_t)tiles_of(lv.g, KIND, A, B) * lv.g.NZ;
    int64_t n = k.ctas > 0 ? k.ctas : (int64_t)s->numSMs * occ;
    n = std::min<int64_t>(std::min<int64_t>(n, work), s->nPartials);
    return (unsigned)std::max<int64_t>(n, 1);
}

}  // namespace

template <typename T, class In, class Out>
void l0_op(top_solver *s, const In &in, const Out &out, Reduce red, const int *done, int nv)
{
    DevLevel &lv = s->L[0];
    const top_solver::L0Kernel &k = s->l0k[prec_slot<T>()];
    const unsigned K = (unsigned)nv;  // right-hand sides (grid y or z)
    if (s->super) {                   // per-element matrices (K_mat), packed on the grid
        const T *Kp;
        if constexpr (sizeof(T) == 8) Kp = lv.KsP64; else Kp = lv.KsP32;
        dim3 gr = coarse_tile_grid(lv.g); gr.z = K;
        launch_k(s, coarse_tile_kernel<T, In, Out>, gr, dim3(kCoarseTileX, 8), 0, s->st, in, out, Kp, lv.g, red, done);
    } else if (k.kind == 1) {
#define TOPGPU_LAUNCH_SHAPE(A, B)                                                                             \
        if (k.ty == A && k.tx == B)                                                                           \
            launch_k(s, l0w_kernel<T, A, B, In, Out>, dim3(l0w_ctas<T, A, B, In, Out, 1>(s, k), K), A * B, 0, s->st,   \
                walshparam<T>(s), in, out, egrid<T>(s), lv.flags, k.mask, lv.g, T(s->p.E0), red, done);
        TOPGPU_WALSH_SHAPES(TOPGPU_LAUNCH_SHAPE)
#undef TOPGPU_LAUNCH_SHAPE
    } else if (k.kind == 3) {
#define TOPGPU_LAUNCH_SHAPE(A, B)                                                                             \
        if (k.ty == A && k.tx == B)                                                                           \
            launch_k(s, l0d_kernel<T, A, B, In, Out>, dim3(l0w_ctas<T, A, B, In, Out, 3>(s, k), K), A * B, 0, s->st,   \
                walshparam<T>(s), in, out, egrid<T>(s), lv.flags, k.mask, lv.g, T(s->p.E0), red, done);
        TOPGPU_WALSH_SHAPES(TOPGPU_LAUNCH_SHAPE)
#undef TOPGPU_LAUNCH_SHAPE
    } else if (k.kind == 5) {        // FP32 only: tensor cores, 16 x 8 element columns
        if constexpr (sizeof(T) == 4) {
            static const bool attr = cudaFuncSetAttribute(l0t_kernel<16, 8, In, Out>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                          tc::kSmemBytes) == cudaSuccess;
            (void)attr;
            launch_k(s, l0t_kernel<16, 8, In, Out>, dim3(l0w_ctas<T, 16, 8, In, Out, 5>(s, k), K), 128, tc::kSmemBytes, s->st, 
                s->tcB, in, out, egrid<T>(s), lv.flags, k.mask, lv.g, T(s->p.E0), red, done, s->tcErr);
        }
    } else if (k.kind == 6) {        // FP32 only: TMA-staged layers, plain FP32 operand vectors
        if constexpr (sizeof(T) == 4 && std::is_same<In, VecIn<float, float>>::value) {
#define TOPGPU_LAUNCH_SHAPE(A, B) if (k.ty == A && k.tx == B) launch_stage<A, B, Out>(s, k, in, out, red, done, nv);
            TOPGPU_WALSH_SHAPES(TOPGPU_LAUNCH_SHAPE)
#undef TOPGPU_LAUNCH_SHAPE
        } else if constexpr (sizeof(T) == 4) {   // another operand type: the direct-load kind, same tile shape
            launch_k(s, l0d_kernel<T, 16, 8, In, Out>, dim3(l0w_ctas<T, 16, 8, In, Out, 3>(s, s->l0kFallback), K), 128, 0, s->st,
                walshparam<T>(s), in, out, egrid<T>(s), lv.flags, s->l0kFallback.mask, lv.g, T(s->p.E0), red, done);
        }
    } else if (k.kind == 4) {        // FP32 only, as kind 2
        if constexpr (sizeof(T) == 4) {
#define TOPGPU_LAUNCH_SHAPE(A, B)                                                                             \
            if (k.ty == A && k.tx == B)                                                                       \
                launch_k(s, l0q_kernel<T, A, B, In, Out>, dim3(l0w_ctas<T, A, B, In, Out, 4>(s, k), K), A * B, 0, s->st,  \
                    walshpair<T>(s), in, out, egrid<T>(s), lv.flags, k.mask, lv.g, T(s->p.E0), red, done);
            TOPGPU_WALSH_SHAPES(TOPGPU_LAUNCH_SHAPE)
#undef TOPGPU_LAUNCH_SHAPE
        }
    } else if (k.kind == 2) {        // FP32 only: the FP64 pair state does not fit in registers
        if constexpr (sizeof(T) == 4) {
#define TOPGPU_LAUNCH_SHAPE(A, B)                                                                             \
            if (k.ty == A && k.tx == B)                                                                       \
                launch_k(s, l0p_kernel<T, A, B, In, Out>, dim3(l0w_ctas<T, A, B, In, Out, 2>(s, k), K), A * B, 0, s->st,  \
                    walshpair<T>(s), in, out, egrid<T>(s), lv.flags, k.mask, lv.g, T(s->p.E0), red, done);
            TOPGPU_WALSH_SHAPES(TOPGPU_LAUNCH_SHAPE)
#undef TOPGPU_LAUNCH_SHAPE
        }
    } else {
        launch_k(s, l0_kernel<T, In, Out>, dim3((unsigned)lv.g.nbx, (unsigned)lv.g.NZ, K), kNodeThreads, 0, s->st, 
            keparam<T>(s), in, out, egrid<T>(s), lv.flags, lv.tileFixed, lv.g, T(s->p.E0), red, done);
    }
    TOPGPU_COUNT_LAUNCH();
}

namespace {
// round an FP32 value to TF32 (nearest, ties away from zero): 10 mantissa bits
float tf32_round(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7F800000u) != 0x7F800000u) u = (u + 0x1000u) & 0xFFFFE000u;
    std::memcpy(&x, &u, 4);
    return x;
}
// Bk for the tensor-core kind: rows n (12 bottom-corner outputs, 12 top,
// 8 zero) x columns k (12 bottom-corner inputs, 4 zero, 12 top, 4 zero),
// corner (by, bx) -> slot 3 (by + 2 bx) + c; Ke's local DOF of corner
// (by, bx, bz), component c is 3 a + c with (cdy, cdx, cdz)(a) = (by, bx, bz)
int tc_operand(top_solver *s)
{
    if (s->tcB) return TOP_OK;
    int corner[2][2][2];
    for (int a = 0; a < 8; ++a) corner[cdy(a)][cdx(a)][cdz(a)] = a;
    auto dof = [&](int j, bool isRow) {        // operand index -> Ke local DOF, or -1 for a pad
        int bz;
        if (isRow) { if (j >= 24) return -1; bz = j / 12; j %= 12; }
        else { if ((j & 15) >= 12) return -1; bz = j >> 4; j &= 15; }
        const int k4 = j / 3, c = j % 3;
        return 3 * corner[k4 & 1][k4 >> 1][bz] + c;
    };
    std::vector<float> img(2 * tc::kBBytes / 4, 0.f);
    for (int n = 0; n < tc::kN; ++n)
        for (int k = 0; k < 32; ++k) {
            const int r = dof(n, true), c = dof(k, false);
            const float v = (r < 0 || c < 0) ? 0.f : s->Ke32.k[r * 24 + c];
            const float hi = tf32_round(v), lo = tf32_round(v - hi);
            const int o = tc::kmajor_off(n, k, 1024) / 4;
            img[o] = hi;
            img[tc::kBBytes / 4 + o] = lo;
        }
    s->tcB = s->dalloc<TcOperandB>(1);
    s->tcErr = s->dalloc<int>(1);
    if (!s->tcB || !s->tcErr) return TOP_ERR_NOMEM;
    if (cudaMemcpy(s->tcB, img.data(), sizeof(float) * img.size(), cudaMemcpyHostToDevice) != cudaSuccess) return TOP_ERR_CUDA;
    return TOP_OK;
}
// pseudo-random values at the active nodes (guard slots stay zero)
__global__ void tc_probe_fill_kernel(float *x, int64_t cs, const int32_t *nodeGrid, int64_t Nn)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < 3 * Nn; i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t h = (uint32_t)(i * 2654435761u) >> 8;
        x[(i % 3) * cs + nodeGrid[i / 3]] = float(h) * (1.f / 16777216.f) - 0.5f;
    }
}
__global__ void tc_probe_diff_kernel(const float *a, const float *b, int64_t n, double *out)
{
    double dd = 0.0, nn = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double d = double(a[i]) - double(b[i]);
        dd += d * d; nn += double(b[i]) * double(b[i]);
    }
    atomicAdd(out, dd); atomicAdd(out + 1, nn);
}
// the tensor-core or staged kind against the dense kernel on one
// pseudo-random vector, with the model's current moduli: relative 2-norm
// difference below 1e-5 and no mbarrier wait gave up
int tc_selftest(top_solver *s, const top_solver::L0Kernel &cand)
{
    DevLevel &l0 = s->L[0];
    const int64_t n = 3 * l0.g.cs;
    const int64_t M = kMargin;
    const Reduce none{nullptr, nullptr, nullptr};
    top_solver::L0Kernel saved = s->l0k[1];
    double *dev = s->scal;                   // two scratch scalars
    cudaMemsetAsync(l0.x32 - M, 0, sizeof(float) * n, s->st);
    tc_probe_fill_kernel<<<512, 256, 0, s->st>>>(l0.x32, l0.g.cs, l0.nodeGrid, l0.Nn);
    cudaMemsetAsync(s->tcErr, 0, sizeof(int), s->st);
    s->l0k[1] = top_solver::L0Kernel{};      // kind 0 (dense), no mask
    l0_op<float>(s, VecIn<float, float>{l0.x32, l0.g.cs}, StoreOut<float, float>{l0.t32, l0.g.cs}, none, nullptr, 1);
    s->l0k[1] = cand; s->l0k[1].mask = saved.mask;
    l0_op<float>(s, VecIn<float, float>{l0.x32, l0.g.cs}, StoreOut<float, float>{s->z32, l0.g.cs}, none, nullptr, 1);
    s->l0k[1] = saved;
    cudaMemsetAsync(dev, 0, 2 * sizeof(double), s->st);
    tc_probe_diff_kernel<<<256, 256, 0, s->st>>>(s->z32 - M, l0.t32 - M, n, dev);
    double h[2] = {0, 0};
    int err = 0;
    if (cudaMemcpyAsync(h, dev, sizeof(h), cudaMemcpyDeviceToHost, s->st) != cudaSuccess ||
        cudaMemcpyAsync(&err, s->tcErr, sizeof(int), cudaMemcpyDeviceToHost, s->st) != cudaSuccess ||
        cudaStreamSynchronize(s->st) != cudaSuccess)
        return TOP_ERR_CUDA;
    cudaMemsetAsync(l0.x32 - M, 0, sizeof(float) * n, s->st);
    if (!err && !(h[1] > 0)) {
        set_error("level-0 kernel kind %d is checked on the model: set the element densities first", cand.kind);
        return TOP_ERR_STATE;
    }
    if (err || !(std::sqrt(h[0] / h[1]) < 1e-5)) {
        set_error("level-0 kernel kind %d failed its self-test (relative difference %.3e, wait error %d)",
                  cand.kind, h[1] > 0 ? std::sqrt(h[0] / h[1]) : -1.0, err);
        return TOP_ERR_CUDA;
    }
    return TOP_OK;
}
}  // namespace

int set_l0_kernel(top_solver *s, int p, int kind, int ty, int tx, int ctas)
{
    top_solver::L0Kernel &k = s->l0k[p];
    if (kind == 0) { k.kind = 0; ++s->opGen; return TOP_OK; }
    DevLevel &l0 = s->L[0];
    if (kind == 5) {                                   // tensor cores: FP32, 16 x 8, any Ke
        if (p != 1 || ty != 16 || tx != 8 || ctas < 0 || s->super) return TOP_ERR_ARGS;
        const int rc = tc_operand(s);
        if (rc != TOP_OK) return rc;
    } else if (kind == 6) {                            // TMA-staged: FP32, Walsh-symmetric Ke
        if (p != 1 || !s->walshOK || !walsh_shape_ok(ty, tx) || ctas < 0 || s->super || !stage_geom_ok(l0.g) || !encode_fn())
            return TOP_ERR_ARGS;
        if (!s->tcErr && !(s->tcErr = s->dalloc<int>(1))) return TOP_ERR_NOMEM;
        if (!s->l0kFallback.mask) {                    // direct-load kind for other operand types
            const int t3 = walsh_tiles(l0.g, 16, 8);
            if (cudaMalloc(&s->l0kFallback.mask, (size_t)t3) != cudaSuccess) { s->l0kFallback.mask = nullptr; return TOP_ERR_NOMEM; }
            walsh_mask_kernel<16, 8><<<t3, 256, 0, s->st>>>(l0.flags, l0.g, s->l0kFallback.mask);
            TOPGPU_COUNT_LAUNCH();
            s->l0kFallback.kind = 3; s->l0kFallback.ty = 16; s->l0kFallback.tx = 8; s->l0kFallback.ctas = 0;
        }
    } else if ((kind != 1 && kind != 3 && !((kind == 2 || kind == 4) && p == 1)) || !s->walshOK || !walsh_shape_ok(ty, tx) || ctas < 0)
        return TOP_ERR_ARGS;
    const int tiles = tiles_of(l0.g, kind, ty, tx);
    if (ctas > s->nPartials) {                         // one reduction partial per CTA and right-hand side
        double *pp = s->dalloc<double>((size_t)ctas * s->kMax);
        if (!pp) return TOP_ERR_NOMEM;
        s->partials = pp; s->nPartials = ctas;
    }
    if (k.mask) { cudaFree(k.mask); k.mask = nullptr; }
    if (cudaMalloc(&k.mask, (size_t)tiles) != cudaSuccess) { k.mask = nullptr; k.kind = 0; return TOP_ERR_NOMEM; }
#define TOPGPU_MASK_SHAPE(A, B)                                                                    \
    if (ty == A && tx == B) {                                                                      \
        if (kind == 2 || kind == 4) walsh_pair_mask_kernel<A, B><<<tiles, 256, 0, s->st>>>(l0.flags, l0.g, k.mask); \
        else if (kind == 6) stage_mask_kernel<A, B><<<tiles, 256, 0, s->st>>>(l0.flags, l0.g, k.mask); \
        else walsh_mask_kernel<A, B><<<tiles, 256, 0, s->st>>>(l0.flags, l0.g, k.mask);            \
    }
    TOPGPU_WALSH_SHAPES(TOPGPU_MASK_SHAPE)
#undef TOPGPU_MASK_SHAPE
    TOPGPU_COUNT_LAUNCH();
    if (cudaGetLastError() != cudaSuccess) return TOP_ERR_CUDA;
    if (kind == 5 || kind == 6) {
        top_solver::L0Kernel cand = k;
        cand.kind = kind; cand.ty = ty; cand.tx = tx; cand.ctas = ctas;
        s->stageErr = false;
        const int rc = tc_selftest(s, cand);
        if (rc != TOP_OK) return rc;
        if (s->stageErr) { set_error("level-0 kernel kind 6: tensor map encoding failed"); return TOP_ERR_CUDA; }
    }
    k.kind = kind; k.ty = ty; k.tx = tx; k.ctas = ctas;
    ++s->opGen;
    return TOP_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: times every level-0 kernel configuration on this model (plain
// y = K u launches on the solver's stream, L2 flushed before each) and keeps
// the fastest per precision.
namespace {
// time per PCG iteration of the level-0 products precision slot p's kernel
// serves, with their epilogues (L2 flushed before each): the outer product
// v = A p with p . v (slot 0, or slot 1 when the outer product runs in FP32),
// and the V-cycle's residual and post-smoothing products (slot 1 in mixed
// precision, slot 0 in FP64).  The epilogues change the registers a kernel
// holds and the bytes it moves, so the fastest configuration is chosen on the
// launches the solver makes.  A slot that serves none times the plain product.
double time_l0(top_solver *s, int p, int nrep, void *flush, size_t flushBytes, cudaEvent_t a, cudaEvent_t b)
{
    DevLevel &l0 = s->L[0];
    const int64_t cs = l0.g.cs;
    const bool mixed = s->p.precision == TOP_PREC_MIXED, outer32 = s->p.outerFP32 != 0;
    const bool outerHere = p == 0 ? !outer32 : outer32;
    const bool vcycleHere = p == 0 ? !mixed : mixed;
    const Reduce none{nullptr, nullptr, nullptr};
    const Reduce dot{s->partials, s->counter, s->scal + 8};
    const float om32 = float(s->p.omega);
    const double om64 = s->p.omega;
    double total = 0.0;
    for (int k = 0; k < nrep + 1; ++k) {
        double t = 0.0;
        bool ok = true;
        auto timed = [&](auto &&launch) {
            if (!ok) return;
            if (flush) cudaMemsetAsync(flush, k & 0xff, flushBytes, s->st);
            cudaEventRecord(a, s->st);
            launch();
            cudaEventRecord(b, s->st);
            if (cudaEventSynchronize(b) != cudaSuccess) { ok = false; return; }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, a, b);
            t += ms;
        };
        if (p == 0) {
            if (outerHere)
                timed([&] { l0_op<double>(s, VecIn<double, double>{s->pv, cs}, DotStoreOut<double, double, double>{s->v, s->pv, cs}, dot, nullptr, 1); });
            if (vcycleHere) {
                timed([&] { l0_op<double>(s, VecIn<double, double>{l0.x64, cs}, ResidOut<double, double, double>{s->r, l0.t64, cs}, none, nullptr, 1); });
                timed([&] { l0_op<double>(s, VecIn<double, double>{l0.x64, cs},
                                          PostSmoothOut<double, double, double>{l0.x64, s->r, l0.invD64, s->z, cs, om64}, dot, nullptr, 1); });
            }
            if (!outerHere && !vcycleHere)
                timed([&] { l0_op<double>(s, VecIn<double, double>{s->pv, cs}, StoreOut<double, double>{s->v, cs}, none, nullptr, 1); });
        } else {
            if (outerHere)
                timed([&] { l0_op<float>(s, VecIn<float, double>{s->pv, cs}, DotStoreOut<float, double, double>{s->v, s->pv, cs}, dot, nullptr, 1); });
            if (vcycleHere) {
                timed([&] { l0_op<float>(s, VecIn<float, float>{l0.x32, cs}, ResidOut<float, double, float>{s->r, l0.t32, cs}, none, nullptr, 1); });
                timed([&] { l0_op<float>(s, VecIn<float, float>{l0.x32, cs},
                                         PostSmoothOut<float, double, float>{l0.x32, s->r, l0.invD32, s->z32, cs, om32}, dot, nullptr, 1); });
            }
            if (!outerHere && !vcycleHere)
                timed([&] { l0_op<float>(s, VecIn<float, float>{l0.x32, cs}, StoreOut<float, float>{l0.t32, cs}, none, nullptr, 1); });
        }
        if (!ok) return -1.0;
        if (k > 0) total += t;              // the first round warms up
    }
    return total / nrep;
}
}  // namespace

int autotune_l0(top_solver *s, int nrep, int64_t flushBytes, double *msBest, int *configs)
{
    if (nrep < 1) return TOP_ERR_ARGS;
    void *flush = nullptr;
    if (flushBytes > 0 && cudaMalloc(&flush, (size_t)flushBytes) != cudaSuccess) return TOP_ERR_NOMEM;
    cudaEvent_t a, b;
    cudaEventCreate(&a); cudaEventCreate(&b);
    static const int shapes[][2] = {{16, 16}, {16, 8}};
    static const std::vector<int> mults = {4, 6, 8, 12, 16};
    static const std::vector<int> stageMults = {1, 2, 3, 4};     // kind 6 CTAs are large (a producer warp + a stage ring)
    int rc = TOP_OK;
    for (int p = 0; p < 2 && rc == TOP_OK; ++p) {
        int best[4] = {0, 16, 16, 0};
        rc = set_l0_kernel(s, p, 0, 16, 16, 0);
        double tBest = rc == TOP_OK ? time_l0(s, p, nrep, flush, (size_t)flushBytes, a, b) : -1.0;
        if (tBest < 0) { rc = TOP_ERR_CUDA; break; }
        if (s->walshOK) {
            for (int kind = 1; kind <= 6 && rc == TOP_OK; ++kind) {
                if ((kind == 2 || kind == 4 || kind == 5 || kind == 6) && p == 0) continue;
                for (const auto &sh : shapes)
                    for (int m : (kind == 6 ? stageMults : mults)) {
                        const int ctas = m * s->numSMs;
                        if (set_l0_kernel(s, p, kind, sh[0], sh[1], ctas) != TOP_OK) continue;
                        const double t = time_l0(s, p, nrep, flush, (size_t)flushBytes, a, b);
                        if (t < 0) { rc = TOP_ERR_CUDA; break; }
                        if (t < tBest) { tBest = t; best[0] = kind; best[1] = sh[0]; best[2] = sh[1]; best[3] = ctas; }
                    }
            }
        }
        if (rc == TOP_OK) rc = set_l0_kernel(s, p, best[0], best[1], best[2], best[3]);
        if (msBest) msBest[p] = tBest;
        if (configs) for (int i = 0; i < 4; ++i) configs[4 * p + i] = best[i];
    }
    cudaEventDestroy(a); cudaEventDestroy(b);
    if (flush) cudaFree(flush);
    return rc;
}

// the operand / epilogue pairs of the solver's level-0 products
using VIdd = VecIn<double, double>;  using VIff = VecIn<float, float>;  using VIfd = VecIn<float, double>;
template void l0_op<double, VIdd, StoreOut<double, double>>(top_solver *, const VIdd &, const StoreOut<double, double> &, Reduce, const int *, int);
template void l0_op<double, VIdd, PostSmoothOut<double, double, double>>(top_solver *, const VIdd &, const PostSmoothOut<double, double, double> &, Reduce, const int *, int);
template void l0_op<double, VIdd, DotStoreOut<double, double, double>>(top_solver *, const VIdd &, const DotStoreOut<double, double, double> &, Reduce, const int *, int);
template void l0_op<double, VIdd, ResidOut<double, double, double>>(top_solver *, const VIdd &, const ResidOut<double, double, double> &, Reduce, const int *, int);
template void l0_op<float, VIff, ResidOut<float, double, float>>(top_solver *, const VIff &, const ResidOut<float, double, float> &, Reduce, const int *, int);
template void l0_op<float, VIff, PostSmoothOut<float, double, double>>(top_solver *, const VIff &, const PostSmoothOut<float, double, double> &, Reduce, const int *, int);
template void l0_op<float, VIff, PostSmoothOut<float, double, float>>(top_solver *, const VIff &, const PostSmoothOut<float, double, float> &, Reduce, const int *, int);
template void l0_op<float, VIfd, DotStoreOut<float, double, double>>(top_solver *, const VIfd &, const DotStoreOut<float, double, double> &, Reduce, const int *, int);
template void l0_op<float, VIfd, StoreOut<float, double>>(top_solver *, const VIfd &, const StoreOut<float, double> &, Reduce, const int *, int);
template void l0_op<float, VIfd, ResidOut<float, double, double>>(top_solver *, const VIfd &, const ResidOut<float, double, double> &, Reduce, const int *, int);
template void l0_op<float, VIff, StoreOut<float, float>>(top_solver *, const VIff &, const StoreOut<float, float> &, Reduce, const int *, int);
template void l0_op<float, VIff, StoreOut<float, double>>(top_solver *, const VIff &, const StoreOut<float, double> &, Reduce, const int *, int);
}  // namespace topgpu
