// topgpu_l0.cu -- level-0 stiffness product dispatch of the fused solver:
// the node-centric kernel with the dense 24x24 Ke (topgpu_grid.cuh) or the
// Walsh-basis tile kernel (topgpu_walsh.cuh), per precision, with the
// operand/epilogue combinations the solver uses instantiated here.
#include <cuda_runtime.h>
#include <algorithm>
#include "topgpu_solver_impl.cuh"

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
    return (kind == 2 || kind == 4) ? walsh_pair_tiles(g, ty, tx) : walsh_tiles(g, ty, tx);
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
        coarse_tile_kernel<T, In, Out><<<gr, dim3(kCoarseTileX, 8), 0, s->st>>>(in, out, Kp, lv.g, red, done);
    } else if (k.kind == 1) {
#define TOPGPU_LAUNCH_SHAPE(A, B)                                                                             \
        if (k.ty == A && k.tx == B)                                                                           \
            l0w_kernel<T, A, B, In, Out><<<dim3(l0w_ctas<T, A, B, In, Out, 1>(s, k), K), A * B, 0, s->st>>>(  \
                walshparam<T>(s), in, out, egrid<T>(s), lv.flags, k.mask, lv.g, T(s->p.E0), red, done);
        TOPGPU_WALSH_SHAPES(TOPGPU_LAUNCH_SHAPE)
#undef TOPGPU_LAUNCH_SHAPE
    } else if (k.kind == 3) {
#define TOPGPU_LAUNCH_SHAPE(A, B)                                                                             \
        if (k.ty == A && k.tx == B)                                                                           \
            l0d_kernel<T, A, B, In, Out><<<dim3(l0w_ctas<T, A, B, In, Out, 3>(s, k), K), A * B, 0, s->st>>>(  \
                walshparam<T>(s), in, out, egrid<T>(s), lv.flags, k.mask, lv.g, T(s->p.E0), red, done);
        TOPGPU_WALSH_SHAPES(TOPGPU_LAUNCH_SHAPE)
#undef TOPGPU_LAUNCH_SHAPE
    } else if (k.kind == 4) {        // FP32 only, as kind 2
        if constexpr (sizeof(T) == 4) {
#define TOPGPU_LAUNCH_SHAPE(A, B)                                                                             \
            if (k.ty == A && k.tx == B)                                                                       \
                l0q_kernel<T, A, B, In, Out><<<dim3(l0w_ctas<T, A, B, In, Out, 4>(s, k), K), A * B, 0, s->st>>>( \
                    walshpair<T>(s), in, out, egrid<T>(s), lv.flags, k.mask, lv.g, T(s->p.E0), red, done);
            TOPGPU_WALSH_SHAPES(TOPGPU_LAUNCH_SHAPE)
#undef TOPGPU_LAUNCH_SHAPE
        }
    } else if (k.kind == 2) {        // FP32 only: the FP64 pair state does not fit in registers
        if constexpr (sizeof(T) == 4) {
#define TOPGPU_LAUNCH_SHAPE(A, B)                                                                             \
            if (k.ty == A && k.tx == B)                                                                       \
                l0p_kernel<T, A, B, In, Out><<<dim3(l0w_ctas<T, A, B, In, Out, 2>(s, k), K), A * B, 0, s->st>>>( \
                    walshpair<T>(s), in, out, egrid<T>(s), lv.flags, k.mask, lv.g, T(s->p.E0), red, done);
            TOPGPU_WALSH_SHAPES(TOPGPU_LAUNCH_SHAPE)
#undef TOPGPU_LAUNCH_SHAPE
        }
    } else {
        l0_kernel<T, In, Out><<<dim3((unsigned)lv.g.nbx, (unsigned)lv.g.NZ, K), kNodeThreads, 0, s->st>>>(
            keparam<T>(s), in, out, egrid<T>(s), lv.flags, lv.tileFixed, lv.g, T(s->p.E0), red, done);
    }
    TOPGPU_COUNT_LAUNCH();
}

int set_l0_kernel(top_solver *s, int p, int kind, int ty, int tx, int ctas)
{
    top_solver::L0Kernel &k = s->l0k[p];
    if (kind == 0) { k.kind = 0; ++s->opGen; return TOP_OK; }
    if ((kind != 1 && kind != 3 && !((kind == 2 || kind == 4) && p == 1)) || !s->walshOK || !walsh_shape_ok(ty, tx) || ctas < 0)
        return TOP_ERR_ARGS;
    DevLevel &l0 = s->L[0];
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
        else walsh_mask_kernel<A, B><<<tiles, 256, 0, s->st>>>(l0.flags, l0.g, k.mask);            \
    }
    TOPGPU_WALSH_SHAPES(TOPGPU_MASK_SHAPE)
#undef TOPGPU_MASK_SHAPE
    TOPGPU_COUNT_LAUNCH();
    if (cudaGetLastError() != cudaSuccess) return TOP_ERR_CUDA;
    k.kind = kind; k.ty = ty; k.tx = tx; k.ctas = ctas;
    ++s->opGen;
    return TOP_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: times every level-0 kernel configuration on this model (plain
// y = K u launches on the solver's stream, L2 flushed before each) and keeps
// the fastest per precision.
namespace {
double time_l0(top_solver *s, int p, int nrep, void *flush, size_t flushBytes, cudaEvent_t a, cudaEvent_t b)
{
    DevLevel &l0 = s->L[0];
    const Reduce none{nullptr, nullptr, nullptr};
    double total = 0.0;
    for (int k = 0; k < nrep + 1; ++k) {
        if (flush) cudaMemsetAsync(flush, k & 0xff, flushBytes, s->st);
        cudaEventRecord(a, s->st);
        if (p == 0) l0_op<double>(s, VecIn<double, double>{s->pv, l0.g.cs}, StoreOut<double, double>{s->v, l0.g.cs}, none, nullptr, 1);
        else l0_op<float>(s, VecIn<float, float>{l0.x32, l0.g.cs}, StoreOut<float, float>{l0.t32, l0.g.cs}, none, nullptr, 1);
        cudaEventRecord(b, s->st);
        if (cudaEventSynchronize(b) != cudaSuccess) return -1.0;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (k > 0) total += ms;              // the first launch warms up
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
    static const int mults[] = {4, 6, 8, 12, 16};
    int rc = TOP_OK;
    for (int p = 0; p < 2 && rc == TOP_OK; ++p) {
        int best[4] = {0, 16, 16, 0};
        rc = set_l0_kernel(s, p, 0, 16, 16, 0);
        double tBest = rc == TOP_OK ? time_l0(s, p, nrep, flush, (size_t)flushBytes, a, b) : -1.0;
        if (tBest < 0) { rc = TOP_ERR_CUDA; break; }
        if (s->walshOK) {
            for (int kind = 1; kind <= 4 && rc == TOP_OK; ++kind) {
                if ((kind == 2 || kind == 4) && p == 0) continue;
                for (const auto &sh : shapes)
                    for (int m : mults) {
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
}  // namespace topgpu
