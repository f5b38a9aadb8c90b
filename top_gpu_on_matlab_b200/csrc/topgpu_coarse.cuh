// topgpu_coarse.cuh -- the coarse part of the V-cycle (every level below the
// finest) as one persistent cooperative kernel.
//
// Below level 0 the grids are small (cfg2: 62 K, 8 K, 1 K nodes and a 336-DOF
// coarsest), so their separate launches are dominated by launch and drain
// time.  This kernel runs the same steps, with the same per-node device code
// and the same summation order (identical results), as one launch: grid-wide
// barriers separate the steps
//   restriction leg, per level:  t = r - K (omega D^-1 r);  r_next = R t
//   coarsest:                    gather r;  t = A^-1 r
//   interpolation leg, per level: x = P t_next + omega D^-1 r;
//                                 t = x + omega D^-1 (r - K x)
// for every right-hand side of a batched solve.
#pragma once
#include <cooperative_groups.h>
#include "topgpu_grid.cuh"

namespace topgpu {

constexpr int kCoarseMaxLevels = 12;
constexpr int kCoarseThreads = kCoarseTileX * 8;

template <typename T> struct CoarseLv {
    Geom g;
    const T *Ks;             // packed Galerkin matrices (not used on the coarsest)
    T *r, *x, *t;            // level vectors, right-hand side k at k * 3 CS
    const T *invD;
    const uint8_t *flags;
};
template <typename T> struct CoarseVc {
    CoarseLv<T> L[kCoarseMaxLevels];   // levels 1 .. nL-1 of the solver; the last is the coarsest
    int n;                             // number of those levels
    T omega;
    const double *Ainv;                // coarsest dense inverse [nC x nC]
    double *cr;                        // coarsest right-hand sides [nv x nC]
    int64_t nC;
    const int32_t *nodeGridC;          // coarsest compact node -> grid slot
    int nv;                            // right-hand sides
};

template <typename T>
__global__ void __launch_bounds__(kCoarseThreads)
coarse_vcycle_kernel(const CoarseVc<T> A, const int *__restrict__ done0)
{
    namespace cgs = cooperative_groups;
    cgs::grid_group grid = cgs::this_grid();
    __shared__ T part[8][3][kCoarseTileX];
    __shared__ int offs[24 * 24];
    __shared__ double red[kCoarsestThreads / 32][4];
    static_assert(kCoarseThreads == kCoarsestThreads, "the coarsest rows use the whole CTA");
    const int tid = threadIdx.x, n = tid % kCoarseTileX, i = tid / kCoarseTileX;
    const int64_t nb = gridDim.x, b = blockIdx.x;
    auto vdone = [&](int vk) { const int *d = done_of(done0, vk); return d && *d; };
    const int NL = A.n;

    // restriction leg
    for (int l = 0; l + 1 < NL; ++l) {
        const CoarseLv<T> &lv = A.L[l], &lc = A.L[l + 1];
        const int64_t vs = 3 * lv.g.cs, vsc = 3 * lc.g.cs;
        coarse_offsets(offs, lv.g, tid, kCoarseThreads);
        __syncthreads();
        const dim3 tg = coarse_tile_grid(lv.g);
        const int64_t per = (int64_t)tg.x * tg.y;
        for (int64_t u = b; u < per * A.nv; u += nb) {
            const int vk = (int)(u / per);
            const int64_t w = u % per;
            if (vdone(vk)) continue;                              // uniform in the CTA
            const JacobiIn<T, T> in(lv.r + vk * vs, lv.invD, lv.g.cs, A.omega);
            const ResidOut<T, T, T> out(lv.r + vk * vs, lv.t + vk * vs, lv.g.cs);
            coarse_tile_unit<T>(in, out, lv.Ks, lv.g, (int)(w % tg.x), (int)(w / tg.x), n, i, part, offs);
        }
        grid.sync();
        const int64_t thr = (int64_t)lc.g.PY * lc.g.NX * lc.g.NZ * RestrictLanes<2>::value;
        const int64_t rper = (thr + kCoarseThreads - 1) / kCoarseThreads;
        for (int64_t u = b; u < rper * A.nv; u += nb) {
            const int vk = (int)(u / rper);
            const int64_t w = u % rper;
            if (vdone(vk)) continue;
            restrict_lanes<T, 2>(lv.t + vk * vs, lv.g, lc.r + vk * vsc, lc.g, lc.flags, w * kCoarseThreads + tid);
        }
        grid.sync();
    }
    // coarsest direct solve: gather the right-hand side, then one CTA per row of A^-1
    {
        const CoarseLv<T> &lc = A.L[NL - 1];
        const int64_t vsc = 3 * lc.g.cs, nC = A.nC;
        for (int64_t e = b * kCoarseThreads + tid; e < nC * A.nv; e += nb * kCoarseThreads) {
            const int vk = (int)(e / nC);
            const int64_t t = e % nC;
            if (vdone(vk)) continue;
            A.cr[vk * nC + t] = double(lc.r[vk * vsc + (t % 3) * lc.g.cs + A.nodeGridC[t / 3]]);
        }
        grid.sync();
        for (int64_t row = b; row < nC; row += nb)
            for (int v0 = 0; v0 < A.nv; v0 += 4) {
                bool act[4];
                bool any = false;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    act[q] = v0 + q < A.nv && !vdone(v0 + q);
                    any = any || act[q];
                }
                if (!any) continue;                               // uniform in the CTA
                double out[4];
                coarsest_row(A.Ainv + nC * row, CompactRhs{A.cr, nC}, nC, v0, act, red, out);
                if (tid == 0)
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (act[q]) lc.t[(v0 + q) * vsc + (row % 3) * lc.g.cs + A.nodeGridC[row / 3]] = T(out[q]);
            }
        grid.sync();
    }
    // interpolation leg
    for (int l = NL - 2; l >= 0; --l) {
        const CoarseLv<T> &lv = A.L[l], &lc = A.L[l + 1];
        const int64_t vs = 3 * lv.g.cs, vsc = 3 * lc.g.cs;
        const int64_t per = (int64_t)lv.g.PY * lv.g.NX, nodes = per * lv.g.NZ;
        for (int64_t e = b * kCoarseThreads + tid; e < nodes * A.nv; e += nb * kCoarseThreads) {
            const int vk = (int)(e / nodes);
            const int64_t w = e % nodes;
            if (vdone(vk)) continue;
            prolong_node<T, 2, T>(lc.t + vk * vsc, lc.g, lv.x + vk * vs, lv.g, lv.flags, lv.r + vk * vs, lv.invD,
                                  A.omega, (int)(w % per), (int)(w / per));
        }
        grid.sync();
        coarse_offsets(offs, lv.g, tid, kCoarseThreads);
        __syncthreads();
        const dim3 tg = coarse_tile_grid(lv.g);
        const int64_t pt = (int64_t)tg.x * tg.y;
        for (int64_t u = b; u < pt * A.nv; u += nb) {
            const int vk = (int)(u / pt);
            const int64_t w = u % pt;
            if (vdone(vk)) continue;
            const VecIn<T, T> in(lv.x + vk * vs, lv.g.cs);
            const PostSmoothOut<T, T, T> out(lv.x + vk * vs, lv.r + vk * vs, lv.invD, lv.t + vk * vs, lv.g.cs, A.omega);
            coarse_tile_unit<T>(in, out, lv.Ks, lv.g, (int)(w % tg.x), (int)(w / tg.x), n, i, part, offs);
        }
        if (l > 0) grid.sync();
    }
}

// CTAs of one cooperative launch: two per SM (fewer CTAs make the grid-wide
// barriers cheaper; level 1 still gives every CTA several tiles), within what
// fits on the GPU at once
template <typename T>
inline int coarse_vcycle_ctas(int numSMs)
{
    static const int occ = [] {
        int o = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, coarse_vcycle_kernel<T>, kCoarseThreads, 0) != cudaSuccess) o = 1;
        return o > 0 ? o : 1;
    }();
    return numSMs * (occ < 2 ? occ : 2);
}

}  // namespace topgpu
