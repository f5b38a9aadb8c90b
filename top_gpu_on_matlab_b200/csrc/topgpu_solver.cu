// topgpu_solver.cu -- fused device solver of libtopgpu.so (sm_100a).
//
// Replaces, for one voxel model resident in HBM, the reference's
// Solving_PCG / Solving_Vcycle / Solving_KbyU_MatrixFree /
// Solving_RestrictResidual / Solving_InterpolationDeviation /
// Solving_AssembleFEAstencil (TOP_GPU.m:602-878, 1033-1267).
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <type_traits>
#include <vector>
#include "topgpu_kernels.cuh"
#include "topgpu_solver_impl.cuh"
#include "topgpu_dense.cuh"
#include "topgpu_coarse.cuh"
#include "topgpu_dense.cuh"

namespace topgpu {
int assemble_level2_f64(double *Ks, const int32_t *upMap, const double *E, const double *K0,
                        const double *Pch, const int32_t *mapUnique, const double *uFree,
                        const double *uFixed, int64_t nElem, int nCh, int64_t nUnique,
                        double *Qscratch, int32_t *eyeScratch, cudaStream_t st,
                        const int32_t *bndList, int64_t nBnd);
int assemble_higher_f64(double *Ks, const int32_t *upMap, const double *KsPrev, const double *Psub,
                        int64_t nElem, int nSub, cudaStream_t st);



// ---------------------------------------------------------------------------
// small kernels
template <typename TI, typename TO>
__global__ void compact_to_grid_kernel(const TI *__restrict__ v, TO *__restrict__ g,
                                       const int32_t *__restrict__ nodeGrid, int64_t Nn, int64_t cs)
{
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Nn) return;
    const int64_t gi = nodeGrid[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) g[c * cs + gi] = TO(v[3 * n + c]);
}
template <typename TI, typename TO>
__global__ void grid_to_compact_kernel(const TI *__restrict__ g, TO *__restrict__ v,
                                       const int32_t *__restrict__ nodeGrid, int64_t Nn, int64_t cs)
{
    const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= Nn) return;
    const int64_t gi = nodeGrid[n];
#pragma unroll
    for (int c = 0; c < 3; ++c) v[3 * n + c] = TO(g[c * cs + gi]);
}
// E (compact, FP64) -> grid slots (FP64 + FP32); SIMP when x != nullptr
__global__ void modulus_kernel(const double *__restrict__ src, int simp, double E0, double Emin, double p,
                               double *__restrict__ Ec, double *__restrict__ Eg, float *__restrict__ Eg32,
                               const int32_t *__restrict__ eleGrid, int64_t Ne)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Ne) return;
    const double v = simp ? Emin + pow(src[e], p) * (E0 - Emin) : src[e];
    Ec[e] = v;
    Eg[eleGrid[e]] = v;
    Eg32[eleGrid[e]] = float(v);
}
// super-element mode: sub-voxel moduli (SIMP when simp != 0), [64 x Ne]
__global__ void modulus_super_kernel(const double *__restrict__ src, int simp, double E0, double Emin, double p,
                                     double *__restrict__ Esub, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) Esub[i] = simp ? Emin + pow(src[i], p) * (E0 - Emin) : src[i];
}
// K_mat(:, e) = I_mat * E_sub(:, e) (TOP_GPU.m:1101-1104); elements with fixed
// DOFs: sum_q Kfree(:, q, uid) E_sub(q, e) + Kfixed(:, uid) (TOP_GPU.m:723-734).
// One CTA per element, one thread per matrix entry.
__global__ void __launch_bounds__(576)
super_kmat_kernel(const double *__restrict__ Imat, const double *__restrict__ Esub, const int32_t *__restrict__ mapUnique,
                  const double *__restrict__ uFree, const double *__restrict__ uFixed, double *__restrict__ Kc)
{
    __shared__ double Ee[64];
    const int64_t e = blockIdx.x;
    const int t = threadIdx.x;
    if (t < 64) Ee[t] = Esub[e * 64 + t];
    __syncthreads();
    const int32_t u = mapUnique[e];
    const double *I = u > 0 ? uFree + (size_t)(u - 1) * 576 * 64 : Imat;
    double acc = 0;
#pragma unroll 8
    for (int q = 0; q < 64; ++q) acc = fma(I[(size_t)q * 576 + t], Ee[q], acc);
    if (u > 0) acc += uFixed[(size_t)(u - 1) * 576 + t];
    Kc[e * 576 + t] = acc;
}
// Level-0 Jacobi diagonal: sum_e E_e diag(Ke) on free components, E0 on
// fixed ones (the element matrices of TOP_GPU.m:1184-1188 summed per node).
__global__ void diag_l0_kernel(const KeParam<double> K, const double *__restrict__ E,
                               const uint8_t *__restrict__ flags, Geom g, double E0,
                               double *__restrict__ diag, double *__restrict__ inv64, float *__restrict__ inv32)
{
    const int q = blockIdx.x * kNodeThreads + threadIdx.x;
    const int Y = q % g.PY, X = q / g.PY, Z = blockIdx.y;
    if (Y >= g.NY || X >= g.NX) return;
    const int64_t idx = g.origin + Y + (int64_t)g.PY * X + g.plane * Z;
    const uint8_t f = flags[idx];
    for (int c = 0; c < 3; ++c) {
        double d = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) d += E[idx - cdy(i) - g.PY * cdx(i) - g.plane * cdz(i)] * K.k[(3 * i + c) * 25];
        if (f & (1 << c)) d = E0;
        const bool on = (f & kActive) && d != 0.0;
        diag[c * g.cs + idx] = d;
        inv64[c * g.cs + idx] = on ? 1.0 / d : 0.0;
        inv32[c * g.cs + idx] = on ? float(1.0 / d) : 0.0f;
    }
}
// Compact element Ks [576 x Ne] -> packed grid slots (FP64 + FP32), 8
// elements per block staged through shared memory (coalesced both ways)
constexpr int kPackE = 8;
__global__ void pack_ks_kernel(const double *__restrict__ KsC, const int32_t *__restrict__ eleGrid, int64_t Ne,
                               double *__restrict__ P64, float *__restrict__ P32, int64_t cs)
{
    __shared__ double sK[kPackE * 576];
    __shared__ int64_t sSlot[kPackE];
    const int64_t e0 = (int64_t)blockIdx.x * kPackE;
    const int ne = (int)((Ne - e0) < kPackE ? (Ne - e0) : kPackE);
    for (int t = threadIdx.x; t < ne * 576; t += blockDim.x) sK[t] = KsC[e0 * 576 + t];
    if (threadIdx.x < ne) sSlot[threadIdx.x] = eleGrid[e0 + threadIdx.x];
    __syncthreads();
    for (int t = threadIdx.x; t < 300 * kPackE; t += blockDim.x) {
        const int el = t % kPackE, p = t / kPackE;
        if (el >= ne) continue;
        int r = 0, base = 0;           // packed index p -> (r, k), r <= k
        while (base + (24 - r) <= p) { base += 24 - r; ++r; }
        const int k = r + (p - base);
        const double v = sK[el * 576 + r + 24 * k];
        P64[ks_off(p, sSlot[el])] = v;
        P32[ks_off(p, sSlot[el])] = float(v);
    }
}
__global__ void diag_coarse_kernel(const double *__restrict__ P64, Geom g, const uint8_t *__restrict__ flags,
                                   double *__restrict__ diag, double *__restrict__ inv64, float *__restrict__ inv32)
{
    const int q = blockIdx.x * kNodeThreads + threadIdx.x;
    const int Y = q % g.PY, X = q / g.PY, Z = blockIdx.y;
    if (Y >= g.NY || X >= g.NX) return;
    const int64_t idx = g.origin + Y + (int64_t)g.PY * X + g.plane * Z;
    for (int c = 0; c < 3; ++c) {
        double d = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) d += P64[ks_off(sym_pack(3 * i + c, 3 * i + c), idx - cdy(i) - g.PY * cdx(i) - g.plane * cdz(i))];
        const bool on = (flags[idx] & kActive) && d != 0.0;
        diag[c * g.cs + idx] = d;
        inv64[c * g.cs + idx] = on ? 1.0 / d : 0.0;
        inv32[c * g.cs + idx] = on ? float(1.0 / d) : 0.0f;
    }
}
// Dense coarsest (or condensed-tail level) matrix, one warp per row (compact
// node n, component c): lanes (j, d), j < 8, d < 3, add the incident element
// i's 24 entries of the row -- 24 different columns -- for i = 0..7 in turn,
// the warp synchronised between elements, so every entry receives its
// additions in the order of a one-thread-per-row loop over i, j, d
// (race-free, deterministic, the same sums).
__global__ void __launch_bounds__(256)
coarsest_assemble_kernel(const double *__restrict__ KsC, const int32_t *__restrict__ nodeGrid,
                         const int32_t *__restrict__ eleCompact, const int32_t *__restrict__ nodeCompact,
                         Geom g, int64_t Nn, double *__restrict__ A)
{
    const int64_t row = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= 3 * Nn) return;                   // whole warps
    const int64_t n = row / 3; const int c = int(row % 3);
    const int64_t nC = 3 * Nn;
    const int64_t idx = nodeGrid[n];
    const int j = lane / 3, d = lane % 3;
    for (int i = 0; i < 8; ++i) {
        const int64_t slot = idx - cdy(i) - g.PY * cdx(i) - g.plane * cdz(i);
        const int32_t e = eleCompact[slot];
        if (e < 0) continue;                     // uniform in the warp
        if (lane < 24) {
            const int32_t m = nodeCompact[slot + cdy(j) + g.PY * cdx(j) + g.plane * cdz(j)];
            A[row + nC * (3 * (int64_t)m + d)] += KsC[(int64_t)e * 576 + (3 * i + c) + 24 * (3 * j + d)];
        }
        __syncwarp();                            // element i's additions before element i + 1's
    }
}
// ---- coarsest level ----
// coarsest solve: x_grid = Ainv * r
// one CTA per row of A^-1, every right-hand side (up to four per pass over the
// row), read from the level's grid vector r in compact order
template <typename T>
__global__ void __launch_bounds__(kCoarsestThreads)
coarsest_gemv_kernel(const double *__restrict__ Ainv, const T *__restrict__ r, int64_t n,
                     T *__restrict__ x, Geom g, const int32_t *__restrict__ nodeGrid,
                     const int *__restrict__ done0, int64_t vs, int nv, int staged)
{
    // staged 1: the right-hand sides gathered from the grid into shared memory;
    // 2 (FP64): read from their compact copy r; 0: read from the grid per term
    pdl_enter();
    __shared__ double red[kCoarsestThreads / 32][4];
    extern __shared__ double rstage[];           // staged: the right-hand sides [4][n]
    const int64_t row = blockIdx.x;
    for (int v0 = 0; v0 < nv; v0 += 4) {
        bool act[4];
        bool any = false;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int *d = done_of(done0, v0 + q);
            act[q] = v0 + q < nv && !(d && *d);
            any = any || act[q];
        }
        if (!any) continue;                      // uniform in the CTA
        double out[4];
        if (staged == 1) {
            // the right-hand sides into shared memory first (all the node-map
            // loads of a thread, then all its value loads), then the same sums
            __syncthreads();                     // the previous group's reads are done
            for (int64_t j0 = threadIdx.x; j0 < n; j0 += (int64_t)kCoarsestThreads * 4) {
                int32_t slot[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int64_t j = j0 + (int64_t)kCoarsestThreads * u;
                    slot[u] = j < n ? nodeGrid[j / 3] : 0;
                }
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int64_t j = j0 + (int64_t)kCoarsestThreads * u;
                    if (j >= n) break;
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        if (act[q]) rstage[q * n + j] = double(r[(v0 + q) * vs + (j % 3) * g.cs + slot[u]]);
                }
            }
            __syncthreads();
            coarsest_row(Ainv + n * row, StagedRhs{rstage, n, v0}, n, v0, act, red, out);
        } else if (staged == 2) {
            // FP64: r is the compact copy the restriction wrote ([k][n], the same values)
            if constexpr (sizeof(T) == 8)
                coarsest_row(Ainv + n * row, CompactRhs{reinterpret_cast<const double *>(r), n}, n, v0, act, red, out);
        } else {
            coarsest_row(Ainv + n * row, GridRhs<T>{r, vs, g.cs, nodeGrid}, n, v0, act, red, out);
        }
        if (threadIdx.x == 0)
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (act[q]) x[(v0 + q) * vs + (row % 3) * g.cs + nodeGrid[row / 3]] = T(out[q]);
    }
}

// ---- the V-cycle's condensed tail: t = M r on one level's active DOFs ----
// M (symmetric) by rows at stride ld (a multiple of four, zero beyond n), in
// the V-cycle's precision T; r in compact order (DOF 3 node + component, zero
// beyond n, right-hand side k at rc + k ld), written by the restriction into
// the level.  One warp per row, kTailRows rows per CTA; each lane reads its
// row and r in 16-byte pieces (r, 8 KB per right-hand side, from L1 after the
// first warp), PB pieces of each in flight, the first batch of M issued before
// the stopping flags are read, and sums in FP64; the lanes combine in a fixed
// shuffle tree.  The result goes to the level's grid vector.
constexpr int kTailRows = 8, kTailThreads = 32 * kTailRows;
__device__ __forceinline__ double tail_piece(const float4 &v, int e) { return double(e == 0 ? v.x : e == 1 ? v.y : e == 2 ? v.z : v.w); }
__device__ __forceinline__ double tail_piece(const double2 &v, int e) { return e == 0 ? v.x : v.y; }
template <typename T, int NQ>
__global__ void __launch_bounds__(kTailThreads)
tail_gemv_kernel(const T *__restrict__ M, int64_t ld, const T *__restrict__ rc, int64_t n, T *__restrict__ x, Geom g,
                 const int32_t *__restrict__ nodeGrid, const int *__restrict__ done0, int64_t vs, int nv)
{
    pdl_enter();
    using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    constexpr int W = 16 / (int)sizeof(T);       // values per piece
    constexpr int PB = NQ == 1 ? 8 : 4;          // pieces of M per lane in flight
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t row = (int64_t)blockIdx.x * kTailRows + warp;
    if (row >= n) return;                        // no barriers below
    const int64_t nw = ld / W;
    const V *Mr = reinterpret_cast<const V *>(M + row * ld);
    V p[PB];
#pragma unroll
    for (int u = 0; u < PB; ++u) {
        const int64_t b = lane + 32 * u;
        if (b < nw) p[u] = __ldg(Mr + b);
    }
    const int64_t out = (row % 3) * g.cs + nodeGrid[row / 3];
    bool first = true;                           // p holds the row's first pieces
    for (int v0 = 0; v0 < nv; v0 += NQ) {
        bool act[NQ];
        bool any = false;
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            const int *d = done_of(done0, v0 + q);
            act[q] = v0 + q < nv && !(d && *d);
            any = any || act[q];
        }
        if (!any) continue;
        double acc[NQ];
#pragma unroll
        for (int q = 0; q < NQ; ++q) acc[q] = 0.0;
        for (int64_t b0 = lane; b0 < nw; b0 += 32 * PB) {
            if (!first || b0 != lane) {
#pragma unroll
                for (int u = 0; u < PB; ++u) {
                    const int64_t b = b0 + 32 * u;
                    if (b < nw) p[u] = __ldg(Mr + b);
                }
            }
            V rv[NQ][PB];
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const V *R = reinterpret_cast<const V *>(rc + (int64_t)(act[q] ? v0 + q : v0) * ld);
#pragma unroll
                for (int u = 0; u < PB; ++u) {
                    const int64_t b = b0 + 32 * u;
                    if (b < nw) rv[q][u] = __ldg(R + b);
                }
            }
#pragma unroll
            for (int u = 0; u < PB; ++u) {
                const int64_t b = b0 + 32 * u;
                if (b >= nw) break;
#pragma unroll
                for (int e = 0; e < W; ++e) {
                    const double mv = tail_piece(p[u], e);
#pragma unroll
                    for (int q = 0; q < NQ; ++q) acc[q] = fma(mv, tail_piece(rv[q][u], e), acc[q]);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NQ; ++q)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        if (lane == 0)
#pragma unroll
            for (int q = 0; q < NQ; ++q)
                if (act[q]) x[(v0 + q) * vs + out] = T(acc[q]);
        first = false;
    }
}

// ---- PCG vector kernels (FP64, level-0 grid arrays) ----
// PCG vector kernels run over whole grid vectors, margins and guard slots
// included (all zero), as one contiguous range of n = 3 CS values
// r -= lambda v, r.r, and the V-cycle's level-0 Jacobi pre-smoothing iterate
// z1 = omega*invD.*r in the V-cycle's precision T (stored in the level-0 x
// vector the V-cycle prolongs into).  x += lambda p is left to the p kernel,
// which reads p anyway (pcg_check records lambda and that it is pending).
// The CTA that completes rr = r . r then runs the iteration's check
// (TOP_GPU.m:630-649) for its right-hand side, in the same launch.
__device__ __forceinline__ void pcg_check_one(PcgState *st)
{
    st->lam = st->rho / st->pv;          // the update's lambda; x += lam p is pending
    st->xPend = 1;
    st->its += 1;
    const double res = sqrt(st->rr) / st->normB;
    st->resnorm = res;
    if (!isfinite(res) || !isfinite(st->rho) || !isfinite(st->pv)) { st->status = TOP_ERR_NAN; st->done = 1; return; }
    if (res < st->tol) { st->done = 1; return; }
    if (st->its >= st->maxIT) { st->status = TOP_ERR_NOT_CONVERGED; st->done = 1; return; }
    st->rhoOld = st->rho;
}
template <typename T>
__global__ void pcg_update_kernel(double *__restrict__ r, const double *__restrict__ v, int64_t n, PcgState *st, Reduce red0,
                                  T *__restrict__ z1, const T *__restrict__ invD, T omega)
{
    pdl_enter();
    const int vk = blockIdx.y;           // right-hand side; vectors at stride n
    st += vk;
    if (st->done) {                      // stopped: nothing pending for the p kernel
        if (blockIdx.x == 0 && threadIdx.x == 0) st->xPend = 0;
        return;
    }
    r += vk * n; v += vk * n;
    z1 += vk * n;
    const Reduce red = red0.at(vk);
    const double lambda = st->rho / st->pv;
    double rr = 0;
    // two consecutive values per access (n and the vector bases are multiples
    // of four values, 16-byte aligned)
    const int64_t n2 = n >> 1, S = (int64_t)gridDim.x * blockDim.x;
    // four grid strides per pass, every load issued before the first store (r
    // is read and written, so the compiler cannot move the next pass's loads
    // up); each thread still adds its rr terms in index order
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n2; j += 4 * S) {
        double ra[4], rb[4], va[4], vb[4];
        T da[4], db[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (j + q * S < n2) {
                ld2(r + 2 * (j + q * S), ra[q], rb[q]);
                ld2(v + 2 * (j + q * S), va[q], vb[q]);
                ld2(invD + 2 * (j + q * S), da[q], db[q]);
            }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (j + q * S < n2) {
                const double a = ra[q] - lambda * va[q], b = rb[q] - lambda * vb[q];
                st2(r + 2 * (j + q * S), a, b);
                st2(z1 + 2 * (j + q * S), T(omega * da[q] * T(a)), T(omega * db[q] * T(b)));
                rr += a * a;
                rr += b * b;
            }
    }
    if (block_sum_last<256>(rr, red.partials, red.counter, red.result, gridDim.x, blockIdx.x)) {
        __threadfence();
        pcg_check_one(st);
    }
}
// z1 = omega*invD.*r on whole grid vectors (n = 3 CS values per right-hand
// side; r at stride vsR, z1 at stride n; invD shared)
template <typename T, typename TR>
__global__ void jacobi_base_kernel(const TR *__restrict__ r, const T *__restrict__ invD, T *__restrict__ z1, T omega,
                                   int64_t n, int64_t vsR, const int *__restrict__ done0)
{
    pdl_enter();
    const int vk = blockIdx.y;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    r += vk * vsR; z1 += vk * n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        z1[i] = omega * invD[i] * T(r[i]);
}
// p = z + beta p (first: p = z), and the pending x += lambda p of the last
// update with the old p (also for a right-hand side that has just stopped).
// beta = rho / rhoOld (the reference's), or with flex the flexible
// (Polak-Ribiere) beta = -sigma / pv, sigma = z . A p_old, pv = p_old . A p_old
template <typename TZ>
__global__ void pcg_p_kernel(double *__restrict__ p, const TZ *__restrict__ z, int64_t n, const PcgState *st, int first,
                             double *__restrict__ x, int flex)
{
    pdl_enter();
    const int vk = blockIdx.y;
    st += vk;
    const bool xp = !first && st->xPend;
    const bool upd = first || !st->done;
    if (!xp && !upd) return;
    p += vk * n; z += vk * n; x += vk * n;
    const double beta = first ? 0.0 : (flex ? -st->sigma / st->pv : st->rho / st->rhoOld);
    const double lam = st->lam;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double po = p[i];
        if (xp) x[i] += lam * po;
        if (upd) p[i] = double(z[i]) + beta * po;
    }
}
// sigma = z . v of every right-hand side that is still iterating (flexible beta)
template <typename TZ>
__global__ void zv_dot_kernel(const TZ *__restrict__ z, const double *__restrict__ v, int64_t n, Reduce red0,
                              const int *__restrict__ done0)
{
    pdl_enter();
    const int vk = blockIdx.y;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    z += vk * n; v += vk * n;
    const Reduce red = red0.at(vk);
    double s = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += double(z[i]) * v[i];
    block_sum_to<256>(s, red.partials, red.counter, red.result, gridDim.x, blockIdx.x);
}
__global__ void dot_kernel(const double *__restrict__ a, const double *__restrict__ b, int64_t n, Reduce red0)
{
    const int vk = blockIdx.y;
    a += vk * n; b += vk * n;
    const Reduce red = red0.at(vk);
    double s = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += a[i] * b[i];
    block_sum_to<256>(s, red.partials, red.counter, red.result, gridDim.x, blockIdx.x);
}
// element energies sum_k w_k u_k' Ke u_k (TOP_GPU.m:580-600) on grid vectors
__global__ void compliance_kernel(const KeParam<double> K, const double *__restrict__ U, int64_t ustride,
                                  int nLoads, const double *__restrict__ w, const int32_t *__restrict__ eleGrid,
                                  int64_t Ne, Geom g, double *__restrict__ ce)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Ne) return;
    const int64_t slot = eleGrid[e];
    double acc = 0;
    for (int k = 0; k < nLoads; ++k) {
        const double *u = U + k * ustride;
        double ue[24];
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
            for (int c = 0; c < 3; ++c) ue[3 * j + c] = u[c * g.cs + slot + cdy(j) + g.PY * cdx(j) + g.plane * cdz(j)];
        double s = 0;
#pragma unroll
        for (int a = 0; a < 24; ++a) {
            double t = 0;
#pragma unroll
            for (int b = 0; b < 24; ++b) t = fma(K.k[a + 24 * b], ue[b], t);
            s = fma(t, ue[a], s);
        }
        acc += s * w[k];
    }
    ce[e] = acc;
}
// super-element mode: ce_e = sum_k w_k u_ke' K_mat_e u_ke (TOP_GPU.m:2622-2645)
__global__ void compliance_kmat_kernel(const double *__restrict__ Kc, const double *__restrict__ U, int64_t ustride,
                                       int nLoads, const double *__restrict__ w, const int32_t *__restrict__ eleGrid,
                                       int64_t Ne, Geom g, double *__restrict__ ce)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Ne) return;
    const int64_t slot = eleGrid[e];
    const double *K = Kc + e * 576;
    double acc = 0;
    for (int k = 0; k < nLoads; ++k) {
        const double *u = U + k * ustride;
        double ue[24];
#pragma unroll
        for (int j = 0; j < 8; ++j)
#pragma unroll
            for (int c = 0; c < 3; ++c) ue[3 * j + c] = u[c * g.cs + slot + cdy(j) + g.PY * cdx(j) + g.plane * cdz(j)];
        double s = 0;
        for (int a = 0; a < 24; ++a) {
            double t = 0;
#pragma unroll
            for (int b = 0; b < 24; ++b) t = fma(K[a + 24 * b], ue[b], t);
            s = fma(t, ue[a], s);
        }
        acc += s * w[k];
    }
    ce[e] = acc;
}

}  // namespace topgpu

using namespace topgpu;

// the V-cycle's condensed tail (defined with the coarsest solve below)
bool tail_on(const top_solver *s);
int build_tail(top_solver *s, cudaStream_t st);

// dynamic shared memory of a GEMV that stages its right-hand sides (up to
// four groups of n FP64 values, at most 96 KB), 0 beyond: those read them
// from the grid
template <typename T>
size_t gemv_stage_bytes(int64_t n, int nv)
{
    constexpr size_t kMax = 96 * 1024;
    static const bool attr = cudaFuncSetAttribute(coarsest_gemv_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMax) == cudaSuccess;
    const size_t b = sizeof(double) * (size_t)(nv < 4 ? nv : 4) * (size_t)n;
    return (attr && b <= kMax) ? b : 0;
}

namespace {

inline dim3 node_grid(const Geom &g) { return dim3((unsigned)g.nbx, (unsigned)g.NZ); }
inline int vec_blocks(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 4096); }

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e__ = (call);                                                                \
        if (e__ != cudaSuccess) { set_error("top_solver: CUDA error %d: %s", (int)e__, cudaGetErrorString(e__)); return TOP_ERR_CUDA; } \
    } while (0)
#define CKL() CK(cudaGetLastError())

Geom make_geom(int ny, int nx, int nz)
{
    Geom g{};
    g.NY = ny + 1; g.NX = nx + 1; g.NZ = nz + 1;
    g.PY = (g.NY + 1 + 3) / 4 * 4;
    const int64_t PX = g.NX + 2, PZ = g.NZ + 2;
    g.plane = (int64_t)g.PY * PX;
    const int64_t ng = g.plane * PZ;
    g.cs = ng + 2 * kMargin;
    g.origin = g.PY + g.plane;   // (Y=0, X'=1, Z'=1)
    g.nbx = (int)(((int64_t)g.PY * g.NX + kNodeThreads - 1) / kNodeThreads);
    return g;
}
inline int64_t gidx(const Geom &g, int Y, int X, int Z) { return g.origin + Y + (int64_t)g.PY * X + g.plane * Z; }

// the device error flag of the two-pass coarse product (a tile copy wait that
// gave up): read, cleared, reported
int op_err_status(top_solver *s)
{
    int e = 0;
    CK(cudaMemcpyAsync(&e, s->opErr, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (e) {
        CK(cudaMemsetAsync(s->opErr, 0, sizeof(int), s->st));
        set_error("coarse product: a packed-matrix tile copy did not complete");
        return TOP_ERR_CUDA;
    }
    return TOP_OK;
}

// ---- level operators ------------------------------------------------------
template <typename T> const T *ks_packed(const DevLevel &l);
template <> const double *ks_packed<double>(const DevLevel &l) { return l.KsP64; }
template <> const float *ks_packed<float>(const DevLevel &l) { return l.KsP32; }
template <typename T> const T *invd(const DevLevel &l);
template <> const double *invd<double>(const DevLevel &l) { return l.invD64; }
template <> const float *invd<float>(const DevLevel &l) { return l.invD32; }
template <typename T> T *vr(DevLevel &l);
template <> double *vr<double>(DevLevel &l) { return l.r64; }
template <> float *vr<float>(DevLevel &l) { return l.r32; }
template <typename T> T *vx(DevLevel &l);
template <> double *vx<double>(DevLevel &l) { return l.x64; }
template <> float *vx<float>(DevLevel &l) { return l.x32; }
template <typename T> T *vt(DevLevel &l);
template <> double *vt<double>(DevLevel &l) { return l.t64; }
template <> float *vt<float>(DevLevel &l) { return l.t32; }

template <typename T> T *wbuf(DevLevel &l);
template <> double *wbuf<double>(DevLevel &l) { return l.W64; }
template <> float *wbuf<float>(DevLevel &l) { return l.W32; }
// resident CTAs per SM of the two-pass product's first pass (its dynamic
// shared memory allowance set once; 0 when that fails)
template <typename T, class In>
int coarse_elem_occ()
{
    static const int occ = [] {
        int n = 0;
        if (cudaFuncSetAttribute(coarse_elem_kernel<T, In>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CoarseElem<T>::kSmem) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, coarse_elem_kernel<T, In>, kElemThreads, CoarseElem<T>::kSmem) != cudaSuccess) {
            (void)cudaGetLastError();
            n = 0;
        }
        return n;
    }();
    return occ;
}
// the first-pass kernels of the V-cycle's coarse products and the coarsest
// GEMV, configured before any launch is captured into a graph
void coarse_elem_setup()
{
    (void)coarse_elem_occ<float, JacobiIn<float, float>>();
    (void)coarse_elem_occ<float, VecIn<float, float>>();
    (void)coarse_elem_occ<double, JacobiIn<double, double>>();
    (void)coarse_elem_occ<double, VecIn<double, double>>();
    (void)gemv_stage_bytes<float>(1, 1);
    (void)gemv_stage_bytes<double>(1, 1);
}

// y-epilogue applied to (K_level in)(node) for every node of a coarse level;
// nv right-hand sides in one launch (vectors at the functors' strides)
template <typename T, class In, class Out>
void coarse_op(top_solver *s, int l, const In &in, const Out &out, Reduce red, const int *done, int nv = 1)
{
    DevLevel &lv = s->L[l];
    int t0 = 0, nt = 0;
    coarse_elem_tiles(lv.g, t0, nt);
    T *W = wbuf<T>(lv);
    if (s->coarseLanes) {
        launch_k(s, coarse_kernel<T, In, Out>, dim3(coarse_blocks(lv.g), (unsigned)nv), kNodeThreads, 0, s->st, in, out, ks_packed<T>(lv), lv.g, red, done);
    } else if (W && s->opErr && nt > 0 && nt >= s->coarseTwoPassMin && coarse_elem_occ<T, In>() > 0) {
        const int64_t wvs = w_alloc_vals(lv.g.cs);
        const unsigned ctas = (unsigned)std::min<int64_t>(nt, (int64_t)s->numSMs * coarse_elem_occ<T, In>());
        launch_k(s, coarse_elem_kernel<T, In>, dim3(ctas, (unsigned)nv), kElemThreads, CoarseElem<T>::kSmem, s->st,
                 in, ks_packed<T>(lv), W, wvs, lv.g, t0, nt, done, s->opErr, s->withholdTile ? 1 : 0);
        s->withholdTile = false;
        TOPGPU_COUNT_LAUNCH();
        launch_k(s, coarse_gather_kernel<T, Out>, dim3((unsigned)lv.g.nbx, (unsigned)lv.g.NZ, (unsigned)nv), kNodeThreads, 0, s->st,
                 out, W, wvs, lv.g, red, done);
    } else {
        dim3 gr = coarse_tile_grid(lv.g); gr.z = (unsigned)nv;
        launch_k(s, coarse_tile_kernel<T, In, Out>, gr, dim3(kCoarseTileX, 8), 0, s->st, in, out, ks_packed<T>(lv), lv.g, red, done);
    }
    TOPGPU_COUNT_LAUNCH();
}
template <typename T> T *rscratch(top_solver *s);
template <> double *rscratch<double>(top_solver *s) { return s->rscr64; }
template <> float *rscratch<float>(top_solver *s) { return s->rscr32; }
// level vectors (r, x, t of each level) hold kMax right-hand sides at stride 3 CS
inline int64_t lvs(const DevLevel &l) { return 3 * l.g.cs; }
// restriction of the level-l residual d onto level l+1 (TOP_GPU.m:817-847);
// d and rc at the level vector strides
template <typename T>
void restrict_op(top_solver *s, int l, const T *d, T *rc, const int *done, int nv = 1, T *cmp = nullptr,
                 const int32_t *slotCmp = nullptr, int64_t vsCmp = 0)
{
    DevLevel &lv = s->L[l], &lc = s->L[l + 1];
    const unsigned K = (unsigned)nv;
    if (lc.span == 4) {
        const int NYc = lc.g.NY, NXf = lv.g.NX, NXc = lc.g.NX, NZf = lv.g.NZ;
        const int64_t nt = (int64_t)NYc * NXf * NZf;
        const int64_t vsS = 3 * nt;                 // scratch per right-hand side
        T *t1 = rscratch<T>(s);
        const dim3 gy((unsigned)((nt + 255) / 256), K);
        if (s->vec4 && vec4_ok(lv.g, {d}, {lvs(lv)}))
            launch_k(s, restrict_y_kernel<T, 4, true>, gy, 256, 0, s->st, d, lv.g, t1, NYc, done, lvs(lv), vsS);
        else
            launch_k(s, restrict_y_kernel<T, 4>, gy, 256, 0, s->st, d, lv.g, t1, NYc, done, lvs(lv), vsS);
        TOPGPU_COUNT_LAUNCH();
        launch_k(s, restrict_xz_kernel<T, 4>, dim3((unsigned)(NXc * lc.g.NZ), (unsigned)((NYc + 31) / 32), K), 32 * 7, 0, s->st,
                 t1, NXf, NZf, rc, lc.g, lc.flags, done, vsS, lvs(lc), cmp, slotCmp, vsCmp);
    } else {
        launch_k(s, restrict_kernel<T, 2>, dim3(restrict_blocks<2>(lc.g), K), kNodeThreads, 0, s->st, d, lv.g, rc, lc.g, lc.flags, done,
                                                                                           lvs(lv), lvs(lc), cmp, slotCmp, vsCmp);
    }
    TOPGPU_COUNT_LAUNCH();
}
// ... of any level (level 0: the configured level-0 kernel, topgpu_l0.cu)
template <typename T, class In, class Out>
void level_op(top_solver *s, int l, const In &in, const Out &out, Reduce red, const int *done)
{
    if (l == 0) l0_op<T>(s, in, out, red, done);
    else coarse_op<T>(s, l, in, out, red, done);
}

// first level of the V-cycle run by the persistent coarse kernel (0: none):
// levels p .. nL-1 when the solver was told so (p = 1 or 2), there are at
// least two of them and every transfer among them is span 2
int coarse_persistent_level(const top_solver *s)
{
    const int p = s->coarsePersistent;
    if (p < 1 || s->nL - p < 2 || s->nL - p > kCoarseMaxLevels) return 0;
    for (int l = p + 1; l < s->nL; ++l)
        if (s->L[l].span != 2) return 0;
    return p;
}

// V-cycle 'Standard' (TOP_GPU.m:766-816) in precision T on the level-0
// residuals r0 (type TR, grid layout, nv right-hand sides at stride vs0);
// writes z0 (type TZ, same stride) and, when zr is set, z0 . r0 into zr
// (per right-hand side: consecutive PcgState's when nv > 1).
// The level-0 Jacobi iterate z1 = omega*invD.*r0 is stored in the level-0 x
// vector first (by this function, or already by the PCG update when
// z1Ready): the first product reads it once per node instead of converting
// r0 and recomputing z1 at every corner load, and the prolongation adds onto
// it.
template <typename T, typename TR, typename TZ>
void vcycle(top_solver *s, const TR *r0, TZ *z0, double *zr, const int *done, int nv = 1, int64_t vs0 = 0,
            bool z1Ready = false)
{
    const int nL = s->nL;
    const T omega = T(s->p.omega);
    const Reduce none{nullptr, nullptr, nullptr};
    const unsigned K = (unsigned)nv;
    // levels pl .. nL-1 as one persistent kernel where their transfers are span 2
    const int pl = coarse_persistent_level(s);
    const bool persist = pl > 0;
    // levels tl .. nL-1 as the condensed tail's one GEMV (0: none); M is held
    // in the precision of the solver's V-cycle
    const bool tailT = sizeof(T) == (s->p.precision == TOP_PREC_MIXED ? 4u : 8u);
    const int tl = (!persist && tailT && s->tailReady && tail_on(s)) ? s->tailL : 0;
    // FP64 coarsest GEMV reading the compact copy of its right-hand sides
    const bool cmpC = sizeof(T) == 8 && !persist && !tl && nv <= s->kMax;
    if (!z1Ready) {
        DevLevel &l0 = s->L[0];
        const int64_t n0 = lvs(l0), M = kMargin;
        launch_k(s, jacobi_base_kernel<T, TR>, dim3((unsigned)vec_blocks(n0), K), 256, 0, s->st, r0 - M, invd<T>(l0) - M, vx<T>(l0) - M,
                                                                                      omega, n0, vs0, done);
        TOPGPU_COUNT_LAUNCH();
    }
    // restriction leg
    for (int l = 0; l < (persist ? pl : (tl ? tl : nL - 1)); ++l) {
        DevLevel &lv = s->L[l], &lc = s->L[l + 1];
        T *d = vt<T>(lv);
        const int64_t vs = lvs(lv);
        if (l == 0)
            l0_op<T>(s, VecIn<T, T>{vx<T>(lv), lv.g.cs, vs}, ResidOut<T, TR, T>{r0, d, lv.g.cs, vs0, vs}, none, done, nv);
        else
            coarse_op<T>(s, l, JacobiIn<T, T>{vr<T>(lv), invd<T>(lv), lv.g.cs, omega, vs}, ResidOut<T, T, T>{vr<T>(lv), d, lv.g.cs, vs},
                         none, done, nv);
        // into the tail's level: r also in compact order, the GEMV's operand;
        // likewise (FP64) into the coarsest level for its GEMV
        if (tl && l + 1 == tl)
            restrict_op<T>(s, l, d, vr<T>(lc), done, nv, static_cast<T *>(s->tailR), s->tailNodeCompact[0], s->tailLd);
        else if (cmpC && l + 1 == nL - 1)
            restrict_op<T>(s, l, d, vr<T>(lc), done, nv, reinterpret_cast<T *>(s->cr), s->nodeCompactC, s->nC);
        else
            restrict_op<T>(s, l, d, vr<T>(lc), done, nv);
    }
    DevLevel &lc = s->L[nL - 1];
    const int64_t n = 3 * lc.Nn;
    if (tl) {
        // t = M r on level tl: the V-cycle of levels tl .. nL-1 in one operator
        DevLevel &lt = s->L[tl];
        const int64_t nt = 3 * lt.Nn;
        const unsigned gt = (unsigned)((nt + kTailRows - 1) / kTailRows);
        if (nv == 1)
            launch_k(s, tail_gemv_kernel<T, 1>, gt, kTailThreads, 0, s->st,
                     (const T *)s->tailMp, s->tailLd, (const T *)s->tailR, nt, vt<T>(lt), lt.g, lt.nodeGrid, done, lvs(lt), nv);
        else
            launch_k(s, tail_gemv_kernel<T, 4>, gt, kTailThreads, 0, s->st,
                     (const T *)s->tailMp, s->tailLd, (const T *)s->tailR, nt, vt<T>(lt), lt.g, lt.nodeGrid, done, lvs(lt), nv);
        TOPGPU_COUNT_LAUNCH();
    } else if (persist) {
        CoarseVc<T> A{};
        A.n = nL - pl;
        for (int l = pl; l < nL; ++l) {
            DevLevel &d = s->L[l];
            A.L[l - pl] = CoarseLv<T>{d.g, l < nL - 1 ? ks_packed<T>(d) : nullptr, vr<T>(d), vx<T>(d), vt<T>(d), invd<T>(d), d.flags};
        }
        A.omega = omega; A.Ainv = s->Ainv; A.cr = s->cr; A.nC = n; A.nodeGridC = lc.nodeGrid; A.nv = nv;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cudaLaunchConfig_t cfg{};
        // from level 2 down the grids are small: one CTA per SM keeps the grid-wide barriers cheap
        cfg.gridDim = dim3((unsigned)(pl >= 2 ? s->numSMs : coarse_vcycle_ctas<T>(s->numSMs)));
        cfg.blockDim = dim3(kCoarseThreads);
        cfg.stream = s->st;
        cfg.attrs = attr; cfg.numAttrs = 1;
        cudaLaunchKernelEx(&cfg, coarse_vcycle_kernel<T>, A, done);
        TOPGPU_COUNT_LAUNCH();
    } else {
        // coarsest direct solve, FP64 (the right-hand side read from the grid by the product)
        const size_t sm = cmpC ? 0 : gemv_stage_bytes<T>(n, nv);
        launch_k(s, coarsest_gemv_kernel<T>, (unsigned)n, kCoarsestThreads, sm, s->st, s->Ainv,
                 cmpC ? reinterpret_cast<const T *>(s->cr) : (const T *)vr<T>(lc), n, vt<T>(lc), lc.g,
                 lc.nodeGrid, done, lvs(lc), nv, cmpC ? 2 : (sm ? 1 : 0));
        TOPGPU_COUNT_LAUNCH();
    }
    // interpolation leg
    for (int l = (persist ? pl - 1 : (tl ? tl - 1 : nL - 2)); l >= 0; --l) {
        DevLevel &lv = s->L[l], &lcn = s->L[l + 1];
        const T *xc = vt<T>(lcn);
        T *x = vx<T>(lv);
        const int64_t vs = lvs(lv), vsc = lvs(lcn);
        dim3 gr = node_grid(lv.g); gr.z = K;
        if (l == 0) {   // x = z1 + P t_c (x holds z1)
            const dim3 g4((unsigned)(((int64_t)((lv.g.NY + 3) / 4) * lv.g.NX * lv.g.NZ + kNodeThreads - 1) / kNodeThreads), K);
            if (lcn.span == 4 && s->vec4 && vec4_ok(lv.g, {x, lv.flags}, {vs}))
                launch_k(s, prolong4_kernel<T, TR, true, true>, g4, kNodeThreads, 0, s->st, xc, lcn.g, x, lv.g, lv.flags, nullptr, nullptr, omega, done, vsc, vs, 0);
            else if (lcn.span == 4)
                launch_k(s, prolong4_kernel<T, TR, true>, g4, kNodeThreads, 0, s->st, xc, lcn.g, x, lv.g, lv.flags, nullptr, nullptr, omega, done, vsc, vs, 0);
            else
                launch_k(s, prolong_kernel<T, 2, TR, true>, gr, kNodeThreads, 0, s->st, xc, lcn.g, x, lv.g, lv.flags, nullptr, nullptr, omega, done, vsc, vs, 0);
            TOPGPU_COUNT_LAUNCH();
            const Reduce rz = zr ? (nv > 1 ? s->redk(zr) : s->red(zr)) : none;
            l0_op<T>(s, VecIn<T, T>{x, lv.g.cs, vs}, PostSmoothOut<T, TR, TZ>{x, r0, invd<T>(lv), z0, lv.g.cs, omega, vs0}, rz, done, nv);
        } else {
            const dim3 g4((unsigned)(((int64_t)((lv.g.NY + 3) / 4) * lv.g.NX * lv.g.NZ + kNodeThreads - 1) / kNodeThreads), K);
            if (lcn.span == 4 && s->vec4 && vec4_ok(lv.g, {x, lv.flags, vr<T>(lv), invd<T>(lv)}, {vs}))
                launch_k(s, prolong4_kernel<T, T, false, true>, g4, kNodeThreads, 0, s->st, xc, lcn.g, x, lv.g, lv.flags, vr<T>(lv), invd<T>(lv), omega, done, vsc, vs, vs);
            else if (lcn.span == 4)
                launch_k(s, prolong4_kernel<T, T, false>, g4, kNodeThreads, 0, s->st, xc, lcn.g, x, lv.g, lv.flags, vr<T>(lv), invd<T>(lv), omega, done, vsc, vs, vs);
            else
                launch_k(s, prolong_kernel<T, 2, T>, gr, kNodeThreads, 0, s->st, xc, lcn.g, x, lv.g, lv.flags, vr<T>(lv), invd<T>(lv), omega, done, vsc, vs, vs);
            TOPGPU_COUNT_LAUNCH();
            coarse_op<T>(s, l, VecIn<T, T>{x, lv.g.cs, vs}, PostSmoothOut<T, T, T>{x, vr<T>(lv), invd<T>(lv), vt<T>(lv), lv.g.cs, omega, vs},
                         none, done, nv);
        }
    }
}

void precond(top_solver *s, const double *r0, double *z0, double *zr, const int *done)
{
    if (s->p.precision == TOP_PREC_MIXED) vcycle<float, double, double>(s, r0, z0, zr, done);
    else vcycle<double, double, double>(s, r0, z0, zr, done);
}

// outer operator v = K0 u on FP64 grid vectors (nv right-hand sides at
// stride vs), u.v into uy.  FP64 unless outerFP32 (the reference's mixed mode
// runs it in single, TOP_GPU.m:683-684).
void outer_op(top_solver *s, const double *u, double *y, double *uy, const int *done, int nv = 1, int64_t vs = 0)
{
    DevLevel &l0 = s->L[0];
    const Reduce red = uy ? (nv > 1 ? s->redk(uy) : s->red(uy)) : Reduce{nullptr, nullptr, nullptr};
    if (s->p.outerFP32)
        l0_op<float>(s, VecIn<float, double>{u, l0.g.cs, vs}, DotStoreOut<float, double, double>{y, u, l0.g.cs, vs}, red, done, nv);
    else
        l0_op<double>(s, VecIn<double, double>{u, l0.g.cs, vs}, DotStoreOut<double, double, double>{y, u, l0.g.cs, vs}, red, done, nv);
}

}  // namespace

// ===========================================================================
extern "C" int top_solver_create(const top_mesh *mesh, const top_solver_params *p, top_solver **out)
{
    if (!mesh || !p || !out) { set_error("top_solver_create: bad arguments"); return TOP_ERR_ARGS; }
    if (!mesh->hasBC) { set_error("top_solver_create: apply boundary conditions first"); return TOP_ERR_STATE; }
    if (p->precision != TOP_PREC_FP64 && p->precision != TOP_PREC_MIXED) { set_error("top_solver_create: bad precision"); return TOP_ERR_ARGS; }
    top_solver *s = new (std::nothrow) top_solver();
    if (!s) return TOP_ERR_NOMEM;
    s->p = *p;
    s->nL = (int)mesh->L.size();
    s->nLoads = mesh->nLoads;
    s->kMax = std::max(1, s->nLoads);   // load cases solve as one batched PCG
    s->L.resize(s->nL);
    auto fail = [&](const char *what) { set_error("top_solver_create: %s", what); top_solver_destroy(s); return TOP_ERR_NOMEM; };
    for (int l = 0; l < s->nL; ++l) {
        const MeshLevel &M = mesh->L[l];
        DevLevel &d = s->L[l];
        d.ny = M.resY; d.nx = M.resX; d.nz = M.resZ; d.span = M.span;
        d.g = make_geom(d.ny, d.nx, d.nz);
        d.Ne = M.Ne; d.Nn = M.Nn; d.ng = d.g.cs - 2 * kMargin;
        const int64_t cs = d.g.cs;
        // 32-bit in-array indices: the vectors of all right-hand sides (batched
        // launches index vector k at k * 3 CS) and the packed coarse matrices
        if ((int64_t)s->kMax * 3 * cs >= (int64_t(1) << 31) - 1 || ((l > 0 || mesh->superElement) && ks_alloc_vals(cs) >= (int64_t(1) << 31))) {
            set_error("top_solver_create: level %d grid too large for 32-bit in-array indices", l); top_solver_destroy(s); return TOP_ERR_SHAPE;
        }
        // host-side flags, node and element maps
        std::vector<uint8_t> fl(cs, 0);
        std::vector<int32_t> ng(M.Nn), eg(M.Ne);
        {   // nodes of this level in its own grid numbering: invert nodMapForward
            const int NY = d.ny + 1, NX = d.nx + 1;
            for (int64_t t = 0; t < (int64_t)M.nodMapForward.size(); ++t) {
                const int32_t c = M.nodMapForward[t];
                if (!c) continue;
                const int Y = int(t % NY), X = int((t / NY) % NX), Z = int(t / ((int64_t)NY * NX));
                const int64_t gi = gidx(d.g, Y, X, Z);
                ng[c - 1] = (int32_t)gi;
                fl[gi + kMargin] = kActive | (l == 0 ? mesh->nodeFixed[c - 1] : 0);
            }
            for (int64_t e = 0; e < M.Ne; ++e) {
                const int64_t gE = M.eleMapBack[e] - 1;
                const int ey = int(gE % d.ny), ex = int((gE / d.ny) % d.nx), ez = int(gE / ((int64_t)d.ny * d.nx));
                eg[e] = (int32_t)gidx(d.g, ey, ex, ez);
            }
        }
        d.flags = s->dalloc<uint8_t>(cs);
        d.nodeGrid = s->dalloc<int32_t>(M.Nn);
        d.eleGrid = s->dalloc<int32_t>(M.Ne);
        if (!d.flags || !d.nodeGrid || !d.eleGrid) return fail("out of device memory");
        cudaMemcpy(d.flags, fl.data(), cs, cudaMemcpyHostToDevice);
        d.flags += kMargin;
        cudaMemcpy(d.nodeGrid, ng.data(), sizeof(int32_t) * M.Nn, cudaMemcpyHostToDevice);
        cudaMemcpy(d.eleGrid, eg.data(), sizeof(int32_t) * M.Ne, cudaMemcpyHostToDevice);
        d.diag = s->galloc<double>(cs, 3);
        d.invD64 = s->galloc<double>(cs, 3);
        d.invD32 = s->galloc<float>(cs, 3);
        const int KM = s->kMax;       // V-cycle vectors of every right-hand side
        d.x64 = s->galloc<double>(cs, 3 * KM); d.t64 = s->galloc<double>(cs, 3 * KM);
        d.x32 = s->galloc<float>(cs, 3 * KM); d.t32 = s->galloc<float>(cs, 3 * KM);
        if (l > 0) {
            d.r64 = s->galloc<double>(cs, 3 * KM); d.r32 = s->galloc<float>(cs, 3 * KM);
            const int nch = M.span * M.span * M.span;
            d.upMap = s->dalloc<int32_t>((size_t)M.Ne * nch);
            d.KsC = s->dalloc<double>((size_t)M.Ne * 576);
            if (!d.upMap || !d.KsC) return fail("out of device memory");
            cudaMemcpy(d.upMap, M.elementUpwardMap.data(), sizeof(int32_t) * M.Ne * nch, cudaMemcpyHostToDevice);
            if (l < s->nL - 1) {
                d.KsP64 = s->ksalloc<double>(cs);
                d.KsP32 = s->ksalloc<float>(cs);
                d.W64 = s->walloc<double>(cs, KM);
                d.W32 = s->walloc<float>(cs, KM);
                if (!d.KsP64 || !d.KsP32 || !d.W64 || !d.W32) return fail("out of device memory");
            }
        }
        if (!d.diag || !d.invD64 || !d.invD32 || !d.x64 || !d.t64 || !d.x32 || !d.t32) return fail("out of device memory");
        if (l == 0) {
            // blocks whose stencil touches a fixed node take the masked path
            std::vector<uint8_t> tf((size_t)d.g.nbx * d.g.NZ, 0);
            const int NY = d.ny + 1, NX = d.nx + 1, NZ = d.nz + 1;
            for (int64_t n = 0; n < M.Nn; ++n) {
                if (!mesh->nodeFixed[n]) continue;
                const int64_t t = M.nodMapBack[n] - 1;
                const int Y = int(t % NY), X = int((t / NY) % NX), Z = int(t / ((int64_t)NY * NX));
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dx = -1; dx <= 1; ++dx)
                        for (int dy = -1; dy <= 1; ++dy) {
                            const int y = Y + dy, x = X + dx, z = Z + dz;
                            if (y < 0 || y >= NY || x < 0 || x >= NX || z < 0 || z >= NZ) continue;
                            const int64_t qq = y + (int64_t)d.g.PY * x;
                            tf[(size_t)(qq / kNodeThreads) + (size_t)d.g.nbx * z] = 1;
                        }
            }
            d.tileFixed = s->dalloc<uint8_t>(tf.size());
            if (!d.tileFixed) return fail("out of device memory");
            cudaMemcpy(d.tileFixed, tf.data(), tf.size(), cudaMemcpyHostToDevice);
        }
    }
    // scratch of the separable span-4 restriction (y-folded fine field)
    {
        int64_t nt = 1;
        for (int l = 0; l + 1 < s->nL; ++l)
            if (s->L[l + 1].span == 4)
                nt = std::max<int64_t>(nt, (int64_t)s->L[l + 1].g.NY * s->L[l].g.NX * s->L[l].g.NZ);
        s->rscr64 = s->dalloc<double>((size_t)3 * nt * s->kMax);
        s->rscr32 = s->dalloc<float>((size_t)3 * nt * s->kMax);
        if (!s->rscr64 || !s->rscr32) return fail("out of device memory");
    }
    // level-0 data
    DevLevel &l0 = s->L[0];
    const MeshLevel &M0 = mesh->L[0];
    for (int t = 0; t < 576; ++t) { s->Ke64.k[t] = M0.Ke[t]; s->Ke32.k[t] = float(M0.Ke[t]); }
    s->walshOK = walsh_blocks(M0.Ke, s->W64) < 1e-12;
    for (int t = 0; t < 8; ++t)
        for (int k = 0; k < 9; ++k) {
            const double b = s->W64.b[t][k];
            s->W32.b[t][k] = float(b);
            s->WP64.b[t][k] = make_double2(b, b);
            s->WP32.b[t][k] = make_float2(float(b), float(b));
        }
    s->KeDev = s->dalloc<double>(576);
    s->Ec = s->dalloc<double>(M0.Ne);
    s->Eg64 = s->galloc<double>(l0.g.cs, 1);
    s->Eg32 = s->galloc<float>(l0.g.cs, 1);
    s->nU = (int64_t)mesh->eleWithFixedDOFs.size();
    s->super = mesh->superElement != 0;
    s->nely = mesh->nely; s->nelx = mesh->nelx; s->nelz = mesh->nelz;
    const int slices = s->super ? 64 : 1;
    s->mapUnique = s->dalloc<int32_t>(M0.Ne);
    s->uFree = s->dalloc<double>((size_t)576 * slices * s->nU);
    if (s->super) {
        s->Esub = s->dalloc<double>((size_t)64 * M0.Ne);
        s->stage = s->dalloc<double>((size_t)64 * M0.Ne);
        s->Imat = s->dalloc<double>((size_t)576 * 64);
        l0.KsC = s->dalloc<double>((size_t)M0.Ne * 576);
        l0.KsP64 = s->ksalloc<double>(l0.g.cs);
        l0.KsP32 = s->ksalloc<float>(l0.g.cs);
        if (!s->Esub || !s->stage || !s->Imat || !l0.KsC || !l0.KsP64 || !l0.KsP32) return fail("out of device memory");
        cudaMemcpy(s->Imat, mesh->I_mat.data(), sizeof(double) * 576 * 64, cudaMemcpyHostToDevice);
    }
    s->uFixed = s->dalloc<double>((size_t)576 * s->nU);
    s->P4 = s->dalloc<double>((size_t)576 * 64);
    s->P2 = s->dalloc<double>((size_t)576 * 8);
    s->Qs = s->dalloc<double>((size_t)576 * 64);
    s->eye = s->dalloc<int32_t>(64 * 64 + 4);
    if (!s->KeDev || !s->Ec || !s->Eg64 || !s->Eg32 || !s->mapUnique || !s->uFree || !s->uFixed || !s->P4 || !s->P2 || !s->Qs || !s->eye)
        return fail("out of device memory");
    cudaMemcpy(s->KeDev, M0.Ke, sizeof(double) * 576, cudaMemcpyHostToDevice);
    if (s->nL > 1) {   // coarse level-1 cells that own a child with fixed DOFs
        const MeshLevel &M1 = mesh->L[1];
        std::vector<int32_t> bl;
        for (int64_t e = 0; e < M1.Ne; ++e)
            for (int c = 0; c < 64; ++c) {
                const int32_t f = M1.elementUpwardMap[e + M1.Ne * c];
                if (f > 0 && mesh->mapUniqueKes[f - 1] > 0) { bl.push_back(int32_t(e)); break; }
            }
        s->nBnd = (int64_t)bl.size();
        if (s->nBnd) {
            s->bndList = s->dalloc<int32_t>(bl.size());
            if (!s->bndList) return fail("out of device memory");
            cudaMemcpy(s->bndList, bl.data(), sizeof(int32_t) * bl.size(), cudaMemcpyHostToDevice);
        }
    }
    cudaMemcpy(s->mapUnique, mesh->mapUniqueKes.data(), sizeof(int32_t) * M0.Ne, cudaMemcpyHostToDevice);
    cudaMemcpy(s->uFree, mesh->uniqueKesFree.data(), sizeof(double) * 576 * slices * s->nU, cudaMemcpyHostToDevice);
    {
        std::vector<double> fx(mesh->uniqueKesFixed);
        for (auto &v : fx) v *= p->E0;     // uniqueKesFixed_ * modulus_ (TOP_GPU.m:1614)
        cudaMemcpy(s->uFixed, fx.data(), sizeof(double) * 576 * s->nU, cudaMemcpyHostToDevice);
    }
    {
        std::vector<double> P((size_t)576 * 64);
        for (int q = 0; q < 64; ++q) child_prolongation(4, q, &P[(size_t)576 * q]);
        cudaMemcpy(s->P4, P.data(), sizeof(double) * 576 * 64, cudaMemcpyHostToDevice);
        for (int q = 0; q < 8; ++q) child_prolongation(2, q, &P[(size_t)576 * q]);
        cudaMemcpy(s->P2, P.data(), sizeof(double) * 576 * 8, cudaMemcpyHostToDevice);
    }
    // PCG vectors
    const int64_t cs0 = l0.g.cs;
    const int KM = s->kMax;           // PCG vectors of every right-hand side
    s->x = s->galloc<double>(cs0, 3 * KM); s->r = s->galloc<double>(cs0, 3 * KM); s->z = s->galloc<double>(cs0, 3 * KM);
    s->z32 = s->galloc<float>(cs0, 3 * KM);
    s->pv = s->galloc<double>(cs0, 3 * KM); s->v = s->galloc<double>(cs0, 3 * KM); s->tmp = s->galloc<double>(cs0, 3 * KM);
    s->b = s->galloc<double>(cs0, 3 * std::max(1, s->nLoads));
    s->weights = s->dalloc<double>(std::max(1, s->nLoads));
    if (!s->x || !s->r || !s->z || !s->z32 || !s->pv || !s->v || !s->tmp || !s->b || !s->weights) return fail("out of device memory");
    cudaMemcpy(s->weights, mesh->weights.data(), sizeof(double) * s->nLoads, cudaMemcpyHostToDevice);
    s->nd0 = 3 * M0.Nn;
    {
        double *Fd = s->dalloc<double>((size_t)s->nd0 * s->nLoads);
        if (!Fd) return fail("out of device memory");
        cudaMemcpy(Fd, mesh->F.data(), sizeof(double) * s->nd0 * s->nLoads, cudaMemcpyHostToDevice);
        for (int k = 0; k < s->nLoads; ++k)
        {
            compact_to_grid_kernel<double, double><<<nb256(M0.Nn), 256>>>(Fd + (size_t)k * s->nd0, s->b + (size_t)k * 3 * cs0, l0.nodeGrid, M0.Nn, cs0);
            TOPGPU_COUNT_LAUNCH();
        }
    }
    // reduction scratch
    // one partial per CTA of every reducing launch: node grids, coarse tiles,
    // per-element kernels (256 elements per CTA)
    int64_t maxBlocks = 4096;
    for (auto &d : s->L) {
        maxBlocks = std::max<int64_t>(maxBlocks, (int64_t)d.g.nbx * d.g.NZ);
        maxBlocks = std::max<int64_t>(maxBlocks, (int64_t)coarse_tile_grid(d.g).x * coarse_tile_grid(d.g).y);
        maxBlocks = std::max<int64_t>(maxBlocks, (d.Ne + 255) / 256 + 1);
    }
    s->nPartials = maxBlocks;
    s->partials = s->dalloc<double>(maxBlocks * s->kMax);
    s->counter = s->dalloc<unsigned>(4 + s->kMax);
    s->scal = s->dalloc<double>(16);
    s->zeroDone = s->dalloc<int>(4);
    s->opErr = s->dalloc<int>(1);
    s->state = s->dalloc<PcgState>(s->kMax);
    if (cudaMallocHost(&s->hstate, sizeof(PcgState) * s->kMax) != cudaSuccess) s->hstate = nullptr;
    if (!s->partials || !s->counter || !s->scal || !s->zeroDone || !s->opErr || !s->state || !s->hstate) return fail("out of memory");
    // coarsest level maps
    {
        DevLevel &lc = s->L[s->nL - 1];
        const MeshLevel &MC = mesh->L[s->nL - 1];
        s->nC = 3 * MC.Nn;
        if (s->nC > 16384) {
            set_error("top_solver_create: coarsest level has %lld DOFs (> 16384); lower coarsestResolutionControl", (long long)s->nC);
            top_solver_destroy(s);
            return TOP_ERR_SHAPE;
        }
        std::vector<int32_t> ec(lc.g.cs, -1), nc(lc.g.cs, -1);
        const int NY = lc.ny + 1, NX = lc.nx + 1;
        for (int64_t t = 0; t < (int64_t)MC.nodMapForward.size(); ++t) {
            const int32_t c = MC.nodMapForward[t];
            if (!c) continue;
            const int Y = int(t % NY), X = int((t / NY) % NX), Z = int(t / ((int64_t)NY * NX));
            nc[gidx(lc.g, Y, X, Z) + kMargin] = c - 1;
        }
        for (int64_t e = 0; e < MC.Ne; ++e) {
            const int64_t gE = MC.eleMapBack[e] - 1;
            const int ey = int(gE % lc.ny), ex = int((gE / lc.ny) % lc.nx), ez = int(gE / ((int64_t)lc.ny * lc.nx));
            ec[gidx(lc.g, ey, ex, ez) + kMargin] = (int32_t)e;
        }
        s->eleCompactC = s->dalloc<int32_t>(lc.g.cs);
        s->nodeCompactC = s->dalloc<int32_t>(lc.g.cs);
        s->Ac = s->dalloc<double>((size_t)s->nC * s->nC);
        s->Ainv = s->dalloc<double>((size_t)s->nC * s->nC);
        s->Wc = s->dalloc<double>((size_t)s->nC * s->nC);
        s->Dc = s->dalloc<double>((size_t)((s->nC + kDb - 1) / kDb) * kDb * kDb);
        s->cr = s->dalloc<double>((size_t)s->nC * s->kMax);
        if (!s->eleCompactC || !s->nodeCompactC || !s->Ac || !s->Ainv || !s->Wc || !s->Dc || !s->cr) return fail("out of device memory");
        cudaMemcpy(s->eleCompactC, ec.data(), sizeof(int32_t) * lc.g.cs, cudaMemcpyHostToDevice);
        cudaMemcpy(s->nodeCompactC, nc.data(), sizeof(int32_t) * lc.g.cs, cudaMemcpyHostToDevice);
        s->eleCompactC += kMargin; s->nodeCompactC += kMargin;
    }
    // the V-cycle's condensed tail: the highest level l >= 1 above the coarsest
    // with at most kTailMaxDofs active DOFs (every level below it is smaller)
    if (std::getenv("TOPGPU_NO_TAIL_OPERATOR")) s->tailMode = 0;
    for (int l = 1; l <= s->nL - 2 && !s->tailL && !s->super; ++l)
        if (3 * mesh->L[l].Nn <= top_solver::kTailMaxDofs) s->tailL = l;
    if (s->tailL) {
        for (int l = s->tailL; l <= s->nL - 2; ++l) {
            const MeshLevel &Mf = mesh->L[l], &Mc = mesh->L[l + 1];
            DevLevel &d = s->L[l];
            const int NYf = d.ny + 1, NXf = d.nx + 1, NZf = d.nz + 1;
            // grid slot -> compact node and element (as for the coarsest level)
            std::vector<int32_t> ecl(d.g.cs, -1), ncl(d.g.cs, -1), nbr((size_t)Mf.Nn * 27, -1);
            for (int64_t t = 0; t < (int64_t)Mf.nodMapForward.size(); ++t) {
                const int32_t c = Mf.nodMapForward[t];
                if (!c) continue;
                const int Y = int(t % NYf), X = int((t / NYf) % NXf), Z = int(t / ((int64_t)NYf * NXf));
                ncl[gidx(d.g, Y, X, Z) + kMargin] = c - 1;
                // the nodes that share an element with it (K's nonzero blocks of the row)
                int q = 0;
                for (int dz = -1; dz <= 1; ++dz)
                    for (int dx = -1; dx <= 1; ++dx)
                        for (int dy = -1; dy <= 1; ++dy, ++q) {
                            const int y = Y + dy, x = X + dx, z = Z + dz;
                            if (y < 0 || y >= NYf || x < 0 || x >= NXf || z < 0 || z >= NZf) continue;
                            const int32_t cn = Mf.nodMapForward[y + (int64_t)NYf * x + (int64_t)NYf * NXf * z];
                            if (cn) nbr[(size_t)(c - 1) * 27 + q] = cn - 1;
                        }
            }
            for (int64_t e = 0; e < Mf.Ne; ++e) {
                const int64_t gE = Mf.eleMapBack[e] - 1;
                const int ey = int(gE % d.ny), ex = int((gE / d.ny) % d.nx), ez = int(gE / ((int64_t)d.ny * d.nx));
                ecl[gidx(d.g, ey, ex, ez) + kMargin] = (int32_t)e;
            }
            // the prolongation from level l+1 on the active DOFs (DOF 3 node + c):
            // the trilinear weights the V-cycle's prolongation applies per component,
            // stored transposed (row k of P contiguous)
            const int S = s->L[l + 1].span, NYc = s->L[l + 1].ny + 1, NXc = s->L[l + 1].nx + 1;
            const int64_t nf = 3 * Mf.Nn, nco = 3 * Mc.Nn;
            std::vector<double> Pt((size_t)(nf * nco), 0.0);
            for (int64_t t = 0; t < (int64_t)Mf.nodMapForward.size(); ++t) {
                const int32_t cf = Mf.nodMapForward[t];
                if (!cf) continue;
                const int Y = int(t % NYf), X = int((t / NYf) % NXf), Z = int(t / ((int64_t)NYf * NXf));
                const int qy = Y / S, ry = Y - qy * S, qx = X / S, rx = X - qx * S, qz = Z / S, rz = Z - qz * S;
                const double wy[2] = {double(S - ry) / S, double(ry) / S};
                const double wx[2] = {double(S - rx) / S, double(rx) / S};
                const double wz[2] = {double(S - rz) / S, double(rz) / S};
                for (int bz = 0; bz < 2; ++bz) {
                    if (bz && rz == 0) continue;
                    for (int bx = 0; bx < 2; ++bx) {
                        if (bx && rx == 0) continue;
                        for (int by = 0; by < 2; ++by) {
                            if (by && ry == 0) continue;
                            const int32_t cc = Mc.nodMapForward[(qy + by) + (int64_t)NYc * (qx + bx) + (int64_t)NYc * NXc * (qz + bz)];
                            if (!cc) continue;
                            const double w = wz[bz] * wx[bx] * wy[by];
                            for (int c = 0; c < 3; ++c) Pt[(size_t)((3 * (cc - 1) + c) + nco * (3 * (cf - 1) + c))] = w;
                        }
                    }
                }
            }
            int32_t *ne = s->dalloc<int32_t>(d.g.cs), *nn = s->dalloc<int32_t>(d.g.cs), *nb = s->dalloc<int32_t>(nbr.size());
            double *Pd = s->dalloc<double>(Pt.size()), *Md = s->dalloc<double>((size_t)(nf * nf));
            if (!ne || !nn || !nb || !Pd || !Md) return fail("out of device memory");
            cudaMemcpy(ne, ecl.data(), sizeof(int32_t) * d.g.cs, cudaMemcpyHostToDevice);
            cudaMemcpy(nn, ncl.data(), sizeof(int32_t) * d.g.cs, cudaMemcpyHostToDevice);
            cudaMemcpy(nb, nbr.data(), sizeof(int32_t) * nbr.size(), cudaMemcpyHostToDevice);
            cudaMemcpy(Pd, Pt.data(), sizeof(double) * Pt.size(), cudaMemcpyHostToDevice);
            s->tailEleCompact.push_back(ne + kMargin);
            s->tailNodeCompact.push_back(nn + kMargin);
            s->tailNbr.push_back(nb);
            s->tailPt.push_back(Pd);
            s->tailMs.push_back(Md);
        }
        // scratch sized by the top tail level (the largest n and m)
        const int64_t n = 3 * mesh->L[s->tailL].Nn, m = 3 * mesh->L[s->tailL + 1].Nn;
        s->tailLd = (n + 3) / 4 * 4;
        s->tailK = s->dalloc<double>((size_t)(n * n));
        s->tailQ = s->dalloc<double>((size_t)(n * m));
        s->tailT = s->dalloc<double>((size_t)(n * m));
        s->tailJ = s->dalloc<double>((size_t)n);
        if (s->p.precision == TOP_PREC_MIXED) {
            s->tailMp = s->dalloc<float>((size_t)(n * s->tailLd));
            s->tailR = s->dalloc<float>((size_t)(s->tailLd * s->kMax));
        } else {
            s->tailMp = s->dalloc<double>((size_t)(n * s->tailLd));
            s->tailR = s->dalloc<double>((size_t)(s->tailLd * s->kMax));
        }
        if (!s->tailK || !s->tailQ || !s->tailT || !s->tailJ || !s->tailMp || !s->tailR) return fail("out of device memory");
    }
    {
        int dev = 0, nsm = 0;
        if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && nsm > 0)
            s->numSMs = nsm;
    }
    coarse_elem_setup();
    // level-0 products in the Walsh basis where Ke allows it (voxel mode)
    if (s->super) s->walshOK = false;
    if (s->walshOK)
        for (int pslot = 0; pslot < 2; ++pslot)
            if (set_l0_kernel(s, pslot, 3, 16, 8, (pslot ? 16 : 12) * s->numSMs) != TOP_OK) return fail("level-0 kernel setup");
    cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) { set_error("top_solver_create: %s", cudaGetErrorString(err)); top_solver_destroy(s); return TOP_ERR_CUDA; }
    *out = s;
    return TOP_OK;
}

extern "C" int top_solver_destroy(top_solver *s)
{
    if (!s) return TOP_OK;
    free_opt_state(s);
    for (auto &G : s->graphs) if (G.exec) cudaGraphExecDestroy(G.exec);
    if (s->capStream) cudaStreamDestroy(s->capStream);
    if (s->capIn) cudaEventDestroy(s->capIn);
    if (s->capOut) cudaEventDestroy(s->capOut);
    for (auto &k : s->l0k) if (k.mask) cudaFree(k.mask);
    if (s->l0kFallback.mask) cudaFree(s->l0kFallback.mask);
    for (void *p : s->allocs) cudaFree(p);
    if (s->hstate) cudaFreeHost(s->hstate);
    delete s;
    return TOP_OK;
}

extern "C" int top_solver_set_l0_kernel(top_solver *s, int fp32, int kind, int ty, int tx, int ctas)
{
    if (!s) return TOP_ERR_ARGS;
    return set_l0_kernel(s, fp32 ? 1 : 0, kind, ty, tx, ctas);
}

extern "C" int top_solver_autotune(top_solver *s, int nrep, int64_t flushBytes, double *msBest2, int *configs8)
{
    if (!s) return TOP_ERR_ARGS;
    const int rc = autotune_l0(s, nrep, flushBytes, msBest2, configs8);
    if (rc != TOP_OK) set_error("top_solver_autotune: failed (%d)", rc);
    return rc;
}

extern "C" int top_solver_set_coarse_persistent(top_solver *s, int on)
{
    if (!s || on < 0 || on > 2) return TOP_ERR_ARGS;
    s->coarsePersistent = on;
    ++s->opGen;                      // captured PCG graphs change
    return TOP_OK;
}

extern "C" int top_solver_set_tail_operator(top_solver *s, int on, int *level)
{
    if (!s || on < -1 || on > 1) { set_error("top_solver_set_tail_operator: bad arguments"); return TOP_ERR_ARGS; }
    s->tailMode = on;
    s->tailReady = false;
    ++s->opGen;                      // captured PCG graphs change
    int rc = TOP_OK;
    if (tail_on(s) && s->assembled) {
        rc = build_tail(s, s->st);
        if (rc == TOP_OK && cudaStreamSynchronize(s->st) != cudaSuccess) { set_error("top_solver_set_tail_operator: CUDA error"); rc = TOP_ERR_CUDA; }
    }
    if (level) *level = tail_on(s) ? s->tailL : 0;
    return rc;
}

extern "C" int top_solver_set_pcg_beta(top_solver *s, int flexible)
{
    if (!s) return TOP_ERR_ARGS;
    s->flexible = flexible != 0;
    ++s->opGen;                      // captured PCG graphs change
    return TOP_OK;
}

extern "C" int top_solver_test_withhold_tile(top_solver *s)
{
    if (!s) return TOP_ERR_ARGS;
    s->withholdTile = true;
    return TOP_OK;
}

extern "C" int top_solver_set_graphs(top_solver *s, int on)
{
    if (!s) return TOP_ERR_ARGS;
    s->useGraphs = on != 0;
    return TOP_OK;
}

extern "C" int top_solver_get_l0_kernel(const top_solver *s, int fp32, int *out4)
{
    if (!s || !out4) return TOP_ERR_ARGS;
    const top_solver::L0Kernel &k = s->l0k[fp32 ? 1 : 0];
    out4[0] = k.kind; out4[1] = k.ty; out4[2] = k.tx; out4[3] = k.ctas;
    return TOP_OK;
}

extern "C" int top_solver_set_stream(top_solver *s, void *stream)
{
    if (!s) return TOP_ERR_ARGS;
    s->st = reinterpret_cast<cudaStream_t>(stream);
    return TOP_OK;
}

extern "C" int top_solver_sizes(const top_solver *s, int64_t *out3)
{
    if (!s || !out3) return TOP_ERR_ARGS;
    out3[0] = s->nL; out3[1] = s->nLoads; out3[2] = s->nd0;
    return TOP_OK;
}

int topgpu::set_modulus_dev(top_solver *s, const double *src, int where, int simp)
{
    if (!s || !src) return TOP_ERR_ARGS;
    const int64_t Ne = s->L[0].Ne;
    const double *d = src;
    if (s->super) {      // [64 x Ne] sub-voxel values
        if (where == 0) {
            CK(cudaMemcpyAsync(s->stage, src, sizeof(double) * 64 * Ne, cudaMemcpyHostToDevice, s->st));
            d = s->stage;
        }
        modulus_super_kernel<<<nb256(64 * Ne), 256, 0, s->st>>>(d, simp, s->p.E0, s->p.Emin, s->p.penal, s->Esub, 64 * Ne);
        TOPGPU_COUNT_LAUNCH();
        CKL();
        s->assembled = false;
        return TOP_OK;
    }
    if (where == 0) {
        CK(cudaMemcpyAsync(s->tmp, src, sizeof(double) * Ne, cudaMemcpyHostToDevice, s->st));
        d = s->tmp;
    }
    modulus_kernel<<<nb256(Ne), 256, 0, s->st>>>(d, simp, s->p.E0, s->p.Emin, s->p.penal, s->Ec, s->Eg64, s->Eg32, s->L[0].eleGrid, Ne);
    TOPGPU_COUNT_LAUNCH();
    CKL();
    s->assembled = false;
    return TOP_OK;
}
extern "C" int top_solver_set_modulus(top_solver *s, const double *E, int where) { return set_modulus_dev(s, E, where, 0); }
extern "C" int top_solver_set_density(top_solver *s, const double *x, int where) { return set_modulus_dev(s, x, where, 1); }

// Cholesky factor and explicit inverse of the coarsest matrix s->Ac (n x n,
// column-major): L over Ac's lower triangle, W = L^-1 in s->Wc, A^-1 in
// s->Ainv (which also serves as the product scratch of the inversion);
// a non-positive pivot sets s->zeroDone[1]
namespace {
void dgemm(cudaStream_t st, bool ta, bool tb, double *C, int64_t ldc, const double *A, int64_t lda, const double *B, int64_t ldb,
           int64_t M, int64_t N, int64_t K, double alpha, double beta, bool lower, bool kFromTile)
{
    if (M <= 0 || N <= 0) return;
    const dim3 g((unsigned)((M + 63) / 64), (unsigned)((N + 63) / 64));
    const int lo = lower ? 1 : 0, kt = kFromTile ? 1 : 0;
    if (!ta && !tb) dgemm_tile_kernel<false, false><<<g, 256, 0, st>>>(C, ldc, A, lda, B, ldb, (int)M, (int)N, (int)K, alpha, beta, lo, kt);
    else if (!ta && tb) dgemm_tile_kernel<false, true><<<g, 256, 0, st>>>(C, ldc, A, lda, B, ldb, (int)M, (int)N, (int)K, alpha, beta, lo, kt);
    else dgemm_tile_kernel<true, true><<<g, 256, 0, st>>>(C, ldc, A, lda, B, ldb, (int)M, (int)N, (int)K, alpha, beta, lo, kt);
}
}  // namespace

// ---- the V-cycle's condensed tail: its operator, at assembly --------------
// The V-cycle at level l (one damped-Jacobi step from zero, residual,
// restriction, the levels below, prolongation onto the Jacobi iterate, one
// damped-Jacobi step) is linear in the level's residual r:
//     t = J r,  x = t + P M' P^T (r - K t),  z = x + J (r - K x)
//     =>  M = 2 J - J K J + Q M' Q^T,   Q = (I - J K) P,   J = omega D^-1,
// M' the operator of the level below (the coarsest level's: its inverse);
// TOP_GPU.m:766-816 in matrix form, the restriction being the prolongation's
// transpose on the active DOFs.  Dense FP64 on the levels' active DOFs (DOF
// 3 node + component), column-major, symmetric.
__global__ void tail_jacobi_kernel(double *__restrict__ J, const double *__restrict__ invD, const int32_t *__restrict__ nodeGrid,
                                   int64_t Nn, int64_t cs, double omega)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3 * Nn) return;
    J[i] = omega * invD[(i % 3) * cs + nodeGrid[i / 3]];
}
// Q = P - diag(J) K P; (K P)(i, j) sums over the 27 nodes that share an
// element with row i's node (K's nonzero blocks of the row), in a fixed order
__global__ void tail_q_kernel(double *__restrict__ Q, const double *__restrict__ Pt, const double *__restrict__ K,
                              const double *__restrict__ J, const int32_t *__restrict__ nbr, int64_t n, int64_t m)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n * m) return;
    const int64_t i = k / m, j = k % m;          // j fastest: the reads of P^T coalesce
    double acc = 0.0;
    for (int t = 0; t < 27; ++t) {
        const int32_t nb = nbr[(i / 3) * 27 + t];
        if (nb < 0) continue;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int64_t c = 3 * (int64_t)nb + d;
            acc = fma(K[i + n * c], Pt[j + m * c], acc);
        }
    }
    Q[i + n * j] = Pt[j + m * i] - J[i] * acc;
}
// M (lower triangle from the GEMM) += 2 diag(J) - diag(J) K diag(J), mirrored
// into the upper triangle: M exactly symmetric
__global__ void tail_m_kernel(double *__restrict__ M, const double *__restrict__ K, const double *__restrict__ J, int64_t n)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n * n) return;
    const int64_t i = k % n, j = k / n;
    if (i < j) return;
    const double v = M[k] + (i == j ? 2.0 * J[i] : 0.0) - J[i] * K[k] * J[j];
    M[k] = v;
    if (i != j) M[j + n * i] = v;
}
// the V-cycle's copy: row i of M (= column i) at stride ld, zero beyond n
template <typename T>
__global__ void tail_pack_kernel(T *__restrict__ Mp, int64_t ld, const double *__restrict__ M, int64_t n)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n * ld) return;
    const int64_t i = k / ld, j = k % ld;
    Mp[k] = j < n ? T(M[j + n * i]) : T(0);
}

bool tail_on(const top_solver *s)
{
    return s->tailL > 0 && (s->tailMode == 1 || (s->tailMode == -1 && s->p.precision == TOP_PREC_MIXED));
}
// M of levels nL-2 .. tailL from the current assembly (after the coarsest inverse)
int build_tail(top_solver *s, cudaStream_t st)
{
    s->tailReady = false;
    if (!tail_on(s)) return TOP_OK;
    const double *Mnext = s->Ainv;
    for (int l = s->nL - 2; l >= s->tailL; --l) {
        const size_t k = (size_t)(l - s->tailL);
        DevLevel &lv = s->L[l];
        const int64_t n = 3 * lv.Nn, m = 3 * s->L[l + 1].Nn;
        double *K = s->tailK, *M = s->tailMs[k];
        CK(cudaMemsetAsync(K, 0, sizeof(double) * n * n, st));
        coarsest_assemble_kernel<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(lv.KsC, lv.nodeGrid, s->tailEleCompact[k], s->tailNodeCompact[k], lv.g, lv.Nn, K);
        tail_jacobi_kernel<<<nb256(n), 256, 0, st>>>(s->tailJ, lv.invD64, lv.nodeGrid, lv.Nn, lv.g.cs, s->p.omega);
        tail_q_kernel<<<nb256(n * m), 256, 0, st>>>(s->tailQ, s->tailPt[k], K, s->tailJ, s->tailNbr[k], n, m);
        dgemm(st, false, true, s->tailT, n, s->tailQ, n, Mnext, m, n, m, m, 1.0, 0.0, false, false);   // T = Q M'
        dgemm(st, false, false, M, n, s->tailT, n, s->tailQ, n, n, n, m, 1.0, 0.0, true, false);      // T Q^T, lower
        tail_m_kernel<<<nb256(n * n), 256, 0, st>>>(M, K, s->tailJ, n);
        s->launches += 6;
        Mnext = M;
    }
    const int64_t n = 3 * s->L[s->tailL].Nn;
    if (s->p.precision == TOP_PREC_MIXED)
        tail_pack_kernel<float><<<nb256(n * s->tailLd), 256, 0, st>>>(static_cast<float *>(s->tailMp), s->tailLd, s->tailMs[0], n);
    else
        tail_pack_kernel<double><<<nb256(n * s->tailLd), 256, 0, st>>>(static_cast<double *>(s->tailMp), s->tailLd, s->tailMs[0], n);
    TOPGPU_COUNT_LAUNCH();
    CKL();
    s->tailReady = true;
    return TOP_OK;
}

int coarsest_inverse(top_solver *s, cudaStream_t st)
{
    const int64_t n = s->nC, nblk = (n + kDb - 1) / kDb;
    double *A = s->Ac;
    for (int64_t b = 0; b < nblk; ++b) {
        const int64_t k0 = b * kDb;
        const int kb = (int)std::min<int64_t>(kDb, n - k0);
        double *D = s->Dc + b * kDb * kDb;
        chol_block_kernel<<<1, 32, 0, st>>>(A, n, k0, kb, D, s->zeroDone + 1);
        TOPGPU_COUNT_LAUNCH();
        const int64_t rest = n - k0 - kb;
        if (rest > 0) {
            double *L21 = A + (k0 + kb) + n * k0;
            dgemm(st, false, false, L21, n, L21, n, D, kDb, rest, kb, kb, 1.0, 0.0, false, false);       // A21 L11^-T
            dgemm(st, false, false, A + (k0 + kb) * (1 + n), n, L21, n, L21, n, rest, rest, kb, -1.0, 1.0, true, false);
            s->launches += 2;
        }
    }
    CK(cudaMemsetAsync(s->Wc, 0, sizeof(double) * n * n, st));
    place_dinv_kernel<<<(unsigned)nblk, kDb * kDb, 0, st>>>(s->Dc, s->Wc, n);
    TOPGPU_COUNT_LAUNCH();
    for (int64_t hs = kDb; hs < n; hs *= 2) {          // bottom-up levels of the block inversion
        const int64_t nodes = (n + 2 * hs - 1) / (2 * hs), tiles = (hs + 63) / 64;
        for (int step = 0; step < 2; ++step) {
            inv_level_kernel<<<dim3((unsigned)tiles, (unsigned)tiles, (unsigned)nodes), 256, 0, st>>>(A, s->Wc, s->Ainv, n, (int)hs, step);
            TOPGPU_COUNT_LAUNCH();
        }
    }
    dgemm(st, true, true, s->Ainv, n, s->Wc, n, s->Wc, n, n, n, n, 1.0, 0.0, false, true);         // W^T W
    TOPGPU_COUNT_LAUNCH();
    return TOP_OK;
}

extern "C" int top_solver_assemble(top_solver *s)
{
    if (!s) return TOP_ERR_ARGS;
    cudaStream_t st = s->st;
    DevLevel &l0 = s->L[0];
    if (s->super) {      // level-0 element matrices, packed copies, diagonal
        super_kmat_kernel<<<(unsigned)l0.Ne, 576, 0, st>>>(s->Imat, s->Esub, s->mapUnique, s->uFree, s->uFixed, l0.KsC);
        TOPGPU_COUNT_LAUNCH();
        pack_ks_kernel<<<(unsigned)((l0.Ne + kPackE - 1) / kPackE), 256, 0, st>>>(l0.KsC, l0.eleGrid, l0.Ne, l0.KsP64, l0.KsP32, l0.g.cs);
        TOPGPU_COUNT_LAUNCH();
        diag_coarse_kernel<<<node_grid(l0.g), kNodeThreads, 0, st>>>(l0.KsP64, l0.g, l0.flags, l0.diag, l0.invD64, l0.invD32);
        TOPGPU_COUNT_LAUNCH();
    }
    // Galerkin Ks (TOP_GPU.m:1054-1147)
    for (int l = 1; l < s->nL; ++l) {
        DevLevel &d = s->L[l];
        int rc;
        if (s->super)    // P_s' K_mat(child) P_s, K_mat with the boundary override (superEle_inplace.cu:70-173)
            rc = assemble_higher_f64(d.KsC, d.upMap, s->L[l - 1].KsC, d.span == 4 ? s->P4 : s->P2, d.Ne,
                                     d.span * d.span * d.span, st);
        else if (l == 1)
            rc = assemble_level2_f64(d.KsC, d.upMap, s->Ec, s->KeDev, s->P4, s->mapUnique, s->uFree, s->uFixed,
                                     d.Ne, 64, s->nU, s->Qs, s->eye, st, s->bndList, s->nBnd);
        else
            rc = assemble_higher_f64(d.KsC, d.upMap, s->L[l - 1].KsC, s->P2, d.Ne, 8, st);
        if (rc) { set_error("top_solver_assemble: Galerkin kernel failed"); return rc; }
        if (l < s->nL - 1) {
            pack_ks_kernel<<<(unsigned)((d.Ne + kPackE - 1) / kPackE), 256, 0, st>>>(d.KsC, d.eleGrid, d.Ne, d.KsP64, d.KsP32, d.g.cs);
            TOPGPU_COUNT_LAUNCH();
            diag_coarse_kernel<<<node_grid(d.g), kNodeThreads, 0, st>>>(d.KsP64, d.g, d.flags, d.diag, d.invD64, d.invD32);
            TOPGPU_COUNT_LAUNCH();
        }
    }
    if (!s->super) {
        diag_l0_kernel<<<node_grid(l0.g), kNodeThreads, 0, st>>>(s->Ke64, s->Eg64, l0.flags, l0.g, s->p.E0, l0.diag, l0.invD64, l0.invD32);
        TOPGPU_COUNT_LAUNCH();
    }
    CKL();
    // coarsest matrix, Cholesky, inverse (TOP_GPU.m:1240-1255)
    DevLevel &lc = s->L[s->nL - 1];
    const int64_t n = s->nC;
    CK(cudaMemsetAsync(s->Ac, 0, sizeof(double) * n * n, st));
    coarsest_assemble_kernel<<<(unsigned)((n + 7) / 8), 256, 0, st>>>(lc.KsC, lc.nodeGrid, s->eleCompactC, s->nodeCompactC, lc.g, lc.Nn, s->Ac);
    TOPGPU_COUNT_LAUNCH();
    CK(cudaMemsetAsync(s->zeroDone, 0, sizeof(int) * 4, st));
    { const int rc = coarsest_inverse(s, st); if (rc) return rc; }
    CKL();
    int flag = 0;
    CK(cudaMemcpyAsync(&flag, s->zeroDone + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (flag) { set_error("top_solver_assemble: coarsest matrix is not positive definite"); return TOP_ERR_NAN; }
    { const int rc = build_tail(s, st); if (rc) return rc; }
    s->assembled = true;
    return TOP_OK;
}

// ---- standalone operators on compact vectors ------------------------------
extern "C" int top_solver_matvec(top_solver *s, int level, const double *u, double *y, int fp32)
{
    if (!s || !u || !y || level < 0 || level >= s->nL) { set_error("top_solver_matvec: bad arguments"); return TOP_ERR_ARGS; }
    if (level > 0 && !s->assembled) { set_error("top_solver_matvec: assemble first"); return TOP_ERR_STATE; }
    if (level == s->nL - 1 && level > 0) { set_error("top_solver_matvec: the coarsest level is solved directly"); return TOP_ERR_ARGS; }
    DevLevel &d = s->L[level];
    const Reduce none{nullptr, nullptr, nullptr};
    CK(cudaMemsetAsync(d.x64 - kMargin, 0, sizeof(double) * 3 * d.g.cs, s->st));
    compact_to_grid_kernel<double, double><<<nb256(d.Nn), 256, 0, s->st>>>(u, d.x64, d.nodeGrid, d.Nn, d.g.cs);
    TOPGPU_COUNT_LAUNCH();
    if (fp32) {                      // the operand rounded to FP32 once (as the V-cycle holds it)
        CK(cudaMemsetAsync(d.x32 - kMargin, 0, sizeof(float) * 3 * d.g.cs, s->st));
        compact_to_grid_kernel<double, float><<<nb256(d.Nn), 256, 0, s->st>>>(u, d.x32, d.nodeGrid, d.Nn, d.g.cs);
        TOPGPU_COUNT_LAUNCH();
        level_op<float>(s, level, VecIn<float, float>{d.x32, d.g.cs}, StoreOut<float, double>{d.t64, d.g.cs}, none, nullptr);
    } else {
        level_op<double>(s, level, VecIn<double, double>{d.x64, d.g.cs}, StoreOut<double, double>{d.t64, d.g.cs}, none, nullptr);
    }
    grid_to_compact_kernel<double, double><<<nb256(d.Nn), 256, 0, s->st>>>(d.t64, y, d.nodeGrid, d.Nn, d.g.cs);
    TOPGPU_COUNT_LAUNCH();
    CKL();
    return op_err_status(s);
}

extern "C" int top_solver_vcycle(top_solver *s, const double *r, double *z)
{
    if (!s || !r || !z) return TOP_ERR_ARGS;
    if (!s->assembled) { set_error("top_solver_vcycle: assemble first"); return TOP_ERR_STATE; }
    DevLevel &l0 = s->L[0];
    CK(cudaMemsetAsync(s->tmp - kMargin, 0, sizeof(double) * 3 * l0.g.cs, s->st));
    compact_to_grid_kernel<double, double><<<nb256(l0.Nn), 256, 0, s->st>>>(r, s->tmp, l0.nodeGrid, l0.Nn, l0.g.cs);
    TOPGPU_COUNT_LAUNCH();
    precond(s, s->tmp, s->z, nullptr, s->zeroDone);
    grid_to_compact_kernel<double, double><<<nb256(l0.Nn), 256, 0, s->st>>>(s->z, z, l0.nodeGrid, l0.Nn, l0.g.cs);
    TOPGPU_COUNT_LAUNCH();
    CKL();
    return op_err_status(s);
}

extern "C" int top_solver_restrict(top_solver *s, int ii, const double *rF, double *rC)
{
    if (!s || ii < 1 || ii >= s->nL) return TOP_ERR_ARGS;
    DevLevel &f = s->L[ii - 1], &c = s->L[ii];
    CK(cudaMemsetAsync(f.x64 - kMargin, 0, sizeof(double) * 3 * f.g.cs, s->st));
    compact_to_grid_kernel<double, double><<<nb256(f.Nn), 256, 0, s->st>>>(rF, f.x64, f.nodeGrid, f.Nn, f.g.cs);
    TOPGPU_COUNT_LAUNCH();
    restrict_op<double>(s, ii - 1, f.x64, c.t64, nullptr);
    grid_to_compact_kernel<double, double><<<nb256(c.Nn), 256, 0, s->st>>>(c.t64, rC, c.nodeGrid, c.Nn, c.g.cs);
    TOPGPU_COUNT_LAUNCH();
    CKL();
    CK(cudaStreamSynchronize(s->st));
    return TOP_OK;
}

extern "C" int top_solver_interpolate(top_solver *s, int ii, const double *xC, double *xF)
{
    if (!s || ii < 1 || ii >= s->nL) return TOP_ERR_ARGS;
    DevLevel &f = s->L[ii - 1], &c = s->L[ii];
    CK(cudaMemsetAsync(c.x64 - kMargin, 0, sizeof(double) * 3 * c.g.cs, s->st));
    compact_to_grid_kernel<double, double><<<nb256(c.Nn), 256, 0, s->st>>>(xC, c.x64, c.nodeGrid, c.Nn, c.g.cs);
    TOPGPU_COUNT_LAUNCH();
    if (c.span == 4)
        prolong_kernel<double, 4, double><<<node_grid(f.g), kNodeThreads, 0, s->st>>>(c.x64, c.g, f.t64, f.g, f.flags, nullptr, nullptr, 0.0, nullptr);
    else
        prolong_kernel<double, 2, double><<<node_grid(f.g), kNodeThreads, 0, s->st>>>(c.x64, c.g, f.t64, f.g, f.flags, nullptr, nullptr, 0.0, nullptr);
    TOPGPU_COUNT_LAUNCH();
    grid_to_compact_kernel<double, double><<<nb256(f.Nn), 256, 0, s->st>>>(f.t64, xF, f.nodeGrid, f.Nn, f.g.cs);
    TOPGPU_COUNT_LAUNCH();
    CKL();
    CK(cudaStreamSynchronize(s->st));
    return TOP_OK;
}

extern "C" int top_solver_get_diag(top_solver *s, int level, double *diag)
{
    if (!s || !diag || level < 0 || level >= s->nL - (s->nL > 1 ? 1 : 0)) return TOP_ERR_ARGS;
    if (!s->assembled) { set_error("top_solver_get_diag: assemble first"); return TOP_ERR_STATE; }
    DevLevel &d = s->L[level];
    grid_to_compact_kernel<double, double><<<nb256(d.Nn), 256, 0, s->st>>>(d.diag, diag, d.nodeGrid, d.Nn, d.g.cs);
    TOPGPU_COUNT_LAUNCH();
    CKL();
    CK(cudaStreamSynchronize(s->st));
    return TOP_OK;
}

extern "C" int top_solver_get_ks(top_solver *s, int level, double *Ks)
{
    if (!s || !Ks || level < (s->super ? 0 : 1) || level >= s->nL) return TOP_ERR_ARGS;   // super: level 0 = K_mat
    if (!s->assembled) { set_error("top_solver_get_ks: assemble first"); return TOP_ERR_STATE; }
    DevLevel &d = s->L[level];
    CK(cudaMemcpyAsync(Ks, d.KsC, sizeof(double) * 576 * d.Ne, cudaMemcpyDeviceToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return TOP_OK;
}

// ---- PCG (Solving_PCG, TOP_GPU.m:602-667) ---------------------------------
__global__ void pcg_init_kernel(PcgState *st, int nv)
{   // ||b|| from the squared norm written by dot_kernel into st->normB
    if ((int)threadIdx.x >= nv) return;
    st += threadIdx.x;
    st->normB = sqrt(st->normB);
    if (st->normB == 0.0) st->done = 1;   // zero load: x = 0, no iterations
}

// The PCG chunk graph for (b, x): captured from `body` (launches on the
// stream it is given) on first use and again when the operator configuration
// changed.  Capture runs on the solver's own non-blocking stream (the
// caller's stream may be the legacy default stream, which cannot be captured).
template <class Body>
static cudaError_t pcg_graph_prepare(top_solver *s, const double *b, double *x, int chunk, int nrhs, Body body,
                                     top_solver::PcgGraph **out)
{
    for (auto &G : s->graphs)
        if (G.exec && G.b == b && G.x == x && G.gen == s->opGen && G.chunk == chunk && G.nrhs == nrhs) { *out = &G; return cudaSuccess; }
    cudaError_t e;
    if (!s->capStream) {
        if ((e = cudaStreamCreateWithFlags(&s->capStream, cudaStreamNonBlocking)) != cudaSuccess) return e;
        if ((e = cudaEventCreateWithFlags(&s->capIn, cudaEventDisableTiming)) != cudaSuccess) return e;
        if ((e = cudaEventCreateWithFlags(&s->capOut, cudaEventDisableTiming)) != cudaSuccess) return e;
    }
    // drop stale graphs and, beyond eight, the oldest
    for (size_t i = 0; i < s->graphs.size();) {
        top_solver::PcgGraph &G = s->graphs[i];
        if (G.gen != s->opGen || (G.b == b && G.x == x && G.nrhs == nrhs) || s->graphs.size() >= 8) {
            if (G.exec) cudaGraphExecDestroy(G.exec);
            s->graphs.erase(s->graphs.begin() + (long)i);
        } else {
            ++i;
        }
    }
    top_solver::PcgGraph G;
    cudaStream_t user = s->st;
    const int64_t before = s->launches;
    s->st = s->capStream;                // every launch helper issues on s->st
    cudaGraph_t graph = nullptr;
    e = cudaStreamBeginCapture(s->capStream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        s->inCapture = true;
        body(s->capStream);
        s->inCapture = false;
        e = cudaStreamEndCapture(s->capStream, &graph);
    }
    s->st = user;
    G.nodes = s->launches - before;      // captured, not run
    s->launches = before;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&G.exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) return e;
    G.b = b; G.x = x; G.gen = s->opGen; G.chunk = chunk; G.nrhs = nrhs;
    s->graphs.push_back(G);
    *out = &s->graphs.back();
    return cudaSuccess;
}

// PCG (TOP_GPU.m:602-667) on nrhs right-hand sides at once: b and x hold
// nrhs level-0 grid vectors at stride 3 CS; every operator runs once per
// iteration for all of them (one launch, the right-hand side in the grid's
// y or z index); each right-hand side keeps its own scalars and stops on its
// own residual.  itsOut / resOut: arrays of nrhs (may be NULL).
int topgpu::pcg_block(top_solver *s, const double *bGrid, double *xg, int nrhs, int warm, int *itsOut, double *resOut)
{
    if (!s->assembled) { set_error("top_solver_pcg: assemble first"); return TOP_ERR_STATE; }
    if (nrhs < 1 || nrhs > s->kMax) { set_error("top_solver_pcg: %d right-hand sides (at most %d)", nrhs, s->kMax); return TOP_ERR_ARGS; }
    DevLevel &l0 = s->L[0];
    const int64_t cs = l0.g.cs, nv = 3 * cs;    // whole grid vectors, margins included
    cudaStream_t st = s->st;
    const int VB = vec_blocks(nv);
    // the residual update: one resident wave of 256-thread CTAs
    static const int updOcc = [] {
        int n32 = 0, n64 = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n32, pcg_update_kernel<float>, 256, 0) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n64, pcg_update_kernel<double>, 256, 0) != cudaSuccess) {
            (void)cudaGetLastError();
            return 4;
        }
        return std::max(1, std::min(n32, n64));
    }();
    const int UB = (int)std::min<int64_t>(std::min<int64_t>((int64_t)updOcc * s->numSMs, (nv / 2 + 255) / 256), s->nPartials);
    const int64_t M = kMargin;
    const unsigned K = (unsigned)nrhs;
    // mixed precision keeps the FP32 V-cycle's output z in FP32
    const bool z32 = s->p.precision == TOP_PREC_MIXED;
    std::vector<PcgState> h0((size_t)nrhs);
    for (auto &h : h0) { h = PcgState{}; h.tol = s->p.tol; h.maxIT = s->p.maxIT; }
    CK(cudaMemcpyAsync(s->state, h0.data(), sizeof(PcgState) * nrhs, cudaMemcpyHostToDevice, st));
    int *done = &s->state->done;
    auto red = [&](double *r) { return nrhs > 1 ? s->redk(r) : s->red(r); };
    dot_kernel<<<dim3(VB, K), 256, 0, st>>>(bGrid - M, bGrid - M, nv, red(&s->state->normB));
    TOPGPU_COUNT_LAUNCH();
    pcg_init_kernel<<<1, 32, 0, st>>>(s->state, nrhs);
    TOPGPU_COUNT_LAUNCH();
    if (!warm) CK(cudaMemsetAsync(xg - kMargin, 0, sizeof(double) * nv * nrhs, st));
    // r = b - A x
    if (s->p.outerFP32)
        l0_op<float>(s, VecIn<float, double>{xg, cs, nv}, ResidOut<float, double, double>{bGrid, s->r, cs, nv},
                     Reduce{nullptr, nullptr, nullptr}, done, nrhs);
    else
        l0_op<double>(s, VecIn<double, double>{xg, cs, nv}, ResidOut<double, double, double>{bGrid, s->r, cs, nv},
                      Reduce{nullptr, nullptr, nullptr}, done, nrhs);
    // z = M r ; rho = z . r ; p = z
    // z = M r, z.r; p = z + beta p (z1Ready: the update kernel stored the V-cycle's Jacobi iterate)
    const int flex = s->flexible ? 1 : 0;
    auto precond_p = [&](cudaStream_t q, int first) {
        if (z32) {
            vcycle<float, double, float>(s, s->r, s->z32, &s->state->rho, done, nrhs, nv, !first);
            if (flex && !first) {
                launch_k(s, zv_dot_kernel<float>, dim3(VB, K), 256, 0, q, s->z32 - M, s->v - M, nv, red(&s->state->sigma), done);
                TOPGPU_COUNT_LAUNCH();
            }
            launch_k(s, pcg_p_kernel<float>, dim3(VB, K), 256, 0, q, s->pv - M, s->z32 - M, nv, s->state, first, xg - M, flex);
        } else {
            vcycle<double, double, double>(s, s->r, s->z, &s->state->rho, done, nrhs, nv, !first);
            if (flex && !first) {
                launch_k(s, zv_dot_kernel<double>, dim3(VB, K), 256, 0, q, s->z - M, s->v - M, nv, red(&s->state->sigma), done);
                TOPGPU_COUNT_LAUNCH();
            }
            launch_k(s, pcg_p_kernel<double>, dim3(VB, K), 256, 0, q, s->pv - M, s->z - M, nv, s->state, first, xg - M, flex);
        }
        TOPGPU_COUNT_LAUNCH();
    };
    precond_p(st, 1);
    CKL();
    static const bool trace = std::getenv("TOPGPU_PCG_TRACE") != nullptr;
    const int chunk = trace ? 1 : 4;
    // one PCG iteration (TOP_GPU.m:620-655); every kernel returns at once for a converged right-hand side
    auto iteration = [&](cudaStream_t q) {
        outer_op(s, s->pv, s->v, &s->state->pv, done, nrhs, nv);                             // v = A p, p.v
        if (z32)
            launch_k(s, pcg_update_kernel<float>, dim3(UB, K), 256, 0, q, s->r - M, s->v - M, nv, s->state, red(&s->state->rr),
                                                                l0.x32 - M, l0.invD32 - M, float(s->p.omega));
        else
            launch_k(s, pcg_update_kernel<double>, dim3(UB, K), 256, 0, q, s->r - M, s->v - M, nv, s->state, red(&s->state->rr),
                                                                 l0.x64 - M, l0.invD64 - M, double(s->p.omega));
        TOPGPU_COUNT_LAUNCH();
        precond_p(q, 0);
    };
    top_solver::PcgGraph *G = nullptr;
    if (s->useGraphs && !trace)
        CK(pcg_graph_prepare(s, bGrid, xg, chunk, nrhs, [&](cudaStream_t q) { for (int k = 0; k < chunk; ++k) iteration(q); }, &G));
    for (int it0 = 0; it0 < s->p.maxIT; it0 += chunk) {
        if (G && it0 + chunk <= s->p.maxIT) {
            CK(cudaEventRecord(s->capIn, st));
            CK(cudaStreamWaitEvent(s->capStream, s->capIn, 0));
            CK(cudaGraphLaunch(G->exec, s->capStream));
            CK(cudaEventRecord(s->capOut, s->capStream));
            CK(cudaStreamWaitEvent(st, s->capOut, 0));
            s->launches += G->nodes;
        } else {
            for (int k = 0; k < chunk && it0 + k < s->p.maxIT; ++k) iteration(st);
        }
        CKL();
        CK(cudaMemcpyAsync(s->hstate, s->state, sizeof(PcgState) * nrhs, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (trace && it0 < 12)
            std::fprintf(stderr, "pcg it %d rho %.6e rhoOld %.6e pv %.6e rr %.6e res %.6e done %d\n", s->hstate->its,
                         s->hstate->rho, s->hstate->rhoOld, s->hstate->pv, s->hstate->rr, s->hstate->resnorm, s->hstate->done);
        bool all = true;
        for (int k = 0; k < nrhs; ++k) all = all && s->hstate[k].done;
        if (all) break;
    }
    int rc = op_err_status(s);
    if (rc != TOP_OK) return rc;
    for (int k = 0; k < nrhs; ++k) {
        const PcgState &f = s->hstate[k];
        if (f.normB == 0.0) CK(cudaMemsetAsync(xg + k * nv - kMargin, 0, sizeof(double) * nv, st));
        if (itsOut) itsOut[k] = f.its;
        if (resOut) resOut[k] = f.resnorm;
        if (f.status == TOP_ERR_NAN) { set_error("top_solver_pcg: non-finite PCG scalar at iteration %d", f.its); rc = TOP_ERR_NAN; }
        else if (f.status == TOP_ERR_NOT_CONVERGED && rc == TOP_OK) {
            set_error("Exceed the maximum iterate numbers (residual %.4e)", f.resnorm); rc = TOP_ERR_NOT_CONVERGED;
        }
    }
    return rc;
}

int topgpu::pcg_grid(top_solver *s, const double *bGrid, double *xg, int warm, int *itsOut, double *resOut)
{
    return pcg_block(s, bGrid, xg, 1, warm, itsOut, resOut);
}

// compact warm start / solution around pcg_grid
static int pcg_run(top_solver *s, const double *bGrid, double *U, int warm, int *itsOut, double *resOut)
{
    DevLevel &l0 = s->L[0];
    const int64_t cs = l0.g.cs;
    CK(cudaMemsetAsync(s->x - kMargin, 0, sizeof(double) * 3 * cs, s->st));
    if (warm) {
        compact_to_grid_kernel<double, double><<<nb256(l0.Nn), 256, 0, s->st>>>(U, s->x, l0.nodeGrid, l0.Nn, cs);
        TOPGPU_COUNT_LAUNCH();
    }
    const int rc = pcg_grid(s, bGrid, s->x, 1, itsOut, resOut);
    if (rc != TOP_OK && rc != TOP_ERR_NOT_CONVERGED) return rc;
    grid_to_compact_kernel<double, double><<<nb256(l0.Nn), 256, 0, s->st>>>(s->x, U, l0.nodeGrid, l0.Nn, cs);
    TOPGPU_COUNT_LAUNCH();
    CKL();
    CK(cudaStreamSynchronize(s->st));
    return rc;
}

extern "C" int top_solver_pcg(top_solver *s, int loadCase, double *U, int warm, int *its, double *relres)
{
    if (!s || !U || loadCase < 0 || loadCase >= s->nLoads) { set_error("top_solver_pcg: bad arguments"); return TOP_ERR_ARGS; }
    return pcg_run(s, s->b + (size_t)loadCase * 3 * s->L[0].g.cs, U, warm, its, relres);
}

extern "C" int top_solver_pcg_all(top_solver *s, double *U, int warm, int *its, double *relres)
{
    if (!s || !U) { set_error("top_solver_pcg_all: bad arguments"); return TOP_ERR_ARGS; }
    DevLevel &l0 = s->L[0];
    const int64_t cs = l0.g.cs, nd = 3 * l0.Nn;
    const int K = s->nLoads;
    CK(cudaMemsetAsync(s->x - kMargin, 0, sizeof(double) * 3 * cs * K, s->st));
    if (warm)
        for (int k = 0; k < K; ++k) {
            compact_to_grid_kernel<double, double><<<nb256(l0.Nn), 256, 0, s->st>>>(U + k * nd, s->x + k * 3 * cs, l0.nodeGrid, l0.Nn, cs);
            TOPGPU_COUNT_LAUNCH();
        }
    const int rc = pcg_block(s, s->b, s->x, K, 1, its, relres);
    if (rc != TOP_OK && rc != TOP_ERR_NOT_CONVERGED) return rc;
    for (int k = 0; k < K; ++k) {
        grid_to_compact_kernel<double, double><<<nb256(l0.Nn), 256, 0, s->st>>>(s->x + k * 3 * cs, U + k * nd, l0.nodeGrid, l0.Nn, cs);
        TOPGPU_COUNT_LAUNCH();
    }
    CKL();
    CK(cudaStreamSynchronize(s->st));
    return rc;
}

extern "C" int top_solver_pcg_rhs(top_solver *s, const double *b, double *U, int warm, int *its, double *relres)
{
    if (!s || !b || !U) return TOP_ERR_ARGS;
    DevLevel &l0 = s->L[0];
    CK(cudaMemsetAsync(s->tmp - kMargin, 0, sizeof(double) * 3 * l0.g.cs, s->st));
    compact_to_grid_kernel<double, double><<<nb256(l0.Nn), 256, 0, s->st>>>(b, s->tmp, l0.nodeGrid, l0.Nn, l0.g.cs);
    TOPGPU_COUNT_LAUNCH();
    CKL();
    return pcg_run(s, s->tmp, U, warm, its, relres);
}

extern "C" int top_solver_unit_compliance(top_solver *s, const double *U, double *ce)
{
    if (!s || !U || !ce) return TOP_ERR_ARGS;
    DevLevel &l0 = s->L[0];
    const int64_t cs = l0.g.cs;
    // U compact [3Nn x nLoads] -> grid; the b array has room for nLoads grid vectors
    double *Ug = s->b;   // overwritten below, so re-upload afterwards would be needed: use tmp for 1 load
    if (s->nLoads != 1) { set_error("top_solver_unit_compliance: multiple load cases not supported in this call"); return TOP_ERR_ARGS; }
    Ug = s->tmp;
    CK(cudaMemsetAsync(Ug - kMargin, 0, sizeof(double) * 3 * cs, s->st));
    compact_to_grid_kernel<double, double><<<nb256(l0.Nn), 256, 0, s->st>>>(U, Ug, l0.nodeGrid, l0.Nn, cs);
    TOPGPU_COUNT_LAUNCH();
    if (s->super)
        compliance_kmat_kernel<<<nb256(l0.Ne), 256, 0, s->st>>>(l0.KsC, Ug, 3 * cs, 1, s->weights, l0.eleGrid, l0.Ne, l0.g, ce);
    else
        compliance_kernel<<<nb256(l0.Ne), 256, 0, s->st>>>(s->Ke64, Ug, 3 * cs, 1, s->weights, l0.eleGrid, l0.Ne, l0.g, ce);
    TOPGPU_COUNT_LAUNCH();
    CKL();
    CK(cudaStreamSynchronize(s->st));
    return TOP_OK;
}

// ---- kernel timing (CUDA events on the solver's stream) -------------------
// which: 0 = level-0 K*u FP64 (the outer PCG operator), 1 = level-0 K*u FP32
// (the V-cycle smoother operator), 2 = one V-cycle, 3 = level-1 K*u FP32,
// 4 = level 0 -> 1 restriction FP32, 5 = level 1 -> 0 prolongation FP32.
// Each launch is preceded by a write of flushBytes to evict L2 (0 = none);
// *msPerLaunch receives the mean event time of the launches alone.
extern "C" int top_solver_time_kernel(top_solver *s, int which, int nrep, int64_t flushBytes, double *msPerLaunch)
{
    if (!s || nrep < 1 || !msPerLaunch) return TOP_ERR_ARGS;
    if (which < 0 || which > 5) { set_error("top_solver_time_kernel: unknown kernel %d", which); return TOP_ERR_ARGS; }
    if (which != 0 && !s->assembled) { set_error("top_solver_time_kernel: assemble first"); return TOP_ERR_STATE; }
    DevLevel &l0 = s->L[0];
    const Reduce none{nullptr, nullptr, nullptr};
    struct Held {                    // released on every return
        void *flush = nullptr;
        cudaEvent_t a = nullptr, b = nullptr;
        ~Held() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); if (flush) cudaFree(flush); }
    } h;
    if (flushBytes > 0) CK(cudaMalloc(&h.flush, (size_t)flushBytes));
    CK(cudaEventCreate(&h.a)); CK(cudaEventCreate(&h.b));
    void *flush = h.flush;
    cudaEvent_t a = h.a, b = h.b;
    double total = 0;
    for (int k = 0; k < nrep; ++k) {
        if (flush) CK(cudaMemsetAsync(flush, k & 0xff, (size_t)flushBytes, s->st));
        CK(cudaEventRecord(a, s->st));
        switch (which) {
        case 0: l0_op<double>(s, VecIn<double, double>{s->pv, l0.g.cs}, StoreOut<double, double>{s->v, l0.g.cs}, none, nullptr); break;
        case 1: l0_op<float>(s, VecIn<float, float>{l0.x32, l0.g.cs}, StoreOut<float, float>{l0.t32, l0.g.cs}, none, nullptr); break;
        case 2: precond(s, s->r, s->z, nullptr, s->zeroDone); break;
        case 4: if (s->nL > 2) {   // level-0 -> level-1 restriction, FP32
            restrict_op<float>(s, 0, s->L[0].t32, s->L[1].r32, nullptr);
        } break;
        case 5: if (s->nL > 2) {   // level-1 -> level-0 prolongation with the Jacobi base, FP32
            DevLevel &f = s->L[0], &c = s->L[1];
            const dim3 g4((unsigned)(((int64_t)((f.g.NY + 3) / 4) * f.g.NX * f.g.NZ + kNodeThreads - 1) / kNodeThreads));
            if (c.span == 4 && s->vec4 && vec4_ok(f.g, {f.x32, f.flags, s->r, f.invD32}, {}))
                prolong4_kernel<float, double, false, true><<<g4, kNodeThreads, 0, s->st>>>(c.t32, c.g, f.x32, f.g, f.flags, s->r, f.invD32, 0.6f, nullptr);
            else if (c.span == 4) prolong4_kernel<float, double, false><<<g4, kNodeThreads, 0, s->st>>>(c.t32, c.g, f.x32, f.g, f.flags, s->r, f.invD32, 0.6f, nullptr);
            else prolong_kernel<float, 2, double><<<node_grid(f.g), kNodeThreads, 0, s->st>>>(c.t32, c.g, f.x32, f.g, f.flags, s->r, f.invD32, 0.6f, nullptr);
            TOPGPU_COUNT_LAUNCH();
        } break;
        case 3: if (s->nL > 2) coarse_op<float>(s, 1, VecIn<float, float>{s->L[1].x32, s->L[1].g.cs}, StoreOut<float, float>{s->L[1].t32, s->L[1].g.cs}, none, nullptr); break;
        default: set_error("top_solver_time_kernel: unknown kernel %d", which); return TOP_ERR_ARGS;
        }
        CK(cudaEventRecord(b, s->st));
        CK(cudaEventSynchronize(b));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, a, b));
        total += ms;
    }
    CKL();
    *msPerLaunch = total / nrep;
    return op_err_status(s);
}
