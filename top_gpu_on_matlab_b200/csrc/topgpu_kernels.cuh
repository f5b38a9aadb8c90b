// topgpu_kernels.cuh -- device kernels shared by the MEX drop-ins and the
// fused solver: Galerkin triple products and the FP64 tensor-core GEMM.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "topgpu_internal.h"

#define TOP_CUDA_CHECK(call, name)                                                   \
    do {                                                                             \
        cudaError_t err__ = (call);                                                  \
        if (err__ != cudaSuccess) {                                                  \
            topgpu::set_error("%s:CUDA CUDA error %d: %s", name, (int)err__,         \
                              cudaGetErrorString(err__));                            \
            return TOP_ERR_CUDA;                                                     \
        }                                                                            \
    } while (0)

namespace topgpu {

// ---------------------------------------------------------------------------
// Kout = sum over children of P_s^T K_s P_s for one coarse element per CTA.
// 64 threads; thread t owns the 3x3 block (rows 3*(t%8).., cols 3*(t/8)..)
// of both T = K_s P_s and Kout, so each shared-memory operand feeds three
// FMAs.  ChildK(f0, i) yields entry i (col-major 24x24) of the child's K;
// the child list is upMap[e + s*nElem] (1-based, <= 0 = skip) and
// skip(f0) excludes children handled elsewhere.
constexpr int kPtkpThreads = 64;

template <typename T, class ChildK, class Skip>
__global__ void __launch_bounds__(kPtkpThreads)
ptkp_kernel(T *__restrict__ Ks, const int32_t *__restrict__ upMap, int64_t nElem, int nCh,
            const T *__restrict__ P, ChildK childK, Skip skip, int accumulate,
            const int32_t *__restrict__ elist)
{
    __shared__ T sK[576], sP[576], sT[576];
    const int64_t e = elist ? (int64_t)elist[blockIdx.x] : (int64_t)blockIdx.x;   // optional subset of elements
    const int t = threadIdx.x, rb = (t % 8) * 3, cb = (t / 8) * 3;
    T acc[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) acc[i][j] = T(0);
    bool any = false;
    for (int s = 0; s < nCh; ++s) {
        const int32_t f1 = upMap[e + (int64_t)s * nElem];
        if (f1 <= 0 || skip(f1 - 1)) continue;   // uniform across the CTA
        any = true;
        for (int i = t; i < 576; i += kPtkpThreads) { sP[i] = P[(size_t)s * 576 + i]; sK[i] = childK(f1 - 1, i); }
        __syncthreads();
        T tt[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) tt[i][j] = T(0);
#pragma unroll 4
        for (int k = 0; k < 24; ++k) {
            T kr[3], pc[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) { kr[i] = sK[(rb + i) + 24 * k]; pc[i] = sP[k + 24 * (cb + i)]; }
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) tt[i][j] = fma(kr[i], pc[j], tt[i][j]);
        }
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) sT[(rb + i) + 24 * (cb + j)] = tt[i][j];
        __syncthreads();
#pragma unroll 4
        for (int k = 0; k < 24; ++k) {
            T pr[3], tc[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) { pr[i] = sP[k + 24 * (rb + i)]; tc[i] = sT[k + 24 * (cb + i)]; }
#pragma unroll
            for (int i = 0; i < 3; ++i)
#pragma unroll
                for (int j = 0; j < 3; ++j) acc[i][j] = fma(pr[i], tc[j], acc[i][j]);
        }
        __syncthreads();
    }
    if (accumulate && !any) return;
    T *out = Ks + (size_t)e * 576;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int idx = (rb + i) + 24 * (cb + j);
            out[idx] = accumulate ? out[idx] + acc[i][j] : acc[i][j];
        }
}

// ---------------------------------------------------------------------------
// FP64 tensor-core GEMM  C[M x N] (row-major, ldc) = A[M x 64] * B[64 x N]
// with mma.sync.m8n8k4.f64 (the FP64 tensor path of sm_100a).  A's rows
// are produced on the fly by ARow (e.g. child moduli of a coarse cell);
// B is row-major [64 x ldb].  CTA tile 64 x 64, 4 warps of 32 x 32.
constexpr int kGemmBM = 64, kGemmBN = 64, kGemmK = 64, kGemmPad = 4;

__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d0), "+d"(d1) : "d"(a), "d"(b));
}

template <class ARow>
__global__ void __launch_bounds__(128)
dgemm_k64_kernel(double *__restrict__ C, int64_t M, int N, int64_t ldc,
                 const double *__restrict__ B, int ldb, ARow arow)
{
    extern __shared__ double smem[];
    double *sA = smem;                                  // [BM][K + pad]
    double *sB = smem + kGemmBM * (kGemmK + kGemmPad);  // [K][BN + pad]
    const int64_t m0 = (int64_t)blockIdx.x * kGemmBM;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // A tile (gathered rows: a few dependent loads each), once per CTA: thread
    // per (row, k) pair, 32 rows per pass
    for (int idx = tid; idx < kGemmBM * kGemmK; idx += 128) {
        const int r = idx % kGemmBM, k = idx / kGemmBM;
        const int64_t m = m0 + r;
        sA[r * (kGemmK + kGemmPad) + k] = (m < M) ? arow(m, k) : 0.0;
    }
    // the CTA's column tiles in turn, the A tile reused from shared memory
    for (int n0 = blockIdx.y * kGemmBN; n0 < N; n0 += gridDim.y * kGemmBN) {
        __syncthreads();                                    // sB free (and sA complete)
        for (int idx = tid; idx < kGemmK * kGemmBN; idx += 128) {
            const int k = idx / kGemmBN, c = idx % kGemmBN;
            sB[k * (kGemmBN + kGemmPad) + c] = (n0 + c < N) ? B[(size_t)k * ldb + n0 + c] : 0.0;
        }
        __syncthreads();
        const int wr = (warp & 1) * 32, wc = (warp >> 1) * 32;
        const int g = lane >> 2, q = lane & 3;
        double acc[4][4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll 4
        for (int k0 = 0; k0 < kGemmK; k0 += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = sA[(wr + 8 * i + g) * (kGemmK + kGemmPad) + k0 + q];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sB[(k0 + q) * (kGemmBN + kGemmPad) + wc + 8 * j + g];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int64_t m = m0 + wr + 8 * i + g;
            if (m >= M) continue;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int n = n0 + wc + 8 * j + 2 * q;
                if (n < N) C[m * ldc + n] = acc[i][j][0];
                if (n + 1 < N) C[m * ldc + n + 1] = acc[i][j][1];
            }
        }
    }
}

constexpr size_t kGemmSmem = sizeof(double) * (kGemmBM * (kGemmK + kGemmPad) + kGemmK * (kGemmBN + kGemmPad));

// ---------------------------------------------------------------------------
// FP64 Galerkin triple products on the tensor cores: Kout = sum over children
// of P_s^T (K_s P_s), one coarse element per warp, every 24 x 24 product as
// 3 x 3 tiles of mma.sync.m8n8k4.f64 (six k-steps each: 108 MMAs per child).
// The child's K_s is gathered into the warp's shared memory (leading dimension
// 25, which spreads a fragment's rows over the banks); T = K_s P_s goes
// through shared memory once; P_s fragments are read straight from global
// memory (one small matrix per child slot, shared by every warp, L1 resident);
// the output tiles accumulate in registers over the children.  Same
// arguments and results as ptkp_kernel (rounding aside).
constexpr int kDmmaWarps = 4;
constexpr int kDmmaLd = 25;

template <class ChildK, class Skip>
__global__ void __launch_bounds__(32 * kDmmaWarps)
ptkp_dmma_kernel(double *__restrict__ Ks, const int32_t *__restrict__ upMap, int64_t nElem, int nCh,
                 const double *__restrict__ P, ChildK childK, Skip skip, int accumulate,
                 const int32_t *__restrict__ elist, int64_t nSel)
{
    __shared__ double smem[kDmmaWarps][2][24 * kDmmaLd];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const int64_t w = (int64_t)blockIdx.x * kDmmaWarps + warp;
    if (w >= nSel) return;                           // whole warps; no CTA-wide barrier below
    const int64_t e = elist ? (int64_t)elist[w] : w;
    double *sK = smem[warp][0], *sT = smem[warp][1];
    double acc[3][3][2];
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
        for (int J = 0; J < 3; ++J) acc[I][J][0] = acc[I][J][1] = 0.0;
    bool any = false;
    for (int s = 0; s < nCh; ++s) {
        const int32_t f1 = upMap[e + (int64_t)s * nElem];
        if (f1 <= 0 || skip(f1 - 1)) continue;     // uniform across the warp
        any = true;
        const double *Ps = P + (size_t)s * 576;
        __syncwarp();                                // the previous child's reads of sK / sT are done
        for (int i = lane; i < 576; i += 32) sK[(i % 24) + kDmmaLd * (i / 24)] = childK(f1 - 1, i);
        __syncwarp();
        // T = K_s P_s: tile (I, J) = sum_kk K[8I.., 4kk..] P[4kk.., 8J..]
#pragma unroll
        for (int I = 0; I < 3; ++I)
#pragma unroll
            for (int J = 0; J < 3; ++J) {
                double d0 = 0.0, d1 = 0.0;
#pragma unroll
                for (int kk = 0; kk < 6; ++kk)
                    dmma_8x8x4(d0, d1, sK[(8 * I + g) + kDmmaLd * (4 * kk + q)], __ldg(Ps + (4 * kk + q) + 24 * (8 * J + g)));
                sT[(8 * I + g) + kDmmaLd * (8 * J + 2 * q)] = d0;
                sT[(8 * I + g) + kDmmaLd * (8 * J + 2 * q + 1)] = d1;
            }
        __syncwarp();
        // Kout += P_s^T T: A = P^T (8I.., 4kk..) = P(4kk.., 8I..), B = T(4kk.., 8J..)
#pragma unroll
        for (int I = 0; I < 3; ++I)
#pragma unroll
            for (int J = 0; J < 3; ++J)
#pragma unroll
                for (int kk = 0; kk < 6; ++kk)
                    dmma_8x8x4(acc[I][J][0], acc[I][J][1], __ldg(Ps + (4 * kk + q) + 24 * (8 * I + g)),
                               sT[(4 * kk + q) + kDmmaLd * (8 * J + g)]);
    }
    if (accumulate && !any) return;
    double *out = Ks + (size_t)e * 576;
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
        for (int J = 0; J < 3; ++J)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int idx = (8 * I + g) + 24 * (8 * J + 2 * q + h);
                out[idx] = accumulate ? out[idx] + acc[I][J][h] : acc[I][J][h];
            }
}
// Many children per coarse element (the 64 of a span-4 cell): one CTA per
// element, its kSplitWarps warps take children w, w + kSplitWarps, ... and the
// warps' partial sums are added in warp order through shared memory
// (deterministic), so a level with few coarse elements still fills the GPU.
constexpr int kSplitWarps = 8;

template <class ChildK, class Skip>
__global__ void __launch_bounds__(32 * kSplitWarps)
ptkp_dmma_split_kernel(double *__restrict__ Ks, const int32_t *__restrict__ upMap, int64_t nElem, int nCh,
                       const double *__restrict__ P, ChildK childK, Skip skip, int accumulate,
                       const int32_t *__restrict__ elist)
{
    extern __shared__ double dsm[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const int64_t e = elist ? (int64_t)elist[blockIdx.x] : (int64_t)blockIdx.x;
    double *sK = dsm + warp * 2 * 24 * kDmmaLd, *sT = sK + 24 * kDmmaLd;
    double *part = dsm + kSplitWarps * 2 * 24 * kDmmaLd;          // [kSplitWarps][576]
    __shared__ int anyW[kSplitWarps];
    double acc[3][3][2];
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
        for (int J = 0; J < 3; ++J) acc[I][J][0] = acc[I][J][1] = 0.0;
    bool any = false;
    for (int s = warp; s < nCh; s += kSplitWarps) {
        const int32_t f1 = upMap[e + (int64_t)s * nElem];
        if (f1 <= 0 || skip(f1 - 1)) continue;     // uniform across the warp
        any = true;
        const double *Ps = P + (size_t)s * 576;
        __syncwarp();
        for (int i = lane; i < 576; i += 32) sK[(i % 24) + kDmmaLd * (i / 24)] = childK(f1 - 1, i);
        __syncwarp();
#pragma unroll
        for (int I = 0; I < 3; ++I)
#pragma unroll
            for (int J = 0; J < 3; ++J) {
                double d0 = 0.0, d1 = 0.0;
#pragma unroll
                for (int kk = 0; kk < 6; ++kk)
                    dmma_8x8x4(d0, d1, sK[(8 * I + g) + kDmmaLd * (4 * kk + q)], __ldg(Ps + (4 * kk + q) + 24 * (8 * J + g)));
                sT[(8 * I + g) + kDmmaLd * (8 * J + 2 * q)] = d0;
                sT[(8 * I + g) + kDmmaLd * (8 * J + 2 * q + 1)] = d1;
            }
        __syncwarp();
#pragma unroll
        for (int I = 0; I < 3; ++I)
#pragma unroll
            for (int J = 0; J < 3; ++J)
#pragma unroll
                for (int kk = 0; kk < 6; ++kk)
                    dmma_8x8x4(acc[I][J][0], acc[I][J][1], __ldg(Ps + (4 * kk + q) + 24 * (8 * I + g)),
                               sT[(4 * kk + q) + kDmmaLd * (8 * J + g)]);
    }
#pragma unroll
    for (int I = 0; I < 3; ++I)
#pragma unroll
        for (int J = 0; J < 3; ++J)
#pragma unroll
            for (int h = 0; h < 2; ++h) part[warp * 576 + (8 * I + g) + 24 * (8 * J + 2 * q + h)] = acc[I][J][h];
    if (lane == 0) anyW[warp] = any ? 1 : 0;
    __syncthreads();
    bool anyC = false;
    for (int w = 0; w < kSplitWarps; ++w) anyC = anyC || anyW[w];
    if (accumulate && !anyC) return;
    double *out = Ks + (size_t)e * 576;
    for (int i = threadIdx.x; i < 576; i += 32 * kSplitWarps) {
        double v = part[i];
        for (int w = 1; w < kSplitWarps; ++w) v += part[w * 576 + i];
        out[i] = accumulate ? out[i] + v : v;
    }
}
constexpr size_t kSplitSmem = sizeof(double) * (kSplitWarps * 2 * 24 * kDmmaLd + kSplitWarps * 576);

// launch over nSel coarse elements (elist, or 0 .. nSel-1): children split
// over the warps of a CTA when a cell has many, one warp per cell otherwise
template <class ChildK, class Skip>
inline void ptkp_f64(cudaStream_t st, double *Ks, const int32_t *upMap, int64_t nElem, int nCh, const double *P,
                     ChildK childK, Skip skip, int accumulate, const int32_t *elist, int64_t nSel)
{
    if (nSel <= 0) return;
    if (nCh >= 2 * kSplitWarps) {
        static const bool attr = cudaFuncSetAttribute(ptkp_dmma_split_kernel<ChildK, Skip>,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSplitSmem) == cudaSuccess;
        (void)attr;
        ptkp_dmma_split_kernel<ChildK, Skip><<<(unsigned)nSel, 32 * kSplitWarps, kSplitSmem, st>>>(
            Ks, upMap, nElem, nCh, P, childK, skip, accumulate, elist);
        return;
    }
    ptkp_dmma_kernel<ChildK, Skip><<<(unsigned)((nSel + kDmmaWarps - 1) / kDmmaWarps), 32 * kDmmaWarps, 0, st>>>(
        Ks, upMap, nElem, nCh, P, childK, skip, accumulate, elist, nSel);
}

}  // namespace topgpu
