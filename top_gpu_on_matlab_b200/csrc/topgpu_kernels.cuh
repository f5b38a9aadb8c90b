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
    const int n0 = blockIdx.y * kGemmBN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // A tile: thread per (row, k) pair, 32 rows per pass
    for (int idx = tid; idx < kGemmBM * kGemmK; idx += 128) {
        const int r = idx % kGemmBM, k = idx / kGemmBM;
        const int64_t m = m0 + r;
        sA[r * (kGemmK + kGemmPad) + k] = (m < M) ? arow(m, k) : 0.0;
    }
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

constexpr size_t kGemmSmem = sizeof(double) * (kGemmBM * (kGemmK + kGemmPad) + kGemmK * (kGemmBN + kGemmPad));

}  // namespace topgpu
