// topgpu_dense.cuh -- dense FP64 linear algebra of the coarsest level: the
// Cholesky factor of the assembled coarsest matrix and its explicit inverse
// (the V-cycle's coarsest solve is one GEMV with it).
//
//   * factorisation: right-looking, 32-column blocks.  One warp factors a
//     diagonal block in registers (lane r holds row r) and forms its
//     triangular inverse; the panel below is a GEMM with that inverse
//     (L21 = A21 L11^-T) and the trailing update a lower-tile GEMM
//     (A22 -= L21 L21^T);
//   * W = L^-1 by 2x2 block inversion, [L11 0; L21 L22]^-1 =
//     [W11 0; -W22 L21 W11  W22], bottom-up from the factorisation's
//     diagonal blocks, every node of a level in one launch;
//   * A^-1 = W^T W, one GEMM that skips the zero blocks of W.
// All products go through one tiled GEMM (64 x 64 tiles, 4 x 4 outputs per
// thread, K steps of 16 staged in shared memory) over column-major matrices.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace topgpu {

constexpr int kDb = 32;          // diagonal block of the factorisation

// C(i, j) = alpha * sum_k a(i, k) b(j, k) + beta * C(i, j) for i < M, j < N,
// a(i, k) = TA ? A[k + lda i] : A[i + lda k] (likewise b).  lower: only tiles
// on or below the diagonal.  kFromTile: a(i, k) = 0 and b(j, k) = 0 for k
// below the tile's first row / column (triangular factors), so K starts at
// max(i0, j0).  C is written after all of a tile's reads, so C may alias A
// when every row block of C reads only its own rows of A.
template <bool TA, bool TB>
__global__ void __launch_bounds__(256)
dgemm_tile_kernel(double *C, int64_t ldc, const double *A, int64_t lda, const double *B, int64_t ldb,
                  int M, int N, int K, double alpha, double beta, int lower, int kFromTile)
{
    __shared__ double As[16][64 + 1], Bs[16][64 + 1];
    const int i0 = blockIdx.x * 64, j0 = blockIdx.y * 64;
    if (lower && j0 > i0) return;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4, t = threadIdx.x;
    double acc[4][4] = {};
    const int kStart = kFromTile ? ((i0 > j0 ? i0 : j0) / 16) * 16 : 0;
    for (int k0 = kStart; k0 < K; k0 += 16) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = t + 256 * q;             // 1024 elements of each 64 x 16 tile
            int ii, kk;
            if (TA) { kk = e % 16; ii = e / 16; } else { ii = e % 64; kk = e / 64; }
            const int i = i0 + ii, k = k0 + kk;
            As[kk][ii] = (i < M && k < K) ? (TA ? A[k + lda * i] : A[i + lda * k]) : 0.0;
            int jj, kb;
            if (TB) { kb = e % 16; jj = e / 16; } else { jj = e % 64; kb = e / 64; }
            const int j = j0 + jj, kq = k0 + kb;
            Bs[kb][jj] = (j < N && kq < K) ? (TB ? B[kq + ldb * j] : B[j + ldb * kq]) : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            double av[4], bv[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) { av[r] = As[kk][tx + 16 * r]; bv[r] = Bs[kk][ty + 16 * r]; }
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = fma(av[r], bv[c], acc[r][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int i = i0 + tx + 16 * r, j = j0 + ty + 16 * c;
            if (i < M && j < N) {
                double *p = C + i + ldc * j;
                *p = alpha * acc[r][c] + (beta != 0.0 ? beta * *p : 0.0);
            }
        }
}

// One level of the bottom-up block inversion of a lower-triangular L (n x n):
// node z covers rows [r0, r0 + 2 hs), r0 = 2 hs z, split at rh = r0 + hs; its
// two products, over blockIdx.z:
//   step 0:  T = L21 W11      (T stored where W21 goes in Tb)
//   step 1:  W21 = -W22 T
// W11 and W22 are complete from the level below.
__global__ void __launch_bounds__(256)
inv_level_kernel(const double *__restrict__ L, double *__restrict__ W, double *__restrict__ Tb, int64_t n, int hs, int step)
{
    const int64_t r0 = (int64_t)blockIdx.z * 2 * hs, rh = r0 + hs;
    if (rh >= n) return;
    const int64_t r1 = r0 + 2 * hs < n ? r0 + 2 * hs : n;
    const int s2 = (int)(r1 - rh);
    if ((int)blockIdx.x * 64 >= s2 || (int)blockIdx.y * 64 >= hs) return;
    __shared__ double As[16][64 + 1], Bs[16][64 + 1];
    const int i0 = blockIdx.x * 64, j0 = blockIdx.y * 64;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4, t = threadIdx.x;
    // step 0: a(i,k) = L[rh+i][r0+k], b(j,k) = W[r0+k][r0+j], K = hs (W11 lower: k >= j)
    // step 1: a(i,k) = W[rh+i][rh+k], b(j,k) = T[rh+k][r0+j], K = s2 (W22 lower: k <= i)
    const int K = step == 0 ? hs : s2;
    const int kBeg = step == 0 ? (j0 / 16) * 16 : 0;
    const int kEnd = step == 0 ? K : (i0 + 64 < K ? i0 + 64 : K);
    double acc[4][4] = {};
    for (int k0 = kBeg; k0 < kEnd; k0 += 16) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = t + 256 * q;
            const int ii = e % 64, kk = e / 64;            // a: column-major, consecutive i
            const int i = i0 + ii, k = k0 + kk;
            double av = 0.0;
            if (i < s2 && k < K) av = step == 0 ? L[(rh + i) + n * (r0 + k)] : W[(rh + i) + n * (rh + k)];
            As[kk][ii] = av;
            const int kb = e % 16, jj = e / 16;             // b: consecutive k
            const int j = j0 + jj, kq = k0 + kb;
            double bv = 0.0;
            if (j < hs && kq < K) bv = step == 0 ? W[(r0 + kq) + n * (r0 + j)] : Tb[(rh + kq) + n * (r0 + j)];
            Bs[kb][jj] = bv;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            double av[4], bv[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) { av[r] = As[kk][tx + 16 * r]; bv[r] = Bs[kk][ty + 16 * r]; }
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = fma(av[r], bv[c], acc[r][c]);
        }
        __syncthreads();
    }
    double *C = step == 0 ? Tb : W;
    const double alpha = step == 0 ? 1.0 : -1.0;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int i = i0 + tx + 16 * r, j = j0 + ty + 16 * c;
            if (i < s2 && j < hs) C[(rh + i) + n * (r0 + j)] = alpha * acc[r][c];
        }
}

// Cholesky of the diagonal block A[k0 .. k0+kb) (kb <= 32) by one warp, lane
// r holding row r; writes L11 over A's lower block and L11^-1 (lower, 32 x 32,
// rows/columns beyond kb the identity) to Dinv.  status: set when a pivot is
// not positive (the pivot is then taken as 1).
__global__ void __launch_bounds__(32) chol_block_kernel(double *A, int64_t n, int64_t k0, int kb, double *Dinv, int *status)
{
    const int r = threadIdx.x;
    double a[kDb];
#pragma unroll
    for (int c = 0; c < kDb; ++c)
        a[c] = (r < kb && c < kb && c <= r) ? A[(k0 + r) + n * (k0 + c)] : (c == r ? 1.0 : 0.0);
#pragma unroll
    for (int j = 0; j < kDb; ++j) {
        double d = __shfl_sync(0xffffffffu, a[j], j);
        if (!(d > 0.0)) { if (r == j) atomicExch(status, 1); d = 1.0; }
        const double ljj = sqrt(d), rl = 1.0 / ljj;    // the same in every lane
        if (r == j) a[j] = ljj;
        else if (r > j) a[j] *= rl;
#pragma unroll
        for (int c = j + 1; c < kDb; ++c) {
            const double lcj = __shfl_sync(0xffffffffu, a[j], c);   // L[c][j]
            if (r >= c) a[c] -= a[j] * lcj;
        }
    }
    // W = L11^-1 in registers, lane r holding row r of W (starting from I):
    // for j in order, row j is scaled by 1 / L[j][j] and then removed from the
    // rows below, w_r -= L[r][j] w_j (row j's entries from lane j by shuffles)
    double w[kDb];
#pragma unroll
    for (int c = 0; c < kDb; ++c) w[c] = c == r ? 1.0 : 0.0;
#pragma unroll
    for (int j = 0; j < kDb; ++j) {
        const double rjj = 1.0 / __shfl_sync(0xffffffffu, a[j], j);   // the same in every lane
        if (r == j)
#pragma unroll
            for (int c = 0; c <= j; ++c) w[c] *= rjj;
#pragma unroll
        for (int c = 0; c <= j; ++c) {
            const double wjc = __shfl_sync(0xffffffffu, w[c], j);
            if (r > j) w[c] -= a[j] * wjc;
        }
    }
    if (r < kb)
#pragma unroll
        for (int c = 0; c < kDb; ++c)
            if (c <= r && c < kb) A[(k0 + r) + n * (k0 + c)] = a[c];
#pragma unroll
    for (int c = 0; c < kDb; ++c) Dinv[r + kDb * c] = w[c];
}

// copy the diagonal blocks' inverses into W's diagonal blocks (upper parts zero)
__global__ void place_dinv_kernel(const double *__restrict__ Dinv, double *__restrict__ W, int64_t n)
{
    const int64_t b = blockIdx.x;
    const int r = threadIdx.x % kDb, c = threadIdx.x / kDb;      // 32 x 32 threads
    const int64_t i = b * kDb + r, j = b * kDb + c;
    if (i < n && j < n) W[i + n * j] = Dinv[b * kDb * kDb + r + kDb * c];
}

}  // namespace topgpu
