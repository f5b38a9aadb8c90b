// topgpu_walsh.cuh -- level-0 stiffness product in the Walsh-Hadamard basis
// of the voxel element.
//
// The 8-node unit-cube element of an isotropic material is invariant under
// the three axis reflections of the cube (a reflection along axis k swaps the
// corner pairs across k and flips the sign of displacement component k).
// Those reflections commute, so they diagonalise together: with the Walsh
// functions w_s(a) = (-1)^(s_y dy(a) + s_x dx(a) + s_z dz(a)) over the
// corners a (s = s_y + 2 s_x + 4 s_z), and U[c][s] = sum_a w_s(a) u[a][c],
//
//     Ke u = W (B U),   (W V)[a][c] = sum_s w_s(a) V[c][s],
//
// where B couples U[c][s] only to U[c'][s'] with s ^ e(c) == s' ^ e(c')
// (e(c) = the bit of component c's own axis): eight 3x3 blocks, one per
// character t = s ^ e(c), with 45 nonzero entries in all (the rest vanish
// by the cube's diagonal symmetries).  The element product then costs two
// 8-point Walsh transforms per component (add/subtract butterflies) plus
// 45 multiply-adds, instead of the 576 multiply-adds of the dense 24x24 Ke.
//
// The kernel marches along z through a 2-D tile of element columns: each
// thread owns one element column, keeps the (y, x) Walsh transform of the
// node layer below it from the previous step (the z butterfly is the only
// part that needs both layers), and sums the Walsh-domain output of the two
// elements sharing a node layer before transforming back.  Node sums across
// the four element columns around a node go through shared memory in a
// fixed order, so results are deterministic.  Tiles overlap by one column:
// a tile of TY x TX element columns produces (TY-1) x (TX-1) node columns.
#pragma once
#include "topgpu_grid.cuh"

namespace topgpu {

template <typename T> struct WalshParam { T b[8][9]; };   // B_t[c][c'] at b[t][3c+c']

// bit of s along the axis of displacement component c (x -> s_x, y -> s_y, z -> s_z)
__host__ __device__ constexpr int walsh_axis_bit(int c) { return c == 0 ? 2 : (c == 1 ? 1 : 4); }
// nonzero entries (bit 3c+c') of block t for the isotropic unit cube
__host__ __device__ constexpr unsigned walsh_pattern(int t)
{
    return t == 0 ? 0x1FFu : t == 1 ? 0x145u : t == 2 ? 0x1B0u : t == 3 ? 0x11Bu
         : t == 4 ? 0x01Bu : t == 5 ? 0x1B1u : t == 6 ? 0x155u : 0x1FFu;
}
__host__ __device__ constexpr int walsh_sign(int s, int a)
{
    return ((((s & 1) * cdy(a)) + (((s >> 1) & 1) * cdx(a)) + (((s >> 2) & 1) * cdz(a))) & 1) ? -1 : 1;
}

// Blocks of Ke (column-major 24x24, corner order of the element node map)
// in the Walsh basis, scaled by 1/64.  Returns the largest entry of Ke's
// Walsh form outside the block pattern relative to max |Ke|: zero up to
// rounding for a cube element of an isotropic material.
inline double walsh_blocks(const double *Ke, WalshParam<double> &P)
{
    double kmax = 0.0, off = 0.0;
    for (int i = 0; i < 576; ++i) kmax = Ke[i] > kmax ? Ke[i] : (-Ke[i] > kmax ? -Ke[i] : kmax);
    for (int s = 0; s < 8; ++s)
        for (int c = 0; c < 3; ++c)
            for (int s2 = 0; s2 < 8; ++s2)
                for (int d = 0; d < 3; ++d) {
                    double m = 0.0;
                    for (int a = 0; a < 8; ++a)
                        for (int b = 0; b < 8; ++b)
                            m += walsh_sign(s, a) * Ke[(3 * a + c) + 24 * (3 * b + d)] * walsh_sign(s2, b);
                    m /= 64.0;
                    const int t = s ^ walsh_axis_bit(c);
                    const bool inBlock = (s2 ^ walsh_axis_bit(d)) == t && ((walsh_pattern(t) >> (3 * c + d)) & 1u);
                    if (inBlock) P.b[t][3 * c + d] = m;
                    else off = (m < 0 ? -m : m) > off ? (m < 0 ? -m : m) : off;
                }
    for (int t = 0; t < 8; ++t)
        for (int k = 0; k < 9; ++k)
            if (!((walsh_pattern(t) >> k) & 1u)) P.b[t][k] = 0.0;
    return kmax > 0 ? off / kmax : 0.0;
}

// (y, x) butterfly of four corner values v[by + 2 bx]; its own inverse up to 1/4
template <typename T>
__device__ __forceinline__ void walsh2(T v[4])
{
    const T p0 = v[0] + v[1], m0 = v[0] - v[1], p1 = v[2] + v[3], m1 = v[2] - v[3];
    v[0] = p0 + p1; v[1] = m0 + m1; v[2] = p0 - p1; v[3] = m0 - m1;
}

template <typename T, int TY, int TX> struct WalshTile {
    static constexpr int NT = TY * TX;                      // threads = element columns
    static constexpr int NS = (TY + 1) * (TX + 1);          // staged node columns
    static constexpr int R = (3 * NS + NT - 1) / NT;        // staged values per thread
    // y stride of a staged column in shared memory, chosen so that the
    // (ty + by, tx + bx) reads of a warp (of a half-warp for 8-byte values)
    // fall in distinct banks
    static constexpr int SY = sizeof(T) == 4 ? (TY < 32 ? TY + 32 : TY + 1) : (TY == 8 ? 24 : TY + 1);
    static constexpr int SC = SY * (TX + 1);                // one component
};

__host__ __device__ inline int walsh_tiles(const Geom &g, int TY, int TX)
{
    return ((g.NY + TY - 2) / (TY - 1)) * ((g.NX + TX - 2) / (TX - 1));
}

// one z-range [z0, z1) of node layers of tile (y0, x0): element layers
// z0-1 .. z1-1 are visited, the first only for its top-layer carry
template <typename T, int TY, int TX, bool MASK, class In, class Out>
__device__ __forceinline__ void l0w_march(const WalshParam<T> &B, const In &in, const Out &out,
                                          const T *__restrict__ E, const uint8_t *__restrict__ flags,
                                          const Geom &g, int y0, int x0, int z0, int z1, T E0,
                                          T *su, T *so, double &dot)
{
    using Tl = WalshTile<T, TY, TX>;
    const int tid = threadIdx.x, ty = tid % TY, tx = tid / TY;
    const int PY = g.PY, PL = (int)g.plane;
    // staged node columns of this thread: (Y, X) = (y0-1+j, x0-1+i); outside
    // [-1, NY] x [-1, NX] they are not guard slots and stage as zero
    int sOff[Tl::R], sComp[Tl::R], sDst[Tl::R];
    bool sOn[Tl::R];
#pragma unroll
    for (int r = 0; r < Tl::R; ++r) {
        const int k = tid + r * Tl::NT;
        const int c = k / Tl::NS, q = k % Tl::NS, j = q % (TY + 1), i = q / (TY + 1);
        const int Y = y0 - 1 + j, X = x0 - 1 + i;
        sOn[r] = k < 3 * Tl::NS && Y <= g.NY && X <= g.NX;
        sComp[r] = c < 3 ? c : 0;
        sDst[r] = k < 3 * Tl::NS ? c * Tl::SC + j + Tl::SY * i : -1;
        sOff[r] = sOn[r] ? (int)(g.origin + Y + (int64_t)PY * X) : 0;
    }
    T pre[Tl::R];
    auto fetch = [&](int z) {
#pragma unroll
        for (int r = 0; r < Tl::R; ++r) {
            T v = T(0);
            if (sOn[r]) {
                const int m = sOff[r] + PL * z;
                v = in(m, sComp[r]);
                if (MASK && (flags[m] & (1 << sComp[r]))) v = T(0);
            }
            pre[r] = v;
        }
    };
    auto stage = [&]() {
#pragma unroll
        for (int r = 0; r < Tl::R; ++r)
            if (sDst[r] >= 0) su[sDst[r]] = pre[r];
    };
    // element column of this thread
    const int ey = y0 - 1 + ty, ex = x0 - 1 + tx;
    const bool eOn = ey <= g.NY - 1 && ex <= g.NX - 1;
    const int eOff = eOn ? (int)(g.origin + ey + (int64_t)PY * ex) : 0;
    // node of this thread (corner (0,0) of its element column) and whether it is an output
    const bool nOut = ty >= 1 && tx >= 1 && ey < g.NY && ex < g.NX;
    auto corners = [&](T h[3][4]) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
            for (int bx = 0; bx < 2; ++bx)
#pragma unroll
                for (int by = 0; by < 2; ++by)
                    h[c][by + 2 * bx] = su[c * Tl::SC + (ty + by) + Tl::SY * (tx + bx)];
            walsh2(h[c]);
        }
    };

    T hb[3][4], gt[3][4];
    fetch(z0 - 1);
    __syncthreads();                     // the previous range's reads of su / so are done
    stage();
    fetch(z0);
    T eNext = eOn ? E[eOff + PL * (z0 - 1)] : T(0);
    __syncthreads();
    corners(hb);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k) gt[c][k] = T(0);

    for (int ez = z0 - 1; ez < z1; ++ez) {
        __syncthreads();                 // every read of su / so of the previous step is done
        stage();                         // node layer ez + 1
        if (ez + 2 <= z1) fetch(ez + 2);
        const T Ee = eNext;
        if (ez + 1 < z1) eNext = eOn ? E[eOff + PL * (ez + 1)] : T(0);
        __syncthreads();
        T ht[3][4];
        corners(ht);
        // z butterfly and modulus: U[c][s], s = sxy + 4 sz
        T U[3][8];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                U[c][k] = Ee * (hb[c][k] + ht[c][k]);
                U[c][k + 4] = Ee * (hb[c][k] - ht[c][k]);
                hb[c][k] = ht[c][k];
            }
        // block products V[c][t ^ e(c)] = sum_c' B_t[c][c'] U[c'][t ^ e(c')]
        T V[3][8];
#pragma unroll
        for (int t = 0; t < 8; ++t)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                T acc = T(0);
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if ((walsh_pattern(t) >> (3 * c + d)) & 1u) acc = fma(B.b[t][3 * c + d], U[d][t ^ walsh_axis_bit(d)], acc);
                V[c][t ^ walsh_axis_bit(c)] = acc;
            }
        // back along z: the bottom layer (ez) is complete with the carry of
        // element ez-1's top layer; this element's top layer is the new carry
        T G[3][4];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                G[c][k] = gt[c][k] + (V[c][k] + V[c][k + 4]);
                gt[c][k] = V[c][k] - V[c][k + 4];
            }
        if (ez < z0) continue;           // first element: its bottom layer is not in this range
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            walsh2(G[c]);
#pragma unroll
            for (int k = 1; k < 4; ++k) so[((k - 1) * 3 + c) * Tl::NT + tid] = G[c][k];
        }
        __syncthreads();
        if (nOut) {
            T y[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                y[c] = G[c][0] + so[(0 * 3 + c) * Tl::NT + tid - 1]          // corner (1,0) of column (ty-1, tx)
                               + so[(1 * 3 + c) * Tl::NT + tid - TY]         // corner (0,1) of column (ty, tx-1)
                               + so[(2 * 3 + c) * Tl::NT + tid - TY - 1];    // corner (1,1) of column (ty-1, tx-1)
            const int idx = eOff + PL * ez;
            if (MASK) {
                const uint8_t f = flags[idx];
#pragma unroll
                for (int c = 0; c < 3; ++c) if (f & (1 << c)) y[c] = E0 * in(idx, c);
            }
            out(idx, y, dot);
        }
    }
}

// Work = (tile, node layer) pairs, tile-major; CTA b takes the contiguous
// share [b W / n, (b+1) W / n) and marches each tile's part of it along z,
// so every CTA gets the same number of layers whatever the grid size.
// resident CTAs per SM the register budget is fitted to
template <typename T, int NT> struct WalshOcc {
    static constexpr int value = sizeof(T) == 4 ? (NT >= 256 ? 3 : 6) : (NT >= 256 ? 1 : 3);
};
// the direct-load kernel keeps its epilogue's prefetched inputs in registers:
// one resident CTA fewer for an FP32 epilogue that prefetches more than
// three values (post-smoothing: x, invD, r), which would spill at 80 registers
template <typename T, int NT, class Out> struct WalshOccD {
    static constexpr int value = WalshOcc<T, NT>::value - ((sizeof(T) == 4 && sizeof(typename Out::Pre) > 24) ? 1 : 0);
};

template <typename T, int TY, int TX, class In, class Out>
__global__ void __launch_bounds__(TY * TX, WalshOcc<T, TY * TX>::value)
l0w_kernel(const WalshParam<T> B, In in0, Out out0, const T *__restrict__ E, const uint8_t *__restrict__ flags,
           const uint8_t *__restrict__ tileMask, Geom g, T E0, Reduce red0, const int *__restrict__ done0)
{
    pdl_enter();
    const int vk = blockIdx.y;          // right-hand side of a batched launch
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    const In in = in0.shift(vk); const Out out = out0.shift(vk); const Reduce red = red0.at(vk);
    using Tl = WalshTile<T, TY, TX>;
    __shared__ T su[3 * Tl::SC];
    __shared__ T so[9 * Tl::NT];
    const int tilesY = (g.NY + TY - 2) / (TY - 1);
    const int64_t total = (int64_t)walsh_tiles(g, TY, TX) * g.NZ;
    int64_t a = total * blockIdx.x / gridDim.x;
    const int64_t b = total * (blockIdx.x + 1) / gridDim.x;
    double dot = 0.0;
    while (a < b) {
        const int tile = (int)(a / g.NZ), z0 = (int)(a % g.NZ);
        const int z1 = (int)(z0 + (b - a) < g.NZ ? z0 + (b - a) : g.NZ);
        const int y0 = (tile % tilesY) * (TY - 1), x0 = (tile / tilesY) * (TX - 1);
        if (tileMask[tile])
            l0w_march<T, TY, TX, true>(B, in, out, E, flags, g, y0, x0, z0, z1, E0, su, so, dot);
        else
            l0w_march<T, TY, TX, false>(B, in, out, E, flags, g, y0, x0, z0, z1, E0, su, so, dot);
        a += z1 - z0;
    }
    if (red.result) block_sum_to<TY * TX>(dot, red.partials, red.counter, red.result, gridDim.x, blockIdx.x);
}

// tileMask[tile] = 1 when a node staged by that tile (any layer) has a fixed component
template <int TY, int TX>
__global__ void __launch_bounds__(256)
walsh_mask_kernel(const uint8_t *__restrict__ flags, Geom g, uint8_t *__restrict__ tileMask)
{
    const int tilesY = (g.NY + TY - 2) / (TY - 1);
    const int y0 = (blockIdx.x % tilesY) * (TY - 1), x0 = (blockIdx.x / tilesY) * (TX - 1);
    int any = 0;
    const int ny = TY + 1, nx = TX + 1;
    for (int k = threadIdx.x; k < ny * nx * g.NZ; k += blockDim.x) {
        const int Y = y0 - 1 + k % ny, X = x0 - 1 + (k / ny) % nx, Z = k / (ny * nx);
        if (Y < 0 || Y >= g.NY || X < 0 || X >= g.NX) continue;
        any |= flags[g.origin + Y + (int64_t)g.PY * X + g.plane * Z] & kFixedMask;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) tileMask[blockIdx.x] = any ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Pair variant: every thread owns two element columns adjacent in y and runs
// the whole Walsh pipeline on (element A, element B) pairs -- in FP32 with
// the sm_100 paired instructions (__fadd2_rn / __fmul2_rn / __ffma2_rn), so
// each add, multiply and multiply-add serves both elements.  A tile of
// TYP x TX threads covers 2 TYP x TX element columns and produces
// (2 TYP - 1) x (TX - 1) node columns.
template <typename T> struct PairOf;
template <> struct PairOf<float> { using type = float2; };
template <> struct PairOf<double> { using type = double2; };

__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ double2 padd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 psub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 pmul(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ double2 pfma(double2 a, double2 b, double2 c) { return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)); }

template <typename T> struct WalshPairParam { typename PairOf<T>::type b[8][9]; };   // (B, B) pairs

template <typename T, int TYP, int TX> struct WalshPairTile {
    static constexpr int NT = TYP * TX;
    static constexpr int EY = 2 * TYP;                      // element rows of a tile
    static constexpr int NS = (EY + 1) * (TX + 1);          // staged node columns
    static constexpr int R = (NS + NT - 1) / NT;            // staged node columns per thread
    static constexpr int SY = EY + 2;                       // even: rows (2ty, 2ty+1) load as one pair
    static constexpr int SC = SY * (TX + 1);
};

__host__ __device__ inline int walsh_pair_tiles(const Geom &g, int TYP, int TX)
{
    return ((g.NY + 2 * TYP - 2) / (2 * TYP - 1)) * ((g.NX + TX - 2) / (TX - 1));
}

template <typename T, int TYP, int TX, bool MASK, class In, class Out>
__device__ __forceinline__ void l0p_march(const WalshPairParam<T> &B, const In &in, const Out &out,
                                          const T *__restrict__ E, const uint8_t *__restrict__ flags,
                                          const Geom &g, int y0, int x0, int z0, int z1, T E0,
                                          T *su, T *so, double &dot)
{
    using P2 = typename PairOf<T>::type;
    using Tl = WalshPairTile<T, TYP, TX>;
    const int tid = threadIdx.x, ty = tid % TYP, tx = tid / TYP;
    const int PY = g.PY, PL = (int)g.plane;
    // staged node columns (Y, X) = (y0-1+j, x0-1+i), all three components
    int sOff[Tl::R], sDst[Tl::R];
#pragma unroll
    for (int r = 0; r < Tl::R; ++r) {
        const int q = tid + r * Tl::NT, j = q % (Tl::EY + 1), i = q / (Tl::EY + 1);
        const int Y = y0 - 1 + j, X = x0 - 1 + i;
        const bool on = q < Tl::NS && Y <= g.NY && X <= g.NX;
        sDst[r] = q < Tl::NS ? j + Tl::SY * i : -1;
        sOff[r] = on ? (int)(g.origin + Y + (int64_t)PY * X) : -1;
    }
    T pre[Tl::R][3];
    auto fetch = [&](int z) {
#pragma unroll
        for (int r = 0; r < Tl::R; ++r) {
            const int m = sOff[r] + PL * z;
            uint8_t f = 0;
            if (MASK && sOff[r] >= 0) f = flags[m];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                T v = T(0);
                if (sOff[r] >= 0) v = in(m, c);
                if (MASK && (f & (1 << c))) v = T(0);
                pre[r][c] = v;
            }
        }
    };
    auto stage = [&]() {
#pragma unroll
        for (int r = 0; r < Tl::R; ++r)
            if (sDst[r] >= 0) {
#pragma unroll
                for (int c = 0; c < 3; ++c) su[c * Tl::SC + sDst[r]] = pre[r][c];
            }
    };
    // element columns (ey, ey + 1) x ex of this thread
    const int ey = y0 - 1 + 2 * ty, ex = x0 - 1 + tx;
    const bool eOnA = ey <= g.NY - 1 && ex <= g.NX - 1, eOnB = ey + 1 <= g.NY - 1 && ex <= g.NX - 1;
    const int eOff = (int)(g.origin + ey + (int64_t)PY * ex);
    // nodes (ey, ex) and (ey + 1, ex): corner (0,0) of elements A and B
    const bool outA = ty >= 1 && tx >= 1 && ey < g.NY && ex < g.NX;
    const bool outB = tx >= 1 && ey + 1 < g.NY && ex < g.NX;
    // (y, x) Walsh transform of the current node layer, as (A, B) pairs
    auto corners = [&](P2 h[3][4]) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
#pragma unroll
            for (int bx = 0; bx < 2; ++bx) {
                const T *col = su + c * Tl::SC + Tl::SY * (tx + bx) + 2 * ty;
                const P2 lo = *reinterpret_cast<const P2 *>(col);     // rows 2ty, 2ty+1
                const T hi = col[2];                                   // row 2ty+2
                h[c][2 * bx] = lo;
                h[c][2 * bx + 1].x = lo.y; h[c][2 * bx + 1].y = hi;
            }
            const P2 p0 = padd(h[c][0], h[c][1]), m0 = psub(h[c][0], h[c][1]);
            const P2 p1 = padd(h[c][2], h[c][3]), m1 = psub(h[c][2], h[c][3]);
            h[c][0] = padd(p0, p1); h[c][1] = padd(m0, m1); h[c][2] = psub(p0, p1); h[c][3] = psub(m0, m1);
        }
    };
    auto eload = [&](int ez) {
        P2 e;
        e.x = eOnA ? E[eOff + PL * ez] : T(0);
        e.y = eOnB ? E[eOff + 1 + PL * ez] : T(0);
        return e;
    };

    P2 hb[3][4], gt[3][4];
    fetch(z0 - 1);
    __syncthreads();                     // the previous range's reads of su / so are done
    stage();
    fetch(z0);
    P2 eNext = eload(z0 - 1);
    __syncthreads();
    corners(hb);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k) { gt[c][k].x = T(0); gt[c][k].y = T(0); }

    for (int ez = z0 - 1; ez < z1; ++ez) {
        __syncthreads();
        stage();                         // node layer ez + 1
        if (ez + 2 <= z1) fetch(ez + 2);
        const P2 Ee = eNext;
        if (ez + 1 < z1) eNext = eload(ez + 1);
        __syncthreads();
        P2 U[3][8];
        {
            P2 ht[3][4];
            corners(ht);
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    U[c][k] = pmul(Ee, padd(hb[c][k], ht[c][k]));
                    U[c][k + 4] = pmul(Ee, psub(hb[c][k], ht[c][k]));
                    hb[c][k] = ht[c][k];
                }
        }
        // block products, in place: block t reads and writes U[c][t ^ e(c)]
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            P2 v[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                P2 acc; acc.x = T(0); acc.y = T(0);
                bool first = true;
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if ((walsh_pattern(t) >> (3 * c + d)) & 1u) {
                        const P2 u = U[d][t ^ walsh_axis_bit(d)];
                        acc = first ? pmul(B.b[t][3 * c + d], u) : pfma(B.b[t][3 * c + d], u, acc);
                        first = false;
                    }
                v[c] = acc;
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) U[c][t ^ walsh_axis_bit(c)] = v[c];
        }
        // back along z with the carry; this element's top layer is the new carry
        P2 G[3][4];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                G[c][k] = padd(gt[c][k], padd(U[c][k], U[c][k + 4]));
                gt[c][k] = psub(U[c][k], U[c][k + 4]);
            }
        if (ez < z0) continue;
        // back in (y, x): corner k = by + 2 bx of (A, B)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const P2 p0 = padd(G[c][0], G[c][1]), m0 = psub(G[c][0], G[c][1]);
            const P2 p1 = padd(G[c][2], G[c][3]), m1 = psub(G[c][2], G[c][3]);
            G[c][0] = padd(p0, p1); G[c][1] = padd(m0, m1); G[c][2] = psub(p0, p1); G[c][3] = psub(m0, m1);
            // to neighbours: X0 = B(1,0) -> (ty+1, tx); (X1, X2) = (A(0,1), B(0,1) + A(1,1)) -> (ty, tx+1);
            // X3 = B(1,1) -> (ty+1, tx+1)
            so[(0 * 3 + c) * Tl::NT + tid] = G[c][1].y;
            P2 x12; x12.x = G[c][2].x; x12.y = G[c][2].y + G[c][3].x;
            reinterpret_cast<P2 *>(so + 3 * Tl::NT)[c * Tl::NT + tid] = x12;
            so[(9 + c) * Tl::NT + tid] = G[c][3].y;
        }
        __syncthreads();
        T yA[3], yB[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            P2 x12; x12.x = T(0); x12.y = T(0);
            if (tx >= 1) x12 = reinterpret_cast<const P2 *>(so + 3 * Tl::NT)[c * Tl::NT + tid - TYP];
            const T x0 = ty >= 1 ? so[(0 * 3 + c) * Tl::NT + tid - 1] : T(0);
            const T x3 = (ty >= 1 && tx >= 1) ? so[(9 + c) * Tl::NT + tid - TYP - 1] : T(0);
            yA[c] = G[c][0].x + x0 + x12.x + x3;
            yB[c] = G[c][0].y + G[c][1].x + x12.y;
        }
        const int idx = eOff + PL * ez;
        if (outA) {
            if (MASK) {
                const uint8_t f = flags[idx];
#pragma unroll
                for (int c = 0; c < 3; ++c) if (f & (1 << c)) yA[c] = E0 * in(idx, c);
            }
            out(idx, yA, dot);
        }
        if (outB) {
            if (MASK) {
                const uint8_t f = flags[idx + 1];
#pragma unroll
                for (int c = 0; c < 3; ++c) if (f & (1 << c)) yB[c] = E0 * in(idx + 1, c);
            }
            out(idx + 1, yB, dot);
        }
    }
}

template <typename T, int NT> struct WalshPairOcc {
    static constexpr int value = NT >= 256 ? 1 : 3;
};

template <typename T, int TYP, int TX, class In, class Out>
__global__ void __launch_bounds__(TYP * TX, WalshPairOcc<T, TYP * TX>::value)
l0p_kernel(const WalshPairParam<T> B, In in0, Out out0, const T *__restrict__ E, const uint8_t *__restrict__ flags,
           const uint8_t *__restrict__ tileMask, Geom g, T E0, Reduce red0, const int *__restrict__ done0)
{
    pdl_enter();
    const int vk = blockIdx.y;          // right-hand side of a batched launch
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    const In in = in0.shift(vk); const Out out = out0.shift(vk); const Reduce red = red0.at(vk);
    using Tl = WalshPairTile<T, TYP, TX>;
    __shared__ __align__(16) T su[3 * Tl::SC];
    __shared__ __align__(16) T so[12 * Tl::NT];
    const int tilesY = (g.NY + 2 * TYP - 2) / (2 * TYP - 1);
    const int64_t total = (int64_t)walsh_pair_tiles(g, TYP, TX) * g.NZ;
    int64_t a = total * blockIdx.x / gridDim.x;
    const int64_t b = total * (blockIdx.x + 1) / gridDim.x;
    double dot = 0.0;
    while (a < b) {
        const int tile = (int)(a / g.NZ), z0 = (int)(a % g.NZ);
        const int z1 = (int)(z0 + (b - a) < g.NZ ? z0 + (b - a) : g.NZ);
        const int y0 = (tile % tilesY) * (2 * TYP - 1), x0 = (tile / tilesY) * (TX - 1);
        if (tileMask[tile])
            l0p_march<T, TYP, TX, true>(B, in, out, E, flags, g, y0, x0, z0, z1, E0, su, so, dot);
        else
            l0p_march<T, TYP, TX, false>(B, in, out, E, flags, g, y0, x0, z0, z1, E0, su, so, dot);
        a += z1 - z0;
    }
    if (red.result) block_sum_to<TYP * TX>(dot, red.partials, red.counter, red.result, gridDim.x, blockIdx.x);
}

// tileMask[tile] for the pair tiling: any staged node with a fixed component
template <int TYP, int TX>
__global__ void __launch_bounds__(256)
walsh_pair_mask_kernel(const uint8_t *__restrict__ flags, Geom g, uint8_t *__restrict__ tileMask)
{
    const int tilesY = (g.NY + 2 * TYP - 2) / (2 * TYP - 1);
    const int y0 = (blockIdx.x % tilesY) * (2 * TYP - 1), x0 = (blockIdx.x / tilesY) * (TX - 1);
    int any = 0;
    const int ny = 2 * TYP + 1, nx = TX + 1;
    for (int k = threadIdx.x; k < ny * nx * g.NZ; k += blockDim.x) {
        const int Y = y0 - 1 + k % ny, X = x0 - 1 + (k / ny) % nx, Z = k / (ny * nx);
        if (Y < 0 || Y >= g.NY || X < 0 || X >= g.NX) continue;
        any |= flags[g.origin + Y + (int64_t)g.PY * X + g.plane * Z] & kFixedMask;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) tileMask[blockIdx.x] = any ? 1 : 0;
}

// ---------------------------------------------------------------------------
// Direct-load variant of the single-column kernel: each thread reads the
// four top corner nodes of its element column straight from global memory
// (L1-cached: every node is read by the four columns around it, two of them
// in the same warp), one layer ahead in registers; the epilogue's inputs at
// the thread's output node are loaded at the start of the layer, so their
// latency hides behind the layer's arithmetic.  Only the node sums go
// through shared memory, double-buffered, so a layer costs one barrier.
template <typename T, int TY, int TX, bool MASK, class In, class Out>
__device__ __forceinline__ void l0d_march(const WalshParam<T> &B, const In &in, const Out &out,
                                          const T *__restrict__ E, const uint8_t *__restrict__ flags,
                                          const Geom &g, int y0, int x0, int z0, int z1, T E0,
                                          T *so, double &dot)
{
    constexpr int NT = TY * TX;
    const int tid = threadIdx.x, ty = tid % TY, tx = tid / TY;
    const int PY = g.PY, PL = (int)g.plane;
    const int ey = y0 - 1 + ty, ex = x0 - 1 + tx;
    // the column's corners (ey + by, ex + bx) lie in [-1, NY] x [-1, NX] (guard
    // slots included) exactly when the column is at most one past the last element
    const bool cOn = ey <= g.NY - 1 && ex <= g.NX - 1;
    const int base = cOn ? (int)(g.origin + ey + (int64_t)PY * ex) : 0;
    const bool nOut = ty >= 1 && tx >= 1 && ey < g.NY && ex < g.NX;
    auto load = [&](int z, T v[3][4]) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int m = base + (k & 1) + PY * (k >> 1) + PL * z;
            uint8_t f = 0;
            if (MASK && cOn) f = flags[m];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                T u = cOn ? in(m, c) : T(0);
                if (MASK && (f & (1 << c))) u = T(0);
                v[c][k] = u;
            }
        }
    };
    auto eload = [&](int z) { return cOn ? E[base + PL * z] : T(0); };

    T hb[3][4], gt[3][4], pre[3][4];
    __syncthreads();                     // the previous range's reads of so are done
    load(z0 - 1, hb);
#pragma unroll
    for (int c = 0; c < 3; ++c) walsh2(hb[c]);
    load(z0, pre);
    T eNext = eload(z0 - 1);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k) gt[c][k] = T(0);

    for (int ez = z0 - 1; ez < z1; ++ez) {
        // this layer's epilogue inputs, loaded now and used after the product
        typename Out::Pre po{};
        if (nOut && ez >= z0) po = out.pre(base + PL * ez);
        T ht[3][4];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 4; ++k) ht[c][k] = pre[c][k];
        if (ez + 2 <= z1) load(ez + 2, pre);
        const T Ee = eNext;
        if (ez + 1 < z1) eNext = eload(ez + 1);
        T U[3][8];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            walsh2(ht[c]);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if constexpr (sizeof(T) == 4) {
                    // FP32: E (hb +- ht) as one multiply and two multiply-adds (12
                    // fewer issued operations per element layer); FP64 keeps the
                    // sum-then-scale rounding of the parity-tested outer product
                    const T a = Ee * ht[c][k];
                    U[c][k] = fma(Ee, hb[c][k], a);
                    U[c][k + 4] = fma(Ee, hb[c][k], -a);
                } else {
                    U[c][k] = Ee * (hb[c][k] + ht[c][k]);
                    U[c][k + 4] = Ee * (hb[c][k] - ht[c][k]);
                }
                hb[c][k] = ht[c][k];
            }
        }
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            T v[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                T acc = T(0);
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if ((walsh_pattern(t) >> (3 * c + d)) & 1u) acc = fma(B.b[t][3 * c + d], U[d][t ^ walsh_axis_bit(d)], acc);
                v[c] = acc;
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) U[c][t ^ walsh_axis_bit(c)] = v[c];
        }
        T G[3][4];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                G[c][k] = gt[c][k] + (U[c][k] + U[c][k + 4]);
                gt[c][k] = U[c][k] - U[c][k + 4];
            }
        if (ez < z0) continue;
        T *buf = so + (ez & 1) * 9 * NT;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            walsh2(G[c]);
#pragma unroll
            for (int k = 1; k < 4; ++k) buf[((k - 1) * 3 + c) * NT + tid] = G[c][k];
        }
        __syncthreads();
        if (nOut) {
            T y[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                y[c] = G[c][0] + buf[(0 * 3 + c) * NT + tid - 1] + buf[(1 * 3 + c) * NT + tid - TY]
                               + buf[(2 * 3 + c) * NT + tid - TY - 1];
            const int idx = base + PL * ez;
            if (MASK) {
                const uint8_t f = flags[idx];
#pragma unroll
                for (int c = 0; c < 3; ++c) if (f & (1 << c)) y[c] = E0 * in(idx, c);
            }
            out.apply(idx, y, po, dot);
        }
    }
}

// FP32 form of l0d_march with displacement components 0 and 1 carried as one
// float2 through every step that treats the components alike (the (y, x)
// and z butterflies, the modulus, the node sums): those run as the paired
// sm_100 instructions (__fadd2_rn / __fmul2_rn / __ffma2_rn), one issue for
// two values; component 2 and the block products, which mix the components,
// stay scalar.  The same operations in the same order as l0d_march, so the
// results are bit-identical; about a quarter fewer floating-point
// instructions per element layer.
__device__ __forceinline__ void walsh2p(float2 v[4])
{
    const float2 p0 = padd(v[0], v[1]), m0 = psub(v[0], v[1]), p1 = padd(v[2], v[3]), m1 = psub(v[2], v[3]);
    v[0] = padd(p0, p1); v[1] = padd(m0, m1); v[2] = psub(p0, p1); v[3] = psub(m0, m1);
}
template <int TY, int TX, bool MASK, class In, class Out>
__device__ __forceinline__ void l0d_march_c2(const WalshParam<float> &B, const In &in, const Out &out,
                                             const float *__restrict__ E, const uint8_t *__restrict__ flags,
                                             const Geom &g, int y0, int x0, int z0, int z1, float E0,
                                             float *so, double &dot)
{
    constexpr int NT = TY * TX;
    const int tid = threadIdx.x, ty = tid % TY, tx = tid / TY;
    const int PY = g.PY, PL = (int)g.plane;
    const int ey = y0 - 1 + ty, ex = x0 - 1 + tx;
    const bool cOn = ey <= g.NY - 1 && ex <= g.NX - 1;
    const int base = cOn ? (int)(g.origin + ey + (int64_t)PY * ex) : 0;
    const bool nOut = ty >= 1 && tx >= 1 && ey < g.NY && ex < g.NX;
    auto load = [&](int z, float2 v01[4], float v2[4]) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int m = base + (k & 1) + PY * (k >> 1) + PL * z;
            uint8_t f = 0;
            if (MASK && cOn) f = flags[m];
            float u0 = cOn ? in(m, 0) : 0.f, u1 = cOn ? in(m, 1) : 0.f, u2 = cOn ? in(m, 2) : 0.f;
            if (MASK) {
                if (f & 1) u0 = 0.f;
                if (f & 2) u1 = 0.f;
                if (f & 4) u2 = 0.f;
            }
            v01[k] = make_float2(u0, u1);
            v2[k] = u2;
        }
    };
    auto eload = [&](int z) { return cOn ? E[base + PL * z] : 0.f; };

    float2 hb01[4], gt01[4], pre01[4];
    float hb2[4], gt2[4], pre2[4];
    __syncthreads();                     // the previous range's reads of so are done
    load(z0 - 1, hb01, hb2);
    walsh2p(hb01);
    walsh2(hb2);
    load(z0, pre01, pre2);
    float eNext = eload(z0 - 1);
#pragma unroll
    for (int k = 0; k < 4; ++k) { gt01[k] = make_float2(0.f, 0.f); gt2[k] = 0.f; }

    for (int ez = z0 - 1; ez < z1; ++ez) {
        typename Out::Pre po{};
        if (nOut && ez >= z0) po = out.pre(base + PL * ez);
        float2 ht01[4];
        float ht2[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) { ht01[k] = pre01[k]; ht2[k] = pre2[k]; }
        if (ez + 2 <= z1) load(ez + 2, pre01, pre2);
        const float Ee = eNext;
        if (ez + 1 < z1) eNext = eload(ez + 1);
        const float2 EE = make_float2(Ee, Ee);
        walsh2p(ht01);
        walsh2(ht2);
        // U[c][k] = E (hb + ht), U[c][k + 4] = E (hb - ht): components 0, 1 paired
        float2 U01[8];
        float U2[8];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 a = pmul(EE, ht01[k]);
            U01[k] = pfma(EE, hb01[k], a);
            U01[k + 4] = pfma(EE, hb01[k], make_float2(-a.x, -a.y));
            hb01[k] = ht01[k];
            const float a2 = Ee * ht2[k];
            U2[k] = fmaf(Ee, hb2[k], a2);
            U2[k + 4] = fmaf(Ee, hb2[k], -a2);
            hb2[k] = ht2[k];
        }
        // block products (mix the components): scalar
        auto Uv = [&](int d, int j) { return d == 0 ? U01[j].x : (d == 1 ? U01[j].y : U2[j]); };
        float2 V01[8];
        float V2[8];
#pragma unroll
        for (int t = 0; t < 8; ++t)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float acc = 0.f;
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if ((walsh_pattern(t) >> (3 * c + d)) & 1u) acc = fmaf(B.b[t][3 * c + d], Uv(d, t ^ walsh_axis_bit(d)), acc);
                const int j = t ^ walsh_axis_bit(c);
                if (c == 0) V01[j].x = acc;
                else if (c == 1) V01[j].y = acc;
                else V2[j] = acc;
            }
        float2 G01[4];
        float G2[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            G01[k] = padd(gt01[k], padd(V01[k], V01[k + 4]));
            gt01[k] = psub(V01[k], V01[k + 4]);
            G2[k] = gt2[k] + (V2[k] + V2[k + 4]);
            gt2[k] = V2[k] - V2[k + 4];
        }
        if (ez < z0) continue;
        walsh2p(G01);
        walsh2(G2);
        float2 *b01 = reinterpret_cast<float2 *>(so + (ez & 1) * 9 * NT);     // [3][NT] pairs
        float *b2 = so + (ez & 1) * 9 * NT + 6 * NT;                          // [3][NT]
#pragma unroll
        for (int k = 1; k < 4; ++k) { b01[(k - 1) * NT + tid] = G01[k]; b2[(k - 1) * NT + tid] = G2[k]; }
        __syncthreads();
        if (nOut) {
            const float2 y01 = padd(padd(padd(G01[0], b01[0 * NT + tid - 1]), b01[1 * NT + tid - TY]), b01[2 * NT + tid - TY - 1]);
            float y[3];
            y[0] = y01.x;
            y[1] = y01.y;
            y[2] = G2[0] + b2[0 * NT + tid - 1] + b2[1 * NT + tid - TY] + b2[2 * NT + tid - TY - 1];
            const int idx = base + PL * ez;
            if (MASK) {
                const uint8_t f = flags[idx];
#pragma unroll
                for (int c = 0; c < 3; ++c) if (f & (1 << c)) y[c] = E0 * in(idx, c);
            }
            out.apply(idx, y, po, dot);
        }
    }
}

template <typename T, int TY, int TX, class In, class Out>
__global__ void __launch_bounds__(TY * TX, (WalshOccD<T, TY * TX, Out>::value))
l0d_kernel(const WalshParam<T> B, In in0, Out out0, const T *__restrict__ E, const uint8_t *__restrict__ flags,
           const uint8_t *__restrict__ tileMask, Geom g, T E0, Reduce red0, const int *__restrict__ done0)
{
    pdl_enter();
    const int vk = blockIdx.y;          // right-hand side of a batched launch
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    const In in = in0.shift(vk); const Out out = out0.shift(vk); const Reduce red = red0.at(vk);
    __shared__ __align__(16) T so[2 * 9 * TY * TX];
    const int tilesY = (g.NY + TY - 2) / (TY - 1);
    const int64_t total = (int64_t)walsh_tiles(g, TY, TX) * g.NZ;
    int64_t a = total * blockIdx.x / gridDim.x;
    const int64_t b = total * (blockIdx.x + 1) / gridDim.x;
    double dot = 0.0;
    while (a < b) {
        const int tile = (int)(a / g.NZ), z0 = (int)(a % g.NZ);
        const int z1 = (int)(z0 + (b - a) < g.NZ ? z0 + (b - a) : g.NZ);
        const int y0 = (tile % tilesY) * (TY - 1), x0 = (tile / tilesY) * (TX - 1);
        if constexpr (sizeof(T) == 4) {
            if (tileMask[tile])
                l0d_march_c2<TY, TX, true>(B, in, out, E, flags, g, y0, x0, z0, z1, E0, so, dot);
            else
                l0d_march_c2<TY, TX, false>(B, in, out, E, flags, g, y0, x0, z0, z1, E0, so, dot);
        } else {
            if (tileMask[tile])
                l0d_march<T, TY, TX, true>(B, in, out, E, flags, g, y0, x0, z0, z1, E0, so, dot);
            else
                l0d_march<T, TY, TX, false>(B, in, out, E, flags, g, y0, x0, z0, z1, E0, so, dot);
        }
        a += z1 - z0;
    }
    if (red.result) block_sum_to<TY * TX>(dot, red.partials, red.counter, red.result, gridDim.x, blockIdx.x);
}

// ---------------------------------------------------------------------------
// Paired direct-load variant (FP32): two element columns per thread as in
// l0p_kernel, paired FP32 arithmetic, and the corner nodes of both columns
// (three rows x two columns) loaded straight from global memory one layer
// ahead, as in l0d_kernel; node sums double-buffered in shared memory.
template <typename T, int TYP, int TX, bool MASK, class In, class Out>
__device__ __forceinline__ void l0q_march(const WalshPairParam<T> &B, const In &in, const Out &out,
                                          const T *__restrict__ E, const uint8_t *__restrict__ flags,
                                          const Geom &g, int y0, int x0, int z0, int z1, T E0,
                                          T *so, double &dot)
{
    using P2 = typename PairOf<T>::type;
    constexpr int NT = TYP * TX;
    const int tid = threadIdx.x, ty = tid % TYP, tx = tid / TYP;
    const int PY = g.PY, PL = (int)g.plane;
    const int ey = y0 - 1 + 2 * ty, ex = x0 - 1 + tx;
    // node rows ey .. ey+2 and columns ex, ex+1: in [-1, NY] x [-1, NX] (guard slots
    // included) when the first element column is at most one past the last element;
    // the third row may then reach NY + 1 only if ey + 1 > NY - 1, i.e. element B void
    const bool cOn = ey <= g.NY - 1 && ex <= g.NX - 1;
    const bool row2 = ey + 2 <= g.NY;
    const int base = cOn ? (int)(g.origin + ey + (int64_t)PY * ex) : 0;
    const bool outA = ty >= 1 && tx >= 1 && ey < g.NY && ex < g.NX;
    const bool outB = tx >= 1 && ey + 1 < g.NY && ex < g.NX;
    auto load = [&](int z, T v[3][2][3]) {      // [comp][column][row]
#pragma unroll
        for (int bx = 0; bx < 2; ++bx)
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const bool on = cOn && (r < 2 || row2);
                const int m = base + r + PY * bx + PL * z;
                uint8_t f = 0;
                if (MASK && on) f = flags[m];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    T u = on ? in(m, c) : T(0);
                    if (MASK && (f & (1 << c))) u = T(0);
                    v[c][bx][r] = u;
                }
            }
    };
    // (y, x) Walsh transform of a node layer as (A, B) pairs
    auto walsh_layer = [&](const T v[3][2][3], P2 h[3][4]) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            P2 w[4];
#pragma unroll
            for (int bx = 0; bx < 2; ++bx) {
                w[2 * bx].x = v[c][bx][0]; w[2 * bx].y = v[c][bx][1];
                w[2 * bx + 1].x = v[c][bx][1]; w[2 * bx + 1].y = v[c][bx][2];
            }
            const P2 p0 = padd(w[0], w[1]), m0 = psub(w[0], w[1]);
            const P2 p1 = padd(w[2], w[3]), m1 = psub(w[2], w[3]);
            h[c][0] = padd(p0, p1); h[c][1] = padd(m0, m1); h[c][2] = psub(p0, p1); h[c][3] = psub(m0, m1);
        }
    };
    auto eload = [&](int z) {
        P2 e;
        e.x = cOn ? E[base + PL * z] : T(0);
        e.y = cOn ? E[base + 1 + PL * z] : T(0);       // element ey+1 <= NY-1 or a guard slot (E = 0)
        return e;
    };

    P2 hb[3][4], gt[3][4];
    T pre[3][2][3];
    __syncthreads();                     // the previous range's reads of so are done
    {
        T v[3][2][3];
        load(z0 - 1, v);
        walsh_layer(v, hb);
    }
    load(z0, pre);
    P2 eNext = eload(z0 - 1);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k) { gt[c][k].x = T(0); gt[c][k].y = T(0); }

    for (int ez = z0 - 1; ez < z1; ++ez) {
        P2 U[3][8];
        {
            P2 ht[3][4];
            walsh_layer(pre, ht);
            if (ez + 2 <= z1) load(ez + 2, pre);
            const P2 Ee = eNext;
            if (ez + 1 < z1) eNext = eload(ez + 1);
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    U[c][k] = pmul(Ee, padd(hb[c][k], ht[c][k]));
                    U[c][k + 4] = pmul(Ee, psub(hb[c][k], ht[c][k]));
                    hb[c][k] = ht[c][k];
                }
        }
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            P2 v[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                P2 acc; acc.x = T(0); acc.y = T(0);
                bool first = true;
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if ((walsh_pattern(t) >> (3 * c + d)) & 1u) {
                        const P2 u = U[d][t ^ walsh_axis_bit(d)];
                        acc = first ? pmul(B.b[t][3 * c + d], u) : pfma(B.b[t][3 * c + d], u, acc);
                        first = false;
                    }
                v[c] = acc;
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) U[c][t ^ walsh_axis_bit(c)] = v[c];
        }
        P2 G[3][4];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                G[c][k] = padd(gt[c][k], padd(U[c][k], U[c][k + 4]));
                gt[c][k] = psub(U[c][k], U[c][k + 4]);
            }
        if (ez < z0) continue;
        T *buf = so + (ez & 1) * 12 * NT;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const P2 p0 = padd(G[c][0], G[c][1]), m0 = psub(G[c][0], G[c][1]);
            const P2 p1 = padd(G[c][2], G[c][3]), m1 = psub(G[c][2], G[c][3]);
            G[c][0] = padd(p0, p1); G[c][1] = padd(m0, m1); G[c][2] = psub(p0, p1); G[c][3] = psub(m0, m1);
            buf[(0 * 3 + c) * NT + tid] = G[c][1].y;                         // B(1,0) -> (ty+1, tx)
            P2 x12; x12.x = G[c][2].x; x12.y = G[c][2].y + G[c][3].x;        // A(0,1), B(0,1)+A(1,1) -> (ty, tx+1)
            reinterpret_cast<P2 *>(buf + 3 * NT)[c * NT + tid] = x12;
            buf[(9 + c) * NT + tid] = G[c][3].y;                             // B(1,1) -> (ty+1, tx+1)
        }
        __syncthreads();
        T yA[3], yB[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            P2 x12; x12.x = T(0); x12.y = T(0);
            if (tx >= 1) x12 = reinterpret_cast<const P2 *>(buf + 3 * NT)[c * NT + tid - TYP];
            const T x0v = ty >= 1 ? buf[(0 * 3 + c) * NT + tid - 1] : T(0);
            const T x3 = (ty >= 1 && tx >= 1) ? buf[(9 + c) * NT + tid - TYP - 1] : T(0);
            yA[c] = G[c][0].x + x0v + x12.x + x3;
            yB[c] = G[c][0].y + G[c][1].x + x12.y;
        }
        const int idx = base + PL * ez;
        if (outA) {
            if (MASK) {
                const uint8_t f = flags[idx];
#pragma unroll
                for (int c = 0; c < 3; ++c) if (f & (1 << c)) yA[c] = E0 * in(idx, c);
            }
            out(idx, yA, dot);
        }
        if (outB) {
            if (MASK) {
                const uint8_t f = flags[idx + 1];
#pragma unroll
                for (int c = 0; c < 3; ++c) if (f & (1 << c)) yB[c] = E0 * in(idx + 1, c);
            }
            out(idx + 1, yB, dot);
        }
    }
}

template <typename T, int TYP, int TX, class In, class Out>
__global__ void __launch_bounds__(TYP * TX, WalshPairOcc<T, TYP * TX>::value)
l0q_kernel(const WalshPairParam<T> B, In in0, Out out0, const T *__restrict__ E, const uint8_t *__restrict__ flags,
           const uint8_t *__restrict__ tileMask, Geom g, T E0, Reduce red0, const int *__restrict__ done0)
{
    pdl_enter();
    const int vk = blockIdx.y;          // right-hand side of a batched launch
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    const In in = in0.shift(vk); const Out out = out0.shift(vk); const Reduce red = red0.at(vk);
    __shared__ __align__(16) T so[2 * 12 * TYP * TX];
    const int tilesY = (g.NY + 2 * TYP - 2) / (2 * TYP - 1);
    const int64_t total = (int64_t)walsh_pair_tiles(g, TYP, TX) * g.NZ;
    int64_t a = total * blockIdx.x / gridDim.x;
    const int64_t b = total * (blockIdx.x + 1) / gridDim.x;
    double dot = 0.0;
    while (a < b) {
        const int tile = (int)(a / g.NZ), z0 = (int)(a % g.NZ);
        const int z1 = (int)(z0 + (b - a) < g.NZ ? z0 + (b - a) : g.NZ);
        const int y0 = (tile % tilesY) * (2 * TYP - 1), x0 = (tile / tilesY) * (TX - 1);
        if (tileMask[tile])
            l0q_march<T, TYP, TX, true>(B, in, out, E, flags, g, y0, x0, z0, z1, E0, so, dot);
        else
            l0q_march<T, TYP, TX, false>(B, in, out, E, flags, g, y0, x0, z0, z1, E0, so, dot);
        a += z1 - z0;
    }
    if (red.result) block_sum_to<TYP * TX>(dot, red.partials, red.counter, red.result, gridDim.x, blockIdx.x);
}

}  // namespace topgpu
