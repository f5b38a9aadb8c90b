// topgpu_stage.cuh -- level-0 FP32 stiffness product with TMA-staged node
// layers (kind 6).
//
// The arithmetic is the Walsh-basis element product of topgpu_walsh.cuh on
// pairs of y-adjacent element columns (sm_100 paired FP32 instructions: one
// add / multiply / multiply-add serves both columns).  What changes is how the
// operands arrive:
//
//  * A producer warp streams every node layer of the CTA's z-march into a
//    ring of shared-memory stages with cp.async.bulk.tensor (one 5-D box of
//    the three displacement components and one 3-D box of the element moduli
//    per layer), completing on a per-stage mbarrier.  It runs up to kStages
//    layers ahead, across the CTA's work items, so the consumers find each
//    layer resident when they reach it: no per-thread global loads and no
//    prefetch registers for the operand.
//  * Consumer threads read their corner nodes from the stage (conflict-free
//    rows), release the stage to the producer with one arrive per warp, and
//    run the product.  Node sums over the four element columns around a node
//    go through a double-buffered exchange in shared memory in a fixed order
//    (deterministic results), one named barrier per layer.
//  * Each thread owns two y-adjacent output nodes (Y even, Y + 1), so the
//    epilogue reads and writes its node vectors with 8-byte (FP32) or 16-byte
//    (FP64) accesses.
//
// Tiles: 2 TYP element rows x TX element columns per CTA, producing
// (2 TYP - 2) x (TX - 1) node columns (the tiles overlap by one element
// column; an even row stride keeps every owned pair aligned).  The TMA box
// starts at the row below the tile rounded down to a multiple of four (the
// 16-byte rule for the innermost coordinate) and spans 2 TYP + 4 rows; rows
// and columns outside the arrays read as zero, like the guard slots.
//
// Every mbarrier wait is bounded: a wait that gives up raises the error flag
// and the kernel finishes its loop without the stage's data (results are then
// invalid and the caller reports the flag), so no thread is left at a barrier.
#pragma once
#include <cuda.h>
#include "topgpu_walsh.cuh"

namespace topgpu {
namespace stg {

constexpr int kStages = 4;
constexpr uint32_t kWaitLimit = 1u << 22;

template <int TYP, int TX> struct Tile {
    static constexpr int NT = TYP * TX;                 // consumer threads
    static constexpr int NTHREADS = NT + 32;            // + the producer warp
    static constexpr int OY = 2 * TYP - 2;              // output node rows per tile
    static constexpr int OX = TX - 1;                   // output node columns per tile
    static constexpr int BY = 2 * TYP + 4;              // staged rows (multiple of 4)
    static constexpr int BXU = TX + 1;                  // staged node columns
    static constexpr int UBYTES = BY * BXU * 3 * 4;     // one node layer, three components
    static constexpr int EBYTES = BY * TX * 4;          // one element layer of moduli
    static constexpr int TXBYTES = UBYTES + EBYTES;     // bytes the two copies deliver
    // a tensor copy's shared-memory destination must be 128-byte aligned:
    // the moduli box starts on the next 128-byte boundary after the node box
    static constexpr int OFF_E = (UBYTES + 127) / 128 * 128;
    static constexpr int SBYTES = (OFF_E + EBYTES + 127) / 128 * 128;
    static constexpr int XN = NT + TYP + 1;             // exchange slots (reads reach tid + TYP + 1)
    static constexpr int XBYTES = 3 * XN * (8 + 4 + 4); // one exchange buffer
    static constexpr int OFF_X = kStages * SBYTES;
    static constexpr int OFF_BAR = OFF_X + 2 * XBYTES;
    static constexpr int SMEM = OFF_BAR + 2 * kStages * 8 + 128;   // + alignment slack of the base
    static_assert(NT % 32 == 0, "whole consumer warps");
    static_assert(OFF_E % 128 == 0 && SBYTES % 128 == 0 && OFF_X % 128 == 0, "128-byte aligned copy destinations");
    static_assert(BY * 4 % 16 == 0, "TMA box rows are a multiple of 16 bytes");
};

__host__ __device__ inline int tiles_y(const Geom &g, int TYP) { return (g.NY + 2 * TYP - 3) / (2 * TYP - 2); }
__host__ __device__ inline int tiles_x(const Geom &g, int TX) { return (g.NX + TX - 2) / (TX - 1); }
__host__ __device__ inline int tiles(const Geom &g, int TYP, int TX) { return tiles_y(g, TYP) * tiles_x(g, TX); }

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void arrive_expect(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(bar) : "memory");
}
// bounded wait for the phase of the given parity; false when the limit ran out
__device__ __forceinline__ bool wait(uint32_t bar, uint32_t parity)
{
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}
__device__ __forceinline__ void tma_load5(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                          int c0, int c1, int c2, int c3, int c4)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
        :: "r"(dst), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar) : "memory");
}
__device__ __forceinline__ void tma_load3(uint32_t dst, const CUtensorMap *map, uint32_t bar, int c0, int c1, int c2)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];"
        :: "r"(dst), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(bar) : "memory");
}
// barrier 1 over the consumer warps only (barrier 0 is __syncthreads)
template <int N> __device__ __forceinline__ void consumers_sync()
{
    asm volatile("bar.sync 1, %0;" :: "n"(N) : "memory");
}

// one (tile, z-range) work item of a CTA's share: (tile, layer) units in
// [a, b) are tile-major, so an item is a tile and a run of its node layers
struct Item { int tile, z0, z1; };
__device__ __forceinline__ Item item_at(int64_t a, int64_t b, int NZ)
{
    Item it;
    it.tile = (int)(a / NZ);
    it.z0 = (int)(a % NZ);
    it.z1 = (int)(it.z0 + (b - a) < NZ ? it.z0 + (b - a) : NZ);
    return it;
}

}  // namespace stg

// consumer state of one CTA: stage ring position, error state, shared memory
struct StageCursor {
    unsigned char *sm;
    uint32_t barFull, barEmpty, cnt;
    int *err, *abortFlag;
    bool ok;
};

// one work item (tile, node layers z0 .. z1-1) on the consumer threads
template <int TYP, int TX, bool MASK, class Out>
__device__ __forceinline__ void l0s_item(StageCursor &S, const WalshPairParam<float> &B, const VecIn<float, float> &in,
                                         const Out &out, const uint8_t *__restrict__ flags, const Geom &g,
                                         const stg::Item &it, int tilesY, float E0, double &dot)
{
    using Tl = stg::Tile<TYP, TX>;
    using P2 = float2;
    constexpr int NT = Tl::NT;
    const int tid = threadIdx.x, ty = tid % TYP, tx = tid / TYP, lane = tid & 31;
    const int PY = g.PY, PL = (int)g.plane;
    float *xch = reinterpret_cast<float *>(S.sm + Tl::OFF_X);
    const int Yo = (it.tile % tilesY) * Tl::OY, Xo = (it.tile / tilesY) * Tl::OX;
    const int ya = (Yo - 1) & ~3, o = (Yo - 1) - ya;
    const int ey = Yo - 1 + 2 * ty, ex = Xo - 1 + tx;
    // owned nodes (ey + 1, ex + 1) and (ey + 2, ex + 1)
    const int Y1 = ey + 1, X1 = ex + 1;
    const bool own = ty <= TYP - 2 && tx <= TX - 2 && X1 < g.NX && Y1 < g.NY;
    const bool own2 = own && Y1 + 1 < g.NY;
    const int idx1 = (int)(g.origin + Y1 + (int64_t)PY * X1);     // + PL * z
    const int urow = o + 2 * ty;                                   // stage row of node row ey
    // the stage of the next layer: bounded wait, then its base
    auto acquire = [&]() -> const float * {
        const int s = (int)(S.cnt % stg::kStages);
        if (S.ok && !stg::wait(S.barFull + 8 * s, (S.cnt / stg::kStages) & 1u)) {
            S.ok = false;
            atomicExch(S.err, 1);
            atomicExch(S.abortFlag, 1);
        }
        return reinterpret_cast<const float *>(S.sm + s * Tl::SBYTES);
    };
    auto release = [&]() {                      // the warp is done reading the stage
        __syncwarp();
        if (lane == 0) stg::arrive(S.barEmpty + 8 * (int)(S.cnt % stg::kStages));
        ++S.cnt;
    };
    // (y, x) Walsh transform of the thread's two columns in node layer z
    // (stage rows urow .. urow + 2, columns tx, tx + 1), as (A, B) pairs
    auto corners = [&](const float *st, int z, P2 h[3][4]) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float v[2][3];
#pragma unroll
            for (int bx = 0; bx < 2; ++bx)
#pragma unroll
                for (int r = 0; r < 3; ++r) v[bx][r] = st[(urow + r) + Tl::BY * ((tx + bx) + Tl::BXU * c)];
            if (MASK) {                              // fixed components read as zero
#pragma unroll
                for (int bx = 0; bx < 2; ++bx)
#pragma unroll
                    for (int r = 0; r < 3; ++r) {
                        const int Y = ey + r, X = ex + bx;
                        if (Y >= 0 && Y < g.NY && X >= 0 && X < g.NX && z >= 0 && z < g.NZ &&
                            (flags[g.origin + Y + (int64_t)PY * X + (int64_t)PL * z] & (1 << c)))
                            v[bx][r] = 0.f;
                    }
            }
            P2 w[4];
#pragma unroll
            for (int bx = 0; bx < 2; ++bx) {
                w[2 * bx].x = v[bx][0]; w[2 * bx].y = v[bx][1];
                w[2 * bx + 1].x = v[bx][1]; w[2 * bx + 1].y = v[bx][2];
            }
            const P2 p0 = padd(w[0], w[1]), m0 = psub(w[0], w[1]);
            const P2 p1 = padd(w[2], w[3]), m1 = psub(w[2], w[3]);
            h[c][0] = padd(p0, p1); h[c][1] = padd(m0, m1); h[c][2] = psub(p0, p1); h[c][3] = psub(m0, m1);
        }
    };

    stg::consumers_sync<NT>();                  // the previous item's exchange reads are done
    P2 hb[3][4], gt[3][4];
    corners(acquire(), it.z0 - 1, hb);
    release();
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int k = 0; k < 4; ++k) { gt[c][k].x = 0.f; gt[c][k].y = 0.f; }
    for (int ez = it.z0 - 1; ez < it.z1; ++ez) {
        typename Out::Pre2 po{};
        if (own && ez >= it.z0) po = out.pre2(idx1 + PL * ez);
        P2 ht[3][4];
        P2 Ee;
        {
            const float *st = acquire();
            corners(st, ez + 1, ht);
            const float *es = st + Tl::OFF_E / 4;      // moduli of element layer ez
            Ee.x = es[urow + Tl::BY * tx];
            Ee.y = es[urow + 1 + Tl::BY * tx];
            release();
        }
        // Element product by block pairs (t, t ^ 4), t = 0..3: the pair reads
        // and writes exactly the z halves U[c][k], U[c][k + 4] of the three
        // (component, Walsh index) combinations k = (t ^ e(c)) & 3, so the z
        // butterfly, both 3 x 3 blocks and the inverse z butterfly with the
        // carry run per pair and only six U values are live at a time.  Same
        // operations in the same order per value as the all-blocks form.
        // The layer's G replaces ht (whose values move into hb).
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            P2 up[3], um[3];                                 // E (hb + ht), E (hb - ht)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int k = (t ^ walsh_axis_bit(c)) & 3;
                const P2 a = pmul(Ee, ht[c][k]);
                P2 na; na.x = -a.x; na.y = -a.y;
                up[c] = pfma(Ee, hb[c][k], a);
                um[c] = pfma(Ee, hb[c][k], na);
            }
            P2 vt[3], v4[3];                                 // blocks t and t ^ 4
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                P2 acc; acc.x = 0.f; acc.y = 0.f;
                bool first = true;
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if ((walsh_pattern(t) >> (3 * c + d)) & 1u) {
                        const P2 u = d == 2 ? um[d] : up[d];     // U[d][t ^ e(d)]: the minus half for z
                        acc = first ? pmul(B.b[t][3 * c + d], u) : pfma(B.b[t][3 * c + d], u, acc);
                        first = false;
                    }
                vt[c] = acc;
                P2 acc4; acc4.x = 0.f; acc4.y = 0.f;
                first = true;
#pragma unroll
                for (int d = 0; d < 3; ++d)
                    if ((walsh_pattern(t ^ 4) >> (3 * c + d)) & 1u) {
                        const P2 u = d == 2 ? up[d] : um[d];     // U[d][t ^ 4 ^ e(d)]
                        acc4 = first ? pmul(B.b[t ^ 4][3 * c + d], u) : pfma(B.b[t ^ 4][3 * c + d], u, acc4);
                        first = false;
                    }
                v4[c] = acc4;
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int k = (t ^ walsh_axis_bit(c)) & 3;
                // V[c][k] (z half 0) and V[c][k + 4]: block t gives the plus half
                // for x and y and the minus half for z, block t ^ 4 the others
                const P2 vp = c == 2 ? v4[c] : vt[c], vm = c == 2 ? vt[c] : v4[c];
                hb[c][k] = ht[c][k];
                ht[c][k] = padd(gt[c][k], padd(vp, vm));
                gt[c][k] = psub(vp, vm);
            }
        }
        P2 (&G)[3][4] = ht;
        if (ez < it.z0) continue;               // uniform: the first layer only seeds the carry
        // back in (y, x): corner k = by + 2 bx of (A, B); publish what the
        // neighbours' nodes need, in a fixed summation order
        float *X = xch + (ez & 1) * (Tl::XBYTES / 4);
        P2 *XP1 = reinterpret_cast<P2 *>(X);                 // [3][XN] pairs for (ty, tx - 1)
        float *XP2 = X + 2 * 3 * Tl::XN;                     // [3][XN] for (ty - 1, tx)
        float *XP3 = XP2 + 3 * Tl::XN;                       // [3][XN] for (ty - 1, tx - 1)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const P2 p0 = padd(G[c][0], G[c][1]), m0 = psub(G[c][0], G[c][1]);
            const P2 p1 = padd(G[c][2], G[c][3]), m1 = psub(G[c][2], G[c][3]);
            G[c][0] = padd(p0, p1); G[c][1] = padd(m0, m1); G[c][2] = psub(p0, p1); G[c][3] = psub(m0, m1);
            P2 x1; x1.x = G[c][1].x + G[c][0].y; x1.y = G[c][1].y;
            XP1[c * Tl::XN + tid] = x1;
            XP2[c * Tl::XN + tid] = G[c][2].x;
            XP3[c * Tl::XN + tid] = G[c][0].x;
        }
        stg::consumers_sync<NT>();
        if (own) {
            float y1[3], y2[3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const P2 r1 = XP1[c * Tl::XN + tid + TYP];             // column tx + 1: A(1,0) + B(0,0), B(1,0)
                const float r2 = XP2[c * Tl::XN + tid + 1];             // row pair ty + 1: A(0,1)
                const float r3 = XP3[c * Tl::XN + tid + TYP + 1];       // (ty + 1, tx + 1): A(0,0)
                y1[c] = (G[c][3].x + G[c][2].y) + r1.x;                 // node (ey + 1, ex + 1)
                y2[c] = ((G[c][3].y + r1.y) + r2) + r3;                 // node (ey + 2, ex + 1)
            }
            const int i1 = idx1 + PL * ez;
            if (MASK) {                          // fixed rows: y = E0 u
                const uint8_t f1 = flags[i1], f2 = own2 ? flags[i1 + 1] : uint8_t(0);
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    if (f1 & (1 << c)) y1[c] = E0 * in(i1, c);
                    if (f2 & (1 << c)) y2[c] = E0 * in(i1 + 1, c);
                }
            }
            out.apply2(i1, y1, y2, own2, po, dot);
        }
    }
}

// resident CTAs per SM the register budget is fitted to (16 x 16: one CTA of
// 288 threads; 16 x 8: two CTAs of 160 threads).  Three 16 x 8 CTAs (128
// registers) spill and measured slower (52 vs 48 us on the 96x192x96 model).
template <int TYP, int TX> struct StageOcc { static constexpr int value = TYP * TX >= 256 ? 1 : 2; };

// kind 6: FP32 level-0 product, node layers staged by TMA (see above)
template <int TYP, int TX, class Out>
__global__ void __launch_bounds__(TYP * TX + 32, (StageOcc<TYP, TX>::value))
l0s_kernel(const __grid_constant__ CUtensorMap mapU, const __grid_constant__ CUtensorMap mapE,
           const WalshPairParam<float> B, VecIn<float, float> in0, Out out0, const uint8_t *__restrict__ flags,
           const uint8_t *__restrict__ tileMask, Geom g, float E0, Reduce red0, const int *__restrict__ done0,
           int *err)
{
    using Tl = stg::Tile<TYP, TX>;
    constexpr int NT = Tl::NT;
    pdl_enter();
    const int vk = blockIdx.y;                          // right-hand side of a batched launch
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    const VecIn<float, float> in = in0.shift(vk);
    const Out out = out0.shift(vk);
    const Reduce red = red0.at(vk);
    extern __shared__ __align__(128) unsigned char smRaw[];
    __shared__ int abortFlag;
    // stage buffers on a 128-byte boundary whatever static shared memory precedes them
    unsigned char *sm = smRaw + ((128u - (stg::smem_u32(smRaw) & 127u)) & 127u);
    const int tid = threadIdx.x;
    const uint32_t barFull = stg::smem_u32(sm + Tl::OFF_BAR), barEmpty = barFull + 8 * stg::kStages;
    if (tid == 0) {
        for (int s = 0; s < stg::kStages; ++s) {
            stg::bar_init(barFull + 8 * s, 1u);
            stg::bar_init(barEmpty + 8 * s, (uint32_t)(NT / 32));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        abortFlag = 0;
    }
    __syncthreads();

    const int tilesY = stg::tiles_y(g, TYP);
    const int64_t total = (int64_t)stg::tiles(g, TYP, TX) * g.NZ;
    const int64_t a0 = total * blockIdx.x / gridDim.x, b0 = total * (blockIdx.x + 1) / gridDim.x;
    double dot = 0.0;

    if (tid >= NT) {
        // ---- producer warp: one lane issues the copies, kStages layers ahead
        if (tid == NT) {
            uint32_t cnt = 0;
            bool ok = true;
            for (int64_t a = a0; a < b0 && ok;) {
                const stg::Item it = stg::item_at(a, b0, g.NZ);
                const int Yo = (it.tile % tilesY) * Tl::OY, Xo = (it.tile / tilesY) * Tl::OX;
                const int ya = (Yo - 1) & ~3;           // box row start: a multiple of four
                for (int L = it.z0 - 1; L <= it.z1; ++L, ++cnt) {
                    const int s = (int)(cnt % stg::kStages);
                    const uint32_t ph = (cnt / stg::kStages) & 1u;
                    if (!stg::wait(barEmpty + 8 * s, ph ^ 1u) || *(volatile int *)&abortFlag) { ok = false; break; }
                    const uint32_t dst = stg::smem_u32(sm + s * Tl::SBYTES);
                    // the copies' alignment rules, checked before issuing: 128-byte
                    // destinations, an innermost coordinate on a 16-byte boundary
                    if ((dst & 127u) || ((dst + Tl::OFF_E) & 127u) || (ya & 3)) { ok = false; break; }
                    stg::arrive_expect(barFull + 8 * s, (uint32_t)Tl::TXBYTES);
                    // node layer L: tensor coordinates (y, x + 1, z + 1, component, right-hand side)
                    stg::tma_load5(dst, &mapU, barFull + 8 * s, ya, Xo, L + 1, 0, vk);
                    // moduli of element layer L - 1: (y, x + 1, z + 1)
                    stg::tma_load3(dst + Tl::OFF_E, &mapE, barFull + 8 * s, ya, Xo, L);
                }
                a += it.z1 - it.z0;
            }
            if (!ok) { atomicExch(err, 1); atomicExch(&abortFlag, 1); }
            // the copies still in flight land before the CTA exits (bounded)
            for (uint32_t c = (cnt > (uint32_t)stg::kStages ? cnt - stg::kStages : 0u); c < cnt; ++c)
                if (!stg::wait(barFull + 8 * (int)(c % stg::kStages), (c / stg::kStages) & 1u)) atomicExch(err, 1);
        }
    } else {
        StageCursor S{sm, barFull, barEmpty, 0u, err, &abortFlag, true};
        for (int64_t a = a0; a < b0;) {
            const stg::Item it = stg::item_at(a, b0, g.NZ);
            if (tileMask[it.tile]) l0s_item<TYP, TX, true>(S, B, in, out, flags, g, it, tilesY, E0, dot);
            else l0s_item<TYP, TX, false>(S, B, in, out, flags, g, it, tilesY, E0, dot);
            a += it.z1 - it.z0;
        }
    }
    if (red.result) block_sum_to<Tl::NTHREADS>(dot, red.partials, red.counter, red.result, gridDim.x, blockIdx.x);
}

// tileMask[tile] = 1 when a node the tile stages (rows Yo-1 .. Yo+2TYP-1,
// columns Xo-1 .. Xo+TX-1, any layer) has a fixed component
template <int TYP, int TX>
__global__ void __launch_bounds__(256)
stage_mask_kernel(const uint8_t *__restrict__ flags, Geom g, uint8_t *__restrict__ tileMask)
{
    using Tl = stg::Tile<TYP, TX>;
    const int tilesY = stg::tiles_y(g, TYP);
    const int Yo = (blockIdx.x % tilesY) * Tl::OY, Xo = (blockIdx.x / tilesY) * Tl::OX;
    int any = 0;
    const int ny = 2 * TYP + 1, nx = TX + 1;
    for (int k = threadIdx.x; k < ny * nx * g.NZ; k += blockDim.x) {
        const int Y = Yo - 1 + k % ny, X = Xo - 1 + (k / ny) % nx, Z = k / (ny * nx);
        if (Y < 0 || Y >= g.NY || X < 0 || X >= g.NX) continue;
        any |= flags[g.origin + Y + (int64_t)g.PY * X + g.plane * Z] & kFixedMask;
    }
    any = __syncthreads_or(any);
    if (threadIdx.x == 0) tileMask[blockIdx.x] = any ? 1 : 0;
}

}  // namespace topgpu
