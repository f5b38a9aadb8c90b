// topgpu_tc.cuh -- level-0 FP32 stiffness product on the 5th-generation
// tensor cores (tcgen05, sm_100a).
//
// The direct-load Walsh kernel (l0d) spends most of its issue slots on the
// element arithmetic.  Here the element products of a tile of 128 element
// columns become one small matrix product per node layer,
//
//     D[e][n] = sum_k A[e][k] Bk[n][k],   y_e = E_e D[e][:]
//
// with A[e][:] the element's 24 corner values (bottom node layer in k 0..11,
// top node layer in k 16..27, zero pads) and Bk = Ke in the same order (rows
// n: the 12 bottom-corner outputs, then the 12 top-corner outputs).  M = 128
// (the CTA's element columns), N = 32 (24 used), K = 32: four K = 8 steps of
// tcgen05.mma kind::tf32 from shared-memory operands into a 32-column TMEM
// accumulator.  FP32 accuracy comes from the split x = hi + lo into TF32
// values: D = A_hi B_hi + A_lo B_hi + A_hi B_lo (the dropped A_lo B_lo is
// ~2^-22 relative), three passes of the four steps.
//
// A node layer is written once, as the top half of the current element layer
// and, in the other buffer of a ping-pong pair, it is the bottom half of the
// next one.  One thread issues the twelve MMAs and commits them to an
// mbarrier; every thread waits on it (bounded), reads its row of D with
// tcgen05.ld and finishes the node sums exactly like l0d (carried top-layer
// outputs, four in-plane columns summed in a fixed order through shared
// memory, fixed-DOF rows, prefetched epilogue inputs).
//
// Shared-memory operands use the K-major layout without swizzle: 8-row x
// 16-byte core matrices, K chunks of 4 TF32 values 128 bytes apart (LBO),
// 8-row groups SBO bytes apart.
#pragma once
#include "topgpu_walsh.cuh"

namespace topgpu {
namespace tc {

constexpr int kRows = 128;                     // element columns per CTA (MMA M)
constexpr int kN = 32;                         // accumulator columns (24 used)
constexpr int kABytes = kRows * 16 * 4;        // one node layer: 128 rows x 16 TF32
constexpr int kBBytes = kN * 32 * 4;           // Bk: 32 rows x 32 TF32
// dynamic shared memory: A hi/lo ping-pong, B hi/lo, node sums, barrier, TMEM address
constexpr int kOffAh = 0, kOffAl = 2 * kABytes, kOffBh = 4 * kABytes, kOffBl = kOffBh + kBBytes;
constexpr int kOffSo = kOffBl + kBBytes;                     // 9 x 128 floats
constexpr int kOffBar = kOffSo + 9 * kRows * 4;              // 8-byte mbarrier
constexpr int kOffTmem = kOffBar + 8;
constexpr int kSmemBytes = kOffTmem + 8;
constexpr uint32_t kWaitLimit = 1u << 22;      // mbarrier polls before the kernel gives up

// byte offset of (row, k) in a K-major no-swizzle operand with the given SBO
__host__ __device__ constexpr int kmajor_off(int row, int k, int sbo)
{
    return (row >> 3) * sbo + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4;
}
// instruction descriptor: D f32, A/B tf32, both K-major, N = 32, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(kN >> 3) << 17) | (uint32_t(kRows >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
// shared-memory matrix descriptor (no swizzle, version 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}
__device__ __forceinline__ uint32_t tf32_rna(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t da, uint64_t db, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :: "r"(dtmem), "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// bounded wait for the given phase parity; false when the limit ran out
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
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
// this warp's 32 TMEM lanes, columns 0..23
__device__ __forceinline__ void tmem_ld24(uint32_t taddr, float v[24])
{
    uint32_t r[24];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23])
                 : "r"(taddr + 16u));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 24; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc

// Bk = Ke in the tensor kernel's order, split into TF32 hi and lo parts, in
// the K-major shared-memory image (Bh then Bl, kBBytes each); built on the host
struct TcOperandB { float img[2 * tc::kBBytes / 4]; };

// state of one CTA's march (shared-memory addresses, TMEM accumulator, phase)
struct TcState {
    unsigned char *sm;
    uint32_t tmem, bar, phase;
    int *err;
    bool ok;
};

template <int TY, int TX, bool MASK, class In, class Out>
__device__ __forceinline__ void l0t_march(TcState &S, const In &in, const Out &out,
                                          const float *__restrict__ E, const uint8_t *__restrict__ flags,
                                          const Geom &g, int y0, int x0, int z0, int z1, float E0, double &dot)
{
    static_assert(TY * TX == tc::kRows, "one element column per accumulator row");
    constexpr int NT = TY * TX;
    const int tid = threadIdx.x, ty = tid % TY, tx = tid / TY, warp = tid >> 5;
    const int PY = g.PY, PL = (int)g.plane;
    const int ey = y0 - 1 + ty, ex = x0 - 1 + tx;
    const bool cOn = ey <= g.NY - 1 && ex <= g.NX - 1;
    const int base = cOn ? (int)(g.origin + ey + (int64_t)PY * ex) : 0;
    const bool nOut = ty >= 1 && tx >= 1 && ey < g.NY && ex < g.NX;
    unsigned char *sm = S.sm;
    float *so = reinterpret_cast<float *>(sm + tc::kOffSo);
    auto load = [&](int z, float v[12]) {      // the column's four corner nodes of layer z, k = 3 (by + 2 bx) + c
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int m = base + (k & 1) + PY * (k >> 1) + PL * z;
            uint8_t f = 0;
            if (MASK && cOn) f = flags[m];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                float u = cOn ? in(m, c) : 0.f;
                if (MASK && (f & (1 << c))) u = 0.f;
                v[3 * k + c] = u;
            }
        }
    };
    auto eload = [&](int z) { return cOn ? E[base + PL * z] : 0.f; };
    auto put = [&](int layer, const float v[12]) {   // hi / lo TF32 rows of node layer `layer`
        unsigned char *ah = sm + tc::kOffAh + (layer & 1) * tc::kABytes;
        unsigned char *al = sm + tc::kOffAl + (layer & 1) * tc::kABytes;
#pragma unroll
        for (int kc = 0; kc < 3; ++kc) {
            uint32_t h[4], l[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                h[j] = tc::tf32_rna(v[4 * kc + j]);
                l[j] = tc::tf32_rna(v[4 * kc + j] - __uint_as_float(h[j]));
            }
            const int off = tc::kmajor_off(tid, 4 * kc, 512);
            *reinterpret_cast<uint4 *>(ah + off) = make_uint4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<uint4 *>(al + off) = make_uint4(l[0], l[1], l[2], l[3]);
        }
    };

    float pre[12], gt[12];
    load(z0 - 1, pre);
    put(z0 - 1, pre);
    load(z0, pre);
    float eNext = eload(z0 - 1);
#pragma unroll
    for (int i = 0; i < 12; ++i) gt[i] = 0.f;

    for (int ez = z0 - 1; ez < z1; ++ez) {
        typename Out::Pre po{};
        if (nOut && ez >= z0) po = out.pre(base + PL * ez);
        put(ez + 1, pre);                                 // top node layer of element layer ez
        if (ez + 2 <= z1) load(ez + 2, pre);
        const float Ee = eNext;
        if (ez + 1 < z1) eNext = eload(ez + 1);
        // operands visible to the tensor core; the previous layer's TMEM reads are done
        tc::fence_proxy_async();
        tc::fence_before();
        __syncthreads();
        tc::fence_after();
        if (tid == 0 && S.ok) {
            const uint32_t aB = tc::smem_u32(sm) + (ez & 1) * tc::kABytes;         // bottom: node layer ez
            const uint32_t aT = tc::smem_u32(sm) + ((ez + 1) & 1) * tc::kABytes;   // top: node layer ez + 1
            const uint32_t bh = tc::smem_u32(sm + tc::kOffBh), bl = tc::smem_u32(sm + tc::kOffBl);
            const uint32_t alo = tc::kOffAl;                                       // lo part offset
#pragma unroll
            for (int pass = 0; pass < 3; ++pass) {
                const uint32_t ao = pass == 1 ? alo : 0u;                          // A_lo in the second pass
                const uint32_t b0 = pass == 2 ? bl : bh;                           // B_lo in the third
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const uint32_t a = (s < 2 ? aB : aT) + ao + (s & 1) * 256;
                    tc::mma_tf32(S.tmem, tc::sdesc(a, 128, 512), tc::sdesc(b0 + s * 256, 128, 1024),
                                 (pass | s) ? 1u : 0u);
                }
            }
            tc::commit(S.bar);
        }
        float D[24];
        {   // a wait that gave up disables the warp as a whole (tcgen05.ld is warp-collective)
            const bool ok = __all_sync(0xffffffffu, S.ok && tc::mbar_wait(S.bar, S.phase));
            if (!ok && S.ok && (tid & 31) == 0) atomicExch(S.err, 1);
            S.ok = ok;
        }
        S.phase ^= 1u;
        tc::fence_after();
        if (S.ok) tc::tmem_ld24(S.tmem + ((uint32_t)(32 * warp) << 16), D);
        else for (int i = 0; i < 24; ++i) D[i] = 0.f;
        float G[12];
#pragma unroll
        for (int i = 0; i < 12; ++i) {
            G[i] = fmaf(Ee, D[i], gt[i]);
            gt[i] = Ee * D[12 + i];
        }
        if (ez < z0) continue;
#pragma unroll
        for (int k = 1; k < 4; ++k)
#pragma unroll
            for (int c = 0; c < 3; ++c) so[((k - 1) * 3 + c) * NT + tid] = G[3 * k + c];
        __syncthreads();
        if (nOut) {
            float y[3];
#pragma unroll
            for (int c = 0; c < 3; ++c)
                y[c] = G[c] + so[(0 * 3 + c) * NT + tid - 1] + so[(1 * 3 + c) * NT + tid - TY] + so[(2 * 3 + c) * NT + tid - TY - 1];
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

// kind 5: FP32 level-0 product on the tensor cores; tiles, work split and
// results' structure as l0d_kernel (16 x 8 element columns per CTA)
template <int TY, int TX, class In, class Out>
__global__ void __launch_bounds__(TY * TX)
l0t_kernel(const TcOperandB *__restrict__ Bimg, In in0, Out out0, const float *__restrict__ E,
           const uint8_t *__restrict__ flags, const uint8_t *__restrict__ tileMask, Geom g, float E0,
           Reduce red0, const int *__restrict__ done0, int *err)
{
    pdl_enter();
    const int vk = blockIdx.y;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    const In in = in0.shift(vk); const Out out = out0.shift(vk); const Reduce red = red0.at(vk);
    extern __shared__ __align__(1024) unsigned char tcsm[];
    const int tid = threadIdx.x;
    // B image and zero pads of the A buffers
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(Bimg->img);
        uint4 *dst = reinterpret_cast<uint4 *>(tcsm + tc::kOffBh);
        for (int i = tid; i < 2 * tc::kBBytes / 16; i += TY * TX) dst[i] = src[i];
        for (int b = 0; b < 4; ++b)        // K chunk 3 (k 12..15) of every row of Ah[0], Ah[1], Al[0], Al[1]
            *reinterpret_cast<uint4 *>(tcsm + b * tc::kABytes + tc::kmajor_off(tid, 12, 512)) = make_uint4(0u, 0u, 0u, 0u);
    }
    TcState S;
    S.sm = tcsm; S.bar = tc::smem_u32(tcsm + tc::kOffBar); S.phase = 0; S.err = err; S.ok = true;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(tcsm + tc::kOffTmem);
    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(tc::smem_u32(tslot)), "r"((uint32_t)tc::kN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(S.bar), "r"(1u) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    S.tmem = *tslot;

    const int tilesY = (g.NY + TY - 2) / (TY - 1);
    const int64_t total = (int64_t)walsh_tiles(g, TY, TX) * g.NZ;
    int64_t a = total * blockIdx.x / gridDim.x;
    const int64_t b = total * (blockIdx.x + 1) / gridDim.x;
    double dot = 0.0;
    while (a < b) {
        const int tile = (int)(a / g.NZ), z0 = (int)(a % g.NZ);
        const int z1 = (int)(z0 + (b - a) < g.NZ ? z0 + (b - a) : g.NZ);
        const int y0 = (tile % tilesY) * (TY - 1), x0 = (tile / tilesY) * (TX - 1);
        if (tileMask[tile]) l0t_march<TY, TX, true>(S, in, out, E, flags, g, y0, x0, z0, z1, E0, dot);
        else l0t_march<TY, TX, false>(S, in, out, E, flags, g, y0, x0, z0, z1, E0, dot);
        a += z1 - z0;
    }
    // every TMEM read is complete before the accumulator is released
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (tid < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(S.tmem), "r"((uint32_t)tc::kN));
    if (red.result) block_sum_to<TY * TX>(dot, red.partials, red.counter, red.result, gridDim.x, blockIdx.x);
}

}  // namespace topgpu
