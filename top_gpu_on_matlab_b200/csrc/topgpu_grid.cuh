// topgpu_grid.cuh -- structured-grid device kernels of the fused solver.
//
// Layout of every level: node (Y, X, Z) of the (ny+1) x (nx+1) x (nz+1) node
// grid lives at  idx = Y + PY*(X+1) + PLANE*(Z+1)  of a zero-guarded array
// (PY >= NY+1, PX = NX+2, PZ = NZ+2, PLANE = PY*PX), one such array per
// displacement component (component stride CS).  Element (ey, ex, ez) is
// stored at the slot of its base node (ey, ex, ez).  All guard slots hold
// zeros, so every stencil access is in bounds and void / outside elements
// contribute nothing.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <initializer_list>
#include "topgpu_internal.h"

namespace topgpu {

constexpr int64_t kMargin = 64;        // elements of zero padding before/after each array
constexpr int kNodeThreads = 256;
constexpr uint8_t kActive = 8;         // flag bit: node belongs to an active element
constexpr uint8_t kFixedMask = 7;      // flag bits 0..2: component fixed (level 0)

struct Geom {
    int NY, NX, NZ;       // node counts
    int PY;               // y pitch
    int nbx;              // node-kernel blocks per z plane
    int64_t plane;        // PY * PX
    int64_t cs;           // component stride
    int64_t origin;       // index of node (0,0,0)
};

// corner j of an element with offsets (dy, dx, dz) in {0,1}
__host__ __device__ constexpr int corner_of(int dy, int dx, int dz)
{
    return 4 * dz + (dy ? (dx ? 1 : 0) : (dx ? 2 : 3));
}
__host__ __device__ constexpr int cdy(int j) { return (j & 3) < 2 ? 1 : 0; }
__host__ __device__ constexpr int cdx(int j) { return ((j & 3) == 1 || (j & 3) == 2) ? 1 : 0; }
__host__ __device__ constexpr int cdz(int j) { return j >> 2; }
// packed upper triangle of a symmetric 24x24 matrix (300 entries)
__host__ __device__ constexpr int sym_pack(int r, int k)
{
    return r <= k ? r * 24 - r * (r - 1) / 2 + (k - r) : k * 24 - k * (k - 1) / 2 + (r - k);
}
// Packed coarse matrices on the grid, tile-interleaved: the element at grid
// slot e keeps entry p at  (e / 32) * 9600 + p * 32 + e % 32, i.e. runs of 32
// consecutive element slots store their 300 entries together (38 KB in FP32),
// so a CTA working on a run of nodes reads a few contiguous blocks instead of
// one 128-byte piece from each of 300 entry planes.  Slot -1 (the guard before
// node (0,0,0)'s elements) falls in a zero tile in front of the array.
constexpr int kKsTile = 32;
constexpr int kKsTileVals = 300 * kKsTile;
__host__ __device__ inline int ks_slot_base(int e) { return (e >> 5) * kKsTileVals + (e & 31); }
__host__ __device__ inline int64_t ks_off(int p, int64_t e) { return (e >> 5) * kKsTileVals + p * kKsTile + (e & 31); }
// values to allocate for a level's packed matrices, and the zero tile in front
inline int64_t ks_alloc_vals(int64_t cs) { return (cs / kKsTile + 3) * (int64_t)kKsTileVals; }
constexpr int64_t kKsFront = kKsTileVals;

template <typename T> struct KeParam { T k[576]; };

// ---------------------------------------------------------------------------
// Deterministic grid-wide sum: per-block partials, the last block to finish
// adds them in index order and writes *result.
template <int NT>
__device__ __forceinline__ void block_sum_to(double v, double *partials, unsigned *counter, double *result,
                                             unsigned nb, unsigned bid);
template <int NT>
__device__ __forceinline__ bool block_sum_last(double v, double *partials, unsigned *counter, double *result,
                                               unsigned nb, unsigned bid);
template <int NT>
__device__ __forceinline__ void block_sum_to(double v, double *partials, unsigned *counter, double *result)
{
    block_sum_to<NT>(v, partials, counter, result, gridDim.x * gridDim.y * gridDim.z,
                     blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z));
}
// nb CTAs (numbered bid) contribute to this sum -- one vector of a batched launch
template <int NT>
__device__ __forceinline__ void block_sum_to(double v, double *partials, unsigned *counter, double *result,
                                             unsigned nb, unsigned bid)
{
    block_sum_last<NT>(v, partials, counter, result, nb, bid);
}
// the same; returns true in thread 0 of the CTA that wrote *result (after
// the write), so that code depending on the whole sum can follow in the
// same launch
template <int NT>
__device__ __forceinline__ bool block_sum_last(double v, double *partials, unsigned *counter, double *result,
                                               unsigned nb, unsigned bid)
{
    __shared__ double red[NT / 32];
    __shared__ bool last;
    // linear thread index: blocks may be 1-, 2- or 3-D (NT threads in all)
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = tid & 31, w = tid >> 5;
    if (lane == 0) red[w] = v;
    __syncthreads();
    if (tid == 0) {
        double s = 0;
        for (int i = 0; i < NT / 32; ++i) s += red[i];
        partials[bid] = s;
        __threadfence();
        last = (atomicAdd(counter, 1u) == nb - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double s = 0;
    for (unsigned i = tid; i < nb; i += NT) s += ((volatile double *)partials)[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) red[w] = s;
    __syncthreads();
    if (tid == 0) {
        double t = 0;
        for (int i = 0; i < NT / 32; ++i) t += red[i];
        *result = t;
        *counter = 0;
        return true;
    }
    return false;
}

// PCG scalars of one right-hand side; batched solves keep one per vector
struct PcgState {
    double normB, rho, rhoOld, pv, rr, resnorm, tol;
    double lam;                      // step length of the last update (x += lam p is applied by the p kernel)
    double sigma;                    // z . A p_old (flexible beta: beta = -sigma / pv)
    int its, maxIT, done, status;
    int xPend, pad_;                 // the last iteration's x update is still to be applied
};
constexpr int kStateInts = int(sizeof(PcgState) / sizeof(int));
constexpr int kStateDoubles = int(sizeof(PcgState) / sizeof(double));
static_assert(sizeof(PcgState) % sizeof(double) == 0, "PcgState packs into doubles");

struct Reduce {             // where a fused dot product goes
    double *partials; unsigned *counter; double *result;
    int64_t pStride = 0;    // batched launches: partials per vector
    int64_t rStride = 0;    //                   result stride (doubles) per vector
    __host__ __device__ Reduce at(int k) const
    {
        if (k == 0) return *this;
        return Reduce{partials + k * pStride, counter + k, result ? result + k * rStride : nullptr, pStride, rStride};
    }
};
// Programmatic dependent launch: kernels the solver launches back to back
// start with this.  The wait returns once the preceding kernel of the stream
// has completed and its writes are visible (at once for an ordinary launch),
// so nothing below it can read a predecessor's output early; the trigger lets
// the next kernel's CTAs be scheduled as this kernel's CTAs finish.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
// per-vector done flag of a batched launch (flags in consecutive PcgState's)
__device__ __forceinline__ const int *done_of(const int *done, int k) { return done ? done + k * kStateInts : nullptr; }

// ---------------------------------------------------------------------------
// Inputs of the node kernels: the value of the operand vector at a node.
// Functors carry one base pointer per component (set on the host), so device
// code indexes each component with 32-bit in-array offsets.
// Batched launches (several right-hand sides) keep the vectors of a level at
// a fixed stride vs (3 CS); shift(k) moves a functor to vector k.  Operand
// functors (read at every corner load of the product) move their pointers;
// epilogues (one call per node) add a 32-bit offset k vs to the index of
// each access instead, so that their many pointers stay kernel parameters
// rather than occupying registers through the whole kernel (the solver
// checks that kMax vs fits).  Vectors shared by all right-hand sides (invD)
// take no offset.
// two adjacent node slots (i, i+1) of a component array, i even and the
// array 16-byte aligned: one 8-byte (float) or 16-byte (double) access
template <typename T> struct Vec2Of;
template <> struct Vec2Of<float> { using type = float2; };
template <> struct Vec2Of<double> { using type = double2; };
template <typename T> __device__ __forceinline__ void ld2(const T *p, T &a, T &b)
{
    const typename Vec2Of<T>::type v = *reinterpret_cast<const typename Vec2Of<T>::type *>(p);
    a = v.x; b = v.y;
}
template <typename T> __device__ __forceinline__ void st2(T *p, T a, T b)
{
    typename Vec2Of<T>::type v; v.x = a; v.y = b;
    *reinterpret_cast<typename Vec2Of<T>::type *>(p) = v;
}

template <typename P> struct Comp3 {
    P p0, p1, p2;
    Comp3() = default;
    __host__ __device__ Comp3(P base, int64_t cs) : p0(base), p1(base + cs), p2(base + 2 * cs) {}
    __device__ __forceinline__ P operator[](int c) const { return c == 0 ? p0 : (c == 1 ? p1 : p2); }
    __device__ __forceinline__ Comp3 shifted(int64_t o) const { Comp3 r = *this; r.p0 += o; r.p1 += o; r.p2 += o; return r; }
};

template <typename T, typename TV>
struct VecIn {
    Comp3<const TV *> u; int64_t vs;
    __host__ __device__ VecIn(const TV *base, int64_t cs, int64_t vstride = 0) : u(base, cs), vs(vstride) {}
    __device__ __forceinline__ VecIn shift(int k) const { VecIn r = *this; if (k) r.u = u.shifted(k * vs); return r; }
    __device__ __forceinline__ T operator()(int m, int c) const { return T(u[c][m]); }
    __device__ __forceinline__ void node3(int m, T v[3]) const { for (int c = 0; c < 3; ++c) v[c] = T(u[c][m]); }
};
// x = omega * invD .* r  (the Jacobi pre-smoothing step, evaluated on the fly)
template <typename T, typename TR>
struct JacobiIn {
    Comp3<const TR *> r; Comp3<const T *> invD; T omega; int64_t vs;
    __host__ __device__ JacobiIn(const TR *rb, const T *ib, int64_t cs, T om, int64_t vstride = 0) : r(rb, cs), invD(ib, cs), omega(om), vs(vstride) {}
    __device__ __forceinline__ JacobiIn shift(int k) const { JacobiIn o = *this; if (k) o.r = r.shifted(k * vs); return o; }
    __device__ __forceinline__ T operator()(int m, int c) const { return omega * invD[c][m] * T(r[c][m]); }
    __device__ __forceinline__ void node3(int m, T v[3]) const { for (int c = 0; c < 3; ++c) v[c] = omega * invD[c][m] * T(r[c][m]); }
};

// Epilogues: what a node kernel does with y = (K u)(node).  pre(i) loads
// the node's epilogue inputs (a kernel may issue it well before y is ready,
// to hide the load latency); apply(i, y, pre, dot) finishes the node;
// operator() does both at once.
template <typename T, typename TY>
struct StoreOut {   // y
    Comp3<TY *> y; int vs, o = 0;
    struct Pre {};
    __host__ __device__ StoreOut(TY *yb, int64_t cs, int64_t vstride = 0) : y(yb, cs), vs((int)vstride) {}
    __device__ __forceinline__ StoreOut shift(int k) const { StoreOut r = *this; r.o = k * vs; return r; }
    __device__ __forceinline__ Pre pre(int) const { return Pre{}; }
    __device__ __forceinline__ void apply(int i, const T yv[3], const Pre &, double &) const
    { for (int c = 0; c < 3; ++c) y[c][i + o] = TY(yv[c]); }
    __device__ __forceinline__ void operator()(int i, const T yv[3], double &dot) const { apply(i, yv, pre(i), dot); }
    // node pair (i, i+1), i even: vector stores; only node i when !both
    struct Pre2 {};
    __device__ __forceinline__ Pre2 pre2(int) const { return Pre2{}; }
    __device__ __forceinline__ void apply2(int i, const T ya[3], const T yb[3], bool both, const Pre2 &, double &) const
    {
        for (int c = 0; c < 3; ++c) {
            if (both) st2(y[c] + i + o, TY(ya[c]), TY(yb[c]));
            else y[c][i + o] = TY(ya[c]);
        }
    }
};
template <typename T, typename TU, typename TY>
struct DotStoreOut { // y, and dot += u . y  (PCG: p . Ap)
    Comp3<TY *> y; Comp3<const TU *> u; int vs, o = 0;
    struct Pre { TU u[3]; };
    __host__ __device__ DotStoreOut(TY *yb, const TU *ub, int64_t cs, int64_t vstride = 0) : y(yb, cs), u(ub, cs), vs((int)vstride) {}
    __device__ __forceinline__ DotStoreOut shift(int k) const { DotStoreOut r = *this; r.o = k * vs; return r; }
    __device__ __forceinline__ Pre pre(int i) const { Pre p; for (int c = 0; c < 3; ++c) p.u[c] = u[c][i + o]; return p; }
    __device__ __forceinline__ void apply(int i, const T yv[3], const Pre &p, double &dot) const
    { for (int c = 0; c < 3; ++c) { y[c][i + o] = TY(yv[c]); dot += double(p.u[c]) * double(yv[c]); } }
    __device__ __forceinline__ void operator()(int i, const T yv[3], double &dot) const { apply(i, yv, pre(i), dot); }
    struct Pre2 { TU a[3], b[3]; };
    __device__ __forceinline__ Pre2 pre2(int i) const
    { Pre2 p; for (int c = 0; c < 3; ++c) ld2(u[c] + i + o, p.a[c], p.b[c]); return p; }
    __device__ __forceinline__ void apply2(int i, const T ya[3], const T yb[3], bool both, const Pre2 &p, double &dot) const
    {
        for (int c = 0; c < 3; ++c) {
            if (both) st2(y[c] + i + o, TY(ya[c]), TY(yb[c]));
            else y[c][i + o] = TY(ya[c]);
            dot += double(p.a[c]) * double(ya[c]);
            if (both) dot += double(p.b[c]) * double(yb[c]);
        }
    }
};
template <typename T, typename TR, typename TD>
struct ResidOut {   // d = r - y
    Comp3<const TR *> r; Comp3<TD *> d; int vsR, vsD, oR = 0, oD = 0;
    struct Pre { TR r[3]; };
    __host__ __device__ ResidOut(const TR *rb, TD *db, int64_t cs, int64_t vsr = 0, int64_t vsd = -1)
        : r(rb, cs), d(db, cs), vsR((int)vsr), vsD((int)(vsd < 0 ? vsr : vsd)) {}
    __device__ __forceinline__ ResidOut shift(int k) const { ResidOut w = *this; w.oR = k * vsR; w.oD = k * vsD; return w; }
    __device__ __forceinline__ Pre pre(int i) const { Pre p; for (int c = 0; c < 3; ++c) p.r[c] = r[c][i + oR]; return p; }
    __device__ __forceinline__ void apply(int i, const T yv[3], const Pre &p, double &) const
    { for (int c = 0; c < 3; ++c) d[c][i + oD] = TD(T(p.r[c]) - yv[c]); }
    __device__ __forceinline__ void operator()(int i, const T yv[3], double &dot) const { apply(i, yv, pre(i), dot); }
    struct Pre2 { TR a[3], b[3]; };
    __device__ __forceinline__ Pre2 pre2(int i) const
    { Pre2 p; for (int c = 0; c < 3; ++c) ld2(r[c] + i + oR, p.a[c], p.b[c]); return p; }
    __device__ __forceinline__ void apply2(int i, const T ya[3], const T yb[3], bool both, const Pre2 &p, double &) const
    {
        for (int c = 0; c < 3; ++c) {
            const TD da = TD(T(p.a[c]) - ya[c]), db = TD(T(p.b[c]) - yb[c]);
            if (both) st2(d[c] + i + oD, da, db);
            else d[c][i + oD] = da;
        }
    }
};
// z = x + omega*invD.*(r - y), optionally dot += z . r  (post-smoothing)
template <typename T, typename TR, typename TZ>
struct PostSmoothOut {
    Comp3<const T *> x; Comp3<const TR *> r; Comp3<const T *> invD; Comp3<TZ *> z; T omega; int vs, o = 0;
    struct Pre { T x[3], d[3]; TR r[3]; };
    __host__ __device__ PostSmoothOut(const T *xb, const TR *rb, const T *ib, TZ *zb, int64_t cs, T om, int64_t vstride = 0)
        : x(xb, cs), r(rb, cs), invD(ib, cs), z(zb, cs), omega(om), vs((int)vstride) {}
    __device__ __forceinline__ PostSmoothOut shift(int k) const { PostSmoothOut w = *this; w.o = k * vs; return w; }
    __device__ __forceinline__ Pre pre(int i) const
    {
        Pre p;
        for (int c = 0; c < 3; ++c) { p.x[c] = x[c][i + o]; p.d[c] = invD[c][i]; p.r[c] = r[c][i + o]; }
        return p;
    }
    __device__ __forceinline__ void apply(int i, const T yv[3], const Pre &p, double &dot) const
    {
        for (int c = 0; c < 3; ++c) {
            const T zv = p.x[c] + omega * p.d[c] * (T(p.r[c]) - yv[c]);
            z[c][i + o] = TZ(zv);
            dot += double(zv) * double(p.r[c]);
        }
    }
    __device__ __forceinline__ void operator()(int i, const T yv[3], double &dot) const { apply(i, yv, pre(i), dot); }
    struct Pre2 { T xa[3], xb[3], da[3], db[3]; TR ra[3], rb[3]; };
    __device__ __forceinline__ Pre2 pre2(int i) const
    {
        Pre2 p;
        for (int c = 0; c < 3; ++c) {
            ld2(x[c] + i + o, p.xa[c], p.xb[c]);
            ld2(invD[c] + i, p.da[c], p.db[c]);
            ld2(r[c] + i + o, p.ra[c], p.rb[c]);
        }
        return p;
    }
    __device__ __forceinline__ void apply2(int i, const T ya[3], const T yb[3], bool both, const Pre2 &p, double &dot) const
    {
        for (int c = 0; c < 3; ++c) {
            const T za = p.xa[c] + omega * p.da[c] * (T(p.ra[c]) - ya[c]);
            const T zb = p.xb[c] + omega * p.db[c] * (T(p.rb[c]) - yb[c]);
            if (both) st2(z[c] + i + o, TZ(za), TZ(zb));
            else z[c][i + o] = TZ(za);
            dot += double(za) * double(p.ra[c]);
            if (both) dot += double(zb) * double(p.rb[c]);
        }
    }
};

// ---------------------------------------------------------------------------
// Level 0: y(node) = sum over the 8 incident elements of E_e * Ke(rows of the
// node) * u_e.  Fixed components: the element matrices have those rows and
// columns removed and E0/nAdj on the diagonal (TOP_GPU.m:1729-1741), which
// summed over the node's elements is y = E0*u for a fixed row and u = 0 in
// every free row -- applied by MASK blocks, the ones whose stencil reaches
// a fixed node.  Ke comes in as a launch parameter (constant bank).
template <typename T, bool MASK, class In, class Out>
__device__ __forceinline__ void l0_node(const KeParam<T> &K, const In &in, const Out &out,
                                        const T *__restrict__ E, const uint8_t *__restrict__ flags,
                                        const Geom &g, int idx, bool valid, T E0, double &dot)
{
    if (!valid) return;
    const int PY = g.PY, PL = (int)g.plane;
    T Ee[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) Ee[i] = E[idx - cdy(i) - PY * cdx(i) - PL * cdz(i)];
    T t[8][3];
#pragma unroll
    for (int i = 0; i < 8; ++i) t[i][0] = t[i][1] = t[i][2] = T(0);
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dx = -1; dx <= 1; ++dx)
#pragma unroll
            for (int dy = -1; dy <= 1; ++dy) {
                const int m = idx + dy + PY * dx + PL * dz;
                T u[3] = {in(m, 0), in(m, 1), in(m, 2)};
                if (MASK) {
                    const uint8_t fm = flags[m];
#pragma unroll
                    for (int c = 0; c < 3; ++c) if (fm & (1 << c)) u[c] = T(0);
                }
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int jy = cdy(i) + dy, jx = cdx(i) + dx, jz = cdz(i) + dz;
                    if (jy < 0 || jy > 1 || jx < 0 || jx > 1 || jz < 0 || jz > 1) continue;
                    const int j = corner_of(jy, jx, jz);
#pragma unroll
                    for (int c = 0; c < 3; ++c)
#pragma unroll
                        for (int d = 0; d < 3; ++d) t[i][c] = fma(K.k[(3 * i + c) + 24 * (3 * j + d)], u[d], t[i][c]);
                }
            }
    T y[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        T s = T(0);
#pragma unroll
        for (int i = 0; i < 8; ++i) s = fma(Ee[i], t[i][c], s);
        y[c] = s;
    }
    if (MASK) {
        const uint8_t f = flags[idx];
#pragma unroll
        for (int c = 0; c < 3; ++c) if (f & (1 << c)) y[c] = E0 * in(idx, c);
    }
    out(idx, y, dot);
}

template <typename T, class In, class Out>
__global__ void __launch_bounds__(kNodeThreads)
l0_kernel(const KeParam<T> K, In in0, Out out0, const T *__restrict__ E, const uint8_t *__restrict__ flags,
          const uint8_t *__restrict__ tileFixed, Geom g, T E0, Reduce red0, const int *__restrict__ done0)
{
    pdl_enter();
    const int vk = blockIdx.z;          // right-hand side of a batched launch
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    const In in = in0.shift(vk); const Out out = out0.shift(vk); const Reduce red = red0.at(vk);
    const int q = blockIdx.x * kNodeThreads + threadIdx.x;
    const int Y = q % g.PY, X = q / g.PY, Z = blockIdx.y;
    const bool valid = Y < g.NY && X < g.NX;
    const int idx = (int)(g.origin + Y + (int64_t)g.PY * X + g.plane * Z);
    double dot = 0.0;
    if (tileFixed[blockIdx.x + (int64_t)g.nbx * Z])
        l0_node<T, true>(K, in, out, E, flags, g, idx, valid, E0, dot);
    else
        l0_node<T, false>(K, in, out, E, flags, g, idx, valid, E0, dot);
    if (red.result) block_sum_to<kNodeThreads>(dot, red.partials, red.counter, red.result, gridDim.x * gridDim.y,
                                               blockIdx.x + gridDim.x * blockIdx.y);
}

// ---------------------------------------------------------------------------
// Coarse levels: y(node) = sum over incident elements of the node's three
// rows of the element's Galerkin matrix Ks (packed upper triangle, entry
// stride CS) times u_e.  Eight lanes per node, lane i taking incident
// element i (the node is its local corner i); a shuffle tree adds them up.
constexpr int kCoarseLanes = 8;

template <typename T, class In, class Out>
__global__ void __launch_bounds__(kNodeThreads)
coarse_kernel(In in0, Out out0, const T *__restrict__ Ks, Geom g, Reduce red0, const int *__restrict__ done0)
{
    pdl_enter();
    const int vk = blockIdx.y;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    const In in = in0.shift(vk); const Out out = out0.shift(vk); const Reduce red = red0.at(vk);
    const int64_t gt = (int64_t)blockIdx.x * kNodeThreads + threadIdx.x;
    const int64_t node = gt / kCoarseLanes;
    const int i = int(gt % kCoarseLanes);
    const int64_t nq = (int64_t)g.PY * g.NX * g.NZ;
    const int64_t nq2 = node < nq ? node : 0;
    const int Y = int(nq2 % g.PY), X = int((nq2 / g.PY) % g.NX), Z = int(nq2 / ((int64_t)g.PY * g.NX));
    const bool valid = node < nq && Y < g.NY;
    const int64_t idx = g.origin + Y + (int64_t)g.PY * X + g.plane * Z;
    T y[3] = {T(0), T(0), T(0)};
    if (valid) {
        const int64_t slot = idx - cdy(i) - g.PY * cdx(i) - g.plane * cdz(i);
        if (Ks[ks_off(sym_pack(3 * i, 3 * i), slot)] != T(0)) {       // void element: all zero
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int m = (int)(slot + cdy(j) + g.PY * cdx(j) + g.plane * cdz(j));
                const T u[3] = {in(m, 0), in(m, 1), in(m, 2)};
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        y[c] = fma(__ldg(Ks + ks_off(sym_pack(3 * i + c, 3 * j + d), slot)), u[d], y[c]);
            }
        }
    }
#pragma unroll
    for (int o = kCoarseLanes / 2; o > 0; o >>= 1)
#pragma unroll
        for (int c = 0; c < 3; ++c) y[c] += __shfl_down_sync(0xffffffffu, y[c], o, kCoarseLanes);
    double dot = 0.0;
    if (valid && i == 0) out((int)idx, y, dot);
    if (red.result) block_sum_to<kNodeThreads>(dot, red.partials, red.counter, red.result, gridDim.x, blockIdx.x);
}
// Tiled variant: a CTA of 32 x 8 threads covers 32 consecutive node slots of
// one (x, z) row; thread (n, i) multiplies the three rows of incident element
// i (the node is its corner i) with u_e, so for a fixed i and entry the 32
// threads of a warp read consecutive element slots (one coalesced run), and
// the eight partial sums of a node are added in a fixed order.
constexpr int kCoarseTileX = 32;
// read-only global load kept in program order with the other such loads
// (so a run of them is issued before the arithmetic that consumes them)
__device__ __forceinline__ float ld_stream(const float *p)
{
    float v;
    asm volatile("ld.global.nc.f32 %0, [%1];" : "=f"(v) : "l"(p));
    return v;
}
// four consecutive values at a 16-byte aligned address (one float4 or two
// double2 accesses).  Grid vectors qualify at every slot Y = 4 m of a column:
// the pitch, plane, origin and component stride are multiples of 4 and the
// arrays start 16-byte aligned (vec4_ok checks it on the host).
__device__ __forceinline__ void ld4(const float *p, float v[4])
{
    const float4 q = *reinterpret_cast<const float4 *>(p);
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4(const double *p, double v[4])
{
    const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void st4(float *p, const float v[4])
{
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(double *p, const double v[4])
{
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
}
inline bool vec4_ok(const Geom &g, std::initializer_list<const void *> ptrs, std::initializer_list<int64_t> strides)
{
    if ((g.PY | g.plane | g.origin | g.cs) & 3) return false;
    for (const void *p : ptrs)
        if (p && (reinterpret_cast<uintptr_t>(p) & 15)) return false;
    for (int64_t v : strides)
        if (v & 3) return false;
    return true;
}
// packed-entry offsets (entry * 32, tile-interleaved layout) of Ks(r, k), in shared memory
__device__ __forceinline__ void coarse_offsets(int *offs, const Geom &, int tid, int nthreads)
{
    for (int k = tid; k < 24 * 24; k += nthreads) offs[k] = sym_pack(k / 24, k % 24) * kKsTile;
}
// One tile: the 32 node slots q = bx*32 .. bx*32+31 of z layer bz; thread
// (n, i) of the 256 takes incident element i of node n.  Every thread of the
// CTA calls it; returns the dot contribution of the epilogue (threads i == 0).
template <typename T, class In, class Out>
__device__ __forceinline__ double coarse_tile_unit(const In &in, const Out &out, const T *__restrict__ Ks, const Geom &g,
                                                   int bx, int bz, int n, int i, T (*part)[3][kCoarseTileX],
                                                   const int *offs)
{
    const int q = bx * kCoarseTileX + n;
    const int Y = q % g.PY, X = q / g.PY, Z = bz;
    const bool valid = Y < g.NY && X < g.NX;
    const int PY = g.PY, PL = (int)g.plane;
    const int idx = (int)(g.origin + Y + (int64_t)g.PY * X + g.plane * Z);
    T y[3] = {T(0), T(0), T(0)};
    if (valid) {
        const int slot = idx - cdy(i) - PY * cdx(i) - PL * cdz(i);
        const T *ke = Ks + ks_slot_base(slot);
        // rows 3i+c, columns 3j+d of the packed symmetric Ks (i is warp-uniform:
        // the offset loads are shared-memory broadcasts)
        if constexpr (sizeof(T) == 4) {
            // FP32: the level's grid is small and the product latency-bound, so
            // all 72 matrix loads of the thread are issued, in order, before any
            // arithmetic uses them (FP64 keeps the interleaved form: 144
            // registers of loads in flight would cost it occupancy)
            T kv[72];
#pragma unroll
            for (int e = 0; e < 72; ++e) kv[e] = ld_stream(ke + offs[(3 * i + e / 24) * 24 + e % 24]);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int m = slot + cdy(j) + PY * cdx(j) + PL * cdz(j);
                const T u[3] = {in(m, 0), in(m, 1), in(m, 2)};
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        y[c] = fma(kv[c * 24 + 3 * j + d], u[d], y[c]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int m = slot + cdy(j) + PY * cdx(j) + PL * cdz(j);
                const T u[3] = {in(m, 0), in(m, 1), in(m, 2)};
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int d = 0; d < 3; ++d)
                        y[c] = fma(__ldg(ke + offs[(3 * i + c) * 24 + 3 * j + d]), u[d], y[c]);
            }
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) part[i][c][n] = y[c];
    __syncthreads();
    double dot = 0.0;
    if (i == 0 && valid) {
        T s[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            s[c] = part[0][c][n];
#pragma unroll
            for (int k = 1; k < 8; ++k) s[c] += part[k][c][n];
        }
        out(idx, s, dot);
    }
    __syncthreads();                     // part is reused by the next tile
    return dot;
}
template <typename T, class In, class Out>
__global__ void __launch_bounds__(kCoarseTileX * 8)
coarse_tile_kernel(In in0, Out out0, const T *__restrict__ Ks, Geom g, Reduce red0, const int *__restrict__ done0)
{
    pdl_enter();
    const int vk = blockIdx.z;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    const In in = in0.shift(vk); const Out out = out0.shift(vk); const Reduce red = red0.at(vk);
    __shared__ T part[8][3][kCoarseTileX];
    __shared__ int offs[24 * 24];
    coarse_offsets(offs, g, threadIdx.x + kCoarseTileX * threadIdx.y, kCoarseTileX * 8);
    __syncthreads();
    const double dot = coarse_tile_unit<T>(in, out, Ks, g, blockIdx.x, blockIdx.y, threadIdx.x, threadIdx.y, part, offs);
    if (red.result) block_sum_to<kCoarseTileX * 8>(dot, red.partials, red.counter, red.result, gridDim.x * gridDim.y,
                                                   blockIdx.x + gridDim.x * blockIdx.y);
}
__host__ __device__ inline dim3 coarse_tile_grid(const Geom &g)
{
    return dim3((unsigned)(((int64_t)g.PY * g.NX + kCoarseTileX - 1) / kCoarseTileX), (unsigned)g.NZ);
}

inline unsigned coarse_blocks(const Geom &g)
{
    const int64_t threads = (int64_t)g.PY * g.NX * g.NZ * kCoarseLanes;
    return (unsigned)((threads + kNodeThreads - 1) / kNodeThreads);
}

// ---------------------------------------------------------------------------
// Two-pass coarse product (the larger coarse levels).  The one-pass tile
// kernel issues 72 scattered scalar loads of packed matrix entries per thread
// and waits on their latency.  Here:
//
//  pass 1 (coarse_elem_kernel): a persistent loop over the packed tiles (32
//    consecutive element slots x 300 entries, contiguous in the
//    tile-interleaved layout).  One thread copies each tile into shared
//    memory with a single bulk copy (cp.async.bulk, completion on an
//    mbarrier), two tiles in flight per CTA, and the CTA forms the outputs
//    w_e = K_e u_e of its 32 elements there: thread (e, i) gathers u at
//    corner i of element slot e, then computes rows 3i..3i+2 (corner i) with
//    the multiply-add order of coarse_tile_unit.  w goes to W, laid out
//    [tile][24][32] like the packed matrices;
//  pass 2 (coarse_gather_kernel): one thread per node slot adds the rows of
//    its corner in its eight incident elements, corners 0..7 in order (the
//    tile kernel's order), and applies the epilogue.
//
// Both passes evaluate the same expressions in the same order as the tile
// kernel, so the products agree bit for bit.  W slots that pass 1 never
// writes (guards before the first and after the last element) stay zero from
// the allocation; slots in its range without an element hold zero matrices.
// Every mbarrier wait is bounded: when one gives up, the CTA stops, raises
// the error flag and waits (bounded) for its copies still in flight.
constexpr int kWTileVals = 24 * kKsTile;
inline int64_t w_alloc_vals(int64_t cs) { return (cs / kKsTile + 3) * (int64_t)kWTileVals; }
constexpr int64_t kWFront = kWTileVals;
constexpr int kElemThreads = 256;                  // 32 element slots x 8 corners

namespace bulk {
constexpr uint32_t kWaitLimit = 1u << 22;           // polls, a backstop to the time limit
constexpr uint64_t kWaitNs = 1000000000ull;         // a wait gives up after one second
__device__ __forceinline__ uint64_t now_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void bar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void arrive_expect(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
}
// bounded wait for the phase of the given parity; false when the limit ran
// out (one second, or kWaitLimit polls)
__device__ __forceinline__ bool wait(uint32_t bar, uint32_t parity)
{
    const uint64_t t0 = now_ns();
    for (uint32_t it = 0; it < kWaitLimit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
        if (ok) return true;
        if (now_ns() - t0 > kWaitNs) return false;
    }
    return false;
}
// bytes (a multiple of 16) from a 16-byte aligned global address into this
// CTA's shared memory (16-byte aligned), completing on the mbarrier
__device__ __forceinline__ void copy(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}
}  // namespace bulk

template <typename T> struct CoarseElem {
    static constexpr uint32_t kTileBytes = (uint32_t)(sizeof(T) * kKsTileVals);   // one packed tile
    static constexpr size_t kOffBar = sizeof(T) * (2 * (size_t)kKsTileVals + kWTileVals);
    static constexpr size_t kSmem = kOffBar + 16;                                 // + two mbarriers
    static_assert(kTileBytes % 16 == 0 && kOffBar % 8 == 0, "bulk copy sizes and mbarrier alignment");
};
// first and count of the packed tiles holding a level's element slots
// (element (Y, X, Z) at its base node's slot, Y < NY - 1, X < NX - 1, Z < NZ - 1)
inline void coarse_elem_tiles(const Geom &g, int &t0, int &nt)
{
    if (g.NY < 2 || g.NX < 2 || g.NZ < 2) { t0 = 0; nt = 0; return; }
    const int64_t lo = g.origin, hi = g.origin + (g.NY - 2) + (int64_t)g.PY * (g.NX - 2) + g.plane * (g.NZ - 2);
    t0 = (int)(lo / kKsTile);
    nt = (int)(hi / kKsTile) - t0 + 1;
}
// rows 3I..3I+2 of element lane e (packed tile ks [300][32], operand us
// [24][32]) into w[(3I + c) * 32], w = the lane's slot of the W tile
template <typename T, int I>
__device__ __forceinline__ void coarse_elem_rows(const T *ks, const T *us, int e, T *w)
{
    T y[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int d = 0; d < 3; ++d)
                y[c] = fma(ks[sym_pack(3 * I + c, 3 * j + d) * kKsTile + e], us[(3 * j + d) * kKsTile + e], y[c]);
#pragma unroll
    for (int c = 0; c < 3; ++c) w[(3 * I + c) * kKsTile] = y[c];
}
template <typename T, class In>
__global__ void __launch_bounds__(kElemThreads)
coarse_elem_kernel(In in0, const T *__restrict__ Ks, T *__restrict__ W0, int64_t wvs, Geom g, int t0, int nt,
                   const int *__restrict__ done0, int *err, int withhold)
{
    pdl_enter();
    const int vk = blockIdx.y;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    const In in = in0.shift(vk);
    T *W = W0 + vk * wvs;
    extern __shared__ __align__(128) unsigned char coarse_smem[];
    T *kbuf = reinterpret_cast<T *>(coarse_smem);          // two packed tiles
    T *us = kbuf + 2 * kKsTileVals;                          // [24][32] element operands
    const uint32_t bar = bulk::smem_addr(coarse_smem + CoarseElem<T>::kOffBar);   // one mbarrier per tile buffer
    const int tid = threadIdx.x, e = tid & 31, i = tid >> 5;
    const int cornerOff = cdy(i) + g.PY * cdx(i) + (int)g.plane * cdz(i);
    if (tid == 0) {
        bulk::bar_init(bar, 1u);
        bulk::bar_init(bar + 8, 1u);
        bulk::fence_init();
    }
    __syncthreads();
    // tile k of this CTA's share into buffer k & 1 (thread 0)
    auto issued = [&](int k) { return blockIdx.x + k * gridDim.x < nt; };
    // withhold: CTA 0 does not issue its first tile (the host's test of the
    // give-up path: that wait runs out and the error flag goes up)
    auto issue = [&](int k) {
        if (!issued(k) || (withhold && blockIdx.x == 0 && k == 0)) return;
        const uint32_t b = bar + 8 * (k & 1);
        bulk::arrive_expect(b, CoarseElem<T>::kTileBytes);
        bulk::copy(bulk::smem_addr(kbuf + (k & 1) * kKsTileVals), Ks + (int64_t)(t0 + blockIdx.x + k * gridDim.x) * kKsTileVals,
                   CoarseElem<T>::kTileBytes, b);
    };
    if (tid == 0) { issue(0); issue(1); }
    // operand of corner i of element slot t*32 + e: node m = t*32 + e + cornerOff
    const int mStep = (int)gridDim.x * kKsTile;
    int m = (t0 + (int)blockIdx.x) * kKsTile + e + cornerOff;
    T u[3] = {T(0), T(0), T(0)};
    if (issued(0)) in.node3(m, u);
    int k = 0;
    bool failed = false;
    for (; issued(k); ++k) {
        const int t = t0 + blockIdx.x + k * gridDim.x;
#pragma unroll
        for (int c = 0; c < 3; ++c) us[(3 * i + c) * kKsTile + e] = u[c];
        const bool got = bulk::wait(bar + 8 * (k & 1), (uint32_t)(k >> 1) & 1u);
        if (!__syncthreads_and(got)) { failed = true; break; }     // uniform: every thread leaves
        m += mStep;
        if (issued(k + 1)) in.node3(m, u);                   // the next tile's operand, loaded during this one
        const T *ks = kbuf + (k & 1) * kKsTileVals;
        T *w = W + (int64_t)t * kWTileVals + e;
        switch (i) {                                         // warp-uniform: immediate entry offsets
        case 0: coarse_elem_rows<T, 0>(ks, us, e, w); break;
        case 1: coarse_elem_rows<T, 1>(ks, us, e, w); break;
        case 2: coarse_elem_rows<T, 2>(ks, us, e, w); break;
        case 3: coarse_elem_rows<T, 3>(ks, us, e, w); break;
        case 4: coarse_elem_rows<T, 4>(ks, us, e, w); break;
        case 5: coarse_elem_rows<T, 5>(ks, us, e, w); break;
        case 6: coarse_elem_rows<T, 6>(ks, us, e, w); break;
        default: coarse_elem_rows<T, 7>(ks, us, e, w); break;
        }
        __syncthreads();                                     // buffer k & 1 and the operands are free
        if (tid == 0) issue(k + 2);
    }
    if (failed && tid == 0) {
        atomicExch(err, 1);
        // tiles k and k + 1 may still be landing: wait for them (bounded)
        for (int kk = k; kk < k + 2; ++kk)
            if (issued(kk) && !(withhold && blockIdx.x == 0 && kk == 0))
                (void)bulk::wait(bar + 8 * (kk & 1), (uint32_t)(kk >> 1) & 1u);
    }
}
template <typename T, class Out>
__global__ void __launch_bounds__(kNodeThreads)
coarse_gather_kernel(Out out0, const T *__restrict__ W0, int64_t wvs, Geom g, Reduce red0, const int *__restrict__ done0)
{
    pdl_enter();
    const int vk = blockIdx.z;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    const Out out = out0.shift(vk); const Reduce red = red0.at(vk);
    const T *W = W0 + vk * wvs;
    const int q = blockIdx.x * kNodeThreads + threadIdx.x;
    const int Y = q % g.PY, X = q / g.PY, Z = blockIdx.y;
    double dot = 0.0;
    if (Y < g.NY && X < g.NX) {
        const int idx = (int)(g.origin + Y + (int64_t)g.PY * X + g.plane * Z);
        T p[8][3];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int slot = idx - cdy(i) - g.PY * cdx(i) - (int)g.plane * cdz(i);
            const T *w = W + (int64_t)(slot >> 5) * kWTileVals + (slot & 31);
#pragma unroll
            for (int c = 0; c < 3; ++c) p[i][c] = w[(3 * i + c) * kKsTile];
        }
        T s[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            s[c] = p[0][c];
#pragma unroll
            for (int k = 1; k < 8; ++k) s[c] += p[k][c];
        }
        out(idx, s, dot);
    }
    if (red.result) block_sum_to<kNodeThreads>(dot, red.partials, red.counter, red.result, gridDim.x * gridDim.y,
                                               blockIdx.x + gridDim.x * blockIdx.y);
}

// ---------------------------------------------------------------------------
// Transfers between level l (fine) and l+1 (coarse), span S.  Prolongation
// is trilinear interpolation of the coarse field at the fine active nodes;
// restriction is its transpose.  (TOP_GPU.m:817-878 express the same
// operators through an intermediate node set with multiplicity weights; for
// every active node the two coincide.)
// One lane group per coarse node (32 lanes for span 4, 8 for span 2): the
// (2S-1)^2 (z, x) tap columns are dealt out over the group, each lane runs
// its columns' 2S-1 y taps, the group adds up with shuffles.
// (a, b, c) of index k = a + na (b + nb c), k < na nb nc: 32-bit unsigned
// division when k fits (every grid here), the 64-bit one otherwise (the
// same results; a 64-bit division by a run-time value is a long sequence)
__device__ __forceinline__ void split3(int64_t k, int na, int nb, int &a, int &b, int &c)
{
    if (k < (int64_t)0xffffffff) {
        const unsigned u = (unsigned)k, q = u / (unsigned)na;
        a = (int)(u - q * (unsigned)na); b = (int)(q % (unsigned)nb); c = (int)(q / (unsigned)nb);
    } else {
        a = (int)(k % na); b = (int)((k / na) % nb); c = (int)(k / ((int64_t)na * nb));
    }
}

template <int S> struct RestrictLanes { static constexpr int value = (S >= 4) ? 32 : 8; };

// lane-group restriction of one coarse node; gt = the thread's index in the
// lane layout (LPN lanes per coarse node; every lane of a warp must call it)
template <typename T, int S>
__device__ __forceinline__ void restrict_lanes(const T *__restrict__ rf, const Geom &gf, T *__restrict__ rc, const Geom &gc,
                                               const uint8_t *__restrict__ flagsC, int64_t gt, T *__restrict__ cmp = nullptr,
                                               const int32_t *__restrict__ slotCmp = nullptr)
{
    constexpr int LPN = RestrictLanes<S>::value, W = 2 * S - 1;
    const int64_t node = gt / LPN;
    const int lane = int(gt % LPN);
    const int64_t nq = (int64_t)gc.PY * gc.NX * gc.NZ;
    const bool inRange = node < nq;
    const int64_t nq2 = inRange ? node : 0;
    int QY, QX, QZ;
    split3(nq2, gc.PY, gc.NX, QY, QX, QZ);
    const bool valid = inRange && QY < gc.NY;
    const int64_t ic = gc.origin + QY + (int64_t)gc.PY * QX + gc.plane * QZ;
    T acc[3] = {T(0), T(0), T(0)};
    if (valid && (flagsC[ic] & kActive)) {
        for (int pr = lane; pr < W * W; pr += LPN) {
            const int oz = pr / W - (S - 1), ox = pr % W - (S - 1);
            const int Z = S * QZ + oz, X = S * QX + ox;
            if (Z < 0 || Z >= gf.NZ || X < 0 || X >= gf.NX) continue;
            const T wzx = (T(S - (oz < 0 ? -oz : oz)) / T(S)) * (T(S - (ox < 0 ? -ox : ox)) / T(S));
            const int64_t base = gf.origin + (int64_t)gf.PY * X + gf.plane * Z;
#pragma unroll
            for (int oy = -(S - 1); oy <= S - 1; ++oy) {
                const int Y = S * QY + oy;
                if (Y < 0 || Y >= gf.NY) continue;
                const T w = wzx * (T(S - (oy < 0 ? -oy : oy)) / T(S));
#pragma unroll
                for (int c = 0; c < 3; ++c) acc[c] = fma(w, rf[c * gf.cs + base + Y], acc[c]);
            }
        }
    }
#pragma unroll
    for (int o = LPN / 2; o > 0; o >>= 1)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[c] += __shfl_down_sync(0xffffffffu, acc[c], o, LPN);
    if (valid && lane == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) rc[c * gc.cs + ic] = acc[c];
        // also in compact order (3 node + c) when asked: the condensed tail's operand
        if (cmp) {
            const int32_t kc = slotCmp[ic];
            if (kc >= 0)
#pragma unroll
                for (int c = 0; c < 3; ++c) cmp[3 * (int64_t)kc + c] = acc[c];
        }
    }
}
template <typename T, int S>
__global__ void __launch_bounds__(kNodeThreads)
restrict_kernel(const T *__restrict__ rf, Geom gf, T *__restrict__ rc, Geom gc,
                const uint8_t *__restrict__ flagsC, const int *__restrict__ done0, int64_t vsF = 0, int64_t vsC = 0,
                T *__restrict__ cmp = nullptr, const int32_t *__restrict__ slotCmp = nullptr, int64_t vsCmp = 0)
{
    pdl_enter();
    const int vk = blockIdx.y;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    rf += vk * vsF; rc += vk * vsC;
    if (cmp) cmp += vk * vsCmp;
    restrict_lanes<T, S>(rf, gf, rc, gc, flagsC, (int64_t)blockIdx.x * kNodeThreads + threadIdx.x, cmp, slotCmp);
}
template <int S>
inline unsigned restrict_blocks(const Geom &gc)
{
    const int64_t threads = (int64_t)gc.PY * gc.NX * gc.NZ * RestrictLanes<S>::value;
    return (unsigned)((threads + kNodeThreads - 1) / kNodeThreads);
}

// Separable restriction (trilinear weights factor per axis): pass A folds the
// fine y taps, t[c][QY][X][Z] = sum_oy w(oy) r_f[c][S QY + oy][X][Z] (dense
// NYc x NXf x NZf per component), passes B and C (one launch) fold x, then z.
// Same weights and clipping as restrict_kernel; every pass reads runs of
// consecutive QY.  V4 (S = 4): the seven taps 4 QY - 3 ..
// 4 QY + 3 come from two aligned four-value loads per component (slots
// 4 QY - 4 .. 4 QY + 3 of the column; the first and any past NY are not used),
// summed in the same order.
template <typename T, int S, bool V4 = false>
__global__ void __launch_bounds__(256)
restrict_y_kernel(const T *__restrict__ rf, Geom gf, T *__restrict__ t, int NYc, const int *__restrict__ done0,
                  int64_t vsF = 0, int64_t vsT = 0)
{
    static_assert(!V4 || S == 4, "vector taps need span 4");
    pdl_enter();
    const int vk = blockIdx.y;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    rf += vk * vsF; t += vk * vsT;
    const int64_t nt = (int64_t)NYc * gf.NX * gf.NZ;
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nt) return;
    int QY, X, Z;
    split3(k, NYc, gf.NX, QY, X, Z);
    const int64_t base = gf.origin + (int64_t)gf.PY * X + gf.plane * Z;
    T acc[3] = {T(0), T(0), T(0)};
    if constexpr (V4) {
        T lo[3][4], hi[3][4];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T *p = rf + c * gf.cs + base + S * QY;
            ld4(p - 4, lo[c]);
            ld4(p, hi[c]);
        }
#pragma unroll
        for (int oy = -(S - 1); oy <= S - 1; ++oy) {
            const int Y = S * QY + oy;
            if (Y < 0 || Y >= gf.NY) continue;
            const T w = T(S - (oy < 0 ? -oy : oy)) / T(S);
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[c] = fma(w, oy < 0 ? lo[c][4 + oy] : hi[c][oy], acc[c]);
        }
    } else {
#pragma unroll
        for (int oy = -(S - 1); oy <= S - 1; ++oy) {
            const int Y = S * QY + oy;
            if (Y < 0 || Y >= gf.NY) continue;
            const T w = T(S - (oy < 0 ? -oy : oy)) / T(S);
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[c] = fma(w, rf[c * gf.cs + base + Y], acc[c]);
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) t[c * nt + k] = acc[c];
}
// passes B and C in one launch: CTA (QX, QZ, 32 coarse y nodes) of 2S-1
// warps; warp w folds the x taps of fine plane Z = S QZ + w - (S-1) (the x
// pass's sum, in its order) into shared memory, then the first warp folds the
// z taps in the z pass's order: the two passes' results, bit for bit, without
// their intermediate array and second launch
template <typename T, int S>
__global__ void __launch_bounds__(32 * (2 * S - 1))
restrict_xz_kernel(const T *__restrict__ t, int NXf, int NZf, T *__restrict__ rc, Geom gc,
                   const uint8_t *__restrict__ flagsC, const int *__restrict__ done0, int64_t vsT = 0, int64_t vsC = 0,
                   T *__restrict__ cmp = nullptr, const int32_t *__restrict__ slotCmp = nullptr, int64_t vsCmp = 0)
{
    pdl_enter();
    const int vk = blockIdx.z;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    t += vk * vsT; rc += vk * vsC;
    if (cmp) cmp += vk * vsCmp;
    const int NYc = gc.NY, NXc = gc.NX;
    const int64_t nt = (int64_t)NYc * NXf * NZf;
    const int QX = (int)(blockIdx.x % NXc), QZ = (int)(blockIdx.x / NXc);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int QY = (int)blockIdx.y * 32 + lane;
    __shared__ T sx[2 * S - 1][3][32];
    const int Z = S * QZ + w - (S - 1);
    T acc[3] = {T(0), T(0), T(0)};
    if (QY < NYc && Z >= 0 && Z < NZf) {
#pragma unroll
        for (int ox = -(S - 1); ox <= S - 1; ++ox) {
            const int X = S * QX + ox;
            if (X < 0 || X >= NXf) continue;
            const T wt = T(S - (ox < 0 ? -ox : ox)) / T(S);
            const int64_t o = QY + (int64_t)NYc * (X + (int64_t)NXf * Z);
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[c] = fma(wt, t[c * nt + o], acc[c]);
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) sx[w][c][lane] = acc[c];
    __syncthreads();
    if (w == 0 && QY < NYc) {
        const int64_t ic = gc.origin + QY + (int64_t)gc.PY * QX + gc.plane * QZ;
        T out[3] = {T(0), T(0), T(0)};
        if (flagsC[ic] & kActive) {
#pragma unroll
            for (int oz = -(S - 1); oz <= S - 1; ++oz) {
                const int Zz = S * QZ + oz;
                if (Zz < 0 || Zz >= NZf) continue;
                const T wt = T(S - (oz < 0 ? -oz : oz)) / T(S);
#pragma unroll
                for (int c = 0; c < 3; ++c) out[c] = fma(wt, sx[oz + S - 1][c][lane], out[c]);
            }
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) rc[c * gc.cs + ic] = out[c];
        if (cmp) {                               // also in compact order (the condensed tail's operand)
            const int32_t kc = slotCmp[ic];
            if (kc >= 0)
#pragma unroll
                for (int c = 0; c < 3; ++c) cmp[3 * (int64_t)kc + c] = out[c];
        }
    }
}

// One row of the coarsest direct solve, x(row) = A^-1(row, :) c, for the
// right-hand sides v0 .. v0+3 whose act flag is set (cr(k, j): entry j of
// right-hand side k).  All kCoarsestThreads threads of the CTA call it: each keeps
// eight loads of the row in flight, the warps reduce by shuffles and thread
// 0 adds the warp sums in a fixed order and returns them in out.
constexpr int kCoarsestThreads = 256;
// coarsest right-hand sides gathered in compact order (k at cr + k n)
struct CompactRhs {
    const double *cr; int64_t n;
    __device__ __forceinline__ double operator()(int k, int64_t j) const { return cr[k * n + j]; }
};
// ... or staged in shared memory ([k - v0][n] for the group starting at v0)
struct StagedRhs {
    const double *s; int64_t n; int v0;
    __device__ __forceinline__ double operator()(int k, int64_t j) const { return s[(k - v0) * n + j]; }
};
// ... or read from the level's grid vector (k at r + k vs)
template <typename T> struct GridRhs {
    const T *r; int64_t vs, cs; const int32_t *nodeGrid;
    __device__ __forceinline__ double operator()(int k, int64_t j) const { return double(r[k * vs + (j % 3) * cs + nodeGrid[j / 3]]); }
};
template <class Rhs>
__device__ __forceinline__ void coarsest_row(const double *__restrict__ a, const Rhs &cr, int64_t n, int v0,
                                             const bool act[4], double (*red)[4], double out[4])
{
    constexpr int U = 8, NW = kCoarsestThreads / 32;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t j0 = tid; j0 < n; j0 += (int64_t)kCoarsestThreads * U) {
        double av[U];
#pragma unroll
        for (int u = 0; u < U; ++u) av[u] = j0 + kCoarsestThreads * u < n ? a[j0 + kCoarsestThreads * u] : 0.0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int64_t j = j0 + kCoarsestThreads * u;
            if (j >= n) break;
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (act[q]) s[q] = fma(av[u], cr(v0 + q, j), s[q]);
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_down_sync(0xffffffffu, s[q], o);
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) red[wid][q] = s[q];
    __syncthreads();
    if (tid == 0)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            double v = red[0][q];
            for (int w = 1; w < NW; ++w) v += red[w][q];
            out[q] = v;
        }
    __syncthreads();                     // red is reused by the next call
}

// Span-4 prolongation, four fine y nodes per thread: the fine nodes
// Y = 4 QY + ry (ry = 0..3) of one fine (X, Z) column share their coarse
// corner values, which are loaded once.  Per node the weights, skipped
// zero-weight corners and the order of the sum are those of prolong_node
// (identical results).  XB: the base is the value xf holds; otherwise
// omega*invD.*r (or 0 when r is null).  V4: the four fine slots of a thread
// are read as one aligned vector per array (slots past NY are y padding of
// the same column, read but not used) and written as one where all four are
// grid nodes (per node otherwise, so padding is never written).
template <typename T, typename TR, bool XB, bool V4 = false>
__global__ void __launch_bounds__(kNodeThreads)
prolong4_kernel(const T *__restrict__ xc, Geom gc, T *__restrict__ xf, Geom gf,
                const uint8_t *__restrict__ flagsF, const TR *__restrict__ r,
                const T *__restrict__ invD, T omega, const int *__restrict__ done0,
                int64_t vsC = 0, int64_t vsF = 0, int64_t vsR = 0)
{
    pdl_enter();
    constexpr int S = 4;
    const int vk = blockIdx.y;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    xc += vk * vsC; xf += vk * vsF;
    if (r) r += vk * vsR;
    const int nqy = (gf.NY + S - 1) / S;
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (int64_t)nqy * gf.NX * gf.NZ) return;
    int qy, X, Z;
    split3(k, nqy, gf.NX, qy, X, Z);
    const int qx = X / S, rx = X - qx * S, qz = Z / S, rz = Z - qz * S;
    const T wx[2] = {T(S - rx) / T(S), T(rx) / T(S)};
    const T wz[2] = {T(S - rz) / T(S), T(rz) / T(S)};
    // coarse corner values [bz][bx][by][c]; by = 1 is read only where some ry > 0 uses it
    T cv[2][2][2][3];
    const bool yNext = S * qy + 1 < gf.NY;
#pragma unroll
    for (int bz = 0; bz < 2; ++bz)
#pragma unroll
        for (int bx = 0; bx < 2; ++bx)
#pragma unroll
            for (int by = 0; by < 2; ++by) {
                const bool need = (bz == 0 || rz != 0) && (bx == 0 || rx != 0) && (by == 0 || yNext);
                const int64_t kc = gc.origin + (qy + by) + (int64_t)gc.PY * (qx + bx) + gc.plane * (qz + bz);
#pragma unroll
                for (int c = 0; c < 3; ++c) cv[bz][bx][by][c] = need ? xc[c * gc.cs + kc] : T(0);
            }
    const int64_t i0 = gf.origin + S * qy + (int64_t)gf.PY * X + gf.plane * Z;
    // every fine load (flags, base) issued before the arithmetic
    // (XB: bs is the stored base; else bs = invD and br = r, combined at the
    // add exactly as prolong_node does)
    uint8_t fl[S];
    T bs[S][3], br[S][3];
    if constexpr (V4) {
        static_assert(S == 4, "vector slots need span 4");
        const uchar4 f4 = *reinterpret_cast<const uchar4 *>(flagsF + i0);
        fl[0] = f4.x; fl[1] = f4.y; fl[2] = f4.z; fl[3] = f4.w;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            T a[S] = {T(0), T(0), T(0), T(0)};
            TR b[S] = {TR(0), TR(0), TR(0), TR(0)};
            if constexpr (XB) ld4(xf + c * gf.cs + i0, a);
            else if (r) { ld4(invD + c * gf.cs + i0, a); ld4(r + c * gf.cs + i0, b); }
#pragma unroll
            for (int ry = 0; ry < S; ++ry) { bs[ry][c] = a[ry]; br[ry][c] = T(b[ry]); }
        }
    } else {
#pragma unroll
        for (int ry = 0; ry < S; ++ry) {
            const bool on = S * qy + ry < gf.NY;
            const int64_t i = i0 + ry;
            fl[ry] = on ? flagsF[i] : uint8_t(0);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                bs[ry][c] = !on ? T(0) : XB ? xf[c * gf.cs + i] : r ? invD[c * gf.cs + i] : T(0);
                br[ry][c] = (!on || XB || !r) ? T(0) : T(r[c * gf.cs + i]);
            }
        }
    }
    T out[S][3];
#pragma unroll
    for (int ry = 0; ry < S; ++ry) {
        if constexpr (!V4) { if (S * qy + ry >= gf.NY) break; }
        const int64_t i = i0 + ry;
        const T wy[2] = {T(S - ry) / T(S), T(ry) / T(S)};
        T v[3] = {T(0), T(0), T(0)};
        if (fl[ry] & kActive) {
#pragma unroll
            for (int bz = 0; bz < 2; ++bz) {
                if (bz && rz == 0) continue;
#pragma unroll
                for (int bx = 0; bx < 2; ++bx) {
                    if (bx && rx == 0) continue;
#pragma unroll
                    for (int by = 0; by < 2; ++by) {
                        if (by && ry == 0) continue;
                        const T w = wz[bz] * wx[bx] * wy[by];
#pragma unroll
                        for (int c = 0; c < 3; ++c) v[c] = fma(w, cv[bz][bx][by][c], v[c]);
                    }
                }
            }
            if (XB) {
#pragma unroll
                for (int c = 0; c < 3; ++c) v[c] += bs[ry][c];
            } else if (r) {
#pragma unroll
                for (int c = 0; c < 3; ++c) v[c] += omega * bs[ry][c] * br[ry][c];
            }
        }
        if constexpr (V4) {
#pragma unroll
            for (int c = 0; c < 3; ++c) out[ry][c] = v[c];
        } else {
#pragma unroll
            for (int c = 0; c < 3; ++c) xf[c * gf.cs + i] = v[c];
        }
    }
    if constexpr (V4) {
        if (S * qy + S <= gf.NY) {
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const T w4[S] = {out[0][c], out[1][c], out[2][c], out[3][c]};
                st4(xf + c * gf.cs + i0, w4);
            }
        } else {
#pragma unroll
            for (int ry = 0; ry < S; ++ry)
                if (S * qy + ry < gf.NY)
#pragma unroll
                    for (int c = 0; c < 3; ++c) xf[c * gf.cs + i0 + ry] = out[ry][c];
        }
    }
}

// the prolongation's value at the grid node (Y, X, Z) = slot i of the fine
// grid (a node of the grid, Y < NY, X < NX): 0 at an inactive node, else
// P xc (span S) plus the base -- the value xf holds there when XB,
// omega*invD.*r when r is set
template <typename T, int S, typename TR, bool XB = false>
__device__ __forceinline__ void prolong_value(const T *__restrict__ xc, const Geom &gc, const T *__restrict__ xf, const Geom &gf,
                                              const uint8_t *__restrict__ flagsF, const TR *__restrict__ r,
                                              const T *__restrict__ invD, T omega, int Y, int X, int Z, int64_t i, T v[3])
{
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = T(0);
    if (flagsF[i] & kActive) {
        const int qy = Y / S, ry = Y - qy * S, qx = X / S, rx = X - qx * S, qz = Z / S, rz = Z - qz * S;
        const T wy[2] = {T(S - ry) / T(S), T(ry) / T(S)};
        const T wx[2] = {T(S - rx) / T(S), T(rx) / T(S)};
        const T wz[2] = {T(S - rz) / T(S), T(rz) / T(S)};
#pragma unroll
        for (int bz = 0; bz < 2; ++bz) {
            if (bz && rz == 0) continue;
#pragma unroll
            for (int bx = 0; bx < 2; ++bx) {
                if (bx && rx == 0) continue;
#pragma unroll
                for (int by = 0; by < 2; ++by) {
                    if (by && ry == 0) continue;
                    const T w = wz[bz] * wx[bx] * wy[by];
                    const int64_t k = gc.origin + (qy + by) + (int64_t)gc.PY * (qx + bx) + gc.plane * (qz + bz);
#pragma unroll
                    for (int c = 0; c < 3; ++c) v[c] = fma(w, xc[c * gc.cs + k], v[c]);
                }
            }
        }
        if (XB) {
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] += xf[c * gf.cs + i];
        } else if (r) {
#pragma unroll
            for (int c = 0; c < 3; ++c) v[c] += omega * invD[c * gf.cs + i] * T(r[c * gf.cs + i]);
        }
    }
}
// one fine node (linear in-plane index q, layer Z) of the prolongation;
// XB: the base omega*invD.*r was stored in xf beforehand (added in place)
template <typename T, int S, typename TR, bool XB = false>
__device__ __forceinline__ void prolong_node(const T *__restrict__ xc, const Geom &gc, T *__restrict__ xf, const Geom &gf,
                                             const uint8_t *__restrict__ flagsF, const TR *__restrict__ r,
                                             const T *__restrict__ invD, T omega, int q, int Z)
{
    const int Y = q % gf.PY, X = q / gf.PY;
    if (Y >= gf.NY || X >= gf.NX) return;
    const int64_t i = gf.origin + Y + (int64_t)gf.PY * X + gf.plane * Z;
    T v[3];
    prolong_value<T, S, TR, XB>(xc, gc, xf, gf, flagsF, r, invD, omega, Y, X, Z, i, v);
#pragma unroll
    for (int c = 0; c < 3; ++c) xf[c * gf.cs + i] = v[c];
}
// x_f = base + P x_c, base = omega*invD.*r when r != nullptr (the pre-smoothed
// iterate of the V-cycle, recomputed), the value x_f holds when XB, else 0.
template <typename T, int S, typename TR, bool XB = false>
__global__ void __launch_bounds__(kNodeThreads)
prolong_kernel(const T *__restrict__ xc, Geom gc, T *__restrict__ xf, Geom gf,
               const uint8_t *__restrict__ flagsF, const TR *__restrict__ r,
               const T *__restrict__ invD, T omega, const int *__restrict__ done0,
               int64_t vsC = 0, int64_t vsF = 0, int64_t vsR = 0)
{
    pdl_enter();
    const int vk = blockIdx.z;
    const int *done = done_of(done0, vk);
    if (done && *done) return;
    xc += vk * vsC; xf += vk * vsF;
    if (r) r += vk * vsR;
    prolong_node<T, S, TR, XB>(xc, gc, xf, gf, flagsF, r, invD, omega, blockIdx.x * kNodeThreads + threadIdx.x, blockIdx.y);
}

}  // namespace topgpu
