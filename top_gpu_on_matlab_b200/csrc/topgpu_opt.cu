// topgpu_opt.cu -- the optimisation steps either side of the FEA solve, on
// the device: element energies and sensitivities (TOP_GPU.m:580-600,
// 168-209), the PDE density/sensitivity filter (880-1031), the OC update
// with bisection (232-253) and the loop that ties them to the solver
// (141-292).
#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include "topgpu_kernels.cuh"
#include "topgpu_solver_impl.cuh"

namespace cg = cooperative_groups;
using namespace topgpu;

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e__ = (call);                                                                \
        if (e__ != cudaSuccess) { set_error("top_opt: CUDA error %d: %s", (int)e__, cudaGetErrorString(e__)); return TOP_ERR_CUDA; } \
    } while (0)

namespace topgpu {

struct OptScalars {          // device-side scalars of one optimisation iteration
    double cObj, vol, sharp, change, lmid, sumE, fval, pad;
};

struct FilterState {
    bool ready = false;
    double rMin = 0;
    KeParam<double> KEF{};   // 8x8 in k[0..63], col-major
    double *act = nullptr;   // element activity on the level-0 element slots (1/0)
    double *invD = nullptr;  // Jacobi of the filter operator, node grid
    double *rhs = nullptr, *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *v = nullptr, *eg = nullptr;
    PcgState *st = nullptr;
    double *part2 = nullptr;           // per-CTA partials of rho = z.r (the update's second sum)
    cudaGraphExec_t chunk = nullptr;   // kChunk filter-PCG iterations as one graph (built on first use)
    int64_t chunkNodes = 0;
};

struct AdjState {
    double *U = nullptr;     // [nLoads][3 x cs] state fields
    double *L = nullptr;     // [3 x cs] adjoint field
    double *e = nullptr;     // [3 x cs] unit load
    double *g = nullptr, *t = nullptr;   // element vectors [Ne]
    double *J = nullptr;     // device scalar
};

// Super-element density filter on the 4x refined sub-voxel grid
// (TOP_GPU.m:113-121, 221-227, 262-265): h = max(0, 4 rMin - dist) over a
// (2R+1)^3 box, R = ceil(4 rMin) - 1, imfilter with zero padding;
// Hs = imfilter(ones, h).
struct SFilterState {
    bool ready = false;
    double rMin = 0;
    int R = 0, fy = 0, fx = 0, fz = 0;
    double *h = nullptr, *Hs = nullptr, *g = nullptr, *t = nullptr;
};

struct OptState {
    bool begun = false;
    top_opt_params prm{};
    double cSolid = 0;
    int loop = 0;
    double change = 1.0, sharp = 1.0;
    double *xd = nullptr, *xPhys = nullptr, *xnew = nullptr, *dc = nullptr, *dv = nullptr, *ce = nullptr, *tmp = nullptr;
    double *U = nullptr;     // [nLoads][3 x cs] grid displacement fields (warm starts)
    OptScalars *sc = nullptr, *hsc = nullptr;
    double *ocPartials = nullptr; int ocBlocks = 0;   // 2 x ocBlocks block sums
    double *ocR = nullptr;                              // -dc./dv of the bisection
    int64_t nv = 0;          // design variables (64 per super-element)
    SFilterState sf;         // super-element density filter
    // passive elements: 1 on the design variables held at 1 (TOP_GPU.m:239, 270;
    // super elements: sub-voxel row Num_ = 4, 247, 273); used when nPassive > 0
    uint8_t *passive = nullptr; int64_t passiveLen = 0, nPassive = 0;
    std::vector<int> caseIts;   // PCG iterations per load case of the last state solves
};

}  // namespace topgpu

namespace {

inline int vb(int64_t n) { return (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096); }

// ---- PDE filter --------------------------------------------------------------
// Nodal Helmholtz kernel of the reference (TOP_GPU.m:888-920): KEF0 sums the
// products of the natural-coordinate shape derivatives over the 2x2x2 Gauss
// points (no Jacobian, unit weights), KEF1 is the lumped-weight mass
// (weights 1/8); iKEF = (rMin/(2*sqrt 3))^2 KEF0 + KEF1.  Local node order
// (s,t,p) = (-1,-1,-1),(1,-1,-1),(1,1,-1),(-1,1,-1), then p = +1.
void filter_kernel_matrix(double rMin, double *K)
{
    static const int sg[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1}};
    const double g = 1.0 / std::sqrt(3.0);
    double K0[64] = {0}, K1[64] = {0};
    for (int q = 0; q < 8; ++q) {
        const double pt[3] = {sg[q][0] * g, sg[q][1] * g, sg[q][2] * g};
        double N[8], dN[8][3];
        for (int a = 0; a < 8; ++a) {
            double f[3], df[3];
            for (int k = 0; k < 3; ++k) { f[k] = 1.0 + sg[a][k] * pt[k]; df[k] = sg[a][k]; }
            N[a] = 0.125 * f[0] * f[1] * f[2];
            dN[a][0] = 0.125 * df[0] * f[1] * f[2];
            dN[a][1] = 0.125 * f[0] * df[1] * f[2];
            dN[a][2] = 0.125 * f[0] * f[1] * df[2];
        }
        for (int a = 0; a < 8; ++a)
            for (int b = 0; b < 8; ++b) {
                K0[a + 8 * b] += dN[a][0] * dN[b][0] + dN[a][1] * dN[b][1] + dN[a][2] * dN[b][2];
                K1[a + 8 * b] += N[a] * (1.0 / 8.0) * N[b];
            }
    }
    const double iR = rMin / 2.0 / std::sqrt(3.0);    // element size 1 (TOP_GPU.m:918)
    for (int t = 0; t < 64; ++t) K[t] = iR * iR * K0[t] + K1[t];
}

// The filter's local node a sits at (s,t,p); the solver's element corner j at
// (dy,dx,dz).  Both are the same eight nodes of the voxel (TOP_GPU.m:2031-2040
// numbering); the filter reuses the element node order of eNodMat.
__global__ void filter_activity_kernel(const int32_t *__restrict__ eleGrid, int64_t Ne, double *__restrict__ act)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < Ne) act[eleGrid[e]] = 1.0;
}
__global__ void filter_diag_kernel(const KeParam<double> K, const double *__restrict__ act, Geom g,
                                   const uint8_t *__restrict__ flags, double *__restrict__ invD)
{
    const int q = blockIdx.x * kNodeThreads + threadIdx.x;
    const int Y = q % g.PY, X = q / g.PY, Z = blockIdx.y;
    if (Y >= g.NY || X >= g.NX) return;
    const int idx = (int)(g.origin + Y + (int64_t)g.PY * X + g.plane * Z);
    double d = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) d += act[idx - cdy(i) - g.PY * cdx(i) - (int)g.plane * cdz(i)] * K.k[9 * i];
    invD[idx] = (flags[idx] & kActive) && d != 0.0 ? 1.0 / d : 0.0;
}
// y = A_filter x (+ dot x.y), node-centric over the 8 incident elements
__global__ void __launch_bounds__(kNodeThreads)
filter_apply_kernel(const KeParam<double> K, const double *__restrict__ act, const double *__restrict__ x,
                    double *__restrict__ y, Geom g, Reduce red, const int *__restrict__ done)
{
    if (done && *done) return;
    const int q = blockIdx.x * kNodeThreads + threadIdx.x;
    const int Y = q % g.PY, X = q / g.PY, Z = blockIdx.y;
    const bool valid = Y < g.NY && X < g.NX;
    const int idx = (int)(g.origin + Y + (int64_t)g.PY * X + g.plane * Z);
    const int PY = g.PY, PL = (int)g.plane;
    double dot = 0.0;
    if (valid) {
        double s = 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int slot = idx - cdy(i) - PY * cdx(i) - PL * cdz(i);
            const double a = act[slot];
            double t = 0.0;
#pragma unroll
            for (int j = 0; j < 8; ++j) t = fma(K.k[i + 8 * j], x[slot + cdy(j) + PY * cdx(j) + PL * cdz(j)], t);
            s = fma(a, t, s);
        }
        y[idx] = s;
        dot = x[idx] * s;
    }
    if (red.result) block_sum_to<kNodeThreads>(dot, red.partials, red.counter, red.result);
}
// element values (compact) -> element slots
__global__ void elem_to_slots_kernel(const double *__restrict__ src, const int32_t *__restrict__ eleGrid,
                                     int64_t Ne, double scale, double *__restrict__ dst)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < Ne) dst[eleGrid[e]] = src[e] * scale;
}
// nodal rhs: sum of the (pre-scaled) values of the incident elements (TOP_GPU.m:975-996)
__global__ void slots_to_nodes_kernel(const double *__restrict__ eg, Geom g, const uint8_t *__restrict__ flags,
                                      double *__restrict__ rhs)
{
    const int q = blockIdx.x * kNodeThreads + threadIdx.x;
    const int Y = q % g.PY, X = q / g.PY, Z = blockIdx.y;
    if (Y >= g.NY || X >= g.NX) return;
    const int idx = (int)(g.origin + Y + (int64_t)g.PY * X + g.plane * Z);
    double s = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) s += eg[idx - cdy(i) - g.PY * cdx(i) - (int)g.plane * cdz(i)];
    rhs[idx] = (flags[idx] & kActive) ? s : 0.0;
}
// node -> element mean (TOP_GPU.m:1004-1005)
__global__ void nodes_to_elem_kernel(const double *__restrict__ xn, const int32_t *__restrict__ eleGrid, Geom g,
                                     int64_t Ne, double *__restrict__ out)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= Ne) return;
    const int slot = eleGrid[e];
    double s = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += xn[slot + cdy(j) + g.PY * cdx(j) + (int)g.plane * cdz(j)];
    out[e] = s * (1.0 / 8.0);
}
// scalar PCG pieces (one component)
__global__ void fpcg_init_kernel(const double *__restrict__ b, double *__restrict__ x, double *__restrict__ r,
                                 double *__restrict__ z, double *__restrict__ p, const double *__restrict__ invD,
                                 int64_t n, Reduce bb)
{   // x = 0, r = b, z = M r, p = z; ||b||^2
    double s1 = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double bi = b[i], zi = invD[i] * bi;
        x[i] = 0.0; r[i] = bi; z[i] = zi; p[i] = zi;
        s1 += bi * bi;
    }
    block_sum_to<256>(s1, bb.partials, bb.counter, bb.result);
}
// the filter-PCG check: same stopping rule as Solving_PCG (TOP_GPU.m:637-649)
__device__ __forceinline__ void fpcg_check(PcgState *st)
{
    st->its += 1;
    const double res = sqrt(st->rr) / st->normB;
    st->resnorm = res;
    if (!isfinite(res)) { st->status = TOP_ERR_NAN; st->done = 1; return; }
    if (res < st->tol) { st->done = 1; return; }
    if (st->its >= st->maxIT) { st->status = TOP_ERR_NOT_CONVERGED; st->done = 1; return; }
    st->rhoOld = st->rho;
}
// one filter-PCG step after v = A p: x += l p, r -= l v, z = M r, rr = r.r
// and rho = z.r in one pass (four grid strides of loads ahead of the stores;
// each thread adds its terms in index order); the CTA that completes both
// sums runs the iteration's check (TOP_GPU.m:637-649) and then stores rho,
// as the separate update, check and z.r launches did (same sums, same order)
__global__ void __launch_bounds__(256)
fpcg_update_kernel(double *__restrict__ x, double *__restrict__ r, double *__restrict__ z,
                   const double *__restrict__ p, const double *__restrict__ v, const double *__restrict__ invD,
                   int64_t n, PcgState *st, double *__restrict__ part1, double *__restrict__ part2, unsigned *counter)
{
    if (st->done) return;
    const double l = st->rho / st->pv;
    double s1 = 0, s2 = 0;
    const int64_t S = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += 4 * S) {
        double xo[4], po[4], ro[4], vo[4], dq[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (i + q * S < n) {
                const int64_t k = i + q * S;
                xo[q] = x[k]; po[q] = p[k]; ro[q] = r[k]; vo[q] = v[k]; dq[q] = invD[k];
            }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (i + q * S < n) {
                const int64_t k = i + q * S;
                x[k] = xo[q] + l * po[q];
                const double ri = ro[q] - l * vo[q];
                r[k] = ri;
                const double zi = dq[q] * ri;
                z[k] = zi;
                s1 += ri * ri;
                s2 += zi * ri;
            }
    }
    // two block sums, each as block_sum_last forms it; the last CTA adds the
    // partials of both in index order
    __shared__ double red[2][8];
    __shared__ bool last;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const unsigned nb = gridDim.x, bid = blockIdx.x;
    for (int o = 16; o > 0; o >>= 1) { s1 += __shfl_down_sync(0xffffffffu, s1, o); s2 += __shfl_down_sync(0xffffffffu, s2, o); }
    if (lane == 0) { red[0][w] = s1; red[1][w] = s2; }
    __syncthreads();
    if (tid == 0) {
        double a = 0, b = 0;
        for (int k = 0; k < 8; ++k) a += red[0][k];
        for (int k = 0; k < 8; ++k) b += red[1][k];
        part1[bid] = a; part2[bid] = b;
        __threadfence();
        last = (atomicAdd(counter, 1u) == nb - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double a = 0, b = 0;
    for (unsigned k = tid; k < nb; k += 256) { a += ((volatile double *)part1)[k]; b += ((volatile double *)part2)[k]; }
    for (int o = 16; o > 0; o >>= 1) { a += __shfl_down_sync(0xffffffffu, a, o); b += __shfl_down_sync(0xffffffffu, b, o); }
    __syncthreads();
    if (lane == 0) { red[0][w] = a; red[1][w] = b; }
    __syncthreads();
    if (tid == 0) {
        double ta = 0, tb = 0;
        for (int k = 0; k < 8; ++k) ta += red[0][k];
        for (int k = 0; k < 8; ++k) tb += red[1][k];
        *counter = 0;
        st->rr = ta;
        // the iteration's check, then rho for the next direction (left as it
        // was once the solve has stopped)
        fpcg_check(st);
        if (!st->done) st->rho = tb;
    }
}
__global__ void fpcg_zr_kernel(const double *__restrict__ z, const double *__restrict__ r, int64_t n, PcgState *st, Reduce red)
{
    if (st->done) return;
    double s = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) s += z[i] * r[i];
    block_sum_to<256>(s, red.partials, red.counter, red.result);
}
__global__ void fpcg_p_kernel(double *__restrict__ p, const double *__restrict__ z, int64_t n, const PcgState *st)
{
    if (st->done) return;
    const double beta = st->rho / st->rhoOld;
    const int64_t S = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += 4 * S) {
        double zo[4], po[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (i + q * S < n) { zo[q] = z[i + q * S]; po[q] = p[i + q * S]; }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (i + q * S < n) p[i + q * S] = zo[q] + beta * po[q];
    }
}
__global__ void fpcg_start_kernel(PcgState *st, double tol, int maxIT)
{
    st->normB = sqrt(st->normB);
    st->tol = tol; st->maxIT = maxIT; st->its = 0; st->status = 0;
    st->done = st->normB == 0.0 ? 1 : 0;
}

// ---- super-element density filter ---------------------------------------------
// sub-voxel (q, e) of the element-major [64 x Ne] layout <-> fine-grid voxel
// (y fastest); q = ly + 4 (lx + 4 lz) (gen_index_mapping, TOP_GPU.m:2673-2697)
__device__ __forceinline__ int64_t sub_to_fine(int64_t i, int ny, int nx, int fy, int fx)
{
    const int64_t e = i / 64; const int q = (int)(i % 64);
    const int ey = (int)(e % ny), ex = (int)((e / ny) % nx), ez = (int)(e / ((int64_t)ny * nx));
    const int y = 4 * ey + (q & 3), x = 4 * ex + ((q >> 2) & 3), z = 4 * ez + (q >> 4);
    return y + (int64_t)fy * (x + (int64_t)fx * z);
}
// mode 0: g = in ./ Hs (sensitivities), mode 1: g = in (densities)
__global__ void sfilt_gather_kernel(const double *__restrict__ in, const double *__restrict__ Hs, int mode, int ny, int nx,
                                    int fy, int fx, int64_t n, double *__restrict__ g)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t f = sub_to_fine(i, ny, nx, fy, fx);
    g[f] = mode == 0 ? in[i] / Hs[f] : in[i];
}
__global__ void sfilt_scatter_kernel(const double *__restrict__ t, const double *__restrict__ Hs, int mode, int ny, int nx,
                                     int fy, int fx, int64_t n, double *__restrict__ out)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t f = sub_to_fine(i, ny, nx, fy, fx);
    out[i] = mode == 1 ? t[f] / Hs[f] : t[f];
}
// t = imfilter(g, h): correlation, zero outside (the kernel is symmetric)
__global__ void sfilt_conv_kernel(const double *__restrict__ g, const double *__restrict__ h, int R, int fy, int fx, int fz,
                                  double *__restrict__ t)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t n = (int64_t)fy * fx * fz;
    if (i >= n) return;
    const int y = (int)(i % fy), x = (int)((i / fy) % fx), z = (int)(i / ((int64_t)fy * fx));
    const int w = 2 * R + 1;
    double s = 0;
    for (int dz = -R; dz <= R; ++dz) {
        const int zz = z + dz;
        if (zz < 0 || zz >= fz) continue;
        for (int dx = -R; dx <= R; ++dx) {
            const int xx = x + dx;
            if (xx < 0 || xx >= fx) continue;
            const double *gr = g + (int64_t)fy * (xx + (int64_t)fx * zz);
            const double *hr = h + w * ((dx + R) + w * (dz + R)) + R;
            for (int dy = -R; dy <= R; ++dy) {
                const int yy = y + dy;
                if (yy < 0 || yy >= fy) continue;
                s = fma(gr[yy], hr[dy], s);
            }
        }
    }
    t[i] = s;
}

// ---- sensitivities ----------------------------------------------------------
// ce_e = sum_k w_k u_ke' Ke u_ke; dc = -p (E0-Emin) x^(p-1) ce / cSolid; dv = 1;
// sums: cObj = sum E_e ce_e / cSolid, sumX = sum xPhys (TOP_GPU.m:191-199)
__global__ void sensitivity_kernel(const KeParam<double> K, const double *__restrict__ U, int64_t ustride, int nLoads,
                                   const double *__restrict__ w, const int32_t *__restrict__ eleGrid, int64_t Ne, Geom g,
                                   const double *__restrict__ xPhys, const double *__restrict__ Ec,
                                   double E0, double Emin, double penal, double cSolid,
                                   double *__restrict__ ce, double *__restrict__ dc, double *__restrict__ dv,
                                   Reduce redC)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double cpart = 0;
    if (e < Ne) {
        const int slot = eleGrid[e];
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
        if (ce) ce[e] = acc;
        const double cn = cSolid > 0 ? acc / cSolid : acc;
        if (dc) {
            const double x = xPhys[e];
            dc[e] = -(penal * (E0 - Emin) * pow(x, penal - 1.0)) * cn;
            dv[e] = 1.0;
        }
        cpart = Ec[e] * cn;
    }
    if (redC.result) block_sum_to<256>(cpart, redC.partials, redC.counter, redC.result);
}
// super-element mode: ce_e = sum_k w_k u_ke' K_mat_e u_ke (TOP_GPU.m:2622-2645),
// dc(q, e) = -p x^(p-1) (E0-Emin) sum_k w_k u_ke' I_q u_ke / cSolid
// (pre_compute_der, 2646-2671); one 64-thread CTA per element, thread = q
__global__ void __launch_bounds__(64)
sensitivity_super_kernel(const double *__restrict__ Imat, const double *__restrict__ Kc, const double *__restrict__ U,
                         int64_t ustride, int nLoads, const double *__restrict__ w, const int32_t *__restrict__ eleGrid,
                         Geom g, const double *__restrict__ xPhys, double E0, double Emin, double penal, double cSolid,
                         double *__restrict__ ce, double *__restrict__ dc, double *__restrict__ dv, Reduce redC)
{
    __shared__ double ue[24];
    __shared__ double part[24];
    const int64_t e = blockIdx.x;
    const int q = threadIdx.x;
    const int slot = eleGrid[e];
    double dq = 0, cp = 0;
    for (int k = 0; k < nLoads; ++k) {
        const double *u = U + k * ustride;
        if (q < 24) {
            const int j = q / 3, c = q % 3;
            ue[q] = u[c * g.cs + slot + cdy(j) + g.PY * cdx(j) + g.plane * cdz(j)];
        }
        __syncthreads();
        const double *I = Imat + (size_t)q * 576;
        double a = 0;
        for (int col = 0; col < 24; ++col) {
            double r = 0;
#pragma unroll
            for (int row = 0; row < 24; ++row) r = fma(I[row + 24 * col], ue[row], r);
            a = fma(r, ue[col], a);
        }
        dq += w[k] * a;
        if (q < 24) {
            const double *K = Kc + e * 576;
            double r = 0;
#pragma unroll
            for (int col = 0; col < 24; ++col) r = fma(K[q + 24 * col], ue[col], r);
            cp += w[k] * r * ue[q];
        }
        __syncthreads();
    }
    if (q < 24) part[q] = cp;
    __syncthreads();
    double cpart = 0;
    if (q == 0) {
        double sc = 0;
        for (int i = 0; i < 24; ++i) sc += part[i];
        if (ce) ce[e] = sc;
        cpart = cSolid > 0 ? sc / cSolid : sc;
    }
    if (dc) {
        const double x = xPhys[e * 64 + q];
        const double dn = cSolid > 0 ? dq / cSolid : dq;
        dc[e * 64 + q] = -(penal * (E0 - Emin) * pow(x, penal - 1.0)) * dn;
        dv[e * 64 + q] = 1.0;
    }
    if (redC.result) block_sum_to<64>(cpart, redC.partials, redC.counter, redC.result);
}

__global__ void sum_scaled_kernel(const double *__restrict__ a, int64_t n, double scale, Reduce red)
{
    double s = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) s += a[i] * scale;
    block_sum_to<256>(s, red.partials, red.counter, red.result);
}
__global__ void sum_kernel(const double *__restrict__ a, int64_t n, int mode, Reduce red)
{   // mode 0: sum a ; mode 1: sum a(1-a)
    double s = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        s += mode ? a[i] * (1.0 - a[i]) : a[i];
    block_sum_to<256>(s, red.partials, red.counter, red.result);
}
__global__ void mul_kernel(const double *__restrict__ a, const double *__restrict__ b, double *__restrict__ c, int64_t n)
{ for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) c[i] = a[i] * b[i]; }
__global__ void div_floor_kernel(const double *__restrict__ a, const double *__restrict__ x, double *__restrict__ c, int64_t n)
{ for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) c[i] = a[i] / fmax(1e-3, x[i]); }

// ---- OC update: bisection on the Lagrange multiplier (TOP_GPU.m:233-253) ----
// One cooperative launch; every block reduces the same per-block partials in
// the same order, so all blocks take identical branches without a broadcast.
// OC update of one element (TOP_GPU.m:236-244) with r = -dc./dv precomputed:
// x .* sqrt(r / lmid) is exactly x .* sqrt(-dc ./ dv / lmid) (same operations)
__device__ __forceinline__ double oc_new(double x, double r, double lmid, double move)
{
    const double cand = x * sqrt(r / lmid);
    // MATLAB's max/min ignore NaN like fmax/fmin
    return fmax(0.0, fmax(x - move, fmin(1.0, fmin(x + move, cand))));
}
// Bisection on the Lagrange multiplier as one cooperative kernel.  r = -dc./dv
// once per element (into rbuf), then per step: every element's x_new - x,
// block sums, one grid-wide barrier, and warp 0 of every CTA adds the block
// sums in the same fixed order (lane-strided, then a shuffle tree) so every
// CTA takes the same branch; block sums alternate between two buffers, so
// the next step cannot overwrite what a slower CTA still reads.
// pin (may be null): design variables held at 1 whatever the multiplier
// (passive elements, TOP_GPU.m:239 / 247)
__global__ void oc_kernel(double *__restrict__ x, const double *__restrict__ dc, const double *__restrict__ dv,
                          double *__restrict__ rbuf, int64_t n, double *__restrict__ partials, OptScalars *sc,
                          double move, int maxSteps, const uint8_t *__restrict__ pin)
{
    cg::grid_group grid = cg::this_grid();
    __shared__ double red[8];
    __shared__ double tot_s;
    const double fval = sc->fval;
    double l1 = 0.0, l2 = 1e9, lmid = 0.5 * (l1 + l2);
    const unsigned nb = gridDim.x;
    const int64_t stride = (int64_t)nb * blockDim.x;
    auto block_reduce = [&](double v, bool isMax) -> double {
        for (int o = 16; o > 0; o >>= 1) {
            const double w = __shfl_down_sync(0xffffffffu, v, o);
            v = isMax ? fmax(v, w) : v + w;
        }
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
        __syncthreads();
        double t = 0.0;
        if (threadIdx.x == 0) {
            for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t = isMax ? fmax(t, red[i]) : t + red[i];
            red[0] = t;
        }
        __syncthreads();
        t = red[0];
        __syncthreads();
        return t;
    };
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) rbuf[i] = -dc[i] / dv[i];
    int step = 0;
    while ((l2 - l1) / (l1 + l2) > 1e-6 && step < maxSteps) {
        lmid = 0.5 * (l2 + l1);
        double s = 0;
        for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
            const double xi = x[i];
            s += ((pin && pin[i]) ? 1.0 : oc_new(xi, rbuf[i], lmid, move)) - xi;
        }
        const double bs = block_reduce(s, false);
        double *pp = partials + (step & 1) * nb;
        if (threadIdx.x == 0) pp[blockIdx.x] = bs;
        grid.sync();
        if (threadIdx.x < 32) {
            double t = 0;
            for (unsigned b = threadIdx.x; b < nb; b += 32) t += pp[b];
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (threadIdx.x == 0) tot_s = t;
        }
        __syncthreads();
        const double gt = fval + tot_s / (double)n;
        if (gt > 0) l1 = lmid; else l2 = lmid;
        ++step;
        __syncthreads();                 // tot_s is rewritten next step
    }
    // xnew from the last multiplier; change = max|xnew - x|; x = xnew
    double mx = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double xn = (pin && pin[i]) ? 1.0 : oc_new(x[i], rbuf[i], lmid, move);
        mx = fmax(mx, fabs(xn - x[i]));
        x[i] = xn;
    }
    const double bm = block_reduce(mx, true);
    double *pp = partials + (step & 1) * nb;
    if (threadIdx.x == 0) pp[blockIdx.x] = bm;
    grid.sync();
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        double c = 0;
        for (unsigned b = 0; b < nb; ++b) c = fmax(c, pp[b]);
        sc->change = c;
        sc->lmid = lmid;
        sc->pad = (double)step;
    }
}

__global__ void copy_kernel(const double *__restrict__ a, double *__restrict__ b, int64_t n)
{ for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) b[i] = a[i]; }
// xPhys(passive) = 1 after the filter (TOP_GPU.m:270 / 273)
__global__ void pin_kernel(double *__restrict__ x, const uint8_t *__restrict__ pin, int64_t n)
{ for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) if (pin[i]) x[i] = 1.0; }
__global__ void fill_kernel(double *__restrict__ a, double v, int64_t n)
{ for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) a[i] = v; }

}  // namespace

// ============================================================================
// solver-attached state
namespace {
FilterState &filt(top_solver *s) { return *reinterpret_cast<FilterState *>(s->filterState); }
OptState &opt(top_solver *s) { return *reinterpret_cast<OptState *>(s->optState); }

int ensure_state(top_solver *s)
{
    if (!s->filterState) s->filterState = new FilterState();
    if (!s->optState) s->optState = new OptState();
    return TOP_OK;
}
}  // namespace

void topgpu::free_opt_state(top_solver *s)
{
    if (s->filterState && filt(s).chunk) cudaGraphExecDestroy(filt(s).chunk);
    delete reinterpret_cast<FilterState *>(s->filterState);
    if (s->optState && opt(s).sf.h) cudaFree(opt(s).sf.h);
    delete reinterpret_cast<OptState *>(s->optState);
    delete reinterpret_cast<AdjState *>(s->adjState);
    s->filterState = s->optState = s->adjState = nullptr;
}

extern "C" int top_solver_filter_setup(top_solver *s, double rMin)
{
    if (!s || !(rMin > 0)) { set_error("top_solver_filter_setup: bad arguments"); return TOP_ERR_ARGS; }
    ensure_state(s);
    FilterState &f = filt(s);
    DevLevel &l0 = s->L[0];
    const int64_t cs = l0.g.cs;
    if (!f.act) {
        f.act = s->galloc<double>(cs, 1); f.invD = s->galloc<double>(cs, 1);
        f.rhs = s->galloc<double>(cs, 1); f.x = s->galloc<double>(cs, 1); f.r = s->galloc<double>(cs, 1);
        f.z = s->galloc<double>(cs, 1); f.p = s->galloc<double>(cs, 1); f.v = s->galloc<double>(cs, 1);
        f.eg = s->galloc<double>(cs, 1);
        f.st = s->dalloc<PcgState>(1);
        f.part2 = s->dalloc<double>(4096);
        if (!f.act || !f.invD || !f.rhs || !f.x || !f.r || !f.z || !f.p || !f.v || !f.eg || !f.st || !f.part2) {
            set_error("top_solver_filter_setup: out of device memory"); return TOP_ERR_NOMEM;
        }
    }
    filter_kernel_matrix(rMin, f.KEF.k);
    if (f.chunk) { cudaGraphExecDestroy(f.chunk); f.chunk = nullptr; }   // the operator is a captured argument
    filter_activity_kernel<<<nb256(l0.Ne), 256, 0, s->st>>>(l0.eleGrid, l0.Ne, f.act);
    TOPGPU_COUNT_LAUNCH();
    filter_diag_kernel<<<dim3(l0.g.nbx, l0.g.NZ), kNodeThreads, 0, s->st>>>(f.KEF, f.act, l0.g, l0.flags, f.invD);
    TOPGPU_COUNT_LAUNCH();
    CK(cudaGetLastError());
    f.rMin = rMin;
    f.ready = true;
    return TOP_OK;
}

// tar = PDE-filter(src), element vectors (device, compact) -- TOP_GPU.m:959-1006
static int filter_apply(top_solver *s, const double *src, double *tar, int *itsOut)
{
    FilterState &f = filt(s);
    DevLevel &l0 = s->L[0];
    const Geom &g = l0.g;
    const int64_t cs = g.cs, ng = l0.ng;
    cudaStream_t st = s->st;
    // nodal rhs: each element adds src/8 to its nodes
    CK(cudaMemsetAsync(f.eg - kMargin, 0, sizeof(double) * cs, st));
    elem_to_slots_kernel<<<nb256(l0.Ne), 256, 0, st>>>(src, l0.eleGrid, l0.Ne, 1.0 / 8.0, f.eg);
    TOPGPU_COUNT_LAUNCH();
    slots_to_nodes_kernel<<<dim3(g.nbx, g.NZ), kNodeThreads, 0, st>>>(f.eg, g, l0.flags, f.rhs);
    TOPGPU_COUNT_LAUNCH();
    // PCG with the filter operator and Jacobi, tol_/10, maxIT_ (TOP_GPU.m:999-1001)
    const int VB = vb(ng);
    fpcg_init_kernel<<<VB, 256, 0, st>>>(f.rhs, f.x, f.r, f.z, f.p, f.invD, ng, s->red(&f.st->normB));
    TOPGPU_COUNT_LAUNCH();
    fpcg_start_kernel<<<1, 1, 0, st>>>(f.st, s->p.tol / 10.0, s->p.maxIT);
    TOPGPU_COUNT_LAUNCH();
    fpcg_zr_kernel<<<VB, 256, 0, st>>>(f.z, f.r, ng, f.st, s->red(&f.st->rho));
    TOPGPU_COUNT_LAUNCH();
    const int *done = &f.st->done;
    const int chunk = 8;
    // one filter-PCG iteration; every kernel returns at once after convergence
    auto iteration = [&](cudaStream_t q) {
        filter_apply_kernel<<<dim3(g.nbx, g.NZ), kNodeThreads, 0, q>>>(f.KEF, f.act, f.p, f.v, g, s->red(&f.st->pv), done);
        TOPGPU_COUNT_LAUNCH();
        fpcg_update_kernel<<<VB, 256, 0, q>>>(f.x, f.r, f.z, f.p, f.v, f.invD, ng, f.st, s->partials, f.part2, s->counter);
        TOPGPU_COUNT_LAUNCH();
        fpcg_p_kernel<<<VB, 256, 0, q>>>(f.p, f.z, ng, f.st);
        TOPGPU_COUNT_LAUNCH();
    };
    // a chunk of iterations as one CUDA graph (its buffers and operator are
    // fixed until the next filter setup), captured on the solver's capture
    // stream and launched there after the caller's stream
    if (s->useGraphs && !f.chunk) {
        if (!s->capStream) {
            CK(cudaStreamCreateWithFlags(&s->capStream, cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&s->capIn, cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&s->capOut, cudaEventDisableTiming));
        }
        const int64_t before = s->launches;
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(s->capStream, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < chunk; ++k) iteration(s->capStream);
        cudaError_t e = cudaStreamEndCapture(s->capStream, &graph);
        f.chunkNodes = s->launches - before;
        s->launches = before;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&f.chunk, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        CK(e);
    }
    PcgState h{};
    for (int it0 = 0; it0 < s->p.maxIT; it0 += chunk) {
        if (f.chunk && s->useGraphs && it0 + chunk <= s->p.maxIT) {
            CK(cudaEventRecord(s->capIn, st));
            CK(cudaStreamWaitEvent(s->capStream, s->capIn, 0));
            CK(cudaGraphLaunch(f.chunk, s->capStream));
            CK(cudaEventRecord(s->capOut, s->capStream));
            CK(cudaStreamWaitEvent(st, s->capOut, 0));
            s->launches += f.chunkNodes;
        } else {
            for (int k = 0; k < chunk && it0 + k < s->p.maxIT; ++k) iteration(st);
        }
        CK(cudaMemcpyAsync(&h, f.st, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (h.done) break;
    }
    nodes_to_elem_kernel<<<nb256(l0.Ne), 256, 0, st>>>(f.x, l0.eleGrid, g, l0.Ne, tar);
    TOPGPU_COUNT_LAUNCH();
    CK(cudaGetLastError());
    if (itsOut) *itsOut = h.its;
    if (h.status == TOP_ERR_NAN) { set_error("PDE filter: non-finite PCG scalar"); return TOP_ERR_NAN; }
    return TOP_OK;
}

extern "C" int top_solver_filter(top_solver *s, const double *src, double *tar, int *its)
{
    if (!s || !src || !tar) return TOP_ERR_ARGS;
    if (!s->filterState || !filt(s).ready) { set_error("top_solver_filter: call top_solver_filter_setup first"); return TOP_ERR_STATE; }
    const int rc = filter_apply(s, src, tar, its);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    return TOP_OK;
}

// ---- super-element density filter (host side) --------------------------------
static int sfilter_setup(top_solver *s, double rMin)
{
    OptState &o = opt(s);
    SFilterState &f = o.sf;
    DevLevel &l0 = s->L[0];
    if ((int64_t)s->nely * s->nelx * s->nelz != l0.Ne) {
        set_error("super-element filter: needs a full box of super-elements"); return TOP_ERR_SHAPE;
    }
    const double r = 4.0 * rMin;
    f.R = (int)std::ceil(r) - 1;
    const int w = 2 * f.R + 1;
    f.fy = 4 * s->nely; f.fx = 4 * s->nelx; f.fz = 4 * s->nelz;
    const int64_t N = (int64_t)f.fy * f.fx * f.fz;
    if (!f.Hs) {
        f.Hs = s->dalloc<double>(N); f.g = s->dalloc<double>(N); f.t = s->dalloc<double>(N);
        if (!f.Hs || !f.g || !f.t) { set_error("super-element filter: out of device memory"); return TOP_ERR_NOMEM; }
    }
    std::vector<double> h((size_t)w * w * w);
    for (int dz = -f.R; dz <= f.R; ++dz)
        for (int dx = -f.R; dx <= f.R; ++dx)
            for (int dy = -f.R; dy <= f.R; ++dy) {
                const double v = r - std::sqrt(double(dx * dx + dy * dy + dz * dz));
                h[(dy + f.R) + w * ((dx + f.R) + w * (dz + f.R))] = v > 0 ? v : 0.0;
            }
    if (f.h) cudaFree(f.h);
    if (cudaMalloc(&f.h, sizeof(double) * h.size()) != cudaSuccess) { f.h = nullptr; return TOP_ERR_NOMEM; }
    CK(cudaMemcpyAsync(f.h, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, s->st));
    fill_kernel<<<vb(N), 256, 0, s->st>>>(f.g, 1.0, N);
    TOPGPU_COUNT_LAUNCH();
    sfilt_conv_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s->st>>>(f.g, f.h, f.R, f.fy, f.fx, f.fz, f.Hs);
    TOPGPU_COUNT_LAUNCH();
    CK(cudaStreamSynchronize(s->st));      // h (host vector) is consumed
    f.rMin = rMin;
    f.ready = true;
    return TOP_OK;
}
// mode 0: out = imfilter(in ./ Hs, h) ; mode 1: out = imfilter(in, h) ./ Hs
static int sfilter_apply(top_solver *s, const double *in, double *out, int mode)
{
    SFilterState &f = opt(s).sf;
    const int64_t n = 64 * s->L[0].Ne, N = (int64_t)f.fy * f.fx * f.fz;
    sfilt_gather_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s->st>>>(in, f.Hs, mode, s->nely, s->nelx, f.fy, f.fx, n, f.g);
    TOPGPU_COUNT_LAUNCH();
    sfilt_conv_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s->st>>>(f.g, f.h, f.R, f.fy, f.fx, f.fz, f.t);
    TOPGPU_COUNT_LAUNCH();
    sfilt_scatter_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s->st>>>(f.t, f.Hs, mode, s->nely, s->nelx, f.fy, f.fx, n, out);
    TOPGPU_COUNT_LAUNCH();
    CK(cudaGetLastError());
    return TOP_OK;
}

extern "C" int top_solver_super_filter_setup(top_solver *s, double rMin)
{
    if (!s || !(rMin > 0)) return TOP_ERR_ARGS;
    if (!s->super) { set_error("top_solver_super_filter_setup: super-element models only"); return TOP_ERR_ARGS; }
    ensure_state(s);
    return sfilter_setup(s, rMin);
}

extern "C" int top_solver_super_filter(top_solver *s, const double *src, double *tar, int mode)
{
    if (!s || !src || !tar || (mode != 0 && mode != 1)) return TOP_ERR_ARGS;
    if (!s->optState || !opt(s).sf.ready) { set_error("top_solver_super_filter: call top_solver_super_filter_setup first"); return TOP_ERR_STATE; }
    const int rc = sfilter_apply(s, src, tar, mode);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    return TOP_OK;
}

// ---- the optimisation loop ---------------------------------------------------
// state solves of all load cases (TOP_GPU.m:181-187) as one batched PCG
static int solve_all(top_solver *s, int warm, int *itsTotal)
{
    OptState &o = opt(s);
    std::vector<int> its((size_t)std::max(1, s->nLoads), 0);
    const int rc = pcg_block(s, s->b, o.U, s->nLoads, warm, its.data(), nullptr);
    if (rc != TOP_OK && rc != TOP_ERR_NOT_CONVERGED) return rc;
    if (rc == TOP_ERR_NOT_CONVERGED) std::fprintf(stderr, "Warning: Exceed the maximum iterate numbers\n");
    int tot = 0;
    for (int k = 0; k < s->nLoads; ++k) tot += its[k];
    if (itsTotal) *itsTotal = tot;
    o.caseIts.assign(its.begin(), its.begin() + s->nLoads);
    return TOP_OK;
}

static int sensitivities(top_solver *s, int withGrad)
{
    OptState &o = opt(s);
    DevLevel &l0 = s->L[0];
    if (s->super) {      // one CTA per element: the objective is summed from ce afterwards
        sensitivity_super_kernel<<<(unsigned)l0.Ne, 64, 0, s->st>>>(
            s->Imat, l0.KsC, o.U, 3 * l0.g.cs, s->nLoads, s->weights, l0.eleGrid, l0.g, o.xPhys,
            s->p.E0, s->p.Emin, s->p.penal, withGrad ? o.cSolid : 0.0, o.ce, withGrad ? o.dc : nullptr, o.dv,
            Reduce{nullptr, nullptr, nullptr});
        TOPGPU_COUNT_LAUNCH();
        sum_scaled_kernel<<<vb(l0.Ne), 256, 0, s->st>>>(o.ce, l0.Ne, withGrad && o.cSolid > 0 ? 1.0 / o.cSolid : 1.0,
                                                        s->red(&o.sc->cObj));
        TOPGPU_COUNT_LAUNCH();
        CK(cudaGetLastError());
        return TOP_OK;
    }
    sensitivity_kernel<<<nb256(l0.Ne), 256, 0, s->st>>>(
        s->Ke64, o.U, 3 * l0.g.cs, s->nLoads, s->weights, l0.eleGrid, l0.Ne, l0.g, o.xPhys, s->Ec,
        s->p.E0, s->p.Emin, s->p.penal, withGrad ? o.cSolid : 0.0, o.ce, withGrad ? o.dc : nullptr, o.dv,
        s->red(&o.sc->cObj));
        TOPGPU_COUNT_LAUNCH();
    CK(cudaGetLastError());
    return TOP_OK;
}

extern "C" int top_solver_set_passive(top_solver *s, const int32_t *ids, int64_t n)
{
    if (!s || n < 0 || (n > 0 && !ids)) { set_error("top_solver_set_passive: bad arguments"); return TOP_ERR_ARGS; }
    ensure_state(s);
    OptState &o = opt(s);
    const int64_t Ne = s->L[0].Ne, nv = Ne * (s->super ? 64 : 1);
    std::vector<uint8_t> mask((size_t)nv, 0);
    for (int64_t k = 0; k < n; ++k) {
        if (ids[k] < 1 || ids[k] > Ne) { set_error("top_solver_set_passive: element %d out of range", (int)ids[k]); return TOP_ERR_ARGS; }
        mask[(size_t)(s->super ? 3 + 64 * (int64_t)(ids[k] - 1) : ids[k] - 1)] = 1;
    }
    if (n > 0 && (!o.passive || o.passiveLen != nv)) {
        o.passive = s->dalloc<uint8_t>((size_t)nv);
        if (!o.passive) { set_error("top_solver_set_passive: out of device memory"); return TOP_ERR_NOMEM; }
        o.passiveLen = nv;
    }
    if (n > 0) {
        CK(cudaMemcpyAsync(o.passive, mask.data(), (size_t)nv, cudaMemcpyHostToDevice, s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    o.nPassive = n;
    return TOP_OK;
}

extern "C" int top_solver_opt_begin(top_solver *s, const top_opt_params *prm, double *cSolidOut)
{
    if (!s || !prm || prm->nLoop < 0 || !(prm->V0 > 0) || (prm->ft != 0 && prm->ft != 1 && prm->ft != 2)) {
        set_error("top_solver_opt_begin: bad arguments"); return TOP_ERR_ARGS;
    }
    if (s->super && prm->ft != 2) {      // TOP_GPU.m:113-121: super-element models filter densities
        set_error("top_solver_opt_begin: super-element models use ft = 2"); return TOP_ERR_ARGS;
    }
    ensure_state(s);
    OptState &o = opt(s);
    DevLevel &l0 = s->L[0];
    const int64_t Ne = l0.Ne, cs = l0.g.cs;
    const int64_t nv = Ne * (s->super ? 64 : 1);
    o.nv = nv;
    if (!o.xd) {
        o.xd = s->dalloc<double>(nv); o.xPhys = s->dalloc<double>(nv); o.xnew = s->dalloc<double>(nv);
        o.dc = s->dalloc<double>(nv); o.dv = s->dalloc<double>(nv); o.ce = s->dalloc<double>(Ne); o.tmp = s->dalloc<double>(nv);
        o.U = s->galloc<double>(cs, 3 * s->nLoads);
        o.sc = s->dalloc<OptScalars>(1);
        if (cudaMallocHost(&o.hsc, sizeof(OptScalars)) != cudaSuccess) o.hsc = nullptr;
        int dev = 0, nsm = 0, perSM = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, oc_kernel, 256, 0);
        o.ocBlocks = std::max(1, std::min<int>(nsm * std::max(1, perSM), (int)((nv + 255) / 256)));
        o.ocPartials = s->dalloc<double>(2 * (size_t)o.ocBlocks);
        o.ocR = s->dalloc<double>((size_t)nv);
        if (!o.xd || !o.xPhys || !o.xnew || !o.dc || !o.dv || !o.ce || !o.tmp || !o.U || !o.sc || !o.hsc || !o.ocPartials || !o.ocR) {
            set_error("top_solver_opt_begin: out of memory"); return TOP_ERR_NOMEM;
        }
    }
    o.prm = *prm;
    if (s->super) { const int rc = sfilter_setup(s, prm->rMin); if (rc) return rc; }
    else if (prm->ft != 0) { const int rc = top_solver_filter_setup(s, prm->rMin); if (rc) return rc; }
    // fully solid solve and its compliance (TOP_GPU.m:142-165)
    fill_kernel<<<vb(nv), 256, 0, s->st>>>(o.tmp, s->p.E0, nv);
    TOPGPU_COUNT_LAUNCH();
    int rc = set_modulus_dev(s, o.tmp, 1, 0);
    if (rc) return rc;
    rc = top_solver_assemble(s);
    if (rc) return rc;
    CK(cudaMemsetAsync(o.U - kMargin, 0, sizeof(double) * 3 * cs * s->nLoads, s->st));
    rc = solve_all(s, 0, nullptr);
    if (rc) return rc;
    o.cSolid = 0;
    rc = sensitivities(s, 0);
    if (rc) return rc;
    CK(cudaMemcpyAsync(o.hsc, o.sc, sizeof(OptScalars), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    o.cSolid = o.hsc->cObj;       // cSolid = E0 * sum(ceList) with E = E0 (super: sum(ceList))
    fill_kernel<<<vb(nv), 256, 0, s->st>>>(o.xd, prm->V0, nv);
    TOPGPU_COUNT_LAUNCH();
    fill_kernel<<<vb(nv), 256, 0, s->st>>>(o.xPhys, prm->V0, nv);
    TOPGPU_COUNT_LAUNCH();
    CK(cudaGetLastError());
    o.loop = 0; o.change = 1.0; o.sharp = 1.0;
    o.begun = true;
    if (cSolidOut) *cSolidOut = o.cSolid;
    return TOP_OK;
}

extern "C" int top_solver_opt_step(top_solver *s, top_opt_record *rec)
{
    if (!s || !s->optState || !opt(s).begun) { set_error("top_solver_opt_step: call top_solver_opt_begin first"); return TOP_ERR_STATE; }
    OptState &o = opt(s);
    const int64_t Ne = o.nv;           // design variables (64 per super-element)
    cudaStream_t st = s->st;
    const int VB = vb(Ne);
    struct PhaseEvents {             // destroyed on every return
        cudaEvent_t e[7] = {};
        ~PhaseEvents() { for (cudaEvent_t x : e) if (x) cudaEventDestroy(x); }
    } pe;
    cudaEvent_t *ev = pe.e;
    for (int k = 0; k < 7; ++k) CK(cudaEventCreate(&ev[k]));
    NvtxRange whole("opt_step");
    CK(cudaEventRecord(ev[0], st));
    // 5.1 SIMP moduli and stencil assembly
    int rc;
    {
        NvtxRange r("opt_step: SIMP + assembly");
        rc = set_modulus_dev(s, o.xPhys, 1, 1);
        if (!rc) rc = top_solver_assemble(s);
    }
    if (rc) return rc;
    CK(cudaEventRecord(ev[1], st));
    // 5.2 state solves, warm-started
    int its = 0;
    {
        NvtxRange r("opt_step: PCG");
        rc = solve_all(s, 1, &its);
    }
    if (rc) return rc;
    CK(cudaEventRecord(ev[2], st));
    // objective and sensitivities, volume
    NvtxRange rest("opt_step: sensitivities, filter, OC");
    rc = sensitivities(s, 1);
    if (rc) return rc;
    sum_kernel<<<VB, 256, 0, st>>>(o.xPhys, Ne, 0, s->red(&o.sc->sumE));
    TOPGPU_COUNT_LAUNCH();
    CK(cudaEventRecord(ev[3], st));
    // 5.3 filtering of the sensitivities
    int fits = 0;
    if (o.prm.ft == 1) {
        mul_kernel<<<VB, 256, 0, st>>>(o.xd, o.dc, o.tmp, Ne);
        TOPGPU_COUNT_LAUNCH();
        rc = filter_apply(s, o.tmp, o.dc, &fits);
        if (rc) return rc;
        div_floor_kernel<<<VB, 256, 0, st>>>(o.dc, o.xd, o.dc, Ne);
        TOPGPU_COUNT_LAUNCH();
    } else if (o.prm.ft == 2 && s->super) {   // dc = imfilter(dc./Hs, h), dv likewise (TOP_GPU.m:221-227)
        rc = sfilter_apply(s, o.dc, o.tmp, 0);
        if (!rc) { copy_kernel<<<VB, 256, 0, st>>>(o.tmp, o.dc, Ne); TOPGPU_COUNT_LAUNCH(); rc = sfilter_apply(s, o.dv, o.tmp, 0); }
        if (rc) return rc;
        copy_kernel<<<VB, 256, 0, st>>>(o.tmp, o.dv, Ne);
        TOPGPU_COUNT_LAUNCH();
    } else if (o.prm.ft == 2) {
        rc = filter_apply(s, o.dc, o.tmp, &fits);
        if (!rc) { copy_kernel<<<VB, 256, 0, st>>>(o.tmp, o.dc, Ne); TOPGPU_COUNT_LAUNCH(); rc = filter_apply(s, o.dv, o.tmp, &fits); }
        if (rc) return rc;
        copy_kernel<<<VB, 256, 0, st>>>(o.tmp, o.dv, Ne);
        TOPGPU_COUNT_LAUNCH();
    }
    CK(cudaEventRecord(ev[4], st));
    // 5.4 OC update; fval = mean(xPhys) - V0
    CK(cudaMemcpyAsync(o.hsc, o.sc, sizeof(OptScalars), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const double cObj = o.hsc->cObj, vol = o.hsc->sumE / (double)Ne;
    OptScalars h = *o.hsc;
    h.fval = vol - o.prm.V0;
    CK(cudaMemcpyAsync(o.sc, &h, sizeof(OptScalars), cudaMemcpyHostToDevice, st));
    {
        double move = 0.2;
        int maxSteps = 256;
        int64_t n = Ne;
        double *xa = o.xd; const double *dca = o.dc, *dva = o.dv; double *ra = o.ocR, *pa = o.ocPartials; OptScalars *sca = o.sc;
        const uint8_t *pin = o.nPassive > 0 ? o.passive : nullptr;
        void *args[] = {&xa, &dca, &dva, &ra, &n, &pa, &sca, &move, &maxSteps, &pin};
        CK(cudaLaunchCooperativeKernel((const void *)oc_kernel, dim3(o.ocBlocks), dim3(256), args, 0, st));
        TOPGPU_COUNT_LAUNCH();
    }
    CK(cudaEventRecord(ev[5], st));
    // xPhys (TOP_GPU.m:256-267): the new design, or its PDE-filtered version
    if (o.prm.ft == 2 && s->super) { rc = sfilter_apply(s, o.xd, o.xPhys, 1); if (rc) return rc; }   // 262-265
    else if (o.prm.ft == 2) { rc = filter_apply(s, o.xd, o.xPhys, &fits); if (rc) return rc; }
    else { copy_kernel<<<VB, 256, 0, st>>>(o.xd, o.xPhys, Ne); TOPGPU_COUNT_LAUNCH(); }
    if (o.nPassive > 0) { pin_kernel<<<VB, 256, 0, st>>>(o.xPhys, o.passive, Ne); TOPGPU_COUNT_LAUNCH(); }
    sum_kernel<<<VB, 256, 0, st>>>(o.xPhys, Ne, 1, s->red(&o.sc->sharp));
    TOPGPU_COUNT_LAUNCH();
    CK(cudaEventRecord(ev[6], st));
    CK(cudaMemcpyAsync(o.hsc, o.sc, sizeof(OptScalars), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    o.loop += 1;
    o.change = o.hsc->change;
    o.sharp = 4.0 * o.hsc->sharp / (double)Ne;
    if (rec) {   // the reference's tHist columns (TOP_GPU.m:283)
        float t[6];
        for (int k = 0; k < 6; ++k) cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]);
        rec->c = cObj * o.cSolid;
        rec->vol = vol;
        rec->sharp = o.sharp;
        rec->cons = h.fval;
        rec->change = o.change;
        rec->pcgIts = its;
        rec->msAssemble = t[0];
        rec->msSolve = t[1];
        rec->msOpt = t[2] + t[4];
        rec->msFilter = t[3] + t[5];
        float tot = 0;
        cudaEventElapsedTime(&tot, ev[0], ev[6]);
        rec->msTotal = tot;
    }
    return TOP_OK;
}

extern "C" int top_solver_opt_case_its(top_solver *s, int *its, int capacity, int *count)
{
    if (!s || capacity < 0 || (capacity > 0 && !its)) { set_error("top_solver_opt_case_its: bad arguments"); return TOP_ERR_ARGS; }
    if (!s->optState) { set_error("top_solver_opt_case_its: no state solves yet"); return TOP_ERR_STATE; }
    const std::vector<int> &v = opt(s).caseIts;
    if (count) *count = (int)v.size();
    for (int k = 0; k < capacity && k < (int)v.size(); ++k) its[k] = v[k];
    return TOP_OK;
}

extern "C" int top_solver_opt_state(top_solver *s, int *loop, double *change, double *sharpness)
{
    if (!s || !s->optState || !opt(s).begun) return TOP_ERR_STATE;
    OptState &o = opt(s);
    if (loop) *loop = o.loop;
    if (change) *change = o.change;
    if (sharpness) *sharpness = o.sharp;
    return TOP_OK;
}

extern "C" int top_solver_get_design(top_solver *s, double *xPhys, double *x)
{
    if (!s || !s->optState || !opt(s).begun) return TOP_ERR_STATE;
    OptState &o = opt(s);
    const int64_t Ne = o.nv;
    if (xPhys) CK(cudaMemcpyAsync(xPhys, o.xPhys, sizeof(double) * Ne, cudaMemcpyDefault, s->st));
    if (x) CK(cudaMemcpyAsync(x, o.xd, sizeof(double) * Ne, cudaMemcpyDefault, s->st));
    CK(cudaStreamSynchronize(s->st));
    return TOP_OK;
}

extern "C" int top_solver_set_design(top_solver *s, const double *xPhys, const double *x)
{
    if (!s || !s->optState || !opt(s).begun) return TOP_ERR_STATE;
    OptState &o = opt(s);
    const int64_t Ne = o.nv;
    if (xPhys) CK(cudaMemcpyAsync(o.xPhys, xPhys, sizeof(double) * Ne, cudaMemcpyDefault, s->st));
    if (x) CK(cudaMemcpyAsync(o.xd, x, sizeof(double) * Ne, cudaMemcpyDefault, s->st));
    return TOP_OK;
}

extern "C" int top_solver_launch_count(const top_solver *s, int64_t *count)
{
    if (!s || !count) return TOP_ERR_ARGS;
    *count = s->launches;
    return TOP_OK;
}

extern "C" int top_solver_optimize(top_solver *s, const top_opt_params *prm, double *xPhysOut,
                                   top_opt_record *hist, int *nIter, double *cSolid)
{
    int rc = top_solver_opt_begin(s, prm, cSolid);
    if (rc) return rc;
    OptState &o = opt(s);
    // TOP_GPU.m:176 -- loop < nLoop && change > 1e-4 && sharpness > 0.01
    while (o.loop < prm->nLoop && o.change > 0.0001 && o.sharp > 0.01) {
        rc = top_solver_opt_step(s, hist ? hist + o.loop : nullptr);
        if (rc) return rc;
    }
    if (nIter) *nIter = o.loop;
    if (xPhysOut) return top_solver_get_design(s, xPhysOut, nullptr);
    return TOP_OK;
}

// ============================================================================
// Adjoint sensitivities.  For K(E(xPhys)) U = F and an objective J(U):
//   compliance J = sum_k w_k F_k' U_k is self-adjoint: dJ/dE_e = -sum_k w_k U_ke' Ke U_ke
//   (the reference's element energies, TOP_GPU.m:580-600, 191-198);
//   a displacement J = U_k[dof] needs the adjoint solve K L = e_dof:
//   dJ/dE_e = -L_e' Ke U_ke.
// Elements with fixed DOFs use E Kfree + Kfixed (TOP_GPU.m:1729-1741); U and L
// vanish on the fixed DOFs, so Ke gives the same products.  dE/dxPhys =
// p xPhys^(p-1) (E0 - Emin) (SIMP, TOP_GPU.m:169).  The chain to the design
// variables follows the filter: ft = 1 the reference's sensitivity filter
// dc = H(x .* dc) / max(1e-3, x) (TOP_GPU.m:213-219), ft = 2 the PDE density
// filter's transpose (the Helmholtz filter is symmetric: H' = H).

namespace {
AdjState &adj(top_solver *s) { return *reinterpret_cast<AdjState *>(s->adjState); }

// dJ[e] = -p x^(p-1) (E0-Emin) sum_k w_k A_ke' Ke B_ke ; J += sum_e E_e sum_k w_k A_ke' Ke B_ke
__global__ void mutual_energy_kernel(const KeParam<double> K, const double *__restrict__ A, int64_t aStride,
                                     const double *__restrict__ B, int64_t bStride, int nPairs,
                                     const double *__restrict__ w, const int32_t *__restrict__ eleGrid, int64_t Ne,
                                     Geom g, const double *__restrict__ xPhys, const double *__restrict__ Ec,
                                     double E0, double Emin, double penal, double *__restrict__ dJ, Reduce redJ)
{
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double jpart = 0;
    if (e < Ne) {
        const int slot = eleGrid[e];
        double acc = 0;
        for (int k = 0; k < nPairs; ++k) {
            const double *a = A + k * aStride, *b = B + k * bStride;
            double ae[24], be[24];
#pragma unroll
            for (int j = 0; j < 8; ++j)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const int64_t o = c * g.cs + slot + cdy(j) + g.PY * cdx(j) + g.plane * cdz(j);
                    ae[3 * j + c] = a[o];
                    be[3 * j + c] = b[o];
                }
            double m = 0;
#pragma unroll
            for (int r = 0; r < 24; ++r) {
                double t = 0;
#pragma unroll
                for (int q = 0; q < 24; ++q) t = fma(K.k[r + 24 * q], be[q], t);
                m = fma(ae[r], t, m);
            }
            acc += (w ? w[k] : 1.0) * m;
        }
        const double x = xPhys[e];
        dJ[e] = -(penal * (E0 - Emin) * pow(x, penal - 1.0)) * acc;
        jpart = Ec[e] * acc;
    }
    if (redJ.result) block_sum_to<256>(jpart, redJ.partials, redJ.counter, redJ.result);
}
__global__ void unit_load_kernel(double *__restrict__ v, const int32_t *__restrict__ nodeGrid, int64_t node, int comp, int64_t cs)
{
    v[comp * cs + nodeGrid[node]] = 1.0;
}
__global__ void pick_dof_kernel(const double *__restrict__ U, const int32_t *__restrict__ nodeGrid, int64_t node, int comp,
                                int64_t cs, double *__restrict__ out)
{
    *out = U[comp * cs + nodeGrid[node]];
}
}  // namespace

extern "C" int top_solver_sensitivity(top_solver *s, const top_sens_params *prm, const double *xPhys, const double *x,
                                      double *dJdx, double *Jout, int *itsOut)
{
    if (!s || !prm || !xPhys || !dJdx) return TOP_ERR_ARGS;
    DevLevel &l0 = s->L[0];
    const int64_t cs = l0.g.cs, Ne = l0.Ne;
    if (prm->objective != 0 && prm->objective != 1) { set_error("top_solver_sensitivity: unknown objective %d", prm->objective); return TOP_ERR_ARGS; }
    if (prm->objective == 1 && (prm->loadCase < 0 || prm->loadCase >= s->nLoads || prm->dof < 0 || prm->dof >= s->nd0)) {
        set_error("top_solver_sensitivity: load case or DOF out of range"); return TOP_ERR_ARGS;
    }
    if (prm->ft < 0 || prm->ft > 2) { set_error("top_solver_sensitivity: ft must be 0, 1 or 2"); return TOP_ERR_ARGS; }
    if (s->super) { set_error("top_solver_sensitivity: voxel (non-super-element) models only"); return TOP_ERR_ARGS; }
    if (prm->ft != 0 && (!s->filterState || !filt(s).ready)) { set_error("top_solver_sensitivity: call top_solver_filter_setup first"); return TOP_ERR_STATE; }
    if (!s->adjState) s->adjState = new AdjState();
    AdjState &a = adj(s);
    if (!a.U) {
        a.U = s->galloc<double>(cs, 3 * s->nLoads); a.L = s->galloc<double>(cs, 3); a.e = s->galloc<double>(cs, 3);
        a.g = s->dalloc<double>(Ne); a.t = s->dalloc<double>(Ne); a.J = s->dalloc<double>(1);
        if (!a.U || !a.L || !a.e || !a.g || !a.t || !a.J) { set_error("top_solver_sensitivity: out of device memory"); return TOP_ERR_NOMEM; }
    }
    cudaStream_t st = s->st;
    int rc = set_modulus_dev(s, xPhys, 1, 1);
    if (rc) return rc;
    rc = top_solver_assemble(s);
    if (rc) return rc;
    const double tolKeep = s->p.tol;
    if (prm->tol > 0) s->p.tol = prm->tol;
    int its = 0, tot = 0;
    // state solves (cold start)
    const int k0 = prm->objective == 0 ? 0 : prm->loadCase, k1 = prm->objective == 0 ? s->nLoads : prm->loadCase + 1;
    for (int k = k0; k < k1 && rc == TOP_OK; ++k) {
        rc = pcg_grid(s, s->b + (size_t)k * 3 * cs, a.U + (size_t)k * 3 * cs, 0, &its, nullptr);
        tot += its;
    }
    double J = 0;
    if (rc == TOP_OK && prm->objective == 0) {
        mutual_energy_kernel<<<nb256(Ne), 256, 0, st>>>(s->Ke64, a.U, 3 * cs, a.U, 3 * cs, s->nLoads, s->weights, l0.eleGrid, Ne,
                                                        l0.g, xPhys, s->Ec, s->p.E0, s->p.Emin, s->p.penal, a.g, s->red(a.J));
        TOPGPU_COUNT_LAUNCH();
        CK(cudaMemcpyAsync(&J, a.J, sizeof(double), cudaMemcpyDeviceToHost, st));
    } else if (rc == TOP_OK) {
        // adjoint: K L = e_dof (the reference's DOF numbering: node-interleaved, compact nodes)
        const int64_t node = prm->dof / 3; const int comp = (int)(prm->dof % 3);
        const double *Uk = a.U + (size_t)prm->loadCase * 3 * cs;
        CK(cudaMemsetAsync(a.e - kMargin, 0, sizeof(double) * 3 * cs, st));
        unit_load_kernel<<<1, 1, 0, st>>>(a.e, l0.nodeGrid, node, comp, cs);
        TOPGPU_COUNT_LAUNCH();
        pick_dof_kernel<<<1, 1, 0, st>>>(Uk, l0.nodeGrid, node, comp, cs, a.J);
        TOPGPU_COUNT_LAUNCH();
        CK(cudaMemcpyAsync(&J, a.J, sizeof(double), cudaMemcpyDeviceToHost, st));
        rc = pcg_grid(s, a.e, a.L, 0, &its, nullptr);
        tot += its;
        if (rc == TOP_OK) {
            mutual_energy_kernel<<<nb256(Ne), 256, 0, st>>>(s->Ke64, a.L, 0, Uk, 0, 1, nullptr, l0.eleGrid, Ne, l0.g, xPhys,
                                                            s->Ec, s->p.E0, s->p.Emin, s->p.penal, a.g, Reduce{nullptr, nullptr, nullptr});
            TOPGPU_COUNT_LAUNCH();
        }
    }
    s->p.tol = tolKeep;
    if (rc != TOP_OK) return rc;
    // chain to the design variables
    const int VB = vb(Ne);
    int fits = 0;
    if (prm->ft == 0) {
        copy_kernel<<<VB, 256, 0, st>>>(a.g, dJdx, Ne);
        TOPGPU_COUNT_LAUNCH();
    } else if (prm->ft == 1) {
        const double *xd = x ? x : xPhys;
        mul_kernel<<<VB, 256, 0, st>>>(xd, a.g, a.t, Ne);
        TOPGPU_COUNT_LAUNCH();
        rc = filter_apply(s, a.t, a.g, &fits);
        if (rc) return rc;
        div_floor_kernel<<<VB, 256, 0, st>>>(a.g, xd, dJdx, Ne);
        TOPGPU_COUNT_LAUNCH();
    } else {
        rc = filter_apply(s, a.g, dJdx, &fits);
        if (rc) return rc;
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    if (Jout) *Jout = J;
    if (itsOut) *itsOut = tot;
    return TOP_OK;
}
