// topgpu_mesh.cpp -- host mesh model of libtopgpu.so: voxel discretisation,
// multigrid hierarchy, element matrices and boundary conditions.
//
// The maps produced here are the ones TOP_GPU.m builds (and are exported
// bit-for-bit through top_mesh_get), but they are computed directly from the
// structured voxel grid: a coarse cell's children, a fine node's parent
// cells and every multiplicity follow from integer grid arithmetic, with no
// per-cell searches.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include "topgpu_internal.h"

namespace topgpu {

static thread_local std::string g_err;
void set_error(const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}

// ---------------------------------------------------------------------------
// Element matrices.
// Node a of an element sits at the unit-cube corner (x, h, z) below, where h
// is the height axis running against the voxel array's y index; degrees of
// freedom are ordered (ux, uh, uz) per node (the reference's Ke layout,
// TOP_GPU.m:1465-1503).
static const int kPos[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};

static void grad_shape(const double p[3], double g[8][3])
{
    for (int a = 0; a < 8; ++a) {
        double f[3], df[3];
        for (int k = 0; k < 3; ++k) {
            f[k] = kPos[a][k] ? p[k] : 1.0 - p[k];
            df[k] = kPos[a][k] ? 1.0 : -1.0;
        }
        g[a][0] = df[0] * f[1] * f[2];
        g[a][1] = f[0] * df[1] * f[2];
        g[a][2] = f[0] * f[1] * df[2];
    }
}

// K += w * B^T D B at point p of the unit cube (isotropic, E = 1)
static void add_bdb(const double p[3], double nu, double w, double *K)
{
    double g[8][3];
    grad_shape(p, g);
    const double lam = nu / ((1 + nu) * (1 - 2 * nu)), mu = 1.0 / (2 * (1 + nu));
    // sigma = lam tr(eps) I + 2 mu eps ; K_(a,c)(b,d) = lam g_ac g_bd + mu g_ad g_bc + mu d_cd (g_a . g_b)
    for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b) {
            double dot = g[a][0] * g[b][0] + g[a][1] * g[b][1] + g[a][2] * g[b][2];
            for (int c = 0; c < 3; ++c)
                for (int d = 0; d < 3; ++d) {
                    double v = lam * g[a][c] * g[b][d] + mu * g[a][d] * g[b][c] + (c == d ? mu * dot : 0.0);
                    K[(3 * a + c) + 24 * (3 * b + d)] += w * v;
                }
        }
}

// Exact stiffness of the unit trilinear brick: 2x2x2 Gauss quadrature
// (exact for the quadratic integrand), times the cell size.
static void element_stiffness(double nu, double cell, double *Ke)
{
    std::memset(Ke, 0, sizeof(double) * 576);
    const double g = 0.5 / std::sqrt(3.0);
    for (int q = 0; q < 8; ++q) {
        double p[3] = {0.5 + ((q & 1) ? g : -g), 0.5 + ((q & 2) ? g : -g), 0.5 + ((q & 4) ? g : -g)};
        add_bdb(p, nu, 0.125, Ke);
    }
    for (int t = 0; t < 576; ++t) Ke[t] *= cell;
}

// Super-element sub-voxel matrices (computeK_ij / hex8_BDB_at,
// TOP_GPU.m:2543-2608): B^T D B at the centre of each of the 4x4x4
// sub-cells, weight 1/64 each, Poisson's ratio 0.30 as in the reference.
// Column q = ly + 4*(lx + 4*lz) for the sub-voxel with array indices
// (ly, lx, lz); h runs against ly.
static void super_imat(double cell, double *I)
{
    std::memset(I, 0, sizeof(double) * 576 * 64);
    for (int lz = 0; lz < 4; ++lz)
        for (int lx = 0; lx < 4; ++lx)
            for (int ly = 0; ly < 4; ++ly) {
                int q = ly + 4 * (lx + 4 * lz);
                double p[3] = {(lx + 0.5) / 4.0, 1.0 - (ly + 0.5) / 4.0, (lz + 0.5) / 4.0};
                add_bdb(p, 0.30, cell / 64.0, I + (size_t)576 * q);
            }
}

// ---------------------------------------------------------------------------
// Transfer weights and Galerkin prolongation blocks.
void child_slot_position(int span, int slot, int *ly, int *lx, int *lz)
{
    if (span == 4) { *ly = slot % 4; *lx = (slot / 4) % 4; *lz = slot / 16; return; }
    // span 2: within each z layer the reference lists the children around
    // the cell, (y,x) = (0,0), (1,0), (1,1), (0,1) (TOP_GPU.m:1941-1948),
    // while elementUpwardMap stores them y-fastest; the Galerkin assembly
    // pairs the two lists slot by slot.
    static const int ring[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
    *lz = slot / 4; *ly = ring[slot % 4][0]; *lx = ring[slot % 4][1];
}

double trilinear_weight(int span, int ly, int lx, int lz, int j)
{
    double wy = kCornerDY[j] ? double(ly) / span : 1.0 - double(ly) / span;
    double wx = kCornerDX[j] ? double(lx) / span : 1.0 - double(lx) / span;
    double wz = kCornerDZ[j] ? double(lz) / span : 1.0 - double(lz) / span;
    return wy * wx * wz;
}

void child_prolongation(int span, int slot, double *P)
{
    int cy, cx, cz;
    child_slot_position(span, slot, &cy, &cx, &cz);
    std::memset(P, 0, sizeof(double) * 576);
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 8; ++j) {
            double w = trilinear_weight(span, cy + kCornerDY[i], cx + kCornerDX[i], cz + kCornerDZ[i], j);
            for (int c = 0; c < 3; ++c) P[(3 * i + c) + 24 * (3 * j + c)] = w;
        }
}

// ---------------------------------------------------------------------------
// Discretisation of one level from its element activity (eleMapForward).
static void discretize(MeshLevel &L, std::vector<int32_t> &nodeGrid)
{
    const int ny = L.resY, nx = L.resX, nz = L.resZ;
    const int NY = ny + 1, NX = nx + 1;
    const int64_t NN = L.gridNodes();
    L.eNodMat.assign((size_t)L.Ne * 8, 0);
    L.nodMapForward.assign(NN, 0);
    std::vector<int32_t> cnt(NN, 0);
    for (int64_t e = 0; e < L.Ne; ++e) {
        int64_t g = L.eleMapBack[e] - 1;
        int ey = int(g % ny), ex = int((g / ny) % nx), ez = int(g / (int64_t(ny) * nx));
        for (int j = 0; j < 8; ++j) {
            int64_t n = (ey + kCornerDY[j]) + int64_t(NY) * ((ex + kCornerDX[j]) + int64_t(NX) * (ez + kCornerDZ[j]));
            L.eNodMat[e + L.Ne * j] = int32_t(n);
            cnt[n]++;
        }
    }
    int64_t Nn = 0;
    nodeGrid.clear();
    for (int64_t n = 0; n < NN; ++n)
        if (cnt[n]) { L.nodMapForward[n] = int32_t(++Nn); nodeGrid.push_back(int32_t(n)); }
    L.Nn = Nn;
    L.nodMapBack.resize(Nn);
    L.nodeCount.resize(Nn);
    L.nodesOnBoundary.clear();
    for (int64_t i = 0; i < Nn; ++i) {
        L.nodMapBack[i] = nodeGrid[i] + 1;
        L.nodeCount[i] = cnt[nodeGrid[i]];
        if (L.nodeCount[i] < 8) L.nodesOnBoundary.push_back(int32_t(i + 1));
    }
    for (auto &v : L.eNodMat) v = L.nodMapForward[v];
}

static int64_t round_div8(int64_t v) { return (v + 4) / 8; }   // MATLAB round(v/8), v >= 0

}  // namespace topgpu

using namespace topgpu;

extern "C" const char *top_last_error(void) { return topgpu::g_err.c_str(); }
extern "C" int top_version(void) { return 1; }

extern "C" int top_mesh_create(const uint8_t *mask, int nely, int nelx, int nelz,
                               int control, double nu, double cellSize, int superElement,
                               top_mesh **out)
{
    if (!mask || !out || control < 1) { set_error("top_mesh_create: bad arguments"); return TOP_ERR_ARGS; }
    if (nelx < 3 || nely < 3 || nelz < 3) {   // TOP_GPU.m:500-502
        set_error("top_mesh_create: Inappropriate Input Model! (at least 3 voxels per axis)");
        return TOP_ERR_SHAPE;
    }
    top_mesh *m = new (std::nothrow) top_mesh();
    if (!m) return TOP_ERR_NOMEM;
    m->nely = nely; m->nelx = nelx; m->nelz = nelz; m->control = control;
    m->nu = nu; m->cellSize = cellSize; m->superElement = superElement;
    // level count and padding (TOP_GPU.m:2044-2063, 1287-1291)
    const int64_t NV = int64_t(nely) * nelx * nelz;
    int64_t nv = 0;
    for (int64_t t = 0; t < NV; ++t) nv += mask[t] != 0;
    int nl = 0;
    while (nv >= control) { ++nl; nv = round_div8(nv); }
    nl = std::max(3, nl);
    const int pad = 1 << nl;
    auto up = [pad](int n) { return (n + pad - 1) / pad * pad; };
    m->L.resize(nl);
    MeshLevel &L0 = m->L[0];
    L0.resX = up(nelx); L0.resY = up(nely); L0.resZ = up(nelz);
    const int64_t NG = L0.gridElems();
    L0.eleMapForward.assign(NG, 0);
    int64_t Ne = 0;
    for (int z = 0; z < L0.resZ; ++z)
        for (int x = 0; x < L0.resX; ++x)
            for (int y = 0; y < L0.resY; ++y) {
                bool on = y < nely && x < nelx && z < nelz && mask[y + int64_t(nely) * (x + int64_t(nelx) * z)];
                if (on) L0.eleMapForward[y + int64_t(L0.resY) * (x + int64_t(L0.resX) * z)] = int32_t(++Ne);
            }
    L0.Ne = Ne;
    L0.eleMapBack.resize(Ne);
    for (int64_t g = 0; g < NG; ++g) if (L0.eleMapForward[g]) L0.eleMapBack[L0.eleMapForward[g] - 1] = int32_t(g + 1);
    std::vector<int32_t> nodeGridPrev;
    discretize(L0, nodeGridPrev);
    // boundary elements: any corner on the boundary (TOP_GPU.m:2110-2116)
    {
        std::vector<uint8_t> bn(L0.Nn, 0);
        for (int32_t n : L0.nodesOnBoundary) bn[n - 1] = 1;
        for (int64_t e = 0; e < Ne; ++e) {
            bool any = false;
            for (int j = 0; j < 8; ++j) any |= bn[L0.eNodMat[e + Ne * j] - 1] != 0;
            if (any) L0.elementsOnBoundary.push_back(int32_t(e + 1));
        }
    }
    element_stiffness(nu, cellSize, L0.Ke);
    // coarser levels
    const int FNY = L0.resY + 1, FNX = L0.resX + 1;
    for (int li = 1; li < nl; ++li) {
        MeshLevel &P = m->L[li - 1], &C = m->L[li];
        const int s = (li == 1) ? 4 : 2, n1 = s + 1, nch = s * s * s, nloc = n1 * n1 * n1;
        C.span = s;
        C.resX = P.resX / s; C.resY = P.resY / s; C.resZ = P.resZ / s;
        const int ny = C.resY, nx = C.resX, nz = C.resZ;
        const int PNY = P.resY + 1, PNX = P.resX + 1;
        const int64_t CG = C.gridElems();
        C.eleMapForward.assign(CG, 0);
        int64_t Nc = 0;
        for (int64_t g = 0; g < CG; ++g) {
            int gy = int(g % ny), gx = int((g / ny) % nx), gz = int(g / (int64_t(ny) * nx));
            bool any = false;
            for (int lz = 0; lz < s && !any; ++lz)
                for (int lx = 0; lx < s && !any; ++lx)
                    for (int ly = 0; ly < s && !any; ++ly)
                        any = P.eleMapForward[(s * gy + ly) + int64_t(P.resY) * ((s * gx + lx) + int64_t(P.resX) * (s * gz + lz))] != 0;
            if (any) C.eleMapForward[g] = int32_t(++Nc);
        }
        C.Ne = Nc;
        C.eleMapBack.resize(Nc);
        for (int64_t g = 0; g < CG; ++g) if (C.eleMapForward[g]) C.eleMapBack[C.eleMapForward[g] - 1] = int32_t(g + 1);
        // children (y-fastest slots) and the fine-node blocks of each cell
        C.elementUpwardMap.assign((size_t)Nc * nch, 0);
        const int64_t PNN = P.gridNodes();
        std::vector<int32_t> intIdx(PNN, 0);
        for (int64_t e = 0; e < Nc; ++e) {
            int64_t g = C.eleMapBack[e] - 1;
            int gy = int(g % ny), gx = int((g / ny) % nx), gz = int(g / (int64_t(ny) * nx));
            for (int lz = 0; lz < s; ++lz)
                for (int lx = 0; lx < s; ++lx)
                    for (int ly = 0; ly < s; ++ly)
                        C.elementUpwardMap[e + Nc * (ly + s * (lx + s * lz))] =
                            P.eleMapForward[(s * gy + ly) + int64_t(P.resY) * ((s * gx + lx) + int64_t(P.resX) * (s * gz + lz))];
            for (int lz = 0; lz <= s; ++lz)
                for (int lx = 0; lx <= s; ++lx)
                    for (int ly = 0; ly <= s; ++ly)
                        intIdx[(s * gy + ly) + int64_t(PNY) * ((s * gx + lx) + int64_t(PNX) * (s * gz + lz))] = 1;
        }
        // intermediate nodes numbered in ascending fine-grid order
        int64_t nInt = 0;
        for (int64_t t = 0; t < PNN; ++t) if (intIdx[t]) intIdx[t] = int32_t(++nInt);
        C.nInt = nInt;
        C.transferMat.resize((size_t)nloc * Nc);
        C.transferMatCoeffi.assign(nInt, 0.0);
        for (int64_t e = 0; e < Nc; ++e) {
            int64_t g = C.eleMapBack[e] - 1;
            int gy = int(g % ny), gx = int((g / ny) % nx), gz = int(g / (int64_t(ny) * nx));
            for (int lz = 0; lz <= s; ++lz)
                for (int lx = 0; lx <= s; ++lx)
                    for (int ly = 0; ly <= s; ++ly) {
                        int32_t v = intIdx[(s * gy + ly) + int64_t(PNY) * ((s * gx + lx) + int64_t(PNX) * (s * gz + lz))];
                        C.transferMat[(ly + n1 * (lx + n1 * lz)) + (size_t)nloc * e] = v;
                        C.transferMatCoeffi[v - 1] += 1.0;
                    }
        }
        C.solidNodeMap.resize(P.Nn);
        for (int64_t n = 0; n < P.Nn; ++n) C.solidNodeMap[n] = intIdx[nodeGridPrev[n]];
        std::vector<int32_t> nodeGrid;
        discretize(C, nodeGrid);
        // nodMapBack in the finest level's node numbering (TOP_GPU.m:1407-1410)
        const int S = 1 << (li + 1);
        for (int64_t n = 0; n < C.Nn; ++n) {
            int64_t t = nodeGrid[n];
            int cy = int(t % (ny + 1)), cx = int((t / (ny + 1)) % (nx + 1)), cz = int(t / (int64_t(ny + 1) * (nx + 1)));
            C.nodMapBack[n] = int32_t(1 + int64_t(cy) * S + int64_t(FNY) * (int64_t(cx) * S + int64_t(FNX) * int64_t(cz) * S));
        }
        C.RI.resize((size_t)nloc * 8);
        for (int lz = 0; lz <= s; ++lz)
            for (int lx = 0; lx <= s; ++lx)
                for (int ly = 0; ly <= s; ++ly)
                    for (int j = 0; j < 8; ++j)
                        C.RI[(ly + n1 * (lx + n1 * lz)) + (size_t)nloc * j] = trilinear_weight(s, ly, lx, lz, j);
        for (int t = 0; t < 576; ++t) C.Ke[t] = P.Ke[t] * s;   // Ke_ii = Ke_{ii-1} * span (TOP_GPU.m:1066)
        nodeGridPrev.swap(nodeGrid);
    }
    if (superElement) {
        m->I_mat.resize((size_t)576 * 64);
        super_imat(cellSize, m->I_mat.data());
    }
    *out = m;
    return TOP_OK;
}

extern "C" int top_mesh_destroy(top_mesh *m) { delete m; return TOP_OK; }

// ---------------------------------------------------------------------------
// Boundary conditions
namespace {
struct Row { int32_t node; double v[3]; size_t ord; };
// rows sorted by node, first occurrence kept (MATLAB unique / setdiff order)
void unique_rows(std::vector<Row> &r)
{
    for (size_t i = 0; i < r.size(); ++i) r[i].ord = i;
    std::sort(r.begin(), r.end(), [](const Row &a, const Row &b) { return a.node != b.node ? a.node < b.node : a.ord < b.ord; });
    size_t k = 0;
    for (size_t i = 0; i < r.size(); ++i) if (k == 0 || r[i].node != r[k - 1].node) r[k++] = r[i];
    r.resize(k);
}
}  // namespace

extern "C" int top_mesh_apply_bc(top_mesh *m, int64_t nFix, const double *fixRows,
                                 int nLoads, const int64_t *nLoadRows,
                                 const double *const *loadRows, const double *weights)
{
    if (!m || nFix < 0 || nLoads < 1 || !nLoadRows || !loadRows || (nFix > 0 && !fixRows)) {
        set_error("top_mesh_apply_bc: bad arguments");
        return TOP_ERR_ARGS;
    }
    MeshLevel &L = m->L[0];
    const int64_t Nn = L.Nn, Ne = L.Ne;
    std::vector<Row> fx((size_t)nFix);
    for (int64_t i = 0; i < nFix; ++i) {
        fx[i].node = int32_t(fixRows[4 * i]);
        for (int c = 0; c < 3; ++c) fx[i].v[c] = fixRows[4 * i + 1 + c];
        if (fx[i].node < 1 || fx[i].node > Nn) { set_error("top_mesh_apply_bc: fixed node %d out of range", fx[i].node); return TOP_ERR_ARGS; }
    }
    // FEA_ApplyBoundaryCondition (TOP_GPU.m:1511-1522): loaded nodes drop out
    // of the fixings; both lists become unique and sorted by node.
    std::vector<std::vector<Row>> ld(nLoads);
    for (int k = 0; k < nLoads; ++k) {
        ld[k].resize((size_t)nLoadRows[k]);
        for (int64_t i = 0; i < nLoadRows[k]; ++i) {
            ld[k][i].node = int32_t(loadRows[k][4 * i]);
            for (int c = 0; c < 3; ++c) ld[k][i].v[c] = loadRows[k][4 * i + 1 + c];
            if (ld[k][i].node < 1 || ld[k][i].node > Nn) { set_error("top_mesh_apply_bc: loaded node %d out of range", ld[k][i].node); return TOP_ERR_ARGS; }
        }
        unique_rows(ld[k]);
        std::vector<uint8_t> loaded(Nn + 1, 0);
        for (auto &r : ld[k]) loaded[r.node] = 1;
        std::vector<Row> keep;
        for (auto &r : fx) if (!loaded[r.node]) keep.push_back(r);
        fx.swap(keep);
        unique_rows(fx);
        if (ld[k].empty()) { set_error("No Loads!"); return TOP_ERR_ARGS; }
        if (fx.empty()) { set_error("No Fixations!"); return TOP_ERR_ARGS; }
    }
    const int64_t nf = (int64_t)fx.size();
    m->nFix = nf;
    m->fixingCond.assign((size_t)nf * 4, 0);
    m->nodeFixed.assign(Nn, 0);
    for (int64_t i = 0; i < nf; ++i) {
        m->fixingCond[i] = fx[i].node;
        for (int c = 0; c < 3; ++c) {
            m->fixingCond[i + nf * (1 + c)] = int32_t(fx[i].v[c]);
            if (fx[i].v[c] == 1.0) m->nodeFixed[fx[i].node - 1] |= uint8_t(1u << c);
        }
    }
    m->nLoads = nLoads;
    m->F.assign((size_t)3 * Nn * nLoads, 0.0);
    m->weights.resize(nLoads);
    for (int k = 0; k < nLoads; ++k) {
        for (auto &r : ld[k])
            for (int c = 0; c < 3; ++c) m->F[(size_t)k * 3 * Nn + 3 * size_t(r.node - 1) + c] = r.v[c];
        m->weights[k] = weights ? weights[k] : 1.0 / nLoads;
    }
    // Fixed-DOF element matrices (Solving_SetupKeWithFixedDOFs, TOP_GPU.m:1566-1614).
    // Elements incident to each node, ascending.
    std::vector<int64_t> ptr(Nn + 1, 0);
    for (int64_t t = 0; t < Ne * 8; ++t) ptr[L.eNodMat[t]]++;
    for (int64_t n = 0; n < Nn; ++n) ptr[n + 1] += ptr[n];
    std::vector<int32_t> inc(ptr[Nn]);
    {
        std::vector<int64_t> fill(ptr.begin(), ptr.end() - 1);
        for (int64_t e = 0; e < Ne; ++e)
            for (int j = 0; j < 8; ++j) inc[fill[L.eNodMat[e + Ne * j] - 1]++] = int32_t(e + 1);
    }
    // Fixed nodes that lie on the boundary, ascending; the reference pairs
    // the i-th of them with the i-th row of fixingCond_ (TOP_GPU.m:1587-1601).
    std::vector<int32_t> fixedSorted(fx.size());
    for (size_t i = 0; i < fx.size(); ++i) fixedSorted[i] = fx[i].node;
    std::vector<int32_t> bfix;
    std::set_intersection(L.nodesOnBoundary.begin(), L.nodesOnBoundary.end(),
                          fixedSorted.begin(), fixedSorted.end(), std::back_inserter(bfix));
    std::vector<uint8_t> hasF(Ne, 0);
    for (int32_t n : bfix)
        for (int64_t t = ptr[n - 1]; t < ptr[n]; ++t) hasF[inc[t] - 1] = 1;
    m->mapUniqueKes.assign(Ne, 0);
    m->eleWithFixedDOFs.clear();
    for (int64_t e = 0; e < Ne; ++e)
        if (hasF[e]) { m->eleWithFixedDOFs.push_back(int32_t(e + 1)); m->mapUniqueKes[e] = int32_t(m->eleWithFixedDOFs.size()); }
    const int64_t nU = (int64_t)m->eleWithFixedDOFs.size();
    const int slices = m->superElement ? 64 : 1;
    const double *base = m->superElement ? m->I_mat.data() : L.Ke;
    m->uniqueKesFree.resize((size_t)576 * slices * nU);
    m->uniqueKesFixed.assign((size_t)576 * nU, 0.0);
    for (int64_t k = 0; k < nU; ++k) std::memcpy(&m->uniqueKesFree[(size_t)k * 576 * slices], base, sizeof(double) * 576 * slices);
    for (size_t ii = 0; ii < bfix.size(); ++ii) {
        const int32_t iNode = m->fixingCond[ii];
        int st[3];
        for (int c = 0; c < 3; ++c) st[c] = m->fixingCond[ii + nf * (1 + c)];
        const int32_t listNode = bfix[ii];
        const int nAdj = int(ptr[listNode] - ptr[listNode - 1]);
        for (int64_t t = ptr[listNode - 1]; t < ptr[listNode]; ++t) {
            const int64_t e = inc[t] - 1;
            const int64_t k = m->mapUniqueKes[e] - 1;
            double *Fr = &m->uniqueKesFree[(size_t)k * 576 * slices];
            double *Fx = &m->uniqueKesFixed[(size_t)k * 576];
            for (int j = 0; j < 8; ++j) {
                if (L.eNodMat[e + Ne * j] != iNode) continue;
                for (int c = 0; c < 3; ++c) {
                    if (st[c] != 1) continue;
                    const int d = 3 * j + c;
                    for (int q = 0; q < slices; ++q)
                        for (int r = 0; r < 24; ++r) { Fr[(size_t)q * 576 + d + 24 * r] = 0; Fr[(size_t)q * 576 + r + 24 * d] = 0; }
                    Fx[d + 24 * d] = 1.0 / nAdj;
                }
            }
        }
    }
    m->hasBC = true;
    return TOP_OK;
}

extern "C" int top_mesh_apply_optcase(top_mesh *m, int optCase)
{
    if (!m) return TOP_ERR_ARGS;
    MeshLevel &L = m->L[0];
    const int NY = L.resY + 1, NX = L.resX + 1;
    const int nely = m->nely, nelx = m->nelx, nelz = m->nelz;
    auto node = [&](int y, int x, int z) { return double(L.nodMapForward[y + int64_t(NY) * (x + int64_t(NX) * z)]); };
    std::vector<double> fix, ld;
    if (optCase == 1) {   // cantilever (TOP_GPU.m:507-516)
        for (int z = 0; z <= nelz; ++z)
            for (int y = 0; y <= nely; ++y) fix.insert(fix.end(), {node(y, 0, z), 1, 1, 1});
        const int zt = int(std::lround(nelz / 6.0 + 1.0));
        std::vector<double> ids;
        for (int z = 0; z < zt; ++z)
            for (int y = 0; y <= nely; ++y) ids.push_back(node(y, nelx, z));
        for (double id : ids) ld.insert(ld.end(), {id, 0.0, 0.0, -1.0 / double(ids.size())});
    } else if (optCase == 2) {   // MBB (TOP_GPU.m:517-529)
        if (nely % 2 || nelx % 2) { set_error("top_mesh_apply_optcase: MBB needs even nely and nelx"); return TOP_ERR_SHAPE; }
        std::vector<int64_t> ids = {0, int64_t(NY) * nelx, nely, nely + int64_t(NY) * nelx};
        std::sort(ids.begin(), ids.end());
        for (int64_t id : ids) fix.insert(fix.end(), {double(L.nodMapForward[id]), 1, 1, 1});
        ld = {node(nely / 2, nelx / 2, nelz), 0.0, 0.0, -1.0};
    } else {
        set_error("top_mesh_apply_optcase: optCase must be 1 or 2");
        return TOP_ERR_ARGS;
    }
    const int64_t nl = int64_t(ld.size() / 4);
    const double *rows[1] = {ld.data()};
    const double w = 1.0;
    return top_mesh_apply_bc(m, int64_t(fix.size() / 4), fix.data(), 1, &nl, rows, &w);
}

extern "C" int top_mesh_info(const top_mesh *m, int64_t *out, int n)
{
    if (!m || !out) return TOP_ERR_ARGS;
    std::vector<int64_t> v;
    v.push_back((int64_t)m->L.size());
    for (size_t l = 0; l < m->L.size(); ++l) {
        const MeshLevel &L = m->L[l];
        v.insert(v.end(), {L.resX, L.resY, L.resZ, L.span, L.Ne, L.Nn, L.nInt,
                           l == 0 ? (int64_t)m->eleWithFixedDOFs.size() : 0});
    }
    for (int i = 0; i < n && i < (int)v.size(); ++i) out[i] = v[i];
    return TOP_OK;
}

extern "C" int top_mesh_get(const top_mesh *m, int level, const char *name, void *dst,
                            int64_t capacity, int64_t *count)
{
    if (!m || !name || level < 0 || level >= (int)m->L.size()) { set_error("top_mesh_get: bad arguments"); return TOP_ERR_ARGS; }
    const MeshLevel &L = m->L[level];
    const void *src = nullptr;
    int64_t n = 0;
    size_t es = 4;
    std::string k(name);
    const std::vector<int32_t> resolution{m->nely, m->nelx, m->nelz};
    auto I = [&](const std::vector<int32_t> &v) { src = v.data(); n = (int64_t)v.size(); es = 4; };
    auto D = [&](const std::vector<double> &v) { src = v.data(); n = (int64_t)v.size(); es = 8; };
    if (k == "eleMapBack") I(L.eleMapBack);
    else if (k == "eleMapForward") I(L.eleMapForward);
    else if (k == "eNodMat") I(L.eNodMat);
    else if (k == "nodMapBack") I(L.nodMapBack);
    else if (k == "nodMapForward") I(L.nodMapForward);
    else if (k == "nodesOnBoundary") I(L.nodesOnBoundary);
    else if (k == "elementsOnBoundary") I(L.elementsOnBoundary);
    else if (k == "elementUpwardMap") I(L.elementUpwardMap);
    else if (k == "transferMat") I(L.transferMat);
    else if (k == "transferMatCoeffi") D(L.transferMatCoeffi);
    else if (k == "solidNodeMapCoarser2Finer") I(L.solidNodeMap);
    else if (k == "RI") D(L.RI);
    else if (k == "Ke") { src = L.Ke; n = 576; es = 8; }
    else if (k == "mapUniqueKes") I(m->mapUniqueKes);
    else if (k == "eleWithFixedDOFs") I(m->eleWithFixedDOFs);
    else if (k == "uniqueKesFree") D(m->uniqueKesFree);
    else if (k == "uniqueKesFixed") D(m->uniqueKesFixed);
    else if (k == "fixingCond") I(m->fixingCond);
    else if (k == "F") D(m->F);
    else if (k == "objWeights") D(m->weights);
    else if (k == "I_mat") D(m->I_mat);
    else if (k == "passiveElements") I(m->passiveElements);
    else if (k == "resolution") I(resolution);
    else if (k == "densityLayout") D(m->densityLayout);
    else { set_error("top_mesh_get: unknown array '%s'", name); return TOP_ERR_ARGS; }
    if (count) *count = n;
    if (dst) {
        if (capacity < n) { set_error("top_mesh_get: buffer too small for '%s' (%lld < %lld)", name, (long long)capacity, (long long)n); return TOP_ERR_SHAPE; }
        if (n) std::memcpy(dst, src, (size_t)n * es);
    }
    return TOP_OK;
}
