/*
 * topo_oracle.c -- FP64 CPU restatement of the TOP_GPU FEA hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see topo_oracle.h).  Line numbers
 * cite mnivan/TOP_GPU_on_matlab: TOP_GPU.m and the six *.cu MEX files.
 *
 * Parity status: the kernel restatements are pinned against the reference
 * CUDA kernels compiled unmodified (oracle/_ref, fixtures in tests/golden);
 * the tables (RI, sub-element node maps) and the element stiffness are
 * pinned against data extracted from TOP_GPU.m (tests/golden); the MATLAB
 * driver logic (hierarchy, PCG, V-cycle, OC) is checked by algebraic
 * identities and scipy direct solves -- "parity unpinned" against outputs of
 * the MATLAB program itself, which cannot run here.
 */
#include "topo_oracle.h"
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KM 576

static void *xc(size_t n, size_t sz) {
    void *p = calloc(n ? n : 1, sz);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}
static int cmp_i32(const void *a, const void *b) {
    int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
    return (x > y) - (x < y);
}

/* ------------------------------------------------------------------------ */
/* Element stiffness (TOP_GPU.m:1465-1503).  The reference writes the closed
 * form of the exactly integrated trilinear-hex stiffness of a unit cube
 * (E = 1) in terms of nine rational constants.  Here the same matrix is
 * formed from its definition, K = lam*Int(dN_c dN_d) + mu*Int(dN_d dN_c) +
 * mu*delta_cd*Int(grad N . grad N), with every integral a product of exact
 * 1-D integrals, then scaled by cellSize (TOP_GPU.m:1502).  Local node
 * numbering: corners (x,h,z) of the unit cube, h = height measured against
 * the y index of the voxel array (TOP_GPU.m:2027-2040).                     */
static const int NODE_POS[8][3] = { /* x, h, z */
    {0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};

void orc_element_stiffness(double nu, double cellSize, double *Ke)
{
    const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu  = 1.0 / (2.0 * (1.0 + nu));
    double Mi[2][2] = {{1.0/3.0, 1.0/6.0},{1.0/6.0, 1.0/3.0}};
    double Di[2][2] = {{1.0, -1.0},{-1.0, 1.0}};
    const double sgn[2] = {-1.0, 1.0};
    /* G(c,d)[a][b] = Int d_c N_a d_d N_b */
    for (int a = 0; a < 8; ++a)
      for (int b = 0; b < 8; ++b) {
        double G[3][3];
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d) {
            double p = 1.0;
            for (int k = 0; k < 3; ++k) {
                int ia = NODE_POS[a][k], ib = NODE_POS[b][k];
                double t;
                if (k == c && k == d) t = Di[ia][ib];
                else if (k == c)      t = sgn[ia] * 0.5;
                else if (k == d)      t = sgn[ib] * 0.5;
                else                  t = Mi[ia][ib];
                p *= t;
            }
            G[c][d] = p;
        }
        double lap = G[0][0] + G[1][1] + G[2][2];
        for (int c = 0; c < 3; ++c)
          for (int d = 0; d < 3; ++d) {
            double v = lam * G[c][d] + mu * G[d][c] + (c == d ? mu * lap : 0.0);
            Ke[(3*a + c) + 24 * (3*b + d)] = v * cellSize;
          }
      }
}

/* Super-element sub-voxel stiffnesses I_mat [576 x 64]
 * (hex8_BDB_at TOP_GPU.m:2543-2588, computeK_ij 2589-2608): B^T D B of the
 * reference hexahedron [-1,1]^3 (E = 1, nu = 0.30 fixed in the reference,
 * detJ = 1/8) at the midpoint of each of the 4x4x4 sub-cells, scaled by
 * 8*cellSize/64.  Column order z, x, y (y reversed), i.e. column
 * q = ly + 4*(lx + 4*lz) for the sub-voxel with array indices (ly,lx,lz).  */
static void hex8_bdb(double xi, double eta, double zeta, double *K)
{
    const double sx[8] = {-1, 1, 1,-1,-1, 1, 1,-1};
    const double sy[8] = {-1,-1, 1, 1,-1,-1, 1, 1};
    const double sz[8] = {-1,-1,-1,-1, 1, 1, 1, 1};
    const double nu = 0.30;
    double B[6][24];
    memset(B, 0, sizeof B);
    for (int a = 0; a < 8; ++a) {
        double dx = 2.0 * 0.125 * sx[a] * (1 + sy[a]*eta) * (1 + sz[a]*zeta);
        double dy = 2.0 * 0.125 * sy[a] * (1 + sx[a]*xi)  * (1 + sz[a]*zeta);
        double dz = 2.0 * 0.125 * sz[a] * (1 + sx[a]*xi)  * (1 + sy[a]*eta);
        int iu = 3*a, iv = iu + 1, iw = iu + 2;
        B[0][iu] = dx; B[1][iv] = dy; B[2][iw] = dz;
        B[3][iv] = dz; B[3][iw] = dy;
        B[4][iu] = dz; B[4][iw] = dx;
        B[5][iu] = dy; B[5][iv] = dx;
    }
    double coef = 1.0 / ((1 + nu) * (1 - 2 * nu));
    double D[6][6];
    memset(D, 0, sizeof D);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) D[i][j] = coef * (i == j ? 1 - nu : nu);
    for (int i = 3; i < 6; ++i) D[i][i] = coef * (1 - 2 * nu) / 2;
    double DB[6][24];
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 24; ++j) {
            double s = 0; for (int k = 0; k < 6; ++k) s += D[i][k] * B[k][j];
            DB[i][j] = s;
        }
    for (int i = 0; i < 24; ++i)
        for (int j = 0; j < 24; ++j) {
            double s = 0; for (int k = 0; k < 6; ++k) s += B[k][i] * DB[k][j];
            K[i + 24 * j] = s * 0.125;
        }
}

void orc_super_Imat(double cellSize, double *I_mat)
{
    const int num = 4;
    double span[4];
    for (int i = 0; i < num; ++i) span[i] = -1.0 + ((i + 1) - 0.5) / num * 2.0;
    int eid = 0;
    for (int z = 0; z < num; ++z)
        for (int x = 0; x < num; ++x)
            for (int y = 0; y < num; ++y) {
                hex8_bdb(span[x], span[num - 1 - y], span[z], I_mat + (size_t)KM * eid);
                ++eid;
            }
    for (int i = 0; i < KM * 64; ++i) I_mat[i] = I_mat[i] / 64.0 * 8.0 * cellSize;
}

/* ------------------------------------------------------------------------ */
/* Restriction/interpolation operator RI [(s+1)^3 x 8]
 * (Solving_Operator4MultiGridRestrictionAndInterpolation, TOP_GPU.m:2165-2328).
 * Row k = ly + (s+1)*(lx + (s+1)*lz) is a fine node of the coarse cell, column
 * j a coarse corner; the entries are the trilinear weights, which the
 * reference tabulates.                                                      */
static double RI2[27 * 8], RI4[125 * 8];
static int32_t SUB2[8 * 8], SUB4[64 * 8];
static int tables_ready = 0;
static const int CORNER_D[8][3] = { /* dy, dx, dz offsets of eNodMat columns */
    {1,0,0},{1,1,0},{0,1,0},{0,0,0},{1,0,1},{1,1,1},{0,1,1},{0,0,1}};

/* Child slot -> child position inside the coarse cell, as listed by
 * Solving_SubEleNodMat (TOP_GPU.m:1938-2017).  For span 4 the slots run
 * y-fastest; for span 2 they run around the cell within each z layer:
 * (y,x) = (0,0),(1,0),(1,1),(0,1).                                          */
static void slot_pos(int span, int s, int *ly, int *lx, int *lz)
{
    if (span == 4) { *ly = s % 4; *lx = (s / 4) % 4; *lz = s / 16; return; }
    static const int ring[4][2] = {{0,0},{1,0},{1,1},{0,1}};
    *lz = s / 4; *ly = ring[s % 4][0]; *lx = ring[s % 4][1];
}

static void build_tables(void)
{
    if (tables_ready) return;
    for (int pass = 0; pass < 2; ++pass) {
        int s = pass ? 4 : 2, n1 = s + 1;
        double *RI = pass ? RI4 : RI2;
        int32_t *SUB = pass ? SUB4 : SUB2;
        for (int lz = 0; lz <= s; ++lz)
            for (int lx = 0; lx <= s; ++lx)
                for (int ly = 0; ly <= s; ++ly) {
                    int k = ly + n1 * (lx + n1 * lz);
                    for (int j = 0; j < 8; ++j) {
                        double wy = CORNER_D[j][0] ? (double)ly / s : 1.0 - (double)ly / s;
                        double wx = CORNER_D[j][1] ? (double)lx / s : 1.0 - (double)lx / s;
                        double wz = CORNER_D[j][2] ? (double)lz / s : 1.0 - (double)lz / s;
                        RI[k + (size_t)n1 * n1 * n1 * j] = wy * wx * wz;
                    }
                }
        for (int c = 0; c < s * s * s; ++c) {
            int ly, lx, lz; slot_pos(s, c, &ly, &lx, &lz);
            for (int i = 0; i < 8; ++i) {
                int Y = ly + CORNER_D[i][0], X = lx + CORNER_D[i][1], Z = lz + CORNER_D[i][2];
                SUB[c * 8 + i] = 1 + Y + n1 * (X + n1 * Z);
            }
        }
    }
    tables_ready = 1;
}
const double *orc_RI_table(int span) { build_tables(); return span == 4 ? RI4 : RI2; }
const int32_t *orc_subele_nodmat(int span) { build_tables(); return span == 4 ? SUB4 : SUB2; }

/* ------------------------------------------------------------------------ */
/* The six MEX kernels, restated on host arrays.                             */
void orc_gather(double *uMat, const double *u, const int32_t *eNod,
                int64_t nElem, int64_t numNodes)
{ /* Gathering_inplace.cu:22-54 */
    (void)numNodes;
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < nElem; ++e)
        for (int c = 0; c < 3; ++c)
            for (int n = 0; n < 8; ++n) {
                int32_t node = eNod[e + n * nElem] - 1;
                uMat[e + (size_t)(3 * n + c) * nElem] = u[node + (size_t)c * numNodes];
            }
}

void orc_scatter(double *Y, const int32_t *eNod, const double *uMat,
                 int64_t Ne, int64_t numNodes)
{ /* Scattering_inplace.cu:45-78 (sequential element order, no atomics) */
    for (int64_t e = 0; e < Ne; ++e)
        for (int c = 0; c < 3; ++c)
            for (int j = 0; j < 8; ++j) {
                int32_t nid = eNod[e + Ne * j] - 1;
                if ((uint32_t)nid < (uint32_t)numNodes)
                    Y[nid + numNodes * c] += uMat[e + Ne * (c + 3 * j)];
            }
}

void orc_scatter_accum3(const int32_t *keys, const double *Tmp, int64_t N,
                        double *xF, int64_t M)
{ /* scatter_accum3_inplace.cu:32-56 */
    for (int64_t i = 0; i < N; ++i) {
        int32_t key = keys[i] - 1;
        if (key < 0 || key >= M) continue;
        for (int c = 0; c < 3; ++c) xF[key + c * M] += Tmp[i + c * N];
    }
}

/* Kout += B^T (Kch B) for one child, the arithmetic of the assembleKs_*
 * kernels (two 24x24 products, k ascending).                                */
static void ptkp_accum(const double *B, const double *Kch, double *Kout)
{
    double T[KM];
    for (int col = 0; col < 24; ++col)
        for (int row = 0; row < 24; ++row) {
            double acc = 0;
            for (int k = 0; k < 24; ++k) acc += Kch[row + 24 * k] * B[k + 24 * col];
            T[row + 24 * col] = acc;
        }
    for (int col = 0; col < 24; ++col)
        for (int row = 0; row < 24; ++row) {
            double acc = 0;
            for (int k = 0; k < 24; ++k) acc += B[k + 24 * row] * T[k + 24 * col];
            Kout[row + 24 * col] += acc;
        }
}

void orc_assemble_ks_level2(double *Ks, const int32_t *upMap, const double *eleModulus,
                            const double *K0, const double *Pch, const int32_t *mapUnique,
                            const double *uFree, const double *uFixed,
                            int64_t nElem, int nCh, int64_t nUnique)
{ /* assembleKs_level2_inplace.cu:58-160 */
    int hasFixed = nUnique > 0 && mapUnique && uFree && uFixed;
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t e = 0; e < nElem; ++e) {
        double Kout[KM], Kch[KM];
        memset(Kout, 0, sizeof Kout);
        for (int s = 0; s < nCh; ++s) {
            int32_t f1 = upMap[e + (size_t)s * nElem];
            if (f1 <= 0) continue;
            int32_t f0 = f1 - 1;
            double mod = eleModulus[f0];
            int32_t uid0 = hasFixed ? mapUnique[f0] - 1 : -1;
            if (uid0 >= 0)
                for (int t = 0; t < KM; ++t)
                    Kch[t] = uFree[(size_t)uid0 * KM + t] * mod + uFixed[(size_t)uid0 * KM + t];
            else
                for (int t = 0; t < KM; ++t) Kch[t] = K0[t] * mod;
            ptkp_accum(Pch + (size_t)s * KM, Kch, Kout);
        }
        memcpy(Ks + (size_t)e * KM, Kout, sizeof Kout);
    }
}

void orc_assemble_ks_higher(double *Ks, const int32_t *upMap, const double *KsPrev,
                            const double *Psub, int64_t nElem, int nSub)
{ /* assembleKs_higherLevel_inplace.cu:59-129 */
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t e = 0; e < nElem; ++e) {
        double Kout[KM];
        memset(Kout, 0, sizeof Kout);
        for (int s = 0; s < nSub; ++s) {
            int32_t f1 = upMap[e + (size_t)s * nElem];
            if (f1 <= 0) continue;
            ptkp_accum(Psub + (size_t)s * KM, KsPrev + (size_t)(f1 - 1) * KM, Kout);
        }
        memcpy(Ks + (size_t)e * KM, Kout, sizeof Kout);
    }
}

void orc_assemble_ks_level2_super(double *Ks, const int32_t *upMap, const double *Ks0,
                            const double *Psub, const int32_t *mapUnique,
                            const double *eleModulus, const double *uFree,
                            const double *uFixed, int64_t nElem, int nSub,
                            int64_t nUnique)
{ /* assembleKs_level2_superEle_inplace.cu:70-173 */
    int hasFixed = nUnique > 0 && mapUnique && uFree && uFixed;
    #pragma omp parallel for schedule(dynamic, 16)
    for (int64_t e = 0; e < nElem; ++e) {
        double Kout[KM], Kch[KM];
        memset(Kout, 0, sizeof Kout);
        for (int s = 0; s < nSub; ++s) {
            int32_t f1 = upMap[e + (size_t)s * nElem];
            if (f1 <= 0) continue;
            int32_t f0 = f1 - 1;
            int32_t uid1 = hasFixed ? mapUnique[f0] : 0;
            if (uid1 > 0) {
                size_t fb = (size_t)(uid1 - 1) * KM * 64, xb = (size_t)(uid1 - 1) * KM;
                for (int t = 0; t < KM; ++t) {
                    double acc = 0;
                    for (int q = 0; q < 64; ++q)
                        acc += uFree[fb + (size_t)q * KM + t] * eleModulus[(size_t)f0 * 64 + q];
                    Kch[t] = acc + uFixed[xb + t];
                }
            } else {
                memcpy(Kch, Ks0 + (size_t)f0 * KM, sizeof Kch);
            }
            ptkp_accum(Psub + (size_t)s * KM, Kch, Kout);
        }
        memcpy(Ks + (size_t)e * KM, Kout, sizeof Kout);
    }
}

/* ------------------------------------------------------------------------ */
/* Mesh construction                                                         */
static void build_incidence(OLevel *L)
{
    int64_t Ne = L->numElements, Nn = L->numNodes;
    L->incPtr = xc(Nn + 1, sizeof(int64_t));
    L->incIdx = xc((size_t)Ne * 8, sizeof(int32_t));
    for (int64_t e = 0; e < Ne; ++e)
        for (int j = 0; j < 8; ++j) L->incPtr[L->eNodMat[e + Ne * j]]++;
    for (int64_t n = 0; n < Nn; ++n) L->incPtr[n + 1] += L->incPtr[n];
    int64_t *fill = xc(Nn, sizeof(int64_t));
    for (int64_t e = 0; e < Ne; ++e)          /* element-ascending per node */
        for (int j = 0; j < 8; ++j) {
            int64_t n = L->eNodMat[e + Ne * j] - 1;
            L->incIdx[L->incPtr[n] + fill[n]++] = (int32_t)(e * 8 + j);
        }
    free(fill);
}

/* eNodMat of a level from its active grid elements; nodMapBack/Forward.
 * TOP_GPU.m:2082-2099 (level 1) and 1389-1406 (coarser levels).            */
static void discretize_level(OLevel *L)
{
    int nx = L->resX, ny = L->resY, nz = L->resZ;
    int64_t Ne = L->numElements;
    int64_t NN = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    int32_t off[8] = {0, ny + 1, ny, -1, 0, 0, 0, 0};
    int32_t plane = (ny + 1) * (nx + 1);
    for (int j = 0; j < 4; ++j) off[4 + j] = plane + off[j];
    L->eNodMat = xc((size_t)Ne * 8, sizeof(int32_t));
    for (int64_t e = 0; e < Ne; ++e) {
        int64_t g = L->eleMapBack[e] - 1;
        int ey = (int)(g % ny), ex = (int)((g / ny) % nx), ez = (int)(g / ((int64_t)ny * nx));
        int32_t base = 1 + (ey + (ny + 1) * (ex + (nx + 1) * ez)) + 1;
        for (int j = 0; j < 8; ++j) L->eNodMat[e + Ne * j] = base + off[j];
    }
    L->nodMapForward = xc(NN, sizeof(int32_t));
    for (int64_t t = 0; t < Ne * 8; ++t) L->nodMapForward[L->eNodMat[t] - 1] = 1;
    int64_t Nn = 0;
    for (int64_t t = 0; t < NN; ++t) if (L->nodMapForward[t]) L->nodMapForward[t] = (int32_t)(++Nn);
    L->numNodes = Nn; L->numDOFs = 3 * Nn;
    L->nodMapBack = xc(Nn, sizeof(int32_t));
    for (int64_t t = 0; t < NN; ++t) if (L->nodMapForward[t]) L->nodMapBack[L->nodMapForward[t] - 1] = (int32_t)(t + 1);
    for (int64_t t = 0; t < Ne * 8; ++t) L->eNodMat[t] = L->nodMapForward[L->eNodMat[t] - 1];
    /* boundary nodes: fewer than 8 incident elements (TOP_GPU.m:2101-2109, 1415-1421) */
    int32_t *cnt = xc(Nn, sizeof(int32_t));
    for (int64_t t = 0; t < Ne * 8; ++t) cnt[L->eNodMat[t] - 1]++;
    int64_t nb = 0;
    for (int64_t n = 0; n < Nn; ++n) if (cnt[n] < 8) ++nb;
    L->nNodesOnBoundary = nb;
    L->nodesOnBoundary = xc(nb, sizeof(int32_t));
    nb = 0;
    for (int64_t n = 0; n < Nn; ++n) if (cnt[n] < 8) L->nodesOnBoundary[nb++] = (int32_t)(n + 1);
    L->numNod2Eles = cnt;
    build_incidence(L);
}

static void build_hierarchy(OModel *m)
{ /* Solving_BuildingMeshHierarchy, TOP_GPU.m:1276-1434 */
    build_tables();
    for (int ii = 1; ii < m->numLevels; ++ii) {
        OLevel *P = &m->L[ii - 1], *L = &m->L[ii];
        int span = (ii == 1) ? 4 : 2;
        int nx = P->resX / span, ny = P->resY / span, nz = P->resZ / span;
        L->resX = nx; L->resY = ny; L->resZ = nz; L->spanWidth = span;
        int n1 = span + 1, nch = span * span * span, nloc = n1 * n1 * n1;
        int64_t NG = (int64_t)nx * ny * nz;
        int PNY = P->resY + 1, PNX = P->resX + 1;
        int64_t PNN = (int64_t)PNY * PNX * (P->resZ + 1);
        /* coarse grid elements with at least one active child (1354) */
        int32_t *upAll = xc((size_t)NG * nch, sizeof(int32_t));
        int32_t *tmAll = xc((size_t)NG * nloc, sizeof(int32_t));
        L->eleMapForward = xc(NG, sizeof(int32_t));
        int64_t Nc = 0;
        for (int64_t g = 0; g < NG; ++g) {
            int gy = (int)(g % ny), gx = (int)((g / ny) % nx), gz = (int)(g / ((int64_t)ny * nx));
            int64_t sum = 0;
            for (int lz = 0; lz < span; ++lz)
                for (int lx = 0; lx < span; ++lx)
                    for (int ly = 0; ly < span; ++ly) {
                        int64_t fg = (span * gy + ly) + (int64_t)P->resY * ((span * gx + lx) + (int64_t)P->resX * (span * gz + lz));
                        int32_t v = P->eleMapForward[fg];
                        upAll[g * nch + ly + span * (lx + span * lz)] = v;
                        sum += v;
                    }
            for (int lz = 0; lz <= span; ++lz)
                for (int lx = 0; lx <= span; ++lx)
                    for (int ly = 0; ly <= span; ++ly)
                        tmAll[g * nloc + ly + n1 * (lx + n1 * lz)] = (int32_t)(1 +
                            (span * gy + ly) + (int64_t)PNY * ((span * gx + lx) + (int64_t)PNX * (span * gz + lz)));
            if (sum > 0) L->eleMapForward[g] = (int32_t)(++Nc);
        }
        L->numElements = Nc;
        L->eleMapBack = xc(Nc, sizeof(int32_t));
        for (int64_t g = 0; g < NG; ++g) if (L->eleMapForward[g]) L->eleMapBack[L->eleMapForward[g] - 1] = (int32_t)(g + 1);
        L->elementUpwardMap = xc((size_t)Nc * nch, sizeof(int32_t));
        for (int64_t e = 0; e < Nc; ++e) {
            int64_t g = L->eleMapBack[e] - 1;
            for (int s = 0; s < nch; ++s) L->elementUpwardMap[e + Nc * s] = upAll[g * nch + s];
        }
        /* intermediate nodes: all fine-grid nodes of all children (void
         * included) of non-empty coarse cells (1355-1360), numbered in
         * ascending fine-grid order (1363).                                 */
        int32_t *temp = xc(PNN, sizeof(int32_t));
        for (int64_t e = 0; e < Nc; ++e) {
            int64_t g = L->eleMapBack[e] - 1;
            for (int k = 0; k < nloc; ++k) temp[tmAll[g * nloc + k] - 1] = 1;
        }
        int64_t nInt = 0;
        for (int64_t t = 0; t < PNN; ++t) if (temp[t]) temp[t] = (int32_t)(++nInt);
        L->intermediateNumNodes = nInt;
        L->transferMat = xc((size_t)nloc * Nc, sizeof(int32_t));
        L->transferMatCoeffi = xc(nInt, sizeof(double));
        for (int64_t e = 0; e < Nc; ++e) {
            int64_t g = L->eleMapBack[e] - 1;
            for (int k = 0; k < nloc; ++k) {
                int32_t v = temp[tmAll[g * nloc + k] - 1];
                L->transferMat[k + (size_t)nloc * e] = v;
            }
        }
        for (int k = 0; k < nloc; ++k)       /* 1366-1370 */
            for (int64_t e = 0; e < Nc; ++e) L->transferMatCoeffi[L->transferMat[k + (size_t)nloc * e] - 1] += 1.0;
        /* solid fine nodes -> intermediate index (1372-1377): the fine level's
         * active nodes in ascending grid order = its compact node order.    */
        L->solidNodeMapCoarser2Finer = xc(P->numNodes, sizeof(int32_t));
        for (int64_t n = 0; n < P->numNodes; ++n) {
            /* P->nodMapForward is indexed by the fine level's own grid ids */
            L->solidNodeMapCoarser2Finer[n] = 0;
        }
        for (int64_t t = 0; t < PNN; ++t) {
            int32_t c = P->nodMapForward[t];
            if (c) L->solidNodeMapCoarser2Finer[c - 1] = temp[t];
        }
        free(temp); free(upAll); free(tmAll);
        /* coarse discretisation (1389-1406) */
        discretize_level(L);
        /* nodMapBack in finest-grid numbering (1407-1410) */
        int stride = 1 << (ii + 1);
        int FNY = m->L[0].resY + 1, FNX = m->L[0].resX + 1;
        for (int64_t n = 0; n < L->numNodes; ++n) {
            int64_t t = L->nodMapBack[n] - 1;
            int cy = (int)(t % (ny + 1)), cx = (int)((t / (ny + 1)) % (nx + 1)), cz = (int)(t / ((int64_t)(ny + 1) * (nx + 1)));
            L->nodMapBack[n] = (int32_t)(1 + cy * stride + (int64_t)FNY * (cx * stride + (int64_t)FNX * cz * stride));
        }
        L->RI = xc((size_t)nloc * 8, sizeof(double));
        memcpy(L->RI, orc_RI_table(span), sizeof(double) * nloc * 8);
        free(L->numNod2Eles); L->numNod2Eles = NULL;
    }
}

OModel *orc_create(const uint8_t *mask, int nely, int nelx, int nelz,
                   int control, double nu, double cellSize, int superElement)
{ /* CreateVoxelFEAmodel (logical branch) + FEA_VoxelBasedDiscretization,
   * TOP_GPU.m:497-503, 2019-2119; FEA_SetupVoxelBased 1444-1463.          */
    if (nelx < 3 || nely < 3 || nelz < 3 || control < 1) return NULL;
    OModel *m = xc(1, sizeof(OModel));
    m->nely = nely; m->nelx = nelx; m->nelz = nelz;
    m->nu = nu; m->cellSize = cellSize; m->control = control;
    m->superElement = superElement;
    m->E0 = 1.0; m->Emin = 1e-6; m->penal = 3.0;        /* TOP_GPU.m:388-391 */
    m->tol = 1e-3; m->maxIT = 800; m->omega = 0.6;       /* 395-397          */
    int64_t nv = 0, NV = (int64_t)nely * nelx * nelz;
    for (int64_t t = 0; t < NV; ++t) nv += mask[t] ? 1 : 0;
    int nl = 0;
    while (nv >= control) { ++nl; nv = (nv + 4) / 8; }   /* round(nv/8)      */
    if (nl < 3) nl = 3;
    int pad = 1 << nl;
    int ax = (nelx + pad - 1) / pad * pad, ay = (nely + pad - 1) / pad * pad, az = (nelz + pad - 1) / pad * pad;
    /* numLevels_ = nl + 1; nonDyadic: numLevels_ - 1 levels (1287-1288)   */
    m->numLevels = nl;
    m->L = xc(m->numLevels, sizeof(OLevel));
    OLevel *L = &m->L[0];
    L->resX = ax; L->resY = ay; L->resZ = az;
    int64_t NG = (int64_t)ax * ay * az;
    L->eleMapForward = xc(NG, sizeof(int32_t));
    int64_t Ne = 0;
    for (int z = 0; z < az; ++z)
        for (int x = 0; x < ax; ++x)
            for (int y = 0; y < ay; ++y) {
                int on = (y < nely && x < nelx && z < nelz) && mask[y + (int64_t)nely * (x + (int64_t)nelx * z)];
                if (on) L->eleMapForward[y + (int64_t)ay * (x + (int64_t)ax * z)] = (int32_t)(++Ne);
            }
    L->numElements = Ne;
    L->eleMapBack = xc(Ne, sizeof(int32_t));
    for (int64_t g = 0; g < NG; ++g) if (L->eleMapForward[g]) L->eleMapBack[L->eleMapForward[g] - 1] = (int32_t)(g + 1);
    discretize_level(L);
    /* boundary elements (2110-2116) */
    uint8_t *bn = xc(L->numNodes, 1);
    for (int64_t i = 0; i < L->nNodesOnBoundary; ++i) bn[L->nodesOnBoundary[i] - 1] = 1;
    int64_t nbe = 0;
    for (int64_t e = 0; e < Ne; ++e) { int any = 0; for (int j = 0; j < 8; ++j) any |= bn[L->eNodMat[e + Ne * j] - 1]; nbe += any; }
    L->nElementsOnBoundary = nbe;
    L->elementsOnBoundary = xc(nbe, sizeof(int32_t));
    nbe = 0;
    for (int64_t e = 0; e < Ne; ++e) { int any = 0; for (int j = 0; j < 8; ++j) any |= bn[L->eNodMat[e + Ne * j] - 1]; if (any) L->elementsOnBoundary[nbe++] = (int32_t)(e + 1); }
    free(bn);
    build_hierarchy(m);
    orc_element_stiffness(nu, cellSize, L->Ke);
    for (int ii = 1; ii < m->numLevels; ++ii)         /* Ke_ii = Ke_{ii-1}*span (1066) */
        for (int t = 0; t < KM; ++t) m->L[ii].Ke[t] = m->L[ii - 1].Ke[t] * m->L[ii].spanWidth;
    if (superElement) {
        m->I_mat = xc((size_t)KM * 64, sizeof(double));
        orc_super_Imat(cellSize, m->I_mat);
        m->eleModulus = xc((size_t)Ne * 64, sizeof(double));
        m->K_mat = xc((size_t)Ne * KM, sizeof(double));
    } else {
        m->eleModulus = xc(Ne, sizeof(double));
    }
    return m;
}

void orc_destroy(OModel *m)
{
    if (!m) return;
    for (int i = 0; i < m->numLevels; ++i) {
        OLevel *L = &m->L[i];
        free(L->eleMapBack); free(L->eleMapForward); free(L->eNodMat);
        free(L->nodMapBack); free(L->nodMapForward); free(L->nodesOnBoundary);
        free(L->elementsOnBoundary); free(L->numNod2Eles); free(L->elementUpwardMap);
        free(L->transferMat); free(L->transferMatCoeffi); free(L->solidNodeMapCoarser2Finer);
        free(L->RI); free(L->Ks); free(L->diagK); free(L->incPtr); free(L->incIdx);
    }
    free(m->passive);
    free(m->L); free(m->fixingCond); free(m->F); free(m->objWeights);
    free(m->mapUniqueKes); free(m->eleWithFixedDOFs); free(m->uniqueKesFree);
    free(m->uniqueKesFixed); free(m->eleModulus); free(m->I_mat); free(m->K_mat);
    free(m->cholL); free(m->diagPrecondF); free(m->filterENod); free(m->fincPtr); free(m->fincIdx);
    free(m);
}

void orc_set_material(OModel *m, double E0, double Emin, double penal)
{ m->E0 = E0; m->Emin = Emin; m->penal = penal; }
void orc_set_solver(OModel *m, double tol, int maxIT, double omega)
{ m->tol = tol; m->maxIT = maxIT; m->omega = omega; }

/* ------------------------------------------------------------------------ */
/* Boundary conditions                                                       */
typedef struct { int32_t node; double v[3]; int64_t ord; } BCRow;
static int cmp_bcrow(const void *a, const void *b) {
    const BCRow *x = a, *y = b;
    if (x->node != y->node) return (x->node > y->node) - (x->node < y->node);
    return (x->ord > y->ord) - (x->ord < y->ord);
}
/* sort by node, keep first occurrence of each node (MATLAB unique / setdiff) */
static int64_t uniq_rows(BCRow *r, int64_t n)
{
    for (int64_t i = 0; i < n; ++i) r[i].ord = i;
    qsort(r, n, sizeof(BCRow), cmp_bcrow);
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) if (k == 0 || r[i].node != r[k - 1].node) r[k++] = r[i];
    return k;
}

static void apply_bc_elemat(double *Free, int nSlices, double *Fixed, const int *dofs, int nd, int nAdj)
{ /* Solving_ApplyBConEleStiffMat_B(_Super), TOP_GPU.m:1729-1741, 2609-2621 */
    for (int q = 0; q < nSlices; ++q) {
        double *K = Free + (size_t)q * KM;
        for (int a = 0; a < nd; ++a)
            for (int t = 0; t < 24; ++t) { K[dofs[a] + 24 * t] = 0; K[t + 24 * dofs[a]] = 0; }
    }
    for (int a = 0; a < nd; ++a) Fixed[dofs[a] + 24 * dofs[a]] = 1.0 / nAdj;
}

int orc_apply_bc(OModel *m, int64_t nFix, const double *fixRows,
                 int nLoads, const int64_t *nLoadRows, const double *const *loadRows,
                 const double *weights)
{ /* FEA_ApplyBoundaryCondition TOP_GPU.m:1505-1546 + Solving_SetupKeWithFixedDOFs 1548-1727 */
    OLevel *L = &m->L[0];
    int64_t Nn = L->numNodes, Ne = L->numElements;
    BCRow *fx = xc(nFix, sizeof(BCRow));
    for (int64_t i = 0; i < nFix; ++i) {
        fx[i].node = (int32_t)fixRows[4 * i];
        for (int c = 0; c < 3; ++c) fx[i].v[c] = fixRows[4 * i + 1 + c];
        if (fx[i].node < 1 || fx[i].node > Nn) { free(fx); return -1; }   /* MATLAB: index error */
    }
    int64_t nf = nFix;
    BCRow **ld = xc(nLoads, sizeof(BCRow *));
    int64_t *nl = xc(nLoads, sizeof(int64_t));
    for (int ii = 0; ii < nLoads; ++ii) {
        ld[ii] = xc(nLoadRows[ii], sizeof(BCRow));
        for (int64_t i = 0; i < nLoadRows[ii]; ++i) {
            ld[ii][i].node = (int32_t)loadRows[ii][4 * i];
            for (int c = 0; c < 3; ++c) ld[ii][i].v[c] = loadRows[ii][4 * i + 1 + c];
            if (ld[ii][i].node < 1 || ld[ii][i].node > Nn) { for (int j = 0; j <= ii; ++j) free(ld[j]); free(ld); free(nl); free(fx); return -1; }
        }
        nl[ii] = uniq_rows(ld[ii], nLoadRows[ii]);
        /* setdiff(fixed nodes, loaded nodes) (1513-1516) */
        int64_t k = 0;
        for (int64_t i = 0; i < nf; ++i) {
            int hit = 0;
            for (int64_t j = 0; j < nl[ii]; ++j) if (ld[ii][j].node == fx[i].node) { hit = 1; break; }
            if (!hit) fx[k++] = fx[i];
        }
        nf = uniq_rows(fx, k);
        if (nl[ii] == 0 || nf == 0) { for (int j = 0; j <= ii; ++j) free(ld[j]); free(ld); free(nl); free(fx); return -1; }
    }
    free(m->fixingCond); free(m->F); free(m->objWeights);
    m->nFix = nf;
    m->fixingCond = xc((size_t)nf * 4, sizeof(int32_t));
    for (int64_t i = 0; i < nf; ++i) {
        m->fixingCond[i] = fx[i].node;
        for (int c = 0; c < 3; ++c) m->fixingCond[i + nf * (1 + c)] = (int32_t)fx[i].v[c];
    }
    m->nLoads = nLoads;
    m->F = xc((size_t)3 * Nn * nLoads, sizeof(double));
    m->objWeights = xc(nLoads, sizeof(double));
    for (int ii = 0; ii < nLoads; ++ii) {
        for (int64_t j = 0; j < nl[ii]; ++j)
            for (int c = 0; c < 3; ++c)
                m->F[(size_t)ii * 3 * Nn + 3 * (size_t)(ld[ii][j].node - 1) + c] = ld[ii][j].v[c];
        m->objWeights[ii] = weights ? weights[ii] : 1.0 / nLoads;
        free(ld[ii]);
    }
    free(ld); free(nl); free(fx);

    /* -- elements with fixed DOFs (1566-1613 / 1648-1692) -- */
    int64_t nbN = L->nNodesOnBoundary;
    int32_t *nodeBidx = xc(Nn, sizeof(int32_t));
    for (int64_t i = 0; i < nbN; ++i) nodeBidx[L->nodesOnBoundary[i] - 1] = (int32_t)(i + 1);
    uint8_t *isBE = xc(Ne, 1);
    for (int64_t i = 0; i < L->nElementsOnBoundary; ++i) isBE[L->elementsOnBoundary[i] - 1] = 1;
    /* nodeBoundaryStruct(node).arr: boundary elements containing it, ascending */
    int64_t *bptr = xc(nbN + 1, sizeof(int64_t));
    for (int64_t e = 0; e < Ne; ++e) if (isBE[e])
        for (int j = 0; j < 8; ++j) { int32_t b = nodeBidx[L->eNodMat[e + Ne * j] - 1]; if (b) bptr[b]++; }
    for (int64_t i = 0; i < nbN; ++i) bptr[i + 1] += bptr[i];
    int32_t *barr = xc(bptr[nbN] + 1, sizeof(int32_t));
    int64_t *bfill = xc(nbN, sizeof(int64_t));
    for (int64_t e = 0; e < Ne; ++e) if (isBE[e])
        for (int j = 0; j < 8; ++j) { int32_t b = nodeBidx[L->eNodMat[e + Ne * j] - 1]; if (b) barr[bptr[b - 1] + bfill[b - 1]++] = (int32_t)(e + 1); }
    /* [~,fixedNodeIndices] = intersect(nodesOnBoundary, fixingCond(:,1)) */
    int32_t *fixSorted = xc(nf, sizeof(int32_t));
    for (int64_t i = 0; i < nf; ++i) fixSorted[i] = m->fixingCond[i];
    qsort(fixSorted, nf, sizeof(int32_t), cmp_i32);
    int64_t nfs = 0;
    int32_t *fni = xc(nbN + 1, sizeof(int32_t));
    for (int64_t i = 0, j = 0; i < nbN && j < nf;) {
        if (L->nodesOnBoundary[i] < fixSorted[j]) ++i;
        else if (L->nodesOnBoundary[i] > fixSorted[j]) ++j;
        else { fni[nfs++] = (int32_t)i; ++i; ++j; while (j < nf && fixSorted[j] == fixSorted[j - 1]) ++j; }
    }
    free(fixSorted);
    /* allElementsWithFixedDOFs = unique([fixedNodesStruct.arr]) */
    uint8_t *hasF = xc(Ne, 1);
    for (int64_t i = 0; i < nfs; ++i)
        for (int64_t t = bptr[fni[i]]; t < bptr[fni[i] + 1]; ++t) hasF[barr[t] - 1] = 1;
    free(m->mapUniqueKes); free(m->eleWithFixedDOFs); free(m->uniqueKesFree); free(m->uniqueKesFixed);
    m->mapUniqueKes = xc(Ne, sizeof(int32_t));
    int64_t nU = 0;
    for (int64_t e = 0; e < Ne; ++e) if (hasF[e]) m->mapUniqueKes[e] = (int32_t)(++nU);
    m->nUnique = nU;
    m->eleWithFixedDOFs = xc(nU, sizeof(int32_t));
    for (int64_t e = 0; e < Ne; ++e) if (hasF[e]) m->eleWithFixedDOFs[m->mapUniqueKes[e] - 1] = (int32_t)(e + 1);
    free(hasF);
    int slices = m->superElement ? 64 : 1;
    m->uniqueKesFree = xc((size_t)KM * slices * nU, sizeof(double));
    m->uniqueKesFixed = xc((size_t)KM * nU, sizeof(double));
    for (int64_t k = 0; k < nU; ++k)
        memcpy(m->uniqueKesFree + (size_t)k * KM * slices, m->superElement ? m->I_mat : L->Ke, sizeof(double) * KM * slices);
    /* for ii = 1:numel(fixedNodesStruct): iFixation = fixingCond_(ii,:) --
     * the ii-th boundary fixed node's element list is paired with the ii-th
     * row of fixingCond_ (1597-1613).                                       */
    for (int64_t ii = 0; ii < nfs; ++ii) {
        int32_t iNode = m->fixingCond[ii];
        int st[3]; for (int c = 0; c < 3; ++c) st[c] = m->fixingCond[ii + nf * (1 + c)];
        int64_t b0 = bptr[fni[ii]], b1 = bptr[fni[ii] + 1];
        int nAdj = (int)(b1 - b0);
        for (int64_t t = b0; t < b1; ++t) {
            int64_t e = barr[t] - 1;
            int dofs[24], nd = 0;
            for (int j = 0; j < 8; ++j)
                if (L->eNodMat[e + Ne * j] == iNode)
                    for (int c = 0; c < 3; ++c) if (st[c] == 1) dofs[nd++] = 3 * j + c;
            int64_t k = m->mapUniqueKes[e] - 1;
            apply_bc_elemat(m->uniqueKesFree + (size_t)k * KM * slices, slices, m->uniqueKesFixed + (size_t)k * KM, dofs, nd, nAdj);
        }
    }
    for (int64_t t = 0; t < (int64_t)KM * nU; ++t) m->uniqueKesFixed[t] *= m->E0;   /* 1614 */
    free(nodeBidx); free(isBE); free(bptr); free(barr); free(bfill); free(fni);
    return 0;
}

int orc_apply_optcase(OModel *m, int optCase)
{ /* TOP_GPU.m:505-534 */
    OLevel *L = &m->L[0];
    int NY = L->resY + 1, NX = L->resX + 1;
    int nely = m->nely, nelx = m->nelx, nelz = m->nelz;
    int64_t cap = (int64_t)(nely + 1) * (nelz + 1) + 8;
    double *fix = xc((size_t)cap * 4, sizeof(double));
    double *ld = xc((size_t)cap * 4, sizeof(double));
    int64_t nF = 0, nLd = 0;
#define NODEID(y, x, z) ((int64_t)(y) + (int64_t)NY * ((x) + (int64_t)NX * (z)))
    if (optCase == 1) {
        for (int z = 0; z <= nelz; ++z)
            for (int y = 0; y <= nely; ++y) {
                fix[4 * nF] = L->nodMapForward[NODEID(y, 0, z)];
                fix[4 * nF + 1] = fix[4 * nF + 2] = fix[4 * nF + 3] = 1; ++nF;
            }
        int zt = (int)round(nelz / 6.0 + 1.0);
        for (int z = 0; z < zt; ++z)
            for (int y = 0; y <= nely; ++y) { ld[4 * nLd] = L->nodMapForward[NODEID(y, nelx, z)]; ++nLd; }
        for (int64_t i = 0; i < nLd; ++i) { ld[4 * i + 1] = 0; ld[4 * i + 2] = 0; ld[4 * i + 3] = -1.0 / nLd; }
    } else if (optCase == 2) {
        if (nely % 2 || nelx % 2) { free(fix); free(ld); return -1; }
        int64_t ids[4] = {NODEID(0, 0, 0), NODEID(0, nelx, 0), NODEID(nely, 0, 0), NODEID(nely, nelx, 0)};
        /* find() order = ascending linear index */
        for (int a = 0; a < 4; ++a) for (int b = a + 1; b < 4; ++b) if (ids[b] < ids[a]) { int64_t t = ids[a]; ids[a] = ids[b]; ids[b] = t; }
        for (int a = 0; a < 4; ++a) { fix[4 * nF] = L->nodMapForward[ids[a]]; fix[4 * nF + 1] = fix[4 * nF + 2] = fix[4 * nF + 3] = 1; ++nF; }
        ld[0] = L->nodMapForward[NODEID(nely / 2, nelx / 2, nelz)]; ld[1] = 0; ld[2] = 0; ld[3] = -1; nLd = 1;
    } else { free(fix); free(ld); return -1; }
#undef NODEID
    const double *rows[1] = {ld};
    double w = 1.0;
    int rc = orc_apply_bc(m, nF, fix, 1, &nLd, rows, &w);
    free(fix); free(ld);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Design state                                                              */
void orc_set_modulus(OModel *m, const double *E)
{
    int64_t n = m->L[0].numElements * (m->superElement ? 64 : 1);
    memcpy(m->eleModulus, E, sizeof(double) * n);
}
void orc_set_density(OModel *m, const double *xPhys)
{ /* SIMP = Emin + xPhys.^p .* (E0 - Emin), TOP_GPU.m:169/172 */
    int64_t n = m->L[0].numElements * (m->superElement ? 64 : 1);
    for (int64_t i = 0; i < n; ++i)
        m->eleModulus[i] = m->Emin + pow(xPhys[i], m->penal) * (m->E0 - m->Emin);
}

/* ------------------------------------------------------------------------ */
/* Matrix-free K*u (Solving_KbyU_MatrixFree, TOP_GPU.m:669-765)              */
static void scatter_level(const OLevel *L, const double *uMat, double *y)
{ /* Scattering_inplace with node-interleaved output; per-node sums run in
   * ascending (element, local node) order -- the same order as the
   * sequential restatement orc_scatter.                                    */
    int64_t Ne = L->numElements, Nn = L->numNodes;
    #pragma omp parallel for schedule(static)
    for (int64_t n = 0; n < Nn; ++n) {
        double s[3] = {0, 0, 0};
        for (int64_t t = L->incPtr[n]; t < L->incPtr[n + 1]; ++t) {
            int64_t e = L->incIdx[t] >> 3; int j = L->incIdx[t] & 7;
            for (int c = 0; c < 3; ++c) s[c] += uMat[e + Ne * (c + 3 * j)];
        }
        for (int c = 0; c < 3; ++c) y[3 * n + c] = s[c];
    }
}

static void boundary_K(const OModel *m, int64_t k, double *K)
{ /* K_free .* Ee + K_fixed (704-711) / sum_q K_free(:,q).*Ee(q) + K_fixed (723-734) */
    int64_t e = m->eleWithFixedDOFs[k] - 1;
    if (!m->superElement) {
        double E = m->eleModulus[e];
        for (int t = 0; t < KM; ++t) K[t] = m->uniqueKesFree[(size_t)k * KM + t] * E + m->uniqueKesFixed[(size_t)k * KM + t];
    } else {
        for (int t = 0; t < KM; ++t) {
            double acc = 0;
            for (int q = 0; q < 64; ++q) acc += m->uniqueKesFree[((size_t)k * 64 + q) * KM + t] * m->eleModulus[e * 64 + q];
            K[t] = acc + m->uniqueKesFixed[(size_t)k * KM + t];
        }
    }
}

void orc_matvec(OModel *m, int level, const double *u, double *y)
{
    const OLevel *L = &m->L[level];
    int64_t Ne = L->numElements, Nn = L->numNodes;
    double *uMat = xc((size_t)Ne * 24, sizeof(double));
    /* gather: uMat[e, 3n+c] = u[3*(eNod-1)+c] */
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; ++e) {
        double ue[24], out[24];
        for (int n = 0; n < 8; ++n)
            for (int c = 0; c < 3; ++c) ue[3 * n + c] = u[3 * (size_t)(L->eNodMat[e + Ne * n] - 1) + c];
        if (level == 0 && !m->superElement) {
            /* uMat*K_0 .* E_e (718) */
            for (int j = 0; j < 24; ++j) {
                double s = 0; for (int k = 0; k < 24; ++k) s += ue[k] * L->Ke[k + 24 * j];
                out[j] = s * m->eleModulus[e];
            }
        } else if (level == 0) {
            /* super: K_mat(e) * u_e (736-740) */
            const double *K = m->K_mat + (size_t)e * KM;
            for (int i = 0; i < 24; ++i) { double s = 0; for (int k = 0; k < 24; ++k) s += K[i + 24 * k] * ue[k]; out[i] = s; }
        } else {
            /* pagemtimes(u(1x24), Ks) (757-760) */
            const double *K = L->Ks + (size_t)e * KM;
            for (int j = 0; j < 24; ++j) { double s = 0; for (int k = 0; k < 24; ++k) s += ue[k] * K[k + 24 * j]; out[j] = s; }
        }
        for (int j = 0; j < 24; ++j) uMat[e + Ne * j] = out[j];
    }
    if (level == 0) {
        /* boundary elements: (E*Kfree + Kfixed) * u_e overrides (712-720) */
        #pragma omp parallel for schedule(static)
        for (int64_t k = 0; k < m->nUnique; ++k) {
            int64_t e = m->eleWithFixedDOFs[k] - 1;
            double K[KM], ue[24];
            boundary_K(m, k, K);
            for (int n = 0; n < 8; ++n)
                for (int c = 0; c < 3; ++c) ue[3 * n + c] = u[3 * (size_t)(L->eNodMat[e + Ne * n] - 1) + c];
            for (int i = 0; i < 24; ++i) { double s = 0; for (int t = 0; t < 24; ++t) s += K[i + 24 * t] * ue[t]; uMat[e + Ne * i] = s; }
        }
    }
    scatter_level(L, uMat, y);
    (void)Nn;
    free(uMat);
}

/* ------------------------------------------------------------------------ */
/* Transfers                                                                 */
void orc_restrict(OModel *m, int ii, const double *rF, double *rC)
{ /* Solving_RestrictResidual TOP_GPU.m:817-847; ii = coarse level (0-based) */
    const OLevel *C = &m->L[ii], *Fl = &m->L[ii - 1];
    int64_t nInt = C->intermediateNumNodes, Nc = C->numElements;
    int nI = (C->spanWidth + 1) * (C->spanWidth + 1) * (C->spanWidth + 1);
    double *r1 = xc((size_t)nInt * 3, sizeof(double));
    for (int64_t n = 0; n < Fl->numNodes; ++n)
        for (int c = 0; c < 3; ++c) r1[(C->solidNodeMapCoarser2Finer[n] - 1) + nInt * c] = rF[3 * n + c];
    for (int64_t t = 0; t < nInt; ++t) for (int c = 0; c < 3; ++c) r1[t + nInt * c] /= C->transferMatCoeffi[t];
    /* P3D(j,e,c) = sum_k RI(k,j) r1(transferMat(k,e),c); P2D row e + Nc*j */
    double *P2D = xc((size_t)Nc * 8 * 3, sizeof(double));
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Nc; ++e)
        for (int c = 0; c < 3; ++c)
            for (int j = 0; j < 8; ++j) {
                double s = 0;
                for (int k = 0; k < nI; ++k) s += C->RI[k + nI * j] * r1[(C->transferMat[k + (size_t)nI * e] - 1) + nInt * c];
                P2D[(e + Nc * j) + (size_t)Nc * 8 * c] = s;
            }
    double *rc = xc((size_t)C->numNodes * 3, sizeof(double));
    orc_scatter_accum3(C->eNodMat, P2D, Nc * 8, rc, C->numNodes);
    for (int64_t n = 0; n < C->numNodes; ++n) for (int c = 0; c < 3; ++c) rC[3 * n + c] = rc[n + C->numNodes * c];
    free(r1); free(P2D); free(rc);
}

void orc_interpolate(OModel *m, int ii, const double *xC, double *xF)
{ /* Solving_InterpolationDeviation TOP_GPU.m:848-878 */
    const OLevel *C = &m->L[ii], *Fl = &m->L[ii - 1];
    int64_t nInt = C->intermediateNumNodes, Nc = C->numElements;
    int nI = (C->spanWidth + 1) * (C->spanWidth + 1) * (C->spanWidth + 1);
    double *Tmp = xc((size_t)nI * Nc * 3, sizeof(double));
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Nc; ++e)
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < nI; ++k) {
                double s = 0;
                for (int j = 0; j < 8; ++j) s += C->RI[k + nI * j] * xC[3 * (size_t)(C->eNodMat[e + Nc * j] - 1) + c];
                Tmp[(k + (size_t)nI * e) + (size_t)nI * Nc * c] = s;
            }
    double *x1 = xc((size_t)nInt * 3, sizeof(double));
    orc_scatter_accum3(C->transferMat, Tmp, (int64_t)nI * Nc, x1, nInt);
    for (int64_t t = 0; t < nInt; ++t) for (int c = 0; c < 3; ++c) x1[t + nInt * c] /= C->transferMatCoeffi[t];
    for (int64_t n = 0; n < Fl->numNodes; ++n)
        for (int c = 0; c < 3; ++c) xF[3 * n + c] = x1[(C->solidNodeMapCoarser2Finer[n] - 1) + nInt * c];
    free(Tmp); free(x1);
}

/* ------------------------------------------------------------------------ */
/* Coarsest level: the reference factors the assembled sparse K with
 * chol(K,'lower') and a fill-reducing permutation (TOP_GPU.m:1240-1255) and
 * solves x = P (L' \ (L \ (P' r))) (796-802).  The oracle uses a dense
 * Cholesky of the same matrix (banded storage, natural node order).         */
void orc_coarsest_solve(OModel *m, const double *r, double *x)
{
    int64_t n = m->nCoarseDOF, bw = m->cholBW;
    const double *Lb = m->cholL;
    double *y = xc(n, sizeof(double));
    for (int64_t i = 0; i < n; ++i) {
        double s = r[i];
        int64_t k0 = i - bw < 0 ? 0 : i - bw;
        for (int64_t k = k0; k < i; ++k) s -= Lb[k * (bw + 1) + (i - k)] * y[k];
        y[i] = s / Lb[i * (bw + 1)];
    }
    for (int64_t i = n - 1; i >= 0; --i) {
        double s = y[i];
        int64_t k1 = i + bw >= n ? n - 1 : i + bw;
        for (int64_t k = i + 1; k <= k1; ++k) s -= Lb[i * (bw + 1) + (k - i)] * x[k];
        x[i] = s / Lb[i * (bw + 1)];
    }
    free(y);
}

static int factor_coarsest(OModel *m)
{
    const OLevel *L = &m->L[m->numLevels - 1];
    int64_t Ne = L->numElements, n = L->numDOFs;
    int64_t bw = 0;
    for (int64_t e = 0; e < Ne; ++e) {
        int32_t lo = INT32_MAX, hi = 0;
        for (int j = 0; j < 8; ++j) { int32_t v = L->eNodMat[e + Ne * j]; if (v < lo) lo = v; if (v > hi) hi = v; }
        if (3 * (int64_t)(hi - lo) + 2 > bw) bw = 3 * (int64_t)(hi - lo) + 2;
    }
    m->cholBW = bw;
    free(m->cholL);
    m->nCoarseDOF = n;
    /* band storage: A(i,j), i>=j, at [j*(bw+1) + (i-j)] */
    double *A = xc((size_t)n * (bw + 1), sizeof(double));
    for (int64_t e = 0; e < Ne; ++e) {
        const double *K = L->Ks + (size_t)e * KM;
        for (int a = 0; a < 24; ++a)
            for (int b = 0; b < 24; ++b) {
                int64_t i = 3 * (int64_t)(L->eNodMat[e + Ne * (a / 3)] - 1) + a % 3;
                int64_t j = 3 * (int64_t)(L->eNodMat[e + Ne * (b / 3)] - 1) + b % 3;
                if (i >= j) A[j * (bw + 1) + (i - j)] += K[a + 24 * b];
            }
    }
    /* left-looking band Cholesky */
    for (int64_t j = 0; j < n; ++j) {
        int64_t k0 = j - bw < 0 ? 0 : j - bw;
        double d = A[j * (bw + 1)];
        for (int64_t k = k0; k < j; ++k) { double l = A[k * (bw + 1) + (j - k)]; d -= l * l; }
        if (!(d > 0)) { m->cholL = A; return -1; }
        double ljj = sqrt(d);
        A[j * (bw + 1)] = ljj;
        int64_t i1 = j + bw >= n ? n - 1 : j + bw;
        #pragma omp parallel for schedule(static) if (i1 - j > 256)
        for (int64_t i = j + 1; i <= i1; ++i) {
            double s = A[j * (bw + 1) + (i - j)];
            int64_t kk = i - bw > k0 ? i - bw : k0;
            for (int64_t k = kk; k < j; ++k) s -= A[k * (bw + 1) + (i - k)] * A[k * (bw + 1) + (j - k)];
            A[j * (bw + 1) + (i - j)] = s / ljj;
        }
    }
    m->cholL = A;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Stencil assembly (Solving_AssembleFEAstencil, TOP_GPU.m:1033-1267)        */
static void build_P(int span, double *P)
{ /* Pch(:,:,s) = interpolatingKe(eDofMat(s,:),:), interpolatingKe = kron(RI,I3)
   * (assembleKs_level2_gpu.m:10-14, TOP_GPU.m:1056-1060)                   */
    const double *RI = orc_RI_table(span);
    const int32_t *SUB = orc_subele_nodmat(span);
    int nI = (span + 1) * (span + 1) * (span + 1), nch = span * span * span;
    memset(P, 0, sizeof(double) * KM * nch);
    for (int s = 0; s < nch; ++s)
        for (int i = 0; i < 8; ++i)
            for (int j = 0; j < 8; ++j) {
                double w = RI[(SUB[s * 8 + i] - 1) + nI * j];
                for (int c = 0; c < 3; ++c) P[(size_t)s * KM + (3 * i + c) + 24 * (3 * j + c)] = w;
            }
}

static void diag_scatter(const OLevel *L, const double *blk /* [Ne x 24] */, double *diag)
{
    scatter_level(L, blk, diag);
}

int orc_assemble(OModel *m)
{
    for (int ii = 1; ii < m->numLevels; ++ii) {
        OLevel *L = &m->L[ii];
        int span = L->spanWidth, nch = span * span * span;
        double *P = xc((size_t)KM * nch, sizeof(double));
        build_P(span, P);
        free(L->Ks);
        L->Ks = xc((size_t)KM * L->numElements, sizeof(double));
        if (ii == 1 && !m->superElement) {
            orc_assemble_ks_level2(L->Ks, L->elementUpwardMap, m->eleModulus, m->L[0].Ke, P,
                                   m->mapUniqueKes, m->uniqueKesFree, m->uniqueKesFixed,
                                   L->numElements, nch, m->nUnique);
        } else if (ii == 1) {
            /* K_mat = I_mat * E_sub (1101-1102) */
            int64_t Ne1 = m->L[0].numElements;
            #pragma omp parallel for schedule(static)
            for (int64_t e = 0; e < Ne1; ++e)
                for (int t = 0; t < KM; ++t) {
                    double s = 0;
                    for (int q = 0; q < 64; ++q) s += m->I_mat[t + (size_t)KM * q] * m->eleModulus[e * 64 + q];
                    m->K_mat[(size_t)e * KM + t] = s;
                }
            orc_assemble_ks_level2_super(L->Ks, L->elementUpwardMap, m->K_mat, P, m->mapUniqueKes,
                                         m->eleModulus, m->uniqueKesFree, m->uniqueKesFixed,
                                         L->numElements, nch, m->nUnique);
        } else {
            orc_assemble_ks_higher(L->Ks, L->elementUpwardMap, m->L[ii - 1].Ks, P, L->numElements, nch);
        }
        free(P);
        if (ii < m->numLevels - 1) {        /* coarse diagK (1149-1164) */
            int64_t Ne = L->numElements;
            double *blk = xc((size_t)Ne * 24, sizeof(double));
            for (int64_t e = 0; e < Ne; ++e) for (int t = 0; t < 24; ++t) blk[e + Ne * t] = L->Ks[(size_t)e * KM + 25 * t];
            free(L->diagK); L->diagK = xc((size_t)L->numDOFs, sizeof(double));
            diag_scatter(L, blk, L->diagK);
            free(blk);
        }
    }
    /* level-1 diagK (1168-1238) */
    OLevel *L = &m->L[0];
    int64_t Ne = L->numElements;
    double *blk = xc((size_t)Ne * 24, sizeof(double));
    if (!m->superElement) {
        for (int64_t e = 0; e < Ne; ++e) for (int t = 0; t < 24; ++t) blk[e + Ne * t] = m->eleModulus[e] * L->Ke[25 * t];
    } else {
        for (int64_t e = 0; e < Ne; ++e) for (int t = 0; t < 24; ++t) blk[e + Ne * t] = m->K_mat[(size_t)e * KM + 25 * t];
    }
    for (int64_t k = 0; k < m->nUnique; ++k) {
        int64_t e = m->eleWithFixedDOFs[k] - 1;
        double K[KM];
        boundary_K(m, k, K);
        for (int t = 0; t < 24; ++t) blk[e + Ne * t] = K[25 * t];
    }
    free(L->diagK); L->diagK = xc((size_t)L->numDOFs, sizeof(double));
    diag_scatter(L, blk, L->diagK);
    free(blk);
    return factor_coarsest(m);
}

/* ------------------------------------------------------------------------ */
/* V-cycle (Solving_Vcycle, 'Standard', TOP_GPU.m:766-816)                    */
void orc_vcycle(OModel *m, const double *r, double *x)
{
    int nL = m->numLevels;
    double **xs = xc(nL, sizeof(double *)), **rs = xc(nL, sizeof(double *));
    rs[0] = (double *)r;
    for (int ii = 0; ii < nL - 1; ++ii) {
        int64_t n = m->L[ii].numDOFs;
        xs[ii] = xc(n, sizeof(double));
        for (int64_t t = 0; t < n; ++t) xs[ii][t] = m->omega * (rs[ii][t] / m->L[ii].diagK[t]);
        double *Ax = xc(n, sizeof(double));
        orc_matvec(m, ii, xs[ii], Ax);
        for (int64_t t = 0; t < n; ++t) Ax[t] = rs[ii][t] - Ax[t];
        rs[ii + 1] = xc(m->L[ii + 1].numDOFs, sizeof(double));
        orc_restrict(m, ii + 1, Ax, rs[ii + 1]);
        free(Ax);
    }
    xs[nL - 1] = xc(m->L[nL - 1].numDOFs, sizeof(double));
    orc_coarsest_solve(m, rs[nL - 1], xs[nL - 1]);
    for (int ii = nL - 2; ii >= 0; --ii) {
        int64_t n = m->L[ii].numDOFs;
        double *dx = xc(n, sizeof(double));
        orc_interpolate(m, ii + 1, xs[ii + 1], dx);
        for (int64_t t = 0; t < n; ++t) xs[ii][t] += dx[t];
        orc_matvec(m, ii, xs[ii], dx);
        for (int64_t t = 0; t < n; ++t) xs[ii][t] += m->omega * (rs[ii][t] - dx[t]) / m->L[ii].diagK[t];
        free(dx);
    }
    memcpy(x, xs[0], sizeof(double) * m->L[0].numDOFs);
    for (int ii = 0; ii < nL; ++ii) { free(xs[ii]); if (ii) free(rs[ii]); }
    free(xs); free(rs);
}

/* ------------------------------------------------------------------------ */
/* PCG (Solving_PCG, TOP_GPU.m:602-667)                                       */
typedef void (*op_fn)(OModel *, const double *, double *);
/* 64 fixed index ranges summed in order: the same value on every run and for
 * any number of threads (an OpenMP reduction combines its partials in no
 * fixed order) */
static double dotp(const double *a, const double *b, int64_t n)
{
    enum { NC = 64 };
    double part[NC];
    #pragma omp parallel for schedule(static)
    for (int c = 0; c < NC; ++c) {
        const int64_t lo = n * c / NC, hi = n * (c + 1) / NC;
        double t = 0;
        for (int64_t i = lo; i < hi; ++i) t += a[i] * b[i];
        part[c] = t;
    }
    double s = 0;
    for (int c = 0; c < NC; ++c) s += part[c];
    return s;
}
static int pcg_generic(OModel *m, op_fn A, op_fn M, int64_t n, const double *b, double *y,
                       int useX0, double tol, int maxIT, double *resOut)
{
    double normB = sqrt(dotp(b, b, n));
    double *r = xc(n, sizeof(double)), *z = xc(n, sizeof(double)), *p = xc(n, sizeof(double)), *v = xc(n, sizeof(double));
    if (!useX0) memset(y, 0, sizeof(double) * n);
    A(m, y, v);
    for (int64_t i = 0; i < n; ++i) r[i] = b[i] - v[i];
    M(m, r, z);
    memcpy(p, z, sizeof(double) * n);
    double x1 = dotp(z, r, n), res = 0;
    int its;
    for (its = 1; its <= maxIT; ++its) {
        A(m, p, v);
        double lambda = x1 / dotp(p, v, n);
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) { y[i] += lambda * p[i]; r[i] -= lambda * v[i]; }
        res = sqrt(dotp(r, r, n)) / normB;
        if (res < tol) break;
        M(m, r, z);
        double x2 = dotp(z, r, n);
        double beta = x2 / x1;
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        x1 = x2;
    }
    if (its > maxIT) its = maxIT;
    if (resOut) *resOut = res;
    free(r); free(z); free(p); free(v);
    return its;
}
static void op_K1(OModel *m, const double *u, double *y) { orc_matvec(m, 0, u, y); }
static void op_V(OModel *m, const double *r, double *x) { orc_vcycle(m, r, x); }
int orc_pcg(OModel *m, const double *b, double *x, int useX0, double tol, int maxIT, double *resOut)
{
    int its = pcg_generic(m, op_K1, op_V, m->L[0].numDOFs, b, x, useX0, tol, maxIT, resOut);
    m->lastPcgIts = its;
    return its;
}

int orc_solve_state(OModel *m, double *U, int warm)
{ /* TOP_GPU.m:155 / 186: one PCG per load case, warm-started from U */
    int tot = 0;
    int64_t n = m->L[0].numDOFs;
    for (int ii = 0; ii < m->nLoads; ++ii)
        tot += orc_pcg(m, m->F + (size_t)ii * n, U + (size_t)ii * n, warm, m->tol, m->maxIT, NULL);
    return tot;
}

/* ------------------------------------------------------------------------ */
/* Sensitivities                                                             */
void orc_unit_compliance(OModel *m, const double *U, double *ce)
{ /* TopOpti_ComputeUnitCompliance TOP_GPU.m:580-600 */
    const OLevel *L = &m->L[0];
    int64_t Ne = L->numElements, n = L->numDOFs;
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; ++e) {
        double acc = 0;
        for (int jj = 0; jj < m->nLoads; ++jj) {
            const double *u = U + (size_t)jj * n;
            double ue[24];
            for (int a = 0; a < 8; ++a) for (int c = 0; c < 3; ++c) ue[3 * a + c] = u[3 * (size_t)(L->eNodMat[e + Ne * a] - 1) + c];
            double s = 0;
            for (int j = 0; j < 24; ++j) { double t = 0; for (int k = 0; k < 24; ++k) t += ue[k] * L->Ke[k + 24 * j]; s += t * ue[j]; }
            acc += s * m->objWeights[jj];
        }
        ce[e] = acc;
    }
}

void orc_unit_compliance_super(OModel *m, const double *U, double *ce)
{ /* TopOpti_ComputeUnitCompliance_Super TOP_GPU.m:2622-2645 (K_mat of the
   * current assembly) */
    const OLevel *L = &m->L[0];
    int64_t Ne = L->numElements, n = L->numDOFs;
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; ++e) {
        double acc = 0;
        const double *K = m->K_mat + (size_t)e * KM;
        for (int jj = 0; jj < m->nLoads; ++jj) {
            const double *u = U + (size_t)jj * n;
            double ue[24];
            for (int a = 0; a < 8; ++a) for (int c = 0; c < 3; ++c) ue[3 * a + c] = u[3 * (size_t)(L->eNodMat[e + Ne * a] - 1) + c];
            double s = 0;
            for (int i = 0; i < 24; ++i) { double t = 0; for (int k = 0; k < 24; ++k) t += K[i + 24 * k] * ue[k]; s += t * ue[i]; }
            acc += s * m->objWeights[jj];
        }
        ce[e] = acc;
    }
}

void orc_pre_compute_der(OModel *m, const double *U, double *dc)
{ /* pre_compute_der TOP_GPU.m:2646-2671: dc(s,e) = sum_w u_e' I_s u_e */
    const OLevel *L = &m->L[0];
    int64_t Ne = L->numElements, n = L->numDOFs;
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; ++e) {
        for (int s = 0; s < 64; ++s) dc[e * 64 + s] = 0;
        for (int jj = 0; jj < m->nLoads; ++jj) {
            const double *u = U + (size_t)jj * n;
            double ue[24];
            for (int a = 0; a < 8; ++a) for (int c = 0; c < 3; ++c) ue[3 * a + c] = u[3 * (size_t)(L->eNodMat[e + Ne * a] - 1) + c];
            for (int s = 0; s < 64; ++s) {
                const double *K = m->I_mat + (size_t)s * KM;
                double acc = 0;
                for (int i = 0; i < 24; ++i) { double t = 0; for (int k = 0; k < 24; ++k) t += K[i + 24 * k] * ue[k]; acc += t * ue[i]; }
                dc[e * 64 + s] += acc * m->objWeights[jj];
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* PDE filter (TOP_GPU.m:880-1031), standard voxel mode                      */
void orc_pde_filter_setup(OModel *m, double rMin)
{
    const double g = 1.0 / sqrt(3.0);
    const double s[8] = {-g, g, g, -g, -g, g, g, -g};
    const double t[8] = {-g, -g, g, g, -g, -g, g, g};
    const double p[8] = {-g, -g, -g, -g, g, g, g, g};
    double N[8][8], dS[24][8];
    for (int q = 0; q < 8; ++q) {
        const double sq = s[q], tq = t[q], pq = p[q];
        N[q][0] = 0.125*(1-sq)*(1-tq)*(1-pq); N[q][1] = 0.125*(1+sq)*(1-tq)*(1-pq);
        N[q][2] = 0.125*(1+sq)*(1+tq)*(1-pq); N[q][3] = 0.125*(1-sq)*(1+tq)*(1-pq);
        N[q][4] = 0.125*(1-sq)*(1-tq)*(1+pq); N[q][5] = 0.125*(1+sq)*(1-tq)*(1+pq);
        N[q][6] = 0.125*(1+sq)*(1+tq)*(1+pq); N[q][7] = 0.125*(1-sq)*(1+tq)*(1+pq);
        const double as[8] = {-1, 1, 1, -1, -1, 1, 1, -1}, at[8] = {-1, -1, 1, 1, -1, -1, 1, 1}, ap[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
        for (int a = 0; a < 8; ++a) {
            dS[3 * q + 0][a] = 0.125 * as[a] * (1 + at[a] * tq) * (1 + ap[a] * pq);
            dS[3 * q + 1][a] = 0.125 * at[a] * (1 + as[a] * sq) * (1 + ap[a] * pq);
            dS[3 * q + 2][a] = 0.125 * ap[a] * (1 + as[a] * sq) * (1 + at[a] * tq);
        }
    }
    double KEF0[64], KEF1[64];
    for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b) {
            double k0 = 0, k1 = 0;
            for (int r = 0; r < 24; ++r) k0 += dS[r][a] * dS[r][b];
            for (int q = 0; q < 8; ++q) k1 += N[q][a] * (1.0 / 8.0) * N[q][b];
            KEF0[a + 8 * b] = k0; KEF1[a + 8 * b] = k1;
        }
    double iR = (rMin * 1.0) / 2.0 / sqrt(3.0);          /* eleSize(1) = 1 (918) */
    for (int i = 0; i < 64; ++i) m->KEF[i] = iR * iR * KEF0[i] + KEF1[i];
    const OLevel *L = &m->L[0];
    free(m->diagPrecondF);
    m->nFilterNodes = L->numNodes;
    m->diagPrecondF = xc(L->numNodes, sizeof(double));
    for (int64_t e = 0; e < L->numElements; ++e)
        for (int a = 0; a < 8; ++a) m->diagPrecondF[L->eNodMat[e + L->numElements * a] - 1] += m->KEF[9 * a];
    for (int64_t n = 0; n < L->numNodes; ++n) m->diagPrecondF[n] = 1.0 / m->diagPrecondF[n];
}

static void op_filterA(OModel *m, const double *u, double *y)
{ /* MatTimesVec_matrixFree_B (1008-1031): accumarray of (u(eNod) * iKEF) */
    const OLevel *L = &m->L[0];
    int64_t Ne = L->numElements;
    double *sub = xc((size_t)Ne * 8, sizeof(double));
    #pragma omp parallel for schedule(static)
    for (int64_t e = 0; e < Ne; ++e)
        for (int b = 0; b < 8; ++b) {
            double s = 0;
            for (int a = 0; a < 8; ++a) s += u[L->eNodMat[e + Ne * a] - 1] * m->KEF[a + 8 * b];
            sub[e + Ne * b] = s;
        }
    #pragma omp parallel for schedule(static)
    for (int64_t n = 0; n < L->numNodes; ++n) {
        double s = 0;
        for (int64_t t = L->incPtr[n]; t < L->incPtr[n + 1]; ++t) s += sub[(L->incIdx[t] >> 3) + Ne * (L->incIdx[t] & 7)];
        y[n] = s;
    }
    free(sub);
}
static void op_filterM(OModel *m, const double *r, double *z)
{
    for (int64_t n = 0; n < m->nFilterNodes; ++n) z[n] = m->diagPrecondF[n] * r[n];
}
int orc_pde_filter(OModel *m, const double *src, double *tar)
{ /* TopOpti_ConductPDEFiltering_matrixFree (959-1006) */
    const OLevel *L = &m->L[0];
    int64_t Ne = L->numElements, Nn = L->numNodes;
    double *rhs = xc(Nn, sizeof(double)), *sol = xc(Nn, sizeof(double));
    /* element -> node: accumarray(eNod(:), repmat(src/8, 8, 1)) */
    for (int64_t n = 0; n < Nn; ++n) {
        double s = 0;
        for (int64_t t = L->incPtr[n]; t < L->incPtr[n + 1]; ++t) s += src[L->incIdx[t] >> 3] * (1.0 / 8.0);
        rhs[n] = s;
    }
    int its = pcg_generic(m, op_filterA, op_filterM, Nn, rhs, sol, 0, m->tol / 10.0, m->maxIT, NULL);
    for (int64_t e = 0; e < Ne; ++e) {
        double s = 0;
        for (int a = 0; a < 8; ++a) s += sol[L->eNodMat[e + Ne * a] - 1];
        tar[e] = s * (1.0 / 8.0);
    }
    free(rhs); free(sol);
    return its;
}

/* ------------------------------------------------------------------------ */
/* Super-element density filter on the 4x refined grid (TOP_GPU.m:113-121,
 * 221-227, 262-265, gen_index_mapping 2673-2697).  imfilter(A, h, 0):
 * correlation, zero outside, same size.                                     */
typedef struct { int R; double *h; double *Hs; int fy, fx, fz; } SFilt;
static void imfilter3(const SFilt *f, const double *A, double *B)
{
    int R = f->R, w = 2 * R + 1, FY = f->fy, FX = f->fx, FZ = f->fz;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int z = 0; z < FZ; ++z)
        for (int x = 0; x < FX; ++x)
            for (int y = 0; y < FY; ++y) {
                double s = 0;
                for (int dz = -R; dz <= R; ++dz) {
                    int zz = z + dz; if (zz < 0 || zz >= FZ) continue;
                    for (int dx = -R; dx <= R; ++dx) {
                        int xx = x + dx; if (xx < 0 || xx >= FX) continue;
                        for (int dy = -R; dy <= R; ++dy) {
                            int yy = y + dy; if (yy < 0 || yy >= FY) continue;
                            s += A[yy + (int64_t)FY * (xx + (int64_t)FX * zz)] * f->h[(dy + R) + w * ((dx + R) + w * (dz + R))];
                        }
                    }
                }
                B[y + (int64_t)FY * (x + (int64_t)FX * z)] = s;
            }
}
/* element-major [64 x Ne] (q = ly + 4(lx + 4 lz)) <-> fine grid y-fastest  */
static int64_t old2new(const OModel *m, int64_t iold)
{
    int64_t nY = 4 * m->nely, nX = 4 * m->nelx;
    int64_t iy = iold % nY, ix = (iold / nY) % nX, iz = iold / (nY * nX);
    int64_t big = iy / 4 + m->nely * (ix / 4 + m->nelx * (iz / 4));
    int64_t loc = iy % 4 + 4 * (ix % 4 + 4 * (iz % 4));
    return loc + 64 * big;
}
static void sfilt_setup(OModel *m, double rMin, SFilt *f)
{
    double r = 4.0 * rMin;
    int c = (int)ceil(r);
    f->R = c - 1;
    int w = 2 * f->R + 1;
    f->h = xc((size_t)w * w * w, sizeof(double));
    for (int dz = -f->R; dz <= f->R; ++dz)
        for (int dx = -f->R; dx <= f->R; ++dx)
            for (int dy = -f->R; dy <= f->R; ++dy) {
                double v = r - sqrt((double)dx * dx + (double)dy * dy + (double)dz * dz);
                f->h[(dy + f->R) + w * ((dx + f->R) + w * (dz + f->R))] = v > 0 ? v : 0;
            }
    f->fy = 4 * m->nely; f->fx = 4 * m->nelx; f->fz = 4 * m->nelz;
    int64_t N = (int64_t)f->fy * f->fx * f->fz;
    double *ones = xc(N, sizeof(double));
    for (int64_t i = 0; i < N; ++i) ones[i] = 1;
    f->Hs = xc(N, sizeof(double));
    imfilter3(f, ones, f->Hs);
    free(ones);
}
/* mode 0: out = filt(in ./ Hs) ; mode 1: out = filt(in) ./ Hs */
static void sfilt_apply(const OModel *m, const SFilt *f, const double *in, double *out, int mode)
{
    int64_t N = (int64_t)f->fy * f->fx * f->fz;
    double *g = xc(N, sizeof(double)), *h = xc(N, sizeof(double));
    for (int64_t i = 0; i < N; ++i) g[i] = in[old2new(m, i)];
    if (mode == 0) for (int64_t i = 0; i < N; ++i) g[i] /= f->Hs[i];
    imfilter3(f, g, h);
    if (mode == 1) for (int64_t i = 0; i < N; ++i) h[i] /= f->Hs[i];
    for (int64_t i = 0; i < N; ++i) out[old2new(m, i)] = h[i];
    free(g); free(h);
}

/* ------------------------------------------------------------------------ */
/* Passive elements (passiveElements_, TOP_GPU.m:125)                         */
int orc_set_passive(OModel *m, const int32_t *ids, int64_t n)
{
    const int64_t Ne = m->L[0].numElements;
    free(m->passive);
    m->passive = NULL;
    if (n <= 0) return 0;
    m->passive = xc(Ne, 1);
    for (int64_t k = 0; k < n; ++k) {
        if (ids[k] < 1 || ids[k] > Ne) { free(m->passive); m->passive = NULL; return -1; }
        m->passive[ids[k] - 1] = 1;
    }
    return 0;
}

/* the design entries a passive element pins to 1: the element (standard
 * voxels) or, as the reference indexes xnew(Num_, passiveElements) and
 * xPhys(Num_, passiveElements) (TOP_GPU.m:247, 273), its sub-voxel row Num_ = 4
 * alone (super elements) */
static void pin_passive(const OModel *m, double *v, int64_t Ne, int sup)
{
    if (!m->passive) return;
    for (int64_t e = 0; e < Ne; ++e)
        if (m->passive[e]) v[sup ? 3 + 64 * e : e] = 1.0;
}

/* ------------------------------------------------------------------------ */
/* Optimisation loop (TOP_GPU.m:122-292)                                      */
int orc_top_opt(OModel *m, double V0, double rMin, int nLoop, int ft,
                double *xPhysOut, double *hist, double *cSolidOut)
{
    const OLevel *L = &m->L[0];
    int sup = m->superElement;
    int64_t Ne = L->numElements, nd = L->numDOFs;
    int64_t nv = Ne * (sup ? 64 : 1);
    if (sup && ft != 2) return -1;
    SFilt sf; memset(&sf, 0, sizeof sf);
    if (!sup) orc_pde_filter_setup(m, rMin); else sfilt_setup(m, rMin, &sf);
    double *x = xc(nv, sizeof(double)), *xPhys = xc(nv, sizeof(double)), *xnew = xc(nv, sizeof(double));
    double *dc = xc(nv, sizeof(double)), *dv = xc(nv, sizeof(double)), *ce = xc(Ne, sizeof(double));
    double *tmp = xc(nv, sizeof(double));
    double *U = xc((size_t)nd * m->nLoads, sizeof(double));
    for (int64_t i = 0; i < nv; ++i) { x[i] = V0; xPhys[i] = V0; }
    /* fully solid solve (141-166) */
    for (int64_t i = 0; i < nv; ++i) m->eleModulus[i] = m->E0;
    if (orc_assemble(m)) return -2;
    orc_solve_state(m, U, 0);
    double cSolid = 0;
    if (!sup) { orc_unit_compliance(m, U, ce); for (int64_t e = 0; e < Ne; ++e) cSolid += m->eleModulus[e] * ce[e]; }
    else { orc_unit_compliance_super(m, U, ce); for (int64_t e = 0; e < Ne; ++e) cSolid += ce[e]; }
    if (cSolidOut) *cSolidOut = cSolid;
    int loop = 0;
    double change = 1.0, sharp = 1.0;
    while (loop < nLoop && change > 0.0001 && sharp > 0.01) {
        ++loop;
        orc_set_density(m, xPhys);
        if (orc_assemble(m)) return -2;
        int its = orc_solve_state(m, U, 1);
        double cObj = 0, V = 0;
        if (!sup) {
            orc_unit_compliance(m, U, ce);
            for (int64_t e = 0; e < Ne; ++e) cObj += m->eleModulus[e] * (ce[e] / cSolid);
            for (int64_t e = 0; e < Ne; ++e) {
                double de = m->penal * (m->E0 - m->Emin) * pow(xPhys[e], m->penal - 1);
                dc[e] = -de * (ce[e] / cSolid); dv[e] = 1.0;
            }
        } else {
            orc_unit_compliance_super(m, U, ce);
            for (int64_t e = 0; e < Ne; ++e) cObj += ce[e] / cSolid;
            orc_pre_compute_der(m, U, dc);
            for (int64_t i = 0; i < nv; ++i) {
                double de = m->penal * (m->E0 - m->Emin) * pow(xPhys[i], m->penal - 1);
                dc[i] = -de * (dc[i] / cSolid); dv[i] = 1.0;
            }
        }
        for (int64_t i = 0; i < nv; ++i) V += xPhys[i];
        V /= (double)nv;
        double cDesign = cObj * cSolid;
        /* filtering (213-229) */
        if (ft == 1) {
            for (int64_t e = 0; e < Ne; ++e) tmp[e] = x[e] * dc[e];
            orc_pde_filter(m, tmp, dc);
            for (int64_t e = 0; e < Ne; ++e) dc[e] = dc[e] / fmax(1e-3, x[e]);
        } else if (ft == 2) {
            if (!sup) { orc_pde_filter(m, dc, tmp); memcpy(dc, tmp, sizeof(double) * nv); orc_pde_filter(m, dv, tmp); memcpy(dv, tmp, sizeof(double) * nv); }
            else { sfilt_apply(m, &sf, dc, tmp, 0); memcpy(dc, tmp, sizeof(double) * nv); sfilt_apply(m, &sf, dv, tmp, 0); memcpy(dv, tmp, sizeof(double) * nv); }
        }
        /* OC bisection (233-251) */
        double fval = 0; for (int64_t i = 0; i < nv; ++i) fval += xPhys[i];
        fval = fval / (double)nv - V0;
        double l1 = 0, l2 = 1e9, move = 0.2;
        while ((l2 - l1) / (l1 + l2) > 1e-6) {
            double lmid = 0.5 * (l2 + l1), sum = 0;
            for (int64_t i = 0; i < nv; ++i) {
                double cand = x[i] * sqrt(-dc[i] / dv[i] / lmid);
                xnew[i] = fmax(0.0, fmax(x[i] - move, fmin(1.0, fmin(x[i] + move, cand))));
            }
            pin_passive(m, xnew, Ne, sup);                        /* 239 / 247 */
            for (int64_t i = 0; i < nv; ++i) sum += xnew[i] - x[i];
            double gt = fval + sum / (double)nv;
            if (gt > 0) l1 = lmid; else l2 = lmid;
        }
        change = 0;
        for (int64_t i = 0; i < nv; ++i) { double d = fabs(xnew[i] - x[i]); if (d > change) change = d; }
        memcpy(x, xnew, sizeof(double) * nv);
        if (ft == 1) memcpy(xPhys, xnew, sizeof(double) * nv);
        else if (ft == 2) { if (!sup) orc_pde_filter(m, xnew, xPhys); else sfilt_apply(m, &sf, xnew, xPhys, 1); }
        pin_passive(m, xPhys, Ne, sup);                           /* 270 / 273 */
        sharp = 0;
        for (int64_t i = 0; i < nv; ++i) sharp += xPhys[i] * (1.0 - xPhys[i]);
        sharp = 4 * sharp / (double)nv;
        if (hist) {
            double *h = hist + (size_t)(loop - 1) * 6;
            h[0] = cDesign; h[1] = V; h[2] = sharp; h[3] = fval; h[4] = change; h[5] = its;
        }
    }
    memcpy(xPhysOut, xPhys, sizeof(double) * nv);
    free(x); free(xPhys); free(xnew); free(dc); free(dv); free(ce); free(tmp); free(U);
    free(sf.h); free(sf.Hs);
    return loop;
}
