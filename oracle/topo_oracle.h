/*
 * topo_oracle.h -- FP64 CPU restatement of the TOP_GPU FEA hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation in top_gpu_on_matlab_b200/.  Only tests/, the smoke() entry
 * and the cpu_baseline / --impl reference legs of bench.py may load it.  The
 * product never links, calls or falls back to it.
 *
 * It restates, in plain C11 + OpenMP, the numerics of mnivan/TOP_GPU_on_matlab:
 *   TOP_GPU.m (voxel discretisation, mesh hierarchy, element matrices,
 *   boundary conditions, matrix-free K*u, V-cycle, transfers, PCG, stencil
 *   assembly, coarsest Cholesky, sensitivities, PDE filter, OC loop) and the
 *   kernel arithmetic of the six MEX files (Gathering_inplace.cu,
 *   Scattering_inplace.cu, scatter_accum3_inplace.cu,
 *   assembleKs_{level2,higherLevel,level2_superEle}_inplace.cu).
 * Each function cites the reference file:line it follows.
 *
 * Storage follows MATLAB: column-major arrays, int32 index arrays holding
 * 1-based values (0 = void / none).
 *
 * Parity pinning: the reference publishes no tests, fixtures or golden
 * vectors and its MATLAB driver cannot run here (no MATLAB).  The oracle is
 * pinned by (a) tables extracted verbatim as data from TOP_GPU.m into
 * tests/golden (restriction operators, sub-element node maps), (b) exact
 * identities of the reference's algebra (Ke rigid-body modes, Galerkin
 * consistency, trilinear partition of unity, transfer multiplicities) and
 * (c) scipy sparse direct solves.  The end-to-end MATLAB path is therefore
 * "parity unpinned" against reference outputs; the MEX kernels are pinned
 * against the reference CUDA sources compiled unmodified (oracle/_ref).
 */
#ifndef TOPO_ORACLE_H
#define TOPO_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int resX, resY, resZ;          /* element grid of this level            */
    int spanWidth;                 /* 0 on level 1                          */
    int64_t numElements, numNodes, numDOFs;
    int32_t *eleMapBack;           /* [Ne]            1-based grid ids       */
    int32_t *eleMapForward;        /* [resX*resY*resZ] 0 / 1-based compact  */
    int32_t *eNodMat;              /* [Ne x 8] col-major, 1-based compact   */
    int32_t *nodMapBack;           /* [Nn]                                  */
    int32_t *nodMapForward;        /* [(resX+1)(resY+1)(resZ+1)]            */
    int64_t nNodesOnBoundary;  int32_t *nodesOnBoundary;
    int64_t nElementsOnBoundary; int32_t *elementsOnBoundary; /* level 1   */
    int32_t *numNod2Eles;          /* [Nn] level 1                          */
    /* levels >= 2 */
    int32_t *elementUpwardMap;     /* [Ne x span^3] col-major               */
    int64_t intermediateNumNodes;
    int32_t *transferMat;          /* [(span+1)^3 x Ne] col-major           */
    double  *transferMatCoeffi;    /* [nInt]                                */
    int32_t *solidNodeMapCoarser2Finer; /* [Nn of level-1]                  */
    double  *RI;                   /* [(span+1)^3 x 8] col-major            */
    /* FEA data */
    double   Ke[576];
    double  *Ks;                   /* [576 x Ne] levels >= 2                */
    double  *diagK;                /* [3 Nn]                                */
    /* node -> (element*8+local) incidence, CSR, for deterministic scatter */
    int64_t *incPtr; int32_t *incIdx;
} OLevel;

typedef struct {
    /* inputs */
    int nely, nelx, nelz;          /* original voxel array size (y,x,z)     */
    double E0, Emin, nu, penal, cellSize;
    double tol, omega; int maxIT;
    int control;                   /* coarsestResolutionControl_            */
    int superElement;              /* 0 / 1 (4x4x4 sub-voxels)              */
    /* mesh */
    int numLevels;
    OLevel *L;
    /* boundary conditions */
    int64_t nFix; int32_t *fixingCond;   /* [nFix x 4] col-major (node,fx,fy,fz) */
    int nLoads; double *F;               /* [3Nn x nLoads]                    */
    double *objWeights;                  /* [nLoads]                          */
    /* elements with fixed DOFs */
    int32_t *mapUniqueKes;               /* [Ne] 0 / 1-based                  */
    int64_t nUnique; int32_t *eleWithFixedDOFs; /* [nUnique] 1-based         */
    double *uniqueKesFree;               /* [576 x nU]  (super: 576x64xnU)    */
    double *uniqueKesFixed;              /* [576 x nU]                        */
    /* design state */
    double *eleModulus;                  /* [Ne] (super: [64 x Ne])           */
    /* super-element data */
    double *I_mat;                       /* [576 x 64]                        */
    double *K_mat;                       /* [576 x Ne]                        */
    /* coarsest direct solver (dense Cholesky, lower, col-major) */
    int64_t nCoarseDOF, cholBW; double *cholL;
    /* PDE filter */
    double KEF[64]; double *diagPrecondF; int64_t nFilterNodes;
    int32_t *filterENod; int64_t nFilterEles; /* super: fine-grid eNodMat    */
    int64_t *fincPtr; int32_t *fincIdx;
    /* statistics */
    int lastPcgIts;
    /* passive elements (TOP_GPU.m:125, 239/247, 270/273): [Ne] 0 / 1, or NULL */
    uint8_t *passive;
} OModel;

/* passive elements, 1-based compact ids (n = 0 clears): in the optimisation
 * loop their design is 1 inside the OC bisection and after the filter */
int orc_set_passive(OModel *m, const int32_t *ids, int64_t n);

/* ---- model construction ------------------------------------------------ */
/* mask: logical [nely x nelx x nelz] col-major (uint8).  Builds level 1,
 * the hierarchy and Ke (TOP_GPU.m:2019-2119, 1276-1442, 1444-1503).        */
OModel *orc_create(const uint8_t *mask, int nely, int nelx, int nelz,
                   int control, double nu, double cellSize, int superElement);
void    orc_destroy(OModel *m);
/* built-in BC generators (TOP_GPU.m:497-535), then FEA_ApplyBoundaryCondition
 * and Solving_SetupKeWithFixedDOFs (TOP_GPU.m:1505-1727).                   */
int     orc_apply_optcase(OModel *m, int optCase);
/* generic BCs: fixing [nFix x 4] (node 1-based compact, 3 flags), loads:
 * per load case [n x 4] (node, fx, fy, fz), row-major double arrays.        */
int     orc_apply_bc(OModel *m, int64_t nFix, const double *fixRows,
                     int nLoads, const int64_t *nLoadRows, const double *const *loadRows,
                     const double *weights);
void    orc_set_material(OModel *m, double E0, double Emin, double penal);
void    orc_set_solver(OModel *m, double tol, int maxIT, double omega);

/* ---- element matrices --------------------------------------------------- */
void    orc_element_stiffness(double nu, double cellSize, double *Ke);   /* 1465-1503 */
void    orc_super_Imat(double cellSize, double *I_mat);                  /* 2543-2608 */
const double *orc_RI_table(int span);      /* 2165-2328, [(s+1)^3 x 8]            */
const int32_t *orc_subele_nodmat(int span);/* 1938-2017, [s^3 x 8] row-major      */

/* ---- the six MEX kernels (CPU restatements) ----------------------------- */
void orc_gather(double *uMat, const double *u, const int32_t *eNod,
                int64_t nElem, int64_t numNodes);                 /* Gathering_inplace.cu:22-54 */
void orc_scatter(double *Y, const int32_t *eNod, const double *uMat,
                 int64_t Ne, int64_t numNodes);                   /* Scattering_inplace.cu:45-78 */
void orc_scatter_accum3(const int32_t *keys, const double *Tmp, int64_t N,
                        double *xF, int64_t M);                   /* scatter_accum3_inplace.cu:32-56 */
void orc_assemble_ks_level2(double *Ks, const int32_t *upMap, const double *eleModulus,
                            const double *K0, const double *Pch, const int32_t *mapUnique,
                            const double *uFree, const double *uFixed,
                            int64_t nElem, int nCh, int64_t nUnique);   /* assembleKs_level2_inplace.cu:58-160 */
void orc_assemble_ks_higher(double *Ks, const int32_t *upMap, const double *KsPrev,
                            const double *Psub, int64_t nElem, int nSub); /* ..._higherLevel_inplace.cu:59-129 */
void orc_assemble_ks_level2_super(double *Ks, const int32_t *upMap, const double *Ks0,
                            const double *Psub, const int32_t *mapUnique,
                            const double *eleModulus, const double *uFree,
                            const double *uFixed, int64_t nElem, int nSub,
                            int64_t nUnique);                     /* ..._superEle_inplace.cu:70-173 */

/* ---- solver ------------------------------------------------------------- */
void orc_set_density(OModel *m, const double *xPhys);   /* SIMP, TOP_GPU.m:169/172, 180 */
void orc_set_modulus(OModel *m, const double *E);       /* direct E per element          */
int  orc_assemble(OModel *m);                           /* TOP_GPU.m:1033-1267            */
/* interleaved DOF vectors [3 Nn(level)] */
void orc_matvec(OModel *m, int level, const double *u, double *y);  /* 669-765 */
void orc_vcycle(OModel *m, const double *r, double *x);             /* 766-816 */
void orc_restrict(OModel *m, int ii, const double *rF, double *rC);  /* 817-847 */
void orc_interpolate(OModel *m, int ii, const double *xC, double *xF); /* 848-878 */
void orc_coarsest_solve(OModel *m, const double *r, double *x);     /* 796-802 */
int  orc_pcg(OModel *m, const double *b, double *x, int useX0, double tol, int maxIT,
             double *resOut);                                       /* 602-667 */
/* ---- optimisation ------------------------------------------------------- */
void orc_unit_compliance(OModel *m, const double *U, double *ce);   /* 580-600 */
void orc_unit_compliance_super(OModel *m, const double *U, double *ce); /* 2622-2645 */
void orc_pre_compute_der(OModel *m, const double *U, double *dc);   /* 2646-2671 */
void orc_pde_filter_setup(OModel *m, double rMin);                  /* 880-957 */
int  orc_pde_filter(OModel *m, const double *src, double *tar);     /* 959-1031 */
/* full loop (TOP_GPU.m:141-292).  hist: per iteration [c, vol, sharp, cons,
 * change, pcgIts]; returns #iterations; xPhysOut [Ne] (super: 64*Ne).      */
int  orc_top_opt(OModel *m, double V0, double rMin, int nLoop, int ft,
                 double *xPhysOut, double *hist, double *cSolidOut);
/* one design iteration pieces, exposed for the bench's CPU arm */
int  orc_solve_state(OModel *m, double *U, int warm);   /* all load cases   */

#ifdef __cplusplus
}
#endif
#endif
