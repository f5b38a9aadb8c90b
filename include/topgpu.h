/*
 * topgpu.h -- C ABI of libtopgpu.so, a B200 (sm_100a) implementation of the
 * TOP_GPU FEA hot path: matrix-free voxel stiffness product, multigrid-
 * preconditioned CG and Galerkin coarse-stiffness assembly.
 *
 * Conventions
 *   - Every function returns a status: TOP_OK (0) or a negative TOP_ERR_*.
 *     top_last_error() returns a message for the calling thread's last error.
 *   - Array arguments are plain pointers.  Unless a function says "host",
 *     pointers are CUDA device pointers on the current device.
 *   - Arrays follow MATLAB layout: column-major, index arrays are int32 (or
 *     uint32 where stated) holding 1-based indices, 0 = void / none.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream, which is what MATLAB's MEX calls use).
 *   - dtype: TOP_F32 (MATLAB single) or TOP_F64 (MATLAB double).
 *
 * Part 1 mirrors the six MEX gateways of mnivan/TOP_GPU_on_matlab one to one
 * (same arguments, same in-place semantics).  Part 2 is the host mesh model
 * (voxel discretisation, mesh hierarchy, boundary conditions) and Part 3 the
 * fused device solver that replaces Solving_PCG / Solving_Vcycle /
 * Solving_KbyU_MatrixFree / Solving_AssembleFEAstencil of TOP_GPU.m.
 */
#ifndef TOPGPU_H
#define TOPGPU_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TOP_OK                 0
#define TOP_ERR_ARGS          -1   /* <Name>:Args / arity                     */
#define TOP_ERR_TYPE          -2   /* <Name>:Type                             */
#define TOP_ERR_SHAPE         -3   /* <Name>:Shape                            */
#define TOP_ERR_CUDA          -4   /* <Name>:CUDA                             */
#define TOP_ERR_NOT_CONVERGED -5   /* PCG reached maxIT (TOP_GPU.m:656-659)   */
#define TOP_ERR_NAN           -6   /* non-finite PCG scalar                   */
#define TOP_ERR_NOMEM         -7
#define TOP_ERR_STATE         -8   /* call out of order (e.g. no assembly)    */

#define TOP_F32 1
#define TOP_F64 2

const char *top_last_error(void);
int top_version(void);

/* ======================================================================= */
/* Part 1 -- drop-in replacements of the MEX kernels                        */
/* ======================================================================= */

/* Gathering_inplace(gUMat, gU, gE)   (Gathering_inplace.cu:75-171)
 * uMat[nElem x 24] (overwritten) = u[eNod(e,n)-1, c] at column 3n+c.
 * u: [nNodes x 3]; eNod: [nElem x 8] int32 (eNodIsU32 = 0) or uint32. */
int top_gather(void *uMat, const void *u, const void *eNod, int eNodIsU32,
               int64_t nElem, int64_t nNodes, int dtype, void *stream);

/* Scattering_inplace(Y, eNodMat, uMat)   (Scattering_inplace.cu:81-146)
 * Y[nNodes x 3] += uMat rows; node ids outside [1, nNodes] are skipped.
 * Synchronises the stream before returning, as the reference does (141). */
int top_scatter(void *Y, const int32_t *eNod, const void *uMat,
                int64_t nElem, int64_t nNodes, int dtype, void *stream);

/* scatter_accum3_inplace(keys, Tmp, xF)   (scatter_accum3_inplace.cu:115-145)
 * xF[key-1, 0..2] += Tmp[i, 0..2]; keys outside [1, M] are skipped. */
int top_scatter_accum3(const int32_t *keys, const void *Tmp, int64_t N,
                       void *xF, int64_t M, int dtype, void *stream);

/* assembleKs_level2_inplace(d_Ks, d_upMap, d_eleModulus, d_K_0, d_Pch,
 *   d_mapUnique, d_uniqueFree, d_uniqueFixed)
 *   (assembleKs_level2_inplace.cu:165-284)
 * Ks[24x24xnElem] = sum_s Pch_s' * Kch_s * Pch_s, Kch = E*K0, or
 * E*uniqueFree(:,uid) + uniqueFixed(:,uid) for children with mapUnique > 0.
 * nUnique = 0 (and NULL free/fixed) disables the boundary branch. */
int top_assemble_ks_level2(void *Ks, const int32_t *upMap, const void *eleModulus,
                           const void *K0, const void *Pch, const int32_t *mapUnique,
                           const void *uniqueFree, const void *uniqueFixed,
                           int64_t nElem, int nCh, int64_t nFine, int64_t nUnique,
                           int dtype, void *stream);

/* Allocation-free top_assemble_ks_level2 (no counterpart in the reference):
 * same arguments and results, but it never calls cudaMalloc/cudaFree.  For
 * callers that cannot let a library allocate device memory mid-call -- a MEX
 * gateway under MATLAB's gpuArray memory pool, or an application that
 * reserves its memory up front and must avoid the device synchronisation of
 * cudaMalloc/cudaFree.  Its FP64 scratch is a fixed device array (~311 KB per
 * GPU, held until exit); nCh is limited to 64 (TOP_ERR_SHAPE above that).
 * The first call on a device, and the first after its context was replaced
 * (cudaDeviceReset), resolves the array's address (make it before any stream
 * capture); concurrent calls on one device race -- serialise them. */
int top_assemble_ks_level2_noalloc(void *Ks, const int32_t *upMap, const void *eleModulus,
                                   const void *K0, const void *Pch, const int32_t *mapUnique,
                                   const void *uniqueFree, const void *uniqueFixed,
                                   int64_t nElem, int nCh, int64_t nFine, int64_t nUnique,
                                   int dtype, void *stream);

/* assembleKs_higherLevel_inplace(d_Ks, d_upMap, d_KsPrev, d_Psub)
 *   (assembleKs_higherLevel_inplace.cu:134-217) */
int top_assemble_ks_higher(void *Ks, const int32_t *upMap, const void *KsPrev,
                           const void *Psub, int64_t nElem, int nSub, int64_t nFine,
                           int dtype, void *stream);

/* assembleKs_level2_superEle_inplace(d_Ks, d_upMap, d_Ks0, d_Psub,
 *   d_mapUnique, d_eleModulus, d_uniqueFree, d_uniqueFixed)
 *   (assembleKs_level2_superEle_inplace.cu:178-325)
 * eleModulus [64 x nFine]; uniqueFree [576 x 64 x nUnique]. */
int top_assemble_ks_level2_super(void *Ks, const int32_t *upMap, const void *Ks0,
                                 const void *Psub, const int32_t *mapUnique,
                                 const void *eleModulus, const void *uniqueFree,
                                 const void *uniqueFixed, int64_t nElem, int nSub,
                                 int64_t nFine, int64_t nUnique, int dtype, void *stream);

/* ======================================================================= */
/* Part 2 -- host mesh model (no GPU needed)                                 */
/* ======================================================================= */
typedef struct top_mesh top_mesh;

/* Voxel discretisation + mesh hierarchy (FEA_VoxelBasedDiscretization
 * TOP_GPU.m:2019-2119, Solving_BuildingMeshHierarchy 1276-1434).
 * mask: host [nely x nelx x nelz] col-major, nonzero = solid.
 * control = coarsestResolutionControl_ (TOP_GPU.m:42, default 20000).
 * cellSize: 1/nelx for logical-array models, 1 for file models. */
int top_mesh_create(const uint8_t *mask, int nely, int nelx, int nelz,
                    int control, double nu, double cellSize, int superElement,
                    top_mesh **out);
int top_mesh_destroy(top_mesh *m);

/* Built-in cantilever (1) / MBB (2) boundary conditions (TOP_GPU.m:505-534),
 * then FEA_ApplyBoundaryCondition (1505-1546) and the fixed-DOF element
 * matrices of Solving_SetupKeWithFixedDOFs (1548-1727). */
int top_mesh_apply_optcase(top_mesh *m, int optCase);
/* Generic BCs (the .TopVoxel semantics, TOP_GPU.m:441-461), host arrays:
 * fixRows [nFix x 4] row-major (node 1-based compact, fixX, fixY, fixZ);
 * loadRows[k] [nLoadRows[k] x 4] row-major (node, fx, fy, fz);
 * weights [nLoads] or NULL for the mean (objWeightingList_). */
int top_mesh_apply_bc(top_mesh *m, int64_t nFix, const double *fixRows,
                      int nLoads, const int64_t *nLoadRows,
                      const double *const *loadRows, const double *weights);

/* A .TopVoxel model file, format version 1.0 (replaces the file branch of
 * CreateVoxelFEAmodel, TOP_GPU.m:416-496): solid voxels, optional per-voxel
 * densities, passive elements, fixations and load cases.  Builds the mesh
 * (cellSize 1, as for file models) and applies the BCs after moving their
 * nodes to the padded grid and the compact numbering (AdaptBCExternalMdl,
 * TOP_GPU.m:1743-1793; one row per node, the first one), load cases weighted
 * equally.  Passive elements (AdaptPassiveElementsExternalMdl, 1795-1813):
 * top_mesh_get(m, 0, "passiveElements", ...) (compact, ascending); the file's
 * densities: "densityLayout".  Errors: TOP_ERR_ARGS with "Incompatible Mesh
 * Data Format!" (a token out of place), "Unsupported Data!" (another
 * version), or a BC node / passive element that touches no solid voxel. */
int top_mesh_create_from_topvoxel(const char *path, int control, double nu, top_mesh **out);

/* Sizes: out[0] numLevels, then per level l (8 values each, from index
 * 1 + 8*l): resX, resY, resZ, spanWidth, numElements, numNodes,
 * intermediateNumNodes, nUnique (level 0 only).  Fills min(n, total). */
int top_mesh_info(const top_mesh *m, int64_t *out, int n);

/* Copy a named array of a level into a host buffer (MATLAB layout).
 * Names: eleMapBack eleMapForward eNodMat nodMapBack nodMapForward
 *   nodesOnBoundary elementsOnBoundary elementUpwardMap transferMat
 *   transferMatCoeffi solidNodeMapCoarser2Finer RI Ke mapUniqueKes
 *   eleWithFixedDOFs uniqueKesFree uniqueKesFixed fixingCond F objWeights
 *   I_mat passiveElements densityLayout, and resolution (int32 nely, nelx,
 *   nelz of the model before padding).  *count receives the element count;
 *   dst may be NULL to query. */
int top_mesh_get(const top_mesh *m, int level, const char *name, void *dst,
                 int64_t capacity, int64_t *count);

/* ======================================================================= */
/* Part 3 -- fused device solver                                            */
/* ======================================================================= */
typedef struct top_solver top_solver;

#define TOP_PREC_FP64  0   /* everything FP64                                 */
#define TOP_PREC_MIXED 1   /* V-cycle FP32, outer PCG / compliance / Cholesky FP64 */

typedef struct {
    double E0, Emin, penal;      /* modulus_, modulusMin_, SIMPpenalty_        */
    double tol;                  /* tol_ (relative residual)                   */
    int    maxIT;                /* maxIT_                                     */
    double omega;                /* weightFactorJacobi_                        */
    int    precision;            /* TOP_PREC_*                                 */
    int    outerFP32;            /* 1: outer matvec in FP32 like the reference's
                                    mixed mode (TOP_GPU.m:683-684)              */
} top_solver_params;

/* Upload a mesh (with BCs applied) to the current CUDA device. */
int top_solver_create(const top_mesh *mesh, const top_solver_params *p, top_solver **out);
int top_solver_destroy(top_solver *s);
int top_solver_set_stream(top_solver *s, void *stream);

/* Element moduli ([64 x Ne] sub-voxel values for super-element models).
 * where: 0 = host pointer, 1 = device pointer.
 * set_density applies SIMP: E = Emin + x^p (E0 - Emin) (TOP_GPU.m:169). */
int top_solver_set_modulus(top_solver *s, const double *E, int where);
int top_solver_set_density(top_solver *s, const double *xPhys, int where);

/* Solving_AssembleFEAstencil (TOP_GPU.m:1033-1267): Galerkin Ks on every
 * coarse level, Jacobi diagonals, coarsest Cholesky (FP64, on the device). */
int top_solver_assemble(top_solver *s);

/* y = K_level u on compact node-interleaved vectors [3 Nn(level)], FP64,
 * device pointers (Solving_KbyU_MatrixFree, TOP_GPU.m:669-765).
 * fp32 = 1 runs the FP32 path used inside the mixed V-cycle. */
int top_solver_matvec(top_solver *s, int level, const double *u, double *y, int fp32);
/* z = V-cycle(r), level-1 compact interleaved FP64 vectors (766-816). */
int top_solver_vcycle(top_solver *s, const double *r, double *z);
/* Restriction (817-847) / prolongation (848-878) between level ii-1 and ii. */
int top_solver_restrict(top_solver *s, int ii, const double *rFine, double *rCoarse);
int top_solver_interpolate(top_solver *s, int ii, const double *xCoarse, double *xFine);
/* Jacobi diagonal (compact interleaved) and coarse Ks [24x24xNe] of a level. */
int top_solver_get_diag(top_solver *s, int level, double *diag);
int top_solver_get_ks(top_solver *s, int level, double *Ks);

/* Solving_PCG (602-667) on load case k: U (device, [3 Nn] compact
 * interleaved) is the warm start when warm = 1 and receives the solution.
 * its / relres may be NULL.  Returns TOP_ERR_NOT_CONVERGED at maxIT. */
int top_solver_pcg(top_solver *s, int loadCase, double *U, int warm, int *its, double *relres);
/* All load cases at once (the state solves of TOP_GPU.m:181-187): one PCG
 * over the nLoads right-hand sides, every operator launched once per
 * iteration for all of them, each with its own recurrence and stopping test
 * (the iterates equal those of top_solver_pcg per load case).  U device
 * [3Nn x nLoads] (warm start when warm != 0); its / relres arrays of nLoads
 * (may be NULL).  No single counterpart in the reference (it loops). */
int top_solver_pcg_all(top_solver *s, double *U, int warm, int *its, double *relres);
/* Same on an explicit right-hand side b (device, compact interleaved). */
int top_solver_pcg_rhs(top_solver *s, const double *b, double *U, int warm, int *its, double *relres);

/* Element energies ce_e = sum_k w_k u_ke' Ke u_ke over the load cases
 * (TopOpti_ComputeUnitCompliance, TOP_GPU.m:580-600), U device [3Nn x nLoads]. */
int top_solver_unit_compliance(top_solver *s, const double *U, double *ce);

/* ---- the optimisation steps around the solve (device resident) ---- */
typedef struct {
    double V0;       /* target volume fraction                                */
    double rMin;     /* filter radius in cells                                */
    int    nLoop;    /* maximum optimisation iterations                       */
    int    ft;       /* 0 none, 1 sensitivity filter, 2 PDE density filter    */
} top_opt_params;
typedef struct {     /* one optimisation iteration (TOP_GPU.m:279-291)         */
    double c, vol, sharp, cons, change;
    int    pcgIts;
    double msAssemble, msSolve, msOpt, msFilter, msTotal;   /* tHist columns */
} top_opt_record;

/* PDE (Helmholtz) filter of TOP_GPU.m:880-1031 on element vectors (device,
 * compact element order): nodal 8x8 kernel, Jacobi-preconditioned CG to
 * tol/10; its may be NULL. */
int top_solver_filter_setup(top_solver *s, double rMin);
int top_solver_filter(top_solver *s, const double *src, double *tar, int *its);
/* Super-element density filter (TOP_GPU.m:113-121, 221-227, 262-265) on
 * [64 x Ne] sub-voxel vectors (device): h = max(0, 4 rMin - dist),
 * Hs = imfilter(ones, h); mode 0: tar = imfilter(src ./ Hs, h) (the
 * sensitivities), mode 1: tar = imfilter(src, h) ./ Hs (the densities).
 * Super-element models on a full box only. */
int top_solver_super_filter_setup(top_solver *s, double rMin);
int top_solver_super_filter(top_solver *s, const double *src, double *tar, int mode);
/* The optimisation loop of TOP_GPU.m:141-292 on the device: opt_begin runs
 * the fully solid solve (cSolid) and sets x = xPhys = V0; each opt_step is
 * one iteration (SIMP, assembly, warm-started PCG per load case,
 * sensitivities, filter, OC bisection, xPhys); optimize loops until
 * nLoop / change <= 1e-4 / sharpness <= 0.01.  Designs are device arrays. */
int top_solver_opt_begin(top_solver *s, const top_opt_params *prm, double *cSolid);
/* Passive elements (passiveElements_, e.g. from a .TopVoxel file): host array
 * of n compact 1-based element ids (n = 0 clears).  In the loop their design
 * is 1 inside the OC bisection and after the filter (TOP_GPU.m:239, 270); for
 * super elements only sub-voxel row Num_ = 4 of each, as the reference
 * indexes it (247, 273). */
int top_solver_set_passive(top_solver *s, const int32_t *ids, int64_t n);
int top_solver_opt_step(top_solver *s, top_opt_record *rec);
int top_solver_opt_state(top_solver *s, int *loop, double *change, double *sharpness);
/* PCG iterations of each load case in the last state solves (the record's
 * pcgIts is their sum; the reference lists them per case, lssIts,
 * TOP_GPU.m:186): copies min(capacity, nLoads) counts, *count = nLoads. */
int top_solver_opt_case_its(top_solver *s, int *its, int capacity, int *count);
/* get/set copy the physical and raw designs (either may be NULL) to/from
 * device or host memory (any pointer CUDA's unified addressing accepts);
 * set_design replaces the state the next opt_step starts from. */
int top_solver_get_design(top_solver *s, double *xPhys, double *x);
int top_solver_set_design(top_solver *s, const double *xPhys, const double *x);
int top_solver_optimize(top_solver *s, const top_opt_params *prm, double *xPhysOut,
                        top_opt_record *hist, int *nIter, double *cSolid);

/* Adjoint sensitivities at the design xPhys (device, [Ne]; x = the design
 * variables for ft = 1, NULL: xPhys).  objective 0: the weighted compliance
 * J = sum_k w_k F_k' U_k, self-adjoint, dJ/dxPhys_e = -p xPhys^(p-1)
 * (E0-Emin) sum_k w_k U_ke' Ke U_ke (the reference's dc times cSolid,
 * TOP_GPU.m:191-198, 580-600); objective 1: the displacement J = U_k[dof]
 * (DOF in the reference's node-interleaved numbering, 0-based), with the
 * adjoint solve K L = e_dof and dJ/dxPhys_e = -p xPhys^(p-1) (E0-Emin)
 * L_e' Ke U_e.  The state (and adjoint) solves start cold and stop at
 * relative residual tol (0: the solver's).  ft chains the result to the
 * design variables: 0 none, 1 the reference's sensitivity filter
 * H(x.*g)/max(1e-3,x), 2 the PDE density filter's transpose (the filter is
 * symmetric); ft != 0 needs top_solver_filter_setup.  Writes dJdx [Ne]
 * (device), J and the summed PCG iterations (either may be NULL).  The
 * reference has the compliance sensitivity only. */
typedef struct {
    int     objective;   /* 0 compliance, 1 displacement                          */
    int     loadCase;    /* objective 1: load case k                              */
    int64_t dof;         /* objective 1: DOF index                                */
    int     ft;          /* 0, 1, 2                                               */
    double  tol;         /* PCG relative residual of the solves (0: solver's)     */
} top_sens_params;
int top_solver_sensitivity(top_solver *s, const top_sens_params *prm, const double *xPhys, const double *x,
                           double *dJdx, double *J, int *pcgIts);

/* Kernel timing with CUDA events on the solver's stream (no host copies):
 * which = 0 level-0 K*u FP64, 1 level-0 K*u FP32, 2 one V-cycle,
 * 3 level-1 K*u FP32, 4 level 0 -> 1 restriction FP32, 5 level 1 -> 0
 * prolongation FP32; L2 is flushed by writing flushBytes before each launch.
 * No counterpart in the reference (its MATLAB driver times with tic/toc). */
int top_solver_time_kernel(top_solver *s, int which, int nrep, int64_t flushBytes, double *msPerLaunch);

/* Level-0 stiffness product kernel, per precision (fp32 = 0: the FP64
 * products, 1: the FP32 V-cycle products).  kind 0 = node-centric product
 * with the dense 24x24 Ke.  Kinds 1-4 use Ke in the Walsh-Hadamard basis of
 * the cube element (eight 3x3 blocks) and march z through tiles of ty x tx
 * threads, each of ctas CTAs taking an equal share of the (tile, z-layer)
 * work (ctas = 0: as many CTAs as fit on the GPU at once): kind 1 stages the
 * node layers in shared memory, kind 2 (FP32 only) gives each thread two
 * element columns and uses paired FP32 arithmetic, kind 3 loads each
 * column's corner nodes directly, kind 4 (FP32 only) combines the two.
 * Tile shapes 16x16 and 16x8.  Kinds 1-4
 * need Ke with the cube's reflection symmetry (always the case for the
 * reference's isotropic voxel); kind 3 is the default then.  Kind 5 (FP32
 * only, 16x8, any Ke) computes the element products on the tensor cores
 * (tcgen05.mma, TF32 hi/lo split to FP32 accuracy, TMEM accumulator); it is
 * checked against kind 0 on the model when set (set the densities first;
 * TOP_ERR_STATE otherwise, TOP_ERR_CUDA if the check fails).  get returns
 * {kind, ty, tx, ctas}.  No counterpart in the reference. */
int top_solver_set_l0_kernel(top_solver *s, int fp32, int kind, int ty, int tx, int ctas);
int top_solver_get_l0_kernel(const top_solver *s, int fp32, int *out4);
/* PCG iterations run as CUDA graphs of four iterations each (captured once
 * per right-hand side / solution pair and operator configuration, launched
 * on a solver-owned stream ordered after the caller's); on = 0 launches the
 * kernels one by one instead.  Default on.  No counterpart in the reference. */
int top_solver_set_graphs(top_solver *s, int on);
/* PCG direction update.  flexible = 0 (default): the reference's
 * beta = rho / rhoOld (TOP_GPU.m:650-653).  flexible = 1: the flexible
 * (Polak-Ribiere) beta = z.(r - r_old) / rhoOld, computed as
 * -z.(A p_old) / (p_old . A p_old) with one extra dot product per iteration;
 * it keeps consecutive directions A-orthogonal when the preconditioner is not
 * exactly symmetric (an FP32 V-cycle on high-contrast designs).  Changes the
 * iterates; compliance and the stopping test are unchanged.  No counterpart
 * in the reference. */
int top_solver_set_pcg_beta(top_solver *s, int flexible);
/* The V-cycle from its highest level with at most 2500 active DOFs (above the
 * coarsest) down, as one operator.  At assembly the library forms, in FP64 on
 * that level's active DOFs, M = 2J - J K J + Q M' Q^T (J = omega D^-1,
 * Q = (I - J K) P, P the prolongation from the level below, M' that level's
 * operator or the coarsest inverse), and every V-cycle applies it with one
 * GEMV (in the V-cycle's precision) instead of the smoothing products,
 * transfers and coarsest solve of those levels.  Equal to those steps in
 * exact arithmetic.  on = 1: use it, 0: do not, -1: the default (in mixed
 * precision, not in FP64).  *level (may be NULL) receives the level it starts
 * at, 0 when not in use (no level qualifies, super-element mode, or off).
 * Takes effect at once on an assembled solver.  No counterpart in the
 * reference. */
int top_solver_set_tail_operator(top_solver *s, int on, int *level);
/* Test of the coarse product's failure path: the next two-pass coarse
 * product withholds one packed-tile copy, so that copy's bounded wait
 * (one second) runs out; the kernel raises its error flag and the calling
 * entry point (top_solver_pcg, _vcycle, _matvec) returns TOP_ERR_CUDA with
 * the message set.  One-shot; the solver stays usable.  No counterpart in
 * the reference. */
int top_solver_test_withhold_tile(top_solver *s);
/* The coarse part of the V-cycle (coarse products, span-2 transfers,
 * coarsest solve) as one persistent cooperative launch with grid-wide
 * barriers: on = 1 from level 1 down, on = 2 from level 2 down (level 1
 * launched per step; one CTA per SM for the small grids), 0 one launch per
 * step (the default); identical results.  No counterpart in the reference. */
int top_solver_set_coarse_persistent(top_solver *s, int on);
/* Autotuner: times each level-0 kernel configuration (kind, tile shape, CTA
 * count; nrep rounds, L2 flushed by writing flushBytes before every launch)
 * on this model and keeps the fastest per precision.  A round is the
 * level-0 products one PCG iteration of this solver makes with that
 * precision's kernel, epilogues included: the outer product with its dot
 * product, and the V-cycle's residual and post-smoothing products (FP32 in
 * mixed precision, FP64 otherwise); a precision that serves none is timed on
 * the plain product.  msBest2 gets {FP64, FP32} ms per round of the winners,
 * configs8 their {kind, ty, tx, ctas} (either may be NULL).  No counterpart
 * in the reference. */
int top_solver_autotune(top_solver *s, int nrep, int64_t flushBytes, double *msBest2, int *configs8);

/* Kernels this solver has launched since it was created (every entry point
 * counts the launches it makes on the solver's stream). */
int top_solver_launch_count(const top_solver *s, int64_t *count);

/* Number of levels / load cases / DOFs of level 0. */
int top_solver_sizes(const top_solver *s, int64_t *out3);

#ifdef __cplusplus
}
#endif
#endif
